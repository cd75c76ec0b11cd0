// ymkh_common.cuh — device helpers shared by the ymkh kernels.
//
// Arithmetic is written operand for operand as in the reference so that,
// compiled with -fmad=false, results are bit-identical to the reference
// kernels built the same way (and to the -ffp-contract=off CPU oracle).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <algorithm>
#include <string>
#include "../../include/ymkh.h"

// Debug build (nvcc -DYMKH_DEBUG=1, built as libymkh_debug.so): the fused
// kernels check every global row copy and every global store against the
// extent of its array, and every staged row against its shared-memory
// slot, before making it.  A failed check sets ERR_BOUNDS in the device
// error word (reported by ymkh_check) and the access is skipped: nothing
// traps or asserts.  Release builds compile the checks away.
#ifndef YMKH_DEBUG
#define YMKH_DEBUG 0
#endif

namespace ymkh {

constexpr unsigned ERR_WAIT = 1u;    // a bounded in-kernel wait ran out of polls
constexpr unsigned ERR_BOUNDS = 2u;  // debug build: an access outside its array was skipped

// true if the access may be made; in a debug build a false `ok` is recorded
__device__ __forceinline__ bool dbg_ok(bool ok, unsigned* err) {
#if YMKH_DEBUG
  if (!ok) {
    if (err) atomicOr(err, ERR_BOUNDS);
    return false;
  }
#else
  (void)ok;
  (void)err;
#endif
  return true;
}

// State order of include/ymkh.h.
enum Field { EX1 = 0, EX2, EX3, EZ1, EZ2, EZ3, BY1, BY2, BY3, AZ1, AZ2, AZ3 };
enum Fluid { FN = 0, FPX, FPZ, FQ1, FQ2, FQ3 };

struct State {
  double* f[YMKH_NFIELDS];
  double* a[YMKH_NFLUID];
  double* b[YMKH_NFLUID];
};

struct StepParams {
  int nx, nz;
  double dx, dz, dt, c2, eps0, alpha;
  int freeze_az1, periodic_x;
  double epsilon, xi_sponge, sigma_sponge, xi_cut, warm_T;
  int suppress_kz0;
  double hyp_diff;
  double rdx, rdz;  // 1/dx and 1/dz rounded to nearest (host division), for div_rn
};

__host__ __device__ __forceinline__ size_t idx2(int x, int z, int nx) {
  return (size_t)x + (size_t)z * (size_t)nx;
}

// s + c += v, Neumaier's compensated summation (A. Neumaier, "Rundungsfehleranalyse
// einiger Verfahren zur Summation endlicher Summen", ZAMM 54, 1974): c gathers the
// rounding error of every addition to s.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double v) {
  const double t = s + v;
  if (fabs(s) >= fabs(v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

// FCT_DeviceMath.cuh:38-46 (compute_eps)
__device__ __forceinline__ double fct_eps(double uL, double uR, double dtdx) {
  double v = 0.5 * (uL + uR);
  return v * dtdx;
}
// FCT_DeviceMath.cuh:52-63 (compute_nu_mu)
// a / b rounded to nearest, for a positive divisor b whose correctly
// rounded reciprocal y = RN(1/b) is known: q = RN(a*y) lies within one ulp
// of a/b, r = a - b*q is exact (one fma), and RN(q + r*y) is the correctly
// rounded quotient (Markstein's Newton-Raphson correction theorem,
// P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  With b > 0 the
// quotient carries a's sign, which restores the sign of an exact zero; an
// infinite a shows as an infinite a*y, which is then the quotient; NaN stays
// NaN.  The theorem needs the remainder in the normal range, so quotients
// below 2^-900 in magnitude (never met by the field differences divided
// here) may differ from a / b in the last bit.  Three FP64 instructions and
// a few selects against a division's ~17, at a quarter of its latency;
// tested bit for bit against a / b for every grid spacing in use.
__device__ __forceinline__ double div_rn(double a, double b, double y) {
  const double q = a * y;
  const double r = fma(-q, b, a);
  const double q1 = copysign(fma(r, y, q), a);
  return isinf(q) ? q : q1;
}

// FP64 min / max written as a compare and a select.  min_sel(x, y) = fmin(x, y) and
// max_sel(x, y) = fmax(x, y) bit for bit, NaN operands included (a NaN
// operand yields the other one), except for zeros of opposite sign, where
// these return x:
//   min_sel(+0, -0) = +0 (fmin: -0),  max_sel(-0, +0) = -0 (fmax: +0).
// Every use below has a nonzero x, or x = +0 in max_sel, or a result whose
// zero sign a later max_sel(+0, .) removes, so each gives CUDA's result.
__device__ __forceinline__ double min_sel(double x, double y) { return (y < x || x != x) ? y : x; }
__device__ __forceinline__ double max_sel(double x, double y) { return (y > x || x != x) ? y : x; }

__device__ __forceinline__ void fct_nu_mu(double eps, double& nu, double& mu) {
  double scrh = min_sel(1.0 / 6.0, fabs(eps));
  scrh = (1.0 / 3.0) * scrh * scrh;
  nu = (1.0 / 6.0) + (1.0 / 3.0) * (eps * eps - scrh * scrh);
  mu = 0.25 - 0.5 * nu;
}

// Periodic / clamped index maps of the shear axis (ymgpu2d/YM_FCT.cu:7-18 pad,
// FCT_Sweeps.cu:68-81 clamped halo loads).
__device__ __forceinline__ int xmap(int x, int nx, int periodic) {
  if (periodic) {
    x %= nx;
    return x < 0 ? x + nx : x;
  }
  return x < 0 ? 0 : (x >= nx ? nx - 1 : x);
}
__device__ __forceinline__ int zclamp(int z, int nz) { return z < 0 ? 0 : (z >= nz ? nz - 1 : z); }
__device__ __forceinline__ int zwrap(int z, int nz) {
  z %= nz;
  return z < 0 ? z + nz : z;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace ymkh

namespace ymkh {

// Up to 24 array pointers passed by value to the column kernels.
struct ArrayList {
  double* p[24];
};

// Arguments of the initial-state kernel (ymgpu2d/YM_Init.cu:32-40).
struct InitArgs {
  int nx, nz;
  double dx, dz;
  int k_mode;
  double perturb_amp, V0, epsilon;
  int run_mode;
  double alpha_YM;
  int init_by1_eq;
  double vz_edge_taper;
  const double* by;
  const double* ex;
  const double* ez;
  const double* az;
  const double* qA;
  const double* qB;
};

// Launchers (one per kernel family).  prepare_* set function attributes
// outside any stream capture.
cudaError_t prepare_fct(int tb);
int fct_ctas_per_sm(int tb);
cudaError_t prepare_maxwell();
int maxwell_ctas_per_sm();
cudaError_t launch_sponge_xicut(const ArrayList& a12, const StepParams& p, int cut, cudaStream_t s);
cudaError_t prepare_column(int nz);
// The z-mean of arrs[0, nmean) removed and arrs[nmean, nmean + nzero) zeroed, in one launch.
cudaError_t launch_zmean(const ArrayList& arrs, int nmean, int nzero, int nx, int nz, cudaStream_t s);
cudaError_t launch_hyperdiff(const ArrayList& a12, int nx, int nz, double mu, cudaStream_t s);
cudaError_t launch_band(const ArrayList& arrs, int narr, const double* W, int ldw, int J, double* C, int nx, int nz,
                        double inv2, cudaStream_t s);
cudaError_t launch_twiddles(double* W, int nz, int lo, int hi, int ldw, cudaStream_t s);
cudaError_t launch_twiddles_f32(float* c, float* sn, int nz, int lo, int hi, cudaStream_t s);
cudaError_t launch_energy(const State& st, size_t N, double* part, double* out, cudaStream_t s);
int energy_nparts(size_t N);
cudaError_t launch_mode_amp(const double* re, const double* im, int nx, int nz, int k, double* colbuf,
                            const double* weight, double* out, cudaStream_t s);
// State snapshots written by host threads (ymkh_snapshot.cu).
class SnapshotQueue;
SnapshotQueue* snapshot_queue_create(int device);
void snapshot_queue_destroy(SnapshotQueue* q);
int snapshot_submit(SnapshotQueue* q, const State& st, int nx, int nz, double dx, double dz, const char* path,
                    int format, cudaStream_t s, std::string& err);
int snapshot_wait(SnapshotQueue* q, std::string& err);
// Non-Abelian Gauss law residual sums (ymkh_diag.cu); part holds
// gauss_nparts(N) * YMKH_GAUSS_NOUT * 2 doubles, out YMKH_GAUSS_NOUT.
int gauss_nparts(size_t N);
cudaError_t launch_gauss(const State& st, int nx, int nz, double dx, double dz, double alpha, double* part,
                         double* out, cudaStream_t s);
cudaError_t launch_init(const State& st, const InitArgs& a, cudaStream_t s);
// 3-pass TF32 band filter on the tensor cores (ymkh_tf32.cu).  Per band:
// the twiddle matrix as TF32 hi/lo tile images for both contractions;
// shared scratch: the G and C^T tile images of the filtered arrays.
struct Tf32BandImages {
  float *a1h, *a1l;  // rows j, k = z: [Jp/128][Zp/32] tiles (Zp = NZ padded to 128)
  float *a2h, *a2l;  // rows z, k = j: [Zp/128][Jp/32] tiles
  int J, Jp;
};
struct Tf32Scratch {
  float *gh, *gl;    // [narr][NT][Zp/32] tiles
  float *ch, *cl;    // [narr][NT][Jp/32] tiles
};
int tf32_ntiles(int nx);
int tf32_jpad(int J);
int tf32_zpad(int nz);
size_t tf32_tile_floats();
cudaError_t prepare_tf32();
cudaError_t launch_tf32_w_images(const double* W, int ldw, int J, int nz, const Tf32BandImages& b, cudaStream_t s);
cudaError_t launch_band_tf32(const ArrayList& arrs, int narr, const Tf32BandImages& b, const Tf32Scratch& w, int nx,
                             int nz, float inv2, unsigned* err, cudaStream_t s);
int capi_error(int code, const char* msg);
void capi_count_launches(int n);

}  // namespace ymkh

namespace ymkh {

// ---- TMA bulk copies (cp.async.bulk, global -> shared, mbarrier completion)

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// Spin on the phase with a bounded number of polls; on timeout the error
// word is set and the caller carries on (the host reports it), so a lost
// completion can never hang the GPU.
__device__ __forceinline__ void mbar_wait(uint64_t* bar, unsigned phase, unsigned* err) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (long it = 0; it < (1L << 26); ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return;
  }
  if (err) atomicOr(err, ERR_WAIT);
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}
// count doubles of a periodic row starting at shear index xs (which may be
// negative or past the end), split at the wrap.  Requires nx even, xs even,
// count even and count <= nx so every piece is 16-byte aligned and sized.
__device__ __forceinline__ void bulk_row_periodic(double* dst, const double* row, int xs, int count, int nx,
                                                  uint64_t* bar) {
  int x = xs % nx;
  if (x < 0) x += nx;
  int done = 0;
  while (done < count) {
    const int len = min(count - done, nx - x);
    bulk_g2s(dst + done, row + x, (unsigned)len * 8u, bar);
    done += len;
    x = 0;
  }
}

}  // namespace ymkh

namespace ymkh {

// How a fused kernel stages its rows (RunDesc::fct_bulk / mx_bulk).
// Measured at 4096 x 8192 (FCT / Maxwell per step): TMA bulk rows issued
// by warp 0 alone 9.0 / 4.5 ms, 16-byte cp.async by every thread 7.8 / 4.1
// ms, bulk rows spread one per thread over all warps 7.3 / 3.9 ms (the form
// kept).
enum RowLoad : int {
  LOAD_ELEM = 0,    // per-element 8-byte cp.async through an x index table (walls, odd nx)
  LOAD_BULK_ALL = 3 // TMA bulk row copies, one per thread spread over all warps
};

// One run of a batch as the fused kernels see it: its start-of-step and
// next-step buffers, its step parameters and its (strip, segment) schedules.
// Items of run i occupy [item0, item0 + nstrips * nsegments) of the batch's
// flattened work lists.
struct RunDesc {
  State in;
  State out;
  State xsw;  // x-swept fluid scratch of the split FCT form (fluid arrays only)
  StepParams p;
  int fct_nstrips, fct_seg, fct_item0, fct_bulk;
  int mx_nstrips, mx_seg, mx_item0, mx_bulk;
  int fx_nstrips, fx_item0;           // split FCT, x pass: items (strip, row, beam)
  int fz_ncols, fz_seg, fz_item0;     // split FCT, z pass: items (column block, segment)
  int pad_;
};

struct RunTable {
  const RunDesc* runs;  // device array, item0 ascending
  int nruns;
  int fct_items, mx_items;
  unsigned* err;  // device error word of the bounded in-kernel waits
  int fx_items, fz_items;
  int fct_contig;  // fused FCT: 1 = contiguous item blocks per CTA (lone run), 0 = round-robin (batches)
};

// Run owning item g of the split FCT's x pass (which = 0) or z pass (1).
__device__ __forceinline__ int find_run_split(const RunDesc* runs, int nruns, int g, int which) {
  int lo = 0, hi = nruns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int i0 = which ? runs[mid].fz_item0 : runs[mid].fx_item0;
    if (i0 <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Index of the run owning flattened item g (binary search on item0).
__device__ __forceinline__ int find_run(const RunDesc* runs, int nruns, int g, bool maxwell) {
  int lo = 0, hi = nruns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int i0 = maxwell ? runs[mid].mx_item0 : runs[mid].fct_item0;
    if (i0 <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Cooperative copy of a run descriptor into shared memory (8-byte words).
__device__ __forceinline__ void load_desc(RunDesc* dst, const RunDesc* src) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(RunDesc) / 8); i += blockDim.x) d[i] = s[i];
}

cudaError_t launch_fct_table(const RunTable& T, int tb, int grid_ctas, cudaStream_t s);
cudaError_t launch_maxwell_table(const RunTable& T, int grid_ctas, cudaStream_t s);
int fct_nstrips(int nx, int tb);
int maxwell_nstrips(int nx);
int fct_bulk_ok(const StepParams& p, int tb);
int maxwell_bulk_ok(const StepParams& p);
cudaError_t launch_fct_split_table(const RunTable& T, int grid_x, int grid_z, cudaStream_t s);
int fct_split_ctas_per_sm(int which);
cudaError_t prepare_fct_split();
int fctx_nstrips(int nx);
int fctz_ncols(int nx);

}  // namespace ymkh
