// ymkh_capi.cu — the extern "C" boundary of include/ymkh.h: context
// lifetime, state binding, the step sequence and the diagnostics.
//
// The step keeps the reference's stage order (ymgpu2d/main_ym.cu:324-455):
//   FCT x+z sweeps of both beams, density floor   -> fct_fused_kernel
//   currents, Ampère, potential, Faraday          -> maxwell_fused_kernel
//   sponge, xi_cut                                -> sponge_xicut_kernel
//   z-mean removal and colour-1 EM zeroing        -> zmean_p2_kernel / zmean_kernel
//   DFT kz bands on the 21 filtered arrays        -> band_coef / band_apply
//   z-hyperdiffusion                              -> hyperdiff_kernel
// The sources of stage 7 are recomputed inside the next FCT launch.
//
// The stencil kernels read start-of-step values of neighbouring tiles, so
// the state alternates between two 24-array buffers: buffer 0 is the state
// the caller binds; buffer 1 is either a second caller-bound set
// (ymkh_bind_state2, zero copy) or allocated here once.  With a library
// buffer, ymkh_step copies back when it ends on buffer 1, so the caller's
// arrays always hold the current state after the call.

#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <atomic>
#include <vector>
#include <algorithm>
#include "ymkh_common.cuh"

#include <nvtx3/nvToolsExt.h>


using namespace ymkh;

namespace {

thread_local int t_err_code = 0;
thread_local char t_err_msg[512] = "";
std::atomic<long long> g_launches{0};

int set_err(int code, const char* fmt, ...) {
  t_err_code = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err_msg, sizeof t_err_msg, fmt, ap);
  va_end(ap);
  return code;
}

// NVTX range for the host timeline of a profiler (header-only NVTX 3: a
// no-op unless a tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

#define CK(call, what)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return set_err(YMKH_ECUDA, "%s: %s", what, cudaGetErrorString(e_)); \
  } while (0)

constexpr int MAX_BANDS = 2 + YMKH_MAX_EXTRA_BANDS;

}  // namespace

struct ymkh_ctx {
  int device = 0;
  int nx = 0, nz = 0;
  size_t N = 0;
  ymkh_params prm{};
  StepParams sp{};
  State buf[2]{};
  bool bound = false;
  bool dual = false;         // second buffer bound by the caller
  double* own = nullptr;     // library second buffer (24*N doubles)
  int cur = 0;
  int nb = 0, lo[MAX_BANDS]{}, hi[MAX_BANDS]{}, J[MAX_BANDS]{};
  double* W[MAX_BANDS]{};
  double* coef = nullptr;    // band coefficients [21][J][nx]
  Tf32BandImages tfb[MAX_BANDS]{};  // TF32 engine: twiddle tile images per band
  Tf32Scratch tfs{};                // TF32 engine: G and C^T tile images
  double* epart = nullptr;   // energy partials
  double* edev = nullptr;    // [0] energy, [1..2] mode amplitudes
  double* mcol = nullptr;    // mode amplitude per-column buffer
  double* mweight = nullptr; // x weights of ymkh_circ_amp (NX doubles, allocated on first use)
  double* gpart = nullptr;   // Gauss residual partials and results (allocated on first use)
  SnapshotQueue* snaps = nullptr;  // snapshot writers (created on first use)
  int fct_tx = 64, fct_seg = 16, fct_grid = 296;  // FCT threads per beam, segment rows, persistent CTAs
  int mx_seg = 16, mx_grid = 148;                   // Maxwell segment rows, persistent CTAs
  int sms = 148;
  bool aligned16 = false;   // every bound array 16-byte aligned: TMA bulk row copies allowed
  unsigned* derr = nullptr; // device error word of the bounded in-kernel waits
  RunDesc* ddesc = nullptr; // device run descriptors for start buffer 0 and 1
  RunDesc hdesc[2]{};       // their host copy, uploaded in stream order by the next step call
  int fct_items = 0, mx_items = 0, fx_items = 0, fz_items = 0;
  bool desc_ok = false;
  bool desc_pending = false; // hdesc not yet uploaded to ddesc
  int fct_mode = YMKH_FCT_FUSED;  // YMKH_FCT_FUSED or YMKH_FCT_SPLIT
  double* xscratch = nullptr;     // 12 x-swept fluid arrays of the split form
  int fz_seg = 128;
  int fx_grid = 0, fz_grid = 0;
  // CUDA graphs of `graph_steps` steps, one per starting buffer
  int graph_steps = 4;
  cudaGraphExec_t gexec[2]{nullptr, nullptr};
  cudaStream_t gstream[2]{nullptr, nullptr};
  long long glaunches[2]{0, 0};  // kernels per captured graph
  // optional per-stage event timing (ymkh_stage_times)
  cudaEvent_t ev[16]{};
  int nev = 0;
  bool timing = false;
};

namespace {

void fill_step_params(ymkh_ctx* c) {
  const ymkh_params& p = c->prm;
  StepParams& s = c->sp;
  s.nx = c->nx; s.nz = c->nz;
  s.dx = p.dx; s.dz = p.dz; s.dt = p.dt_step;
  s.rdx = 1.0 / p.dx; s.rdz = 1.0 / p.dz;  // IEEE division: correctly rounded
  s.c2 = p.c * p.c; s.eps0 = p.eps_0; s.alpha = p.alpha_YM;
  s.freeze_az1 = p.freeze_az1; s.periodic_x = p.periodic_x;
  s.epsilon = p.epsilon; s.xi_sponge = p.xi_sponge; s.sigma_sponge = p.sigma_sponge;
  s.xi_cut = p.xi_cut; s.warm_T = p.warm_T; s.suppress_kz0 = p.suppress_kz0;
  s.hyp_diff = p.hyp_diff_coeff;
}

int band_list(const ymkh_params& p, int* lo, int* hi) {
  int n = 0;
  if (p.kz_suppress_max >= 1) { lo[n] = 1; hi[n] = p.kz_suppress_max; ++n; }
  if (p.kz_suppress_hi > p.kz_suppress_max + 1) { lo[n] = p.kz_suppress_max + 2; hi[n] = p.kz_suppress_hi; ++n; }
  for (int i = 0; i < p.n_extra_bands && i < YMKH_MAX_EXTRA_BANDS; ++i) {
    lo[n] = p.extra_band_lo[i]; hi[n] = p.extra_band_hi[i]; ++n;
  }
  return n;
}

void drop_graphs(ymkh_ctx* c) {
  for (int k = 0; k < 2; ++k)
    if (c->gexec[k]) { cudaGraphExecDestroy(c->gexec[k]); c->gexec[k] = nullptr; c->gstream[k] = nullptr; }
}

void free_bands(ymkh_ctx* c) {
  for (int b = 0; b < MAX_BANDS; ++b) {
    if (c->W[b]) { cudaFree(c->W[b]); c->W[b] = nullptr; }
    for (float** q : {&c->tfb[b].a1h, &c->tfb[b].a1l, &c->tfb[b].a2h, &c->tfb[b].a2l})
      if (*q) { cudaFree(*q); *q = nullptr; }
  }
  for (float** q : {&c->tfs.gh, &c->tfs.gl, &c->tfs.ch, &c->tfs.cl})
    if (*q) { cudaFree(*q); *q = nullptr; }
  if (c->coef) { cudaFree(c->coef); c->coef = nullptr; }
  c->nb = 0;
}

// TF32 engine set-up: twiddle tile images per band and the shared scratch.
int setup_tf32(ymkh_ctx* c) {
  CK(prepare_tf32(), "TF32 GEMM shared-memory attribute");
  const size_t zp = (size_t)tf32_zpad(c->nz);
  const size_t tf = tf32_tile_floats();
  const size_t nt = (size_t)tf32_ntiles(c->nx);
  int maxJp = 0;
  for (int b = 0; b < c->nb; ++b) {
    Tf32BandImages& t = c->tfb[b];
    t.J = c->J[b];
    t.Jp = tf32_jpad(c->J[b]);
    maxJp = std::max(maxJp, t.Jp);
    const size_t n = (size_t)t.Jp * zp;  // floats per image
    for (float** q : {&t.a1h, &t.a1l, &t.a2h, &t.a2l}) CK(cudaMalloc(q, n * sizeof(float)), "cudaMalloc TF32 twiddle images");
    CK(launch_tf32_w_images(c->W[b], c->J[b], c->J[b], c->nz, t, 0), "TF32 twiddle images");
    g_launches++;
  }
  const size_t ng = 21 * nt * (zp / 32) * tf, nc = 21 * nt * (size_t)(maxJp / 32) * tf;
  CK(cudaMalloc(&c->tfs.gh, ng * sizeof(float)), "cudaMalloc TF32 G images");
  CK(cudaMalloc(&c->tfs.gl, ng * sizeof(float)), "cudaMalloc TF32 G images");
  CK(cudaMalloc(&c->tfs.ch, nc * sizeof(float)), "cudaMalloc TF32 coefficient images");
  CK(cudaMalloc(&c->tfs.cl, nc * sizeof(float)), "cudaMalloc TF32 coefficient images");
  return 0;
}

int setup_params(ymkh_ctx* c, const ymkh_params* p) {
  if (p->dt_step <= 0 || p->dx <= 0 || p->dz <= 0) return set_err(YMKH_EINVAL, "dx, dz, dt_step must be > 0");
  if (p->filter_engine != YMKH_FILTER_DFT && p->filter_engine != YMKH_FILTER_TF32X3)
    return set_err(YMKH_EINVAL, "unknown filter_engine %d", p->filter_engine);
  if (p->suppress_kz0 && (c->nz & (c->nz - 1)) != 0)
    return set_err(YMKH_EINVAL, "suppress_kz0 requires NZ a power of 2 (got %d)", c->nz);
  if (p->n_extra_bands < 0 || p->n_extra_bands > YMKH_MAX_EXTRA_BANDS)
    return set_err(YMKH_EINVAL, "n_extra_bands out of range");
  int lo[MAX_BANDS], hi[MAX_BANDS];
  const int nb = band_list(*p, lo, hi);
  for (int b = 0; b < nb; ++b)
    if (lo[b] < 0 || hi[b] < lo[b] || hi[b] > 1 << 20) return set_err(YMKH_EINVAL, "bad band [%d, %d]", lo[b], hi[b]);
  drop_graphs(c);
  free_bands(c);
  c->prm = *p;
  fill_step_params(c);
  size_t maxJ = 0;
  for (int b = 0; b < nb; ++b) {
    c->lo[b] = lo[b]; c->hi[b] = hi[b]; c->J[b] = 2 * (hi[b] - lo[b] + 1);
    CK(cudaMalloc(&c->W[b], (size_t)c->nz * c->J[b] * sizeof(double)), "cudaMalloc twiddles");
    CK(launch_twiddles(c->W[b], c->nz, lo[b], hi[b], c->J[b], 0), "twiddle kernel");
    g_launches++;
    maxJ = std::max(maxJ, (size_t)c->J[b]);
  }
  c->nb = nb;
  if (nb && p->filter_engine == YMKH_FILTER_TF32X3) {
    int rc = setup_tf32(c);
    if (rc) return rc;
  } else if (nb) {
    CK(cudaMalloc(&c->coef, 21 * maxJ * (size_t)c->nx * sizeof(double)), "cudaMalloc band coefficients");
  }
  // the twiddle tables and images are built on the legacy default stream:
  // wait for that stream only, not for other streams' work in flight (a
  // server creates runs while others step)
  CK(cudaStreamSynchronize(0), "twiddle setup");
  return 0;
}

// Segment length for persistent CTAs taking (strip, segment) items
// round-robin: the smallest per-CTA item count whose last round is nearly
// full, with segments of at least 16 rows.
int pick_segment(int nz, int nstrips, int grid) {
  int best_seg = nz, best_cost = 1 << 30;
  for (int nseg = 1; nseg <= std::max(1, nz / 16); ++nseg) {
    const int seg = (nz + nseg - 1) / nseg;
    const int items = nstrips * ((nz + seg - 1) / seg);
    const int rounds = (items + grid - 1) / grid;
    // cost in rows per CTA, each item paying its 6-row start-up
    const int cost = rounds * (seg + 6);
    if (cost < best_cost) { best_cost = cost; best_seg = seg; }
  }
  return best_seg;
}

// One-row segments: a CTA's contiguous block then ends at any row, so the
// blocks differ by at most one row (at 1024 x 2048 on B200 the step took
// 0.523 ms against 0.529 ms with 16-row segments, 7.38 against 7.40 ms at
// 4096 x 8192).  Maxwell keeps round-robin segments: its contiguous form
// measured slower (7.49 ms).
constexpr int kFctSegment = 1;

void choose_launch_shape(ymkh_ctx* c) {
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  // 128-wide strips from NX = 1024 up: at 4096 x 8192 on B200 the step's FCT
  // + Maxwell take 6.97 + 2.80 ms against 7.31 + 3.09 ms with 64-wide strips
  c->fct_tx = c->nx >= 1024 ? 128 : (c->nx >= 128 ? 64 : 32);
  const int fct_per_sm = std::max(1, fct_ctas_per_sm(c->fct_tx));
  c->fct_grid = c->sms * fct_per_sm;
  // segments are the FCT's unit of load balance: each CTA runs a contiguous
  // block of them, a strip's part as one piece (ymkh_fct.cu)
  c->fct_seg = std::min(c->nz, kFctSegment);
  const int mx_per_sm = std::max(1, maxwell_ctas_per_sm());
  c->mx_grid = c->sms * mx_per_sm;
  c->mx_seg = pick_segment(c->nz, maxwell_nstrips(c->nx), c->mx_grid);
  c->fx_grid = c->sms * std::max(1, fct_split_ctas_per_sm(0)) * 4;
  c->fz_grid = c->sms * std::max(1, fct_split_ctas_per_sm(1)) * 4;
}

// Row staging of the fused kernels when every bound array is 16-byte aligned
// and x is periodic with nx even: TMA bulk row copies issued one per thread
// across all warps (RowLoad).
constexpr int kAlignedRowLoad = LOAD_BULK_ALL;

RunDesc make_desc(const ymkh_ctx* c, int start, int tb, int fct_item0, int mx_item0) {
  RunDesc d{};
  d.in = c->buf[start];
  d.out = c->buf[1 - start];
  d.p = c->sp;
  d.fct_nstrips = fct_nstrips(c->nx, tb);
  d.fct_seg = c->fct_seg;
  d.fct_item0 = fct_item0;
  d.fct_bulk = (c->aligned16 && fct_bulk_ok(c->sp, tb)) ? kAlignedRowLoad : (int)LOAD_ELEM;
  d.mx_nstrips = maxwell_nstrips(c->nx);
  d.mx_seg = c->mx_seg;
  d.mx_item0 = mx_item0;
  d.mx_bulk = (c->aligned16 && maxwell_bulk_ok(c->sp)) ? kAlignedRowLoad : (int)LOAD_ELEM;
  if (c->xscratch)
    for (int i = 0; i < 6; ++i) {
      d.xsw.a[i] = c->xscratch + (size_t)i * c->N;
      d.xsw.b[i] = c->xscratch + (size_t)(6 + i) * c->N;
    }
  d.fx_nstrips = fctx_nstrips(c->nx);
  d.fz_ncols = fctz_ncols(c->nx);
  d.fz_seg = std::min(c->nz, c->fz_seg);
  return d;
}

int items_fx(const RunDesc& d, int nz) { return d.fx_nstrips * nz * 2; }
int items_fz(const RunDesc& d, int nz) { return d.fz_ncols * ((nz + d.fz_seg - 1) / d.fz_seg); }

// The split FCT form needs a 12-array scratch for the x-swept fluid.
int ensure_xscratch(ymkh_ctx* c) {
  if (c->fct_mode != YMKH_FCT_SPLIT || c->xscratch) return 0;
  if (cudaMalloc(&c->xscratch, (size_t)12 * c->N * sizeof(double)) != cudaSuccess)
    return set_err(YMKH_ENOMEM, "cudaMalloc x-sweep scratch (%zu bytes)", (size_t)12 * c->N * sizeof(double));
  return 0;
}

int items_fct(const RunDesc& d, int nz) { return d.fct_nstrips * ((nz + d.fct_seg - 1) / d.fct_seg); }
int items_mx(const RunDesc& d, int nz) { return d.mx_nstrips * ((nz + d.mx_seg - 1) / d.mx_seg); }

// Device descriptors of this run for both start buffers (single-run tables).
int upload_desc(ymkh_ctx* c) {
  c->desc_ok = false;
  if (!c->bound) return 0;
  if (!c->ddesc) CK(cudaMalloc(&c->ddesc, 2 * sizeof(RunDesc)), "cudaMalloc run descriptors");
  { int rc = ensure_xscratch(c); if (rc) return rc; }
  RunDesc* h = c->hdesc;
  h[0] = make_desc(c, 0, c->fct_tx, 0, 0);
  h[1] = make_desc(c, 1, c->fct_tx, 0, 0);
  for (int i = 0; i < 2; ++i) h[i].fx_item0 = h[i].fz_item0 = 0;
  c->fct_items = items_fct(h[0], c->nz);
  c->mx_items = items_mx(h[0], c->nz);
  c->fx_items = items_fx(h[0], c->nz);
  c->fz_items = items_fz(h[0], c->nz);
  c->desc_pending = true;  // uploaded by the next step call, on its stream
  c->desc_ok = true;
  return 0;
}

// Table uploads are ordered on the stream of the step call that follows a
// change, after the steps already queued there, so a table is never
// rewritten under a kernel in flight on that stream.  Inside a stream
// capture (where a pageable copy cannot be captured) the copy is synchronous.
cudaError_t upload_table(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (s) cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone) return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
}

int flush_desc(ymkh_ctx* c, cudaStream_t s) {
  if (!c->desc_ok) { int rc = upload_desc(c); if (rc) return rc; }
  if (c->desc_pending) {
    CK(upload_table(c->ddesc, c->hdesc, sizeof c->hdesc, s), "upload run descriptors");
    c->desc_pending = false;
  }
  return 0;
}

// The list l without its first k arrays.
ArrayList drop_front(const ArrayList& l, int k) {
  ArrayList r{};
  for (int i = 0; i + k < 24; ++i) r.p[i] = l.p[i + k];
  return r;
}

ArrayList list21(const State& s) {
  ArrayList l{};
  double* v[21] = {s.f[BY1], s.f[EX1], s.f[EZ1], s.f[BY2], s.f[BY3], s.f[EX2], s.f[EX3],
                   s.f[EZ2], s.f[EZ3], s.f[AZ2], s.f[AZ3], s.a[FQ2], s.a[FQ3], s.b[FQ2],
                   s.b[FQ3], s.a[FPZ], s.b[FPZ], s.a[FPX], s.b[FPX], s.a[FN], s.b[FN]};
  for (int i = 0; i < 21; ++i) l.p[i] = v[i];
  return l;
}
ArrayList list12(const State& s) {
  ArrayList l{};
  double* v[12] = {s.f[BY2], s.f[BY3], s.f[EX2], s.f[EX3], s.f[EZ2], s.f[EZ3],
                   s.f[AZ2], s.f[AZ3], s.a[FQ2], s.a[FQ3], s.b[FQ2], s.b[FQ3]};
  for (int i = 0; i < 12; ++i) l.p[i] = v[i];
  return l;
}

// One reference iteration from buffer c->cur into buffer 1 - c->cur.
enum Stage { ST_FCT = 0, ST_MAXWELL, ST_POINTWISE, ST_ZMEAN, ST_BANDS, ST_HYPER, ST_ZERO, ST_COUNT };

void mark(ymkh_ctx* c, int stage, cudaStream_t s) {
  if (c->timing) cudaEventRecord(c->ev[stage], s);
}

// Stages after the fused FCT and Maxwell launches, on the run's new buffer.
int post_stages(ymkh_ctx* c, const State& out, cudaStream_t s) {
  mark(c, ST_POINTWISE, s);
  if (c->prm.xi_sponge > 0.0) { CK(launch_sponge_xicut(list12(out), c->sp, 0, s), "sponge"); g_launches++; }
  if (c->prm.xi_cut > 0.0) { CK(launch_sponge_xicut(list12(out), c->sp, 1, s), "xi_cut"); g_launches++; }
  // With suppress_kz0 the step ends by zeroing By1, Ex1 and Ez1, the first
  // three arrays of list21 (main_ym.cu:443-447).  The z-mean and the band
  // filters treat every array on its own and hyperdiffusion does not touch
  // colour 1, so the z-mean launch zeroes those three and the later stages
  // skip them: the state after the step is the same bit for bit.
  const int skip = c->prm.suppress_kz0 ? 3 : 0;
  const ArrayList l21 = list21(out);
  const ArrayList filt = drop_front(l21, skip);
  mark(c, ST_ZMEAN, s);
  if (c->prm.suppress_kz0) {
    ArrayList zl = filt;  // 12 arrays lose their z-mean, then By1, Ex1, Ez1 are zeroed
    for (int i = 0; i < 3; ++i) zl.p[12 + i] = l21.p[i];
    CK(launch_zmean(zl, 12, 3, c->nx, c->nz, s), "zmean");
    g_launches++;
  }
  mark(c, ST_BANDS, s);
  const double inv2 = (double)(2.0f / (float)c->nz);
  for (int b = 0; b < c->nb; ++b) {
    if (c->prm.filter_engine == YMKH_FILTER_TF32X3) {
      CK(launch_band_tf32(filt, 21 - skip, c->tfb[b], c->tfs, c->nx, c->nz, 2.0f / (float)c->nz, c->derr, s),
         "band filter (TF32 tensor cores)");
      g_launches += 3;
    } else {
      CK(launch_band(filt, 21 - skip, c->W[b], c->J[b], c->J[b], c->coef, c->nx, c->nz, inv2, s), "band filter");
      g_launches += 2;
    }
  }
  mark(c, ST_HYPER, s);
  if (c->prm.hyp_diff_coeff > 0.0) {
    CK(launch_hyperdiff(list12(out), c->nx, c->nz, c->prm.hyp_diff_coeff, s), "hyperdiffusion");
    g_launches++;
  }
  mark(c, ST_ZERO, s);  // colour-1 zeroing: done by the z-mean launch above
  mark(c, ST_COUNT, s);
  return 0;
}

// One reference iteration from buffer c->cur into buffer 1 - c->cur.
int step_once(ymkh_ctx* c, cudaStream_t s) {
  { int rc = flush_desc(c, s); if (rc) return rc; }
  RunTable T{c->ddesc + c->cur, 1, c->fct_items, c->mx_items, c->derr, c->fx_items, c->fz_items, 1};
  mark(c, ST_FCT, s);
  {
    NvtxRange r("ymkh fct");
    if (c->fct_mode == YMKH_FCT_SPLIT) {
      CK(launch_fct_split_table(T, c->fx_grid, c->fz_grid, s), "fct_x/fct_z kernels");
      g_launches++;
    } else {
      CK(launch_fct_table(T, c->fct_tx, c->fct_grid, s), "fct_fused_kernel");
    }
  }
  mark(c, ST_MAXWELL, s);
  {
    NvtxRange r("ymkh maxwell");
    CK(launch_maxwell_table(T, c->mx_grid, s), "maxwell_fused_kernel");
  }
  g_launches += 2;
  NvtxRange r("ymkh column stages");
  int rc = post_stages(c, c->buf[1 - c->cur], s);
  if (rc) return rc;
  c->cur = 1 - c->cur;
  return 0;
}

int copy_back(ymkh_ctx* c, cudaStream_t s) {
  const size_t bytes = c->N * sizeof(double);
  const State& a = c->buf[1];
  const State& b = c->buf[0];
  for (int i = 0; i < 12; ++i) CK(cudaMemcpyAsync(b.f[i], a.f[i], bytes, cudaMemcpyDeviceToDevice, s), "copy back");
  for (int i = 0; i < 6; ++i) {
    CK(cudaMemcpyAsync(b.a[i], a.a[i], bytes, cudaMemcpyDeviceToDevice, s), "copy back");
    CK(cudaMemcpyAsync(b.b[i], a.b[i], bytes, cudaMemcpyDeviceToDevice, s), "copy back");
  }
  c->cur = 0;
  return 0;
}

int run_graph(ymkh_ctx* c, cudaStream_t s) {
  const int start = c->cur;
  if (!c->gexec[start] || c->gstream[start] != s) {
    if (c->gexec[start]) { cudaGraphExecDestroy(c->gexec[start]); c->gexec[start] = nullptr; }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = 0;
    const long long l0 = g_launches.load();
    for (int k = 0; k < c->graph_steps && !rc; ++k) rc = step_once(c, s);
    c->glaunches[start] = g_launches.load() - l0;
    g_launches -= c->glaunches[start];  // counted when the graph runs
    cudaError_t ec = cudaStreamEndCapture(s, &g);
    c->cur = start;  // capture did not execute anything
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    CK(ec, "end capture");
    cudaError_t ei = cudaGraphInstantiate(&c->gexec[start], g, 0);
    cudaGraphDestroy(g);
    CK(ei, "graph instantiate");
    c->gstream[start] = s;
  }
  CK(cudaGraphLaunch(c->gexec[start], s), "graph launch");
  g_launches += c->glaunches[start];
  // graph_steps is even: the state ends in the buffer it started from
  return 0;
}

}  // namespace

extern "C" {

int ymkh_last_error(char* buf, size_t n) {
  if (buf && n) {
    strncpy(buf, t_err_msg, n - 1);
    buf[n - 1] = 0;
  }
  return t_err_code;
}

long long ymkh_launch_count(void) { return g_launches.load(); }

int ymkh_build_flags(void) { return YMKH_DEBUG ? YMKH_BUILD_DEBUG : 0; }

int ymkh_create(const ymkh_grid* grid, const ymkh_params* params, ymkh_ctx** out) {
  if (!grid || !params || !out) return set_err(YMKH_EINVAL, "null argument");
  if (grid->nx < 4 || grid->nz < 4) return set_err(YMKH_EINVAL, "grid too small (%d x %d)", grid->nx, grid->nz);
  if ((size_t)grid->nx * grid->nz > ((size_t)1 << 34)) return set_err(YMKH_EINVAL, "grid too large");
  ymkh_ctx* c = new ymkh_ctx();
  // failures after this point release the context and what it holds
#define CK_CREATE(call, what)                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      const int rc_ = set_err(YMKH_ECUDA, "%s: %s", what, cudaGetErrorString(e_));            \
      ymkh_destroy(c);                                                                        \
      return rc_;                                                                             \
    }                                                                                         \
  } while (0)
  CK_CREATE(cudaGetDevice(&c->device), "cudaGetDevice");
  c->nx = grid->nx; c->nz = grid->nz; c->N = (size_t)grid->nx * grid->nz;
  int rc = setup_params(c, params);
  if (rc) { free_bands(c); delete c; return rc; }
  CK_CREATE(prepare_fct(32), "FCT kernel attributes");
  CK_CREATE(prepare_fct(64), "FCT kernel attributes");
  CK_CREATE(prepare_fct(128), "FCT kernel attributes");
  CK_CREATE(prepare_maxwell(), "Maxwell kernel attributes");
  CK_CREATE(prepare_fct_split(), "split FCT kernel attributes");
  choose_launch_shape(c);
  CK_CREATE(prepare_column(c->nz), "column kernel attributes");
#undef CK_CREATE
  const int np = energy_nparts(c->N);
  if (cudaMalloc(&c->epart, (size_t)2 * np * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->edev, 4 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->mcol, (size_t)2 * c->nx * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->derr, sizeof(unsigned)) != cudaSuccess || cudaMemset(c->derr, 0, sizeof(unsigned)) != cudaSuccess) {
    ymkh_destroy(c);
    return set_err(YMKH_ENOMEM, "cudaMalloc diagnostics");
  }
  *out = c;
  return 0;
}

int ymkh_set_params(ymkh_ctx* c, const ymkh_params* p) {
  if (!c || !p) return set_err(YMKH_EINVAL, "null argument");
  int rc = setup_params(c, p);
  if (rc) return rc;
  return upload_desc(c);
}

static State make_state(double* const f[12], double* const a[6], double* const b[6]) {
  State s{};
  for (int i = 0; i < 12; ++i) s.f[i] = f[i];
  for (int i = 0; i < 6; ++i) { s.a[i] = a[i]; s.b[i] = b[i]; }
  return s;
}

static bool aligned16(const State& s) {
  for (int i = 0; i < 12; ++i) if (reinterpret_cast<uintptr_t>(s.f[i]) % 16) return false;
  for (int i = 0; i < 6; ++i)
    if (reinterpret_cast<uintptr_t>(s.a[i]) % 16 || reinterpret_cast<uintptr_t>(s.b[i]) % 16) return false;
  return true;
}

static bool state_ok(const State& s) {
  for (int i = 0; i < 12; ++i) if (!s.f[i]) return false;
  for (int i = 0; i < 6; ++i) if (!s.a[i] || !s.b[i]) return false;
  return true;
}

int ymkh_bind_state(ymkh_ctx* c, double* const fields[YMKH_NFIELDS], double* const fluidA[YMKH_NFLUID],
                    double* const fluidB[YMKH_NFLUID]) {
  if (!c || !fields || !fluidA || !fluidB) return set_err(YMKH_EINVAL, "null argument");
  State s = make_state(fields, fluidA, fluidB);
  if (!state_ok(s)) return set_err(YMKH_EINVAL, "null state array");
  drop_graphs(c);
  c->buf[0] = s;
  if (!c->own) {
    if (cudaMalloc(&c->own, 24 * c->N * sizeof(double)) != cudaSuccess)
      return set_err(YMKH_ENOMEM, "cudaMalloc second state buffer (%zu bytes)", 24 * c->N * sizeof(double));
  }
  for (int i = 0; i < 12; ++i) c->buf[1].f[i] = c->own + (size_t)i * c->N;
  for (int i = 0; i < 6; ++i) {
    c->buf[1].a[i] = c->own + (size_t)(12 + i) * c->N;
    c->buf[1].b[i] = c->own + (size_t)(18 + i) * c->N;
  }
  c->dual = false;
  c->cur = 0;
  c->bound = true;
  c->aligned16 = aligned16(c->buf[0]) && aligned16(c->buf[1]);
  return upload_desc(c);
}

// Zero-copy form: the caller provides both buffers; after ymkh_step the
// current state is in buffer ymkh_current_buffer().
int ymkh_bind_state2(ymkh_ctx* c, double* const* state0, double* const* state1) {
  if (!c || !state0 || !state1) return set_err(YMKH_EINVAL, "null argument");
  State s0 = make_state(state0, state0 + 12, state0 + 18);
  State s1 = make_state(state1, state1 + 12, state1 + 18);
  if (!state_ok(s0) || !state_ok(s1)) return set_err(YMKH_EINVAL, "null state array");
  drop_graphs(c);
  if (c->own) { cudaFree(c->own); c->own = nullptr; }
  c->buf[0] = s0;
  c->buf[1] = s1;
  c->dual = true;
  c->cur = 0;
  c->bound = true;
  c->aligned16 = aligned16(s0) && aligned16(s1);
  return upload_desc(c);
}

// Reads (and clears) the device error word set by in-kernel waits that ran
// out of polls; synchronises the stream.
int ymkh_check(ymkh_ctx* c, void* stream) {
  if (!c) return set_err(YMKH_EINVAL, "null context");
  unsigned h = 0;
  CK(cudaMemcpyAsync(&h, c->derr, sizeof h, cudaMemcpyDeviceToHost, (cudaStream_t)stream), "error word D2H");
  CK(cudaStreamSynchronize((cudaStream_t)stream), "error word sync");
  if (h) {
    cudaMemsetAsync(c->derr, 0, sizeof(unsigned), (cudaStream_t)stream);
    return set_err(YMKH_ECUDA, "%s (error word %u); results of that step are invalid",
                   (h & ERR_BOUNDS) ? "a checked access was out of range and skipped" : "a bounded in-kernel wait timed out",
                   h);
  }
  return 0;
}

int ymkh_current_buffer(ymkh_ctx* c) { return c ? c->cur : -1; }

int ymkh_set_current_buffer(ymkh_ctx* c, int which) {
  if (!c || (which != 0 && which != 1)) return set_err(YMKH_EINVAL, "bad buffer index");
  if (!c->dual && which == 1) return set_err(YMKH_ESTATE, "buffer 1 is library-owned");
  c->cur = which;
  return 0;
}

int ymkh_init(ymkh_ctx* c, const ymkh_init_params* ip, void* stream) {
  if (!c || !ip) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  cudaStream_t s = (cudaStream_t)stream;
  InitArgs a{};
  a.nx = c->nx; a.nz = c->nz; a.dx = c->prm.dx; a.dz = c->prm.dz;
  a.k_mode = ip->k_mode; a.perturb_amp = ip->perturb_amp; a.V0 = ip->V0; a.epsilon = ip->epsilon;
  a.run_mode = ip->run_mode; a.alpha_YM = (double)(float)ip->alpha_YM;
  a.init_by1_eq = ip->init_by1_eq; a.vz_edge_taper = ip->vz_edge_taper;
  const double* hs[6] = {ip->seed_by, ip->seed_ex, ip->seed_ez, ip->seed_az, ip->seed_qA, ip->seed_qB};
  const double** ds[6] = {&a.by, &a.ex, &a.ez, &a.az, &a.qA, &a.qB};
  double* seedbuf = nullptr;
  int nseed = 0;
  for (int k = 0; k < 6; ++k) if (hs[k]) ++nseed;
  if (nseed) {
    CK(cudaMalloc(&seedbuf, (size_t)6 * c->nx * sizeof(double)), "cudaMalloc seed");
    for (int k = 0; k < 6; ++k) {
      if (!hs[k]) continue;
      double* d = seedbuf + (size_t)k * c->nx;
      CK(cudaMemcpyAsync(d, hs[k], c->nx * sizeof(double), cudaMemcpyHostToDevice, s), "seed upload");
      *ds[k] = d;
    }
  }
  c->cur = 0;
  cudaError_t e = launch_init(c->buf[0], a, s);
  g_launches++;
  if (seedbuf) {
    cudaStreamSynchronize(s);
    cudaFree(seedbuf);
  }
  CK(e, "init kernel");
  return 0;
}

int ymkh_step(ymkh_ctx* c, int nsteps, void* stream) {
  if (!c) return set_err(YMKH_EINVAL, "null context");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  if (nsteps < 0) return set_err(YMKH_EINVAL, "negative step count");
  NvtxRange range("ymkh_step");
  cudaStream_t s = (cudaStream_t)stream;
  { int rc = flush_desc(c, s); if (rc) return rc; }  // before any capture of the steps
  int done = 0;
  const bool graphs = s != nullptr && c->graph_steps >= 2 && (c->graph_steps % 2) == 0;
  if (graphs) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (cs == cudaStreamCaptureStatusNone) {
      while (nsteps - done >= c->graph_steps) {
        int rc = run_graph(c, s);
        if (rc) return rc;
        done += c->graph_steps;
      }
    }
  }
  for (; done < nsteps; ++done) {
    int rc = step_once(c, s);
    if (rc) return rc;
  }
  if (!c->dual && c->cur == 1) return copy_back(c, s);
  return 0;
}

int ymkh_set_graph_steps(ymkh_ctx* c, int n) {
  if (!c || n < 0 || (n % 2) != 0) return set_err(YMKH_EINVAL, "graph step count must be even and >= 0");
  drop_graphs(c);
  c->graph_steps = n;
  return 0;
}

int ymkh_set_fct_shape(ymkh_ctx* c, int tx, int seg) {
  if (!c || (tx != 32 && tx != 64 && tx != 128) || seg < 1) return set_err(YMKH_EINVAL, "bad FCT launch shape");
  drop_graphs(c);
  c->fct_tx = tx;
  c->fct_seg = seg;
  c->fct_grid = c->sms * std::max(1, fct_ctas_per_sm(tx));
  return upload_desc(c);
}

int ymkh_set_fct_mode(ymkh_ctx* c, int mode) {
  if (!c || (mode != YMKH_FCT_FUSED && mode != YMKH_FCT_SPLIT)) return set_err(YMKH_EINVAL, "bad FCT mode");
  drop_graphs(c);
  c->fct_mode = mode;
  return upload_desc(c);
}

int ymkh_get_fct_shape(ymkh_ctx* c, int* tx, int* seg) {
  if (!c) return set_err(YMKH_EINVAL, "null context");
  if (tx) *tx = c->fct_tx;
  if (seg) *seg = c->fct_seg;
  return 0;
}

// Runs nsteps plain (uncaptured) steps with an event between stages and
// accumulates the device time of each stage into out_ms[0..ST_COUNT).
int ymkh_stage_times(ymkh_ctx* c, int nsteps, void* stream, float* out_ms, int nout) {
  if (!c || !out_ms || nout < ST_COUNT) return set_err(YMKH_EINVAL, "bad arguments");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i <= ST_COUNT; ++i) CK(cudaEventCreate(&c->ev[i]), "cudaEventCreate");
  for (int i = 0; i < ST_COUNT; ++i) out_ms[i] = 0.f;
  c->timing = true;
  int rc = 0;
  for (int k = 0; k < nsteps && !rc; ++k) {
    rc = step_once(c, s);
    if (rc) break;
    cudaError_t e = cudaEventSynchronize(c->ev[ST_COUNT]);
    if (e != cudaSuccess) { rc = set_err(YMKH_ECUDA, "stage timing: %s", cudaGetErrorString(e)); break; }
    for (int i = 0; i < ST_COUNT; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]);
      out_ms[i] += ms;
    }
  }
  c->timing = false;
  for (int i = 0; i <= ST_COUNT; ++i) cudaEventDestroy(c->ev[i]);
  if (!rc && !c->dual && c->cur == 1) rc = copy_back(c, s);
  return rc;
}

int ymkh_energy_async(ymkh_ctx* c, double* dev_out, void* stream) {
  if (!c || !dev_out) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  CK(launch_energy(c->buf[c->cur], c->N, c->epart, dev_out, (cudaStream_t)stream), "energy kernels");
  g_launches += 2;
  return 0;
}

int ymkh_energy(ymkh_ctx* c, double* host_out, void* stream) {
  if (!host_out) return set_err(YMKH_EINVAL, "null argument");
  int rc = ymkh_energy_async(c, c ? c->edev : nullptr, stream);
  if (rc) return rc;
  CK(cudaMemcpyAsync(host_out, c->edev, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream), "energy D2H");
  return ymkh_check(c, stream);
}

int ymkh_mode_amp(ymkh_ctx* c, int k, double* host_out2, void* stream) {
  return ymkh_circ_amp(c, YMKH_PAIR_AZ, k, nullptr, host_out2, stream);
}

int ymkh_circ_amp(ymkh_ctx* c, int pair, int k, const double* host_weight, double* host_out2, void* stream) {
  if (!c || !host_out2) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  static const int re_of[4] = {AZ2, BY2, EX2, EZ2};
  if (pair < 0 || pair > 3) return set_err(YMKH_EINVAL, "pair %d not in 0..3", pair);
  cudaStream_t s = (cudaStream_t)stream;
  const State& st = c->buf[c->cur];
  const double* w = nullptr;
  if (host_weight) {
    if (!c->mweight && cudaMalloc(&c->mweight, (size_t)c->nx * sizeof(double)) != cudaSuccess)
      return set_err(YMKH_ENOMEM, "cudaMalloc mode weights");
    CK(cudaMemcpyAsync(c->mweight, host_weight, (size_t)c->nx * sizeof(double), cudaMemcpyHostToDevice, s),
       "mode weights H2D");
    w = c->mweight;
  }
  CK(launch_mode_amp(st.f[re_of[pair]], st.f[re_of[pair] + 1], c->nx, c->nz, k, c->mcol, w, c->edev + 1, s),
     "mode amplitude kernels");
  g_launches += 2;
  CK(cudaMemcpyAsync(host_out2, c->edev + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, s), "mode amp D2H");
  CK(cudaStreamSynchronize(s), "mode amp sync");
  return 0;
}

int ymkh_gauss(ymkh_ctx* c, double* host_out, void* stream) {
  if (!c || !host_out) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  const int np = gauss_nparts(c->N);
  const size_t n = (size_t)np * YMKH_GAUSS_NOUT * 2 + YMKH_GAUSS_NOUT;
  if (!c->gpart && cudaMalloc(&c->gpart, n * sizeof(double)) != cudaSuccess)
    return set_err(YMKH_ENOMEM, "cudaMalloc Gauss partials");
  cudaStream_t s = (cudaStream_t)stream;
  double* dout = c->gpart + (size_t)np * YMKH_GAUSS_NOUT * 2;
  CK(launch_gauss(c->buf[c->cur], c->nx, c->nz, c->prm.dx, c->prm.dz, c->prm.alpha_YM, c->gpart, dout, s),
     "Gauss residual kernels");
  g_launches += 2;
  CK(cudaMemcpyAsync(host_out, dout, YMKH_GAUSS_NOUT * sizeof(double), cudaMemcpyDeviceToHost, s), "Gauss D2H");
  CK(cudaStreamSynchronize(s), "Gauss sync");
  return 0;
}

int ymkh_snapshot(ymkh_ctx* c, const char* path, int format, void* stream) {
  if (!c || !path) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "state not bound");
  if (format != YMKH_SNAP_CSV && format != YMKH_SNAP_FP64) return set_err(YMKH_EINVAL, "snapshot format %d", format);
  if (!c->snaps) c->snaps = snapshot_queue_create(c->device);
  std::string err;
  const int rc = snapshot_submit(c->snaps, c->buf[c->cur], c->nx, c->nz, c->prm.dx, c->prm.dz, path, format,
                                 (cudaStream_t)stream, err);
  return rc ? set_err(rc, "%s", err.c_str()) : 0;
}

int ymkh_snapshot_wait(ymkh_ctx* c) {
  if (!c) return set_err(YMKH_EINVAL, "null context");
  if (!c->snaps) return 0;
  std::string err;
  const int rc = snapshot_wait(c->snaps, err);
  return rc ? set_err(rc, "%s", err.c_str()) : 0;
}

int ymkh_destroy(ymkh_ctx* c) {
  if (!c) return 0;
  if (c->snaps) snapshot_queue_destroy(c->snaps);  // waits for its writers
  drop_graphs(c);
  free_bands(c);
  if (c->own) cudaFree(c->own);
  if (c->epart) cudaFree(c->epart);
  if (c->edev) cudaFree(c->edev);
  if (c->mcol) cudaFree(c->mcol);
  if (c->mweight) cudaFree(c->mweight);
  if (c->gpart) cudaFree(c->gpart);
  if (c->derr) cudaFree(c->derr);
  if (c->ddesc) cudaFree(c->ddesc);
  if (c->xscratch) cudaFree(c->xscratch);
  delete c;
  return 0;
}

int ymkh_twiddles(int nz, int m_lo, int m_hi, float* cos_out, float* sin_out) {
  if (nz < 1 || m_lo < 0 || m_hi < m_lo || !cos_out || !sin_out) return set_err(YMKH_EINVAL, "bad arguments");
  const size_t n = (size_t)(m_hi - m_lo + 1) * nz;
  float *dc = nullptr, *ds = nullptr;
  CK(cudaMalloc(&dc, n * sizeof(float)), "cudaMalloc");
  CK(cudaMalloc(&ds, n * sizeof(float)), "cudaMalloc");
  cudaError_t e = launch_twiddles_f32(dc, ds, nz, m_lo, m_hi, 0);
  g_launches++;
  if (e == cudaSuccess) e = cudaMemcpy(cos_out, dc, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(sin_out, ds, n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dc);
  cudaFree(ds);
  CK(e, "twiddle table");
  return 0;
}

// ------------------------------------------------------------------ batches
// Runs of any sizes advance together: one FCT and one Maxwell launch per step
// cover the (run, strip, segment) items of every member; the post-Maxwell
// stages are launched per member.  Steps can be captured as CUDA graphs.

struct ymkh_batch {
  std::vector<ymkh_ctx*> runs;
  RunDesc* ddesc = nullptr;  // [2][cap]: tables for the members' current / next buffers
  int cap = 0;
  int fct_items = 0, mx_items = 0, fx_items = 0, fz_items = 0;
  int tb = 64, fct_grid = 0, mx_grid = 0, fx_grid = 0, fz_grid = 0;
  int fct_mode = YMKH_FCT_FUSED;
  unsigned* derr = nullptr;
  bool dirty = true;
  int parity = 0;            // steps taken since the tables were built, mod 2
  int graph_steps = 4;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  long long glaunches = 0;
  // The members' column stages (z-mean, band filters, ...) are independent
  // run to run: they fork onto auxiliary streams after the fused launches
  // and join back before the next step (also inside a captured graph).
  static constexpr int kAux = 8;
  cudaStream_t aux[kAux]{};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[kAux]{};
};

namespace {

void batch_drop_graph(ymkh_batch* b) {
  if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; b->gstream = nullptr; }
}

int batch_build(ymkh_batch* b, cudaStream_t s) {
  const int n = (int)b->runs.size();
  if (n > b->cap) {
    if (b->ddesc) cudaFree(b->ddesc);
    b->cap = std::max(n, 2 * b->cap);
    CK(cudaMalloc(&b->ddesc, 2 * (size_t)b->cap * sizeof(RunDesc)), "cudaMalloc batch descriptors");
  }
  std::vector<RunDesc> h(2 * (size_t)std::max(n, 1));
  int f0 = 0, m0 = 0, x0 = 0, z0 = 0;
  for (int i = 0; i < n; ++i) {
    ymkh_ctx* c = b->runs[i];
    if (b->fct_mode == YMKH_FCT_SPLIT && !c->xscratch) {
      const int keep = c->fct_mode;
      c->fct_mode = YMKH_FCT_SPLIT;
      int rc = ensure_xscratch(c);
      c->fct_mode = keep;
      if (rc) return rc;
    }
    RunDesc d0 = make_desc(c, c->cur, b->tb, f0, m0);
    RunDesc d1 = make_desc(c, 1 - c->cur, b->tb, f0, m0);
    d0.fx_item0 = d1.fx_item0 = x0;
    d0.fz_item0 = d1.fz_item0 = z0;
    x0 += items_fx(d0, c->nz);
    z0 += items_fz(d0, c->nz);
    // batches take 128-row FCT segments round-robin (RunTable::fct_contig = 0)
    d0.fct_seg = d1.fct_seg = std::min(c->nz, 128);
    d0.mx_seg = d1.mx_seg = std::min(c->nz, 128);
    d0.fct_item0 = d1.fct_item0 = f0;
    d0.mx_item0 = d1.mx_item0 = m0;
    h[i] = d0;
    h[n + i] = d1;
    f0 += items_fct(d0, c->nz);
    m0 += items_mx(d0, c->nz);
  }
  b->fct_items = f0;
  b->mx_items = m0;
  b->fx_items = x0;
  b->fz_items = z0;
  if (n) {
    // in stream order after the steps already queued on s (a pageable
    // source is staged before the call returns)
    CK(upload_table(b->ddesc, h.data(), (size_t)n * sizeof(RunDesc), s), "upload batch table");
    CK(upload_table(b->ddesc + b->cap, h.data() + n, (size_t)n * sizeof(RunDesc), s), "upload batch table");
  }
  b->parity = 0;
  b->dirty = false;
  batch_drop_graph(b);
  return 0;
}

int batch_step_once(ymkh_batch* b, cudaStream_t s) {
  const int n = (int)b->runs.size();
  if (!n) return 0;
  RunTable T{b->ddesc + (size_t)b->parity * b->cap, n, b->fct_items, b->mx_items, b->derr, b->fx_items, b->fz_items, 0};
  if (b->fct_mode == YMKH_FCT_SPLIT)
    CK(launch_fct_split_table(T, b->fx_grid, b->fz_grid, s), "fct_x/fct_z kernels (batch)");
  else
    CK(launch_fct_table(T, b->tb, b->fct_grid, s), "fct_fused_kernel (batch)");
  CK(launch_maxwell_table(T, b->mx_grid, s), "maxwell_fused_kernel (batch)");
  g_launches += 2;
  const int na = b->aux[0] ? std::min(n, (int)ymkh_batch::kAux) : 1;
  if (na > 1) {
    CK(cudaEventRecord(b->fork_ev, s), "batch fork");
    for (int i = 0; i < na; ++i) CK(cudaStreamWaitEvent(b->aux[i], b->fork_ev, 0), "batch fork");
  }
  for (int j = 0; j < n; ++j) {
    ymkh_ctx* c = b->runs[j];
    int rc = post_stages(c, c->buf[1 - c->cur], na > 1 ? b->aux[j % na] : s);
    if (rc) return rc;
    c->cur = 1 - c->cur;
  }
  if (na > 1) {
    for (int i = 0; i < na; ++i) {
      CK(cudaEventRecord(b->join_ev[i], b->aux[i]), "batch join");
      CK(cudaStreamWaitEvent(s, b->join_ev[i], 0), "batch join");
    }
  }
  b->parity ^= 1;
  return 0;
}

}  // namespace

int ymkh_batch_create(ymkh_batch** out) {
  if (!out) return set_err(YMKH_EINVAL, "null argument");
  ymkh_batch* b = new ymkh_batch();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  for (int tb : {32, 64, 128}) prepare_fct(tb);
  prepare_maxwell();
  prepare_fct_split();
  b->fct_grid = sms * std::max(1, fct_ctas_per_sm(b->tb));
  b->mx_grid = sms * std::max(1, maxwell_ctas_per_sm());
  b->fx_grid = sms * std::max(1, fct_split_ctas_per_sm(0)) * 4;
  b->fz_grid = sms * std::max(1, fct_split_ctas_per_sm(1)) * 4;
  bool ok = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < ymkh_batch::kAux; ++i)
    ok = cudaStreamCreateWithFlags(&b->aux[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->join_ev[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok || cudaMalloc(&b->derr, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(b->derr, 0, sizeof(unsigned)) != cudaSuccess) {
    for (int i = 0; i < ymkh_batch::kAux; ++i) {
      if (b->aux[i]) cudaStreamDestroy(b->aux[i]);
      if (b->join_ev[i]) cudaEventDestroy(b->join_ev[i]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    delete b;
    return set_err(YMKH_ENOMEM, "batch streams, events or error word");
  }
  *out = b;
  return 0;
}

int ymkh_batch_add(ymkh_batch* b, ymkh_ctx* c) {
  if (!b || !c) return set_err(YMKH_EINVAL, "null argument");
  if (!c->bound) return set_err(YMKH_ESTATE, "run state not bound");
  for (ymkh_ctx* r : b->runs) if (r == c) return set_err(YMKH_EINVAL, "run already in the batch");
  b->runs.push_back(c);
  b->dirty = true;
  return 0;
}

int ymkh_batch_remove(ymkh_batch* b, ymkh_ctx* c) {
  if (!b || !c) return set_err(YMKH_EINVAL, "null argument");
  auto it = std::find(b->runs.begin(), b->runs.end(), c);
  if (it == b->runs.end()) return set_err(YMKH_EINVAL, "run not in the batch");
  b->runs.erase(it);
  b->dirty = true;
  return 0;
}

int ymkh_batch_size(ymkh_batch* b) { return b ? (int)b->runs.size() : -1; }

int ymkh_batch_set_graph_steps(ymkh_batch* b, int n) {
  if (!b || n < 0 || (n % 2) != 0) return set_err(YMKH_EINVAL, "graph step count must be even and >= 0");
  batch_drop_graph(b);
  b->graph_steps = n;
  return 0;
}

int ymkh_batch_step(ymkh_batch* b, int nsteps, void* stream) {
  if (!b) return set_err(YMKH_EINVAL, "null batch");
  if (nsteps < 0) return set_err(YMKH_EINVAL, "negative step count");
  NvtxRange range("ymkh_batch_step");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->dirty) { int rc = batch_build(b, s); if (rc) return rc; }
  int done = 0;
  const bool graphs = s != nullptr && b->graph_steps >= 2 && !b->runs.empty();
  if (graphs) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    if (cs == cudaStreamCaptureStatusNone) {
      // the captured graph starts from the tables' first parity
      if (b->parity != 0 && nsteps - done > b->graph_steps) {
        int rc = batch_step_once(b, s);
        if (rc) return rc;
        ++done;
      }
      while (b->parity == 0 && nsteps - done >= b->graph_steps) {
        if (!b->gexec || b->gstream != s) {
          batch_drop_graph(b);
          std::vector<int> cur0;
          for (ymkh_ctx* c : b->runs) cur0.push_back(c->cur);
          cudaGraph_t g = nullptr;
          CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
          const long long l0 = g_launches.load();
          int rc = 0;
          for (int k = 0; k < b->graph_steps && !rc; ++k) rc = batch_step_once(b, s);
          b->glaunches = g_launches.load() - l0;
          g_launches -= b->glaunches;
          cudaError_t ec = cudaStreamEndCapture(s, &g);
          for (size_t i = 0; i < b->runs.size(); ++i) b->runs[i]->cur = cur0[i];  // nothing ran yet
          b->parity = 0;
          if (rc) { if (g) cudaGraphDestroy(g); return rc; }
          CK(ec, "end capture");
          cudaError_t ei = cudaGraphInstantiate(&b->gexec, g, 0);
          cudaGraphDestroy(g);
          CK(ei, "graph instantiate");
          b->gstream = s;
        }
        CK(cudaGraphLaunch(b->gexec, s), "graph launch");
        g_launches += b->glaunches;
        done += b->graph_steps;  // even: every member ends in the buffer it started from
      }
    }
  }
  for (; done < nsteps; ++done) {
    int rc = batch_step_once(b, s);
    if (rc) return rc;
  }
  bool moved = false;
  for (ymkh_ctx* c : b->runs)
    if (!c->dual && c->cur == 1) { int rc = copy_back(c, s); if (rc) return rc; moved = true; }
  // A member moved back to buffer 0 no longer matches the tables of the
  // current parity (built for it starting in buffer 1): rebuild them from
  // every member's current buffer before the next step.
  if (moved) b->dirty = true;
  return 0;
}

int ymkh_batch_check(ymkh_batch* b, void* stream) {
  if (!b) return set_err(YMKH_EINVAL, "null batch");
  unsigned h = 0;
  CK(cudaMemcpyAsync(&h, b->derr, sizeof h, cudaMemcpyDeviceToHost, (cudaStream_t)stream), "error word D2H");
  CK(cudaStreamSynchronize((cudaStream_t)stream), "error word sync");
  if (h) {
    cudaMemsetAsync(b->derr, 0, sizeof(unsigned), (cudaStream_t)stream);
    return set_err(YMKH_ECUDA, "%s (error word %u)",
                   (h & ERR_BOUNDS) ? "a checked access was out of range and skipped" : "a bounded in-kernel wait timed out",
                   h);
  }
  return 0;
}

int ymkh_batch_set_fct_mode(ymkh_batch* b, int mode) {
  if (!b || (mode != YMKH_FCT_FUSED && mode != YMKH_FCT_SPLIT)) return set_err(YMKH_EINVAL, "bad FCT mode");
  b->fct_mode = mode;
  b->dirty = true;
  return 0;
}

int ymkh_batch_destroy(ymkh_batch* b) {
  if (!b) return 0;
  batch_drop_graph(b);
  if (b->ddesc) cudaFree(b->ddesc);
  if (b->derr) cudaFree(b->derr);
  for (int i = 0; i < ymkh_batch::kAux; ++i) {
    if (b->aux[i]) cudaStreamDestroy(b->aux[i]);
    if (b->join_ev[i]) cudaEventDestroy(b->join_ev[i]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  delete b;
  return 0;
}

}  // extern "C"

namespace ymkh {
// Error reporting and launch counting for entry points defined in other
// translation units (ymkh_noalloc.cu).
int capi_error(int code, const char* msg) { return set_err(code, "%s", msg); }
void capi_count_launches(int n) { g_launches += n; }
}  // namespace ymkh
