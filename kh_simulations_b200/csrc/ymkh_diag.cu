// ymkh_diag.cu — the non-Abelian Gauss law residual on the device.
//
// The reference checks the constraint offline, from 6-digit CSV snapshots
// (ymgpu2d/analysis/gauss_check.py:40-110):
//   G^a = (Ex^a - Ex^a[x-1]) / dx + (Ez^a - Ez^a[z-1]) / dz
//       + alpha (Az x Ezc)^a - (Q^a_A nA + Q^a_B nB),
//   Ezc^a = (Ez^a + Ez^a[z-1]) / 2, neighbours wrapping around in x and z.
// Here it runs on the FP64 state.  Each cell's terms are evaluated operand
// for operand as that script writes them; the sums of squares are
// compensated (Neumaier) in a fixed order: warp shuffles, then the warps of
// a CTA, then one pass over the CTA partials in index order.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

constexpr int GA_THREADS = 256;
constexpr int GA_PER_THREAD = 8;
constexpr int GA_NV = YMKH_GAUSS_NOUT;
// value slots: [0..2] G, [3..5] div E, [6..8] alpha (Az x Ezc), [9..11] rho,
// [12..14] div E + alpha (Az x Ezc), [15] |Ex1|+|Ex2|+|Ex3|+|Ez1|+|Ez2|+|Ez3|

__device__ __forceinline__ void add_sq(double* s, double* c, int v, double x) { neumaier_add(s[v], c[v], x * x); }

__global__ void __launch_bounds__(GA_THREADS)
    gauss_partial_kernel(const __grid_constant__ State st, int nx, int nz, double dx, double dz, double alpha,
                         double* __restrict__ part) {
  double s[GA_NV], c[GA_NV];
#pragma unroll
  for (int v = 0; v < GA_NV; ++v) s[v] = c[v] = 0.0;
  const size_t N = (size_t)nx * (size_t)nz;
  const size_t base = (size_t)blockIdx.x * GA_THREADS * GA_PER_THREAD;
  for (int k = 0; k < GA_PER_THREAD; ++k) {
    const size_t i = base + (size_t)k * GA_THREADS + threadIdx.x;
    if (i >= N) break;
    const int z = (int)(i / (size_t)nx);
    const int x = (int)(i - (size_t)z * (size_t)nx);
    const size_t iw = (x == 0) ? i + (size_t)(nx - 1) : i - 1;
    const size_t is = (z == 0) ? i + (size_t)(nz - 1) * (size_t)nx : i - (size_t)nx;
    double de[3], ezc[3];
    double alle = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double* ex = st.f[EX1 + a];
      const double* ez = st.f[EZ1 + a];
      const double ezi = ez[i], ezs = ez[is];
      de[a] = (ex[i] - ex[iw]) / dx + (ezi - ezs) / dz;
      ezc[a] = 0.5 * (ezi + ezs);
    }
    alle = fabs(st.f[EX1][i]) + fabs(st.f[EX2][i]);
    alle = alle + fabs(st.f[EX3][i]);
    alle = alle + fabs(st.f[EZ1][i]);
    alle = alle + fabs(st.f[EZ2][i]);
    alle = alle + fabs(st.f[EZ3][i]);
    const double az1 = st.f[AZ1][i], az2 = st.f[AZ2][i], az3 = st.f[AZ3][i];
    double nab[3];
    nab[0] = alpha * (az2 * ezc[2] - az3 * ezc[1]);
    nab[1] = alpha * (az3 * ezc[0] - az1 * ezc[2]);
    nab[2] = alpha * (az1 * ezc[1] - az2 * ezc[0]);
    const double nA = st.a[FN][i], nB = st.b[FN][i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double rho = st.a[FQ1 + a][i] * nA + st.b[FQ1 + a][i] * nB;
      const double lhs = de[a] + nab[a];
      add_sq(s, c, a, lhs - rho);
      add_sq(s, c, 3 + a, de[a]);
      add_sq(s, c, 6 + a, nab[a]);
      add_sq(s, c, 9 + a, rho);
      add_sq(s, c, 12 + a, lhs);
    }
    add_sq(s, c, 15, alle);
  }
  // warp: butterfly in a fixed pattern
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int v = 0; v < GA_NV; ++v) {
      const double so = __shfl_xor_sync(0xffffffffu, s[v], off);
      const double co = __shfl_xor_sync(0xffffffffu, c[v], off);
      c[v] += co;
      neumaier_add(s[v], c[v], so);
    }
  }
  __shared__ double ws[GA_THREADS / 32][GA_NV][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < GA_NV; ++v) {
      ws[warp][v][0] = s[v];
      ws[warp][v][1] = c[v];
    }
  }
  __syncthreads();
  if (threadIdx.x < GA_NV) {
    const int v = threadIdx.x;
    double a = 0.0, ca = 0.0;
    for (int w = 0; w < GA_THREADS / 32; ++w) {
      ca += ws[w][v][1];
      neumaier_add(a, ca, ws[w][v][0]);
    }
    part[((size_t)blockIdx.x * GA_NV + v) * 2] = a;
    part[((size_t)blockIdx.x * GA_NV + v) * 2 + 1] = ca;
  }
}

// One thread per value: the CTA partials in index order, then the
// root-mean-square over the N cells.
__global__ void gauss_final_kernel(const double* __restrict__ part, int nparts, double n_cells, double* out) {
  const int v = threadIdx.x;
  if (v >= GA_NV) return;
  double s = 0.0, c = 0.0;
  for (int b = 0; b < nparts; ++b) {
    c += part[((size_t)b * GA_NV + v) * 2 + 1];
    neumaier_add(s, c, part[((size_t)b * GA_NV + v) * 2]);
  }
  out[v] = sqrt((s + c) / n_cells);
}

}  // namespace

int gauss_nparts(size_t N) { return (int)((N + GA_THREADS * GA_PER_THREAD - 1) / (GA_THREADS * GA_PER_THREAD)); }

cudaError_t launch_gauss(const State& st, int nx, int nz, double dx, double dz, double alpha, double* part,
                         double* out, cudaStream_t s) {
  const size_t N = (size_t)nx * (size_t)nz;
  const int np = gauss_nparts(N);
  gauss_partial_kernel<<<np, GA_THREADS, 0, s>>>(st, nx, nz, dx, dz, alpha, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  gauss_final_kernel<<<1, 32, 0, s>>>(part, np, (double)N, out);
  return cudaGetLastError();
}

}  // namespace ymkh
