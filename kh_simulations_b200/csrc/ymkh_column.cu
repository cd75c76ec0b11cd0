// ymkh_column.cu — post-Maxwell stages that act along z or pointwise:
// sponge (YM_Physics.cu:161-182), xi_cut (:192-210), z-mean removal
// (:272-327), the DFT kz band filters (:349-584), z-hyperdiffusion (:228-259)
// and the colour-1 zeroing (ymgpu2d/main_ym.cu:443-447).  All update the new
// state buffer in place; none reads a neighbour another CTA writes.
//
// The band filter is written as two dense FP64 contractions per band, over
// all filtered arrays at once (21 arrays: the 15 EM/colour arrays of
// YM_Physics.cu:373-379 and n, px, pz of both beams):
//   C[j, x] = inv2 * sum_z W[z, j] G[z, x]          (coefficients A_m, B_m)
//   G[z, x] = G[z, x] - sum_j W[z, j] C[j, x]       (subtract the band)
// with W[z, 2i] = cosf(phase), W[z, 2i+1] = sinf(phase) the reference's FP32
// twiddles (YM_Physics.cu:387-388) widened to double and inv2 = 2.0f/nz
// (:425), summed in the reference's order (its warp-shuffle tree), so the
// filtered step is bit-identical to the reference's -fmad=false build.

#include "ymkh_common.cuh"

#include <mutex>

namespace ymkh {

// ---------------------------------------------------------------- twiddles
// W[z * ldw + 2*(m-lo) + {0,1}] for m in [lo, hi].
__global__ void twiddle_kernel(double* W, int nz, int lo, int hi, int ldw) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = lo + blockIdx.y;
  if (z >= nz || m > hi) return;
  float phase = 2.0f * (float)M_PI * m * z / (float)nz;
  float cz = cosf(phase), sz = sinf(phase);
  W[(size_t)z * ldw + 2 * (m - lo)] = (double)cz;
  W[(size_t)z * ldw + 2 * (m - lo) + 1] = (double)sz;
}

__global__ void twiddle_f32_kernel(float* c, float* s, int nz, int lo, int hi) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = lo + blockIdx.y;
  if (z >= nz || m > hi) return;
  float phase = 2.0f * (float)M_PI * m * z / (float)nz;
  c[(size_t)(m - lo) * nz + z] = cosf(phase);
  s[(size_t)(m - lo) * nz + z] = sinf(phase);
}

cudaError_t launch_twiddles(double* W, int nz, int lo, int hi, int ldw, cudaStream_t s) {
  dim3 grid((nz + 127) / 128, hi - lo + 1);
  twiddle_kernel<<<grid, 128, 0, s>>>(W, nz, lo, hi, ldw);
  return cudaGetLastError();
}
cudaError_t launch_twiddles_f32(float* c, float* sn, int nz, int lo, int hi, cudaStream_t s) {
  dim3 grid((nz + 127) / 128, hi - lo + 1);
  twiddle_f32_kernel<<<grid, 128, 0, s>>>(c, sn, nz, lo, hi);
  return cudaGetLastError();
}


// ---------------------------------------------------------- sponge / xicut
__global__ void sponge_xicut_kernel(const __grid_constant__ ArrayList a12, StepParams p, int cut) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  if (x >= p.nx) return;
  const double xc = (p.nx * p.dx) * 0.5;
  const double xi = fabs((x * p.dx - xc) / p.epsilon);
  const size_t i = idx2(x, z, p.nx);
  if (cut) {
    if (xi <= p.xi_cut) return;
#pragma unroll
    for (int k = 0; k < 12; ++k) a12.p[k][i] = 0.0;
  } else {
    if (xi <= p.xi_sponge) return;
    const double sig = p.sigma_sponge * (xi - p.xi_sponge);
    const double dec = exp(-sig * p.dt);
#pragma unroll
    for (int k = 0; k < 12; ++k) a12.p[k][i] *= dec;
  }
}

cudaError_t launch_sponge_xicut(const ArrayList& a12, const StepParams& p, int cut, cudaStream_t s) {
  dim3 grid((p.nx + 127) / 128, p.nz);
  sponge_xicut_kernel<<<grid, 128, 0, s>>>(a12, p, cut);
  return cudaGetLastError();
}

// -------------------------------------------------------------- z-mean
// Arrays [0, nmean) lose their z-mean; arrays [nmean, gridDim.y) are set to
// zero (the colour-1 fields, which the step zeroes once the z-mean is done:
// ymgpu2d/main_ym.cu:443-447; no stage in between reads or writes them).
// One CTA per (4 columns, array).  The column sum uses the reference's
// halving tree (YM_Physics.cu:301-308) so the mean is bit-identical.
constexpr int ZM_CX = 4;
constexpr size_t kColumnSmemMax = 200 * 1024;  // shared memory of the staged-column kernels
__global__ void zmean_kernel(const __grid_constant__ ArrayList arrs, int nx, int nz, int nmean) {
  extern __shared__ double sm[];  // [nz][ZM_CX]
  const int x0 = blockIdx.x * ZM_CX;
  double* g = arrs.p[blockIdx.y];
  if ((int)blockIdx.y >= nmean) {
    for (int i = threadIdx.x; i < nz * ZM_CX; i += blockDim.x) {
      const int z = i / ZM_CX, c = i - z * ZM_CX;
      if (x0 + c < nx) g[idx2(x0 + c, z, nx)] = 0.0;
    }
    return;
  }
  for (int i = threadIdx.x; i < nz * ZM_CX; i += blockDim.x) {
    const int z = i / ZM_CX, c = i - z * ZM_CX;
    sm[i] = (x0 + c < nx) ? g[idx2(x0 + c, z, nx)] : 0.0;
  }
  __syncthreads();
  for (int st = nz >> 1; st > 0; st >>= 1) {
    for (int i = threadIdx.x; i < st * ZM_CX; i += blockDim.x) sm[i] += sm[i + st * ZM_CX];
    __syncthreads();
  }
  const double inv = 1.0 / (double)nz;
  for (int i = threadIdx.x; i < nz * ZM_CX; i += blockDim.x) {
    const int z = i / ZM_CX, c = i - z * ZM_CX;
    if (x0 + c < nx) {
      const size_t gi = idx2(x0 + c, z, nx);
      g[gi] -= sm[c] * inv;
    }
  }
}

// Power-of-two NZ = 32 M: one CTA per (32 columns, array), warp l holding the
// rows z = l + 32 j of its lane's column, so every load is one coalesced row
// segment.  The halving tree pairs z with z + NZ/2, then z + NZ/4, ...: its
// levels down to stride 32 stay inside a residue class z mod 32, where they
// form the same halving tree over j; each thread sums its class in that order
// with a pairwise binary counter over the leaves in bit-reversed j order
// (T(y) = T(y_even) + T(y_odd)), and the last five levels (strides 16 .. 1)
// are a shuffle tree over the 32 class sums.  The sum is therefore the
// halving tree's, bit for bit; the columns are then re-read (mostly from L2)
// and the mean subtracted.
template <int LOGM>
__global__ void __launch_bounds__(1024) zmean_p2_kernel(const __grid_constant__ ArrayList arrs, int nx, int nmean) {
  constexpr int M = 1 << LOGM;
  __shared__ double part[32][33];
  __shared__ double mean[32];
  const int lane = threadIdx.x & 31, l = threadIdx.x >> 5;
  const int x = blockIdx.x * 32 + lane;
  double* g = arrs.p[blockIdx.y];
  const bool in = x < nx;
  if ((int)blockIdx.y >= nmean) {  // an array the step zeroes (zmean_kernel)
    if (in)
#pragma unroll 8
      for (int j = 0; j < M; ++j) g[(size_t)(l + 32 * j) * nx + x] = 0.0;
    return;
  }
  double st[LOGM + 1];
#pragma unroll
  for (int jj = 0; jj < M; ++jj) {
    int j = 0;
#pragma unroll
    for (int b = 0; b < LOGM; ++b) j |= ((jj >> b) & 1) << (LOGM - 1 - b);
    double carry = in ? g[(size_t)(l + 32 * j) * nx + x] : 0.0;
    int k = 0;
#pragma unroll
    for (int b = 0; b < LOGM; ++b) {
      if (((jj >> b) & 1) == 0) break;
      carry = st[b] + carry;
      k = b + 1;
    }
    st[k] = carry;
  }
  part[l][lane] = st[LOGM];
  __syncthreads();
  {
    double v = part[lane][l];  // warp l: column l of the tile, lane = residue class
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, d);
    if (lane == 0) mean[l] = v * (1.0 / (double)(32 * M));
  }
  __syncthreads();
  if (in) {
    const double mu = mean[lane];
#pragma unroll 8
    for (int j = 0; j < M; ++j) {
      const size_t gi = (size_t)(l + 32 * j) * nx + x;
      g[gi] -= mu;
    }
  }
}

cudaError_t launch_zmean(const ArrayList& arrs, int nmean, int nzero, int nx, int nz, cudaStream_t s) {
  const int narr = nmean + nzero;
  const dim3 g32((nx + 31) / 32, narr);
  switch (nz) {
    case 128: zmean_p2_kernel<2><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 256: zmean_p2_kernel<3><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 512: zmean_p2_kernel<4><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 1024: zmean_p2_kernel<5><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 2048: zmean_p2_kernel<6><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 4096: zmean_p2_kernel<7><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    case 8192: zmean_p2_kernel<8><<<g32, 1024, 0, s>>>(arrs, nx, nmean); return cudaGetLastError();
    default: break;
  }
  const size_t smem = (size_t)nz * ZM_CX * sizeof(double);
  if (smem > kColumnSmemMax) return cudaErrorInvalidValue;  // NZ > 6400 without a coalesced form
  dim3 grid((nx + ZM_CX - 1) / ZM_CX, narr);
  zmean_kernel<<<grid, 256, smem, s>>>(arrs, nx, nz, nmean);
  return cudaGetLastError();
}

// ---------------------------------------------------------- hyperdiffusion
// Race-free form of YM_Physics.cu:228-259: every stencil reads the values
// from before the update (the reference's in-place version reads a mix).
constexpr int HD_CX = 4;
__global__ void hyperdiff_kernel(const __grid_constant__ ArrayList a12, int nx, int nz, double mu) {
  extern __shared__ double sm[];  // [nz][HD_CX]
  const int x0 = blockIdx.x * HD_CX;
  double* g = a12.p[blockIdx.y];
  for (int i = threadIdx.x; i < nz * HD_CX; i += blockDim.x) {
    const int z = i / HD_CX, c = i - z * HD_CX;
    sm[i] = (x0 + c < nx) ? g[idx2(x0 + c, z, nx)] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nz * HD_CX; i += blockDim.x) {
    const int z = i / HD_CX, c = i - z * HD_CX;
    if (x0 + c >= nx) continue;
    const int zm1 = (z == 0) ? nz - 1 : z - 1;
    const int zm2 = (z <= 1) ? z - 2 + nz : z - 2;
    const int zp1 = (z == nz - 1) ? 0 : z + 1;
    const int zp2 = (z >= nz - 2) ? z + 2 - nz : z + 2;
    const double d4 = sm[zm2 * HD_CX + c] - 4.0 * sm[zm1 * HD_CX + c] + 6.0 * sm[i] - 4.0 * sm[zp1 * HD_CX + c] +
                      sm[zp2 * HD_CX + c];
    g[idx2(x0 + c, z, nx)] = sm[i] - mu * d4;
  }
}

// NZ a multiple of 32 (at least 64): one 1024-thread CTA per (32 columns,
// array); lane c holds column c and warp w the rows [w L, (w+1) L), L = NZ/32,
// so every access is a coalesced 256-byte row segment.  Each warp first reads
// the two rows on either side of its segment (periodic in z), then the CTA
// synchronises, and each warp updates its own rows in place from a five-row
// window of values read before any write: every stencil sees the values from
// before the update, as hyperdiff_kernel's shared copy gives, with the same
// arithmetic, so the result is the same bit for bit.
__global__ void __launch_bounds__(1024) hyperdiff_seg_kernel(const __grid_constant__ ArrayList a12, int nx, int nz,
                                                             double mu) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = blockIdx.x * 32 + lane;
  const bool in = x < nx;
  double* g = a12.p[blockIdx.y];
  const int L = nz >> 5, z0 = w * L;
  auto at = [&](int z) -> double {
    z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
    return in ? g[(size_t)z * nx + x] : 0.0;
  };
  const double h0 = at(z0 - 2), h1 = at(z0 - 1);        // rows below the segment
  const double t0 = at(z0 + L), t1 = at(z0 + L + 1);    // rows above it
  __syncthreads();  // every warp holds its neighbours' rows before any write
  double w0 = h0, w1 = h1, w2 = at(z0), w3 = at(z0 + 1);
#pragma unroll 4
  for (int k = 0; k < L; ++k) {
    const double w4 = (k + 2 < L) ? at(z0 + k + 2) : (k + 2 == L ? t0 : t1);
    const double d4 = w0 - 4.0 * w1 + 6.0 * w2 - 4.0 * w3 + w4;
    if (in) g[(size_t)(z0 + k) * nx + x] = w2 - mu * d4;
    w0 = w1;
    w1 = w2;
    w2 = w3;
    w3 = w4;
  }
}

cudaError_t launch_hyperdiff(const ArrayList& a12, int nx, int nz, double mu, cudaStream_t s) {
  if (nz % 32 == 0 && nz >= 64) {
    hyperdiff_seg_kernel<<<dim3((nx + 31) / 32, 12), 1024, 0, s>>>(a12, nx, nz, mu);
    return cudaGetLastError();
  }
  const size_t smem = (size_t)nz * HD_CX * sizeof(double);
  if (smem > kColumnSmemMax) return cudaErrorInvalidValue;  // NZ > 6400 and not a multiple of 32
  dim3 grid((nx + HD_CX - 1) / HD_CX, 12);
  hyperdiff_kernel<<<grid, 256, smem, s>>>(a12, nx, nz, mu);
  return cudaGetLastError();
}

// The staged-column kernels (zmean_kernel, hyperdiff_kernel) keep a block of
// whole columns in shared memory.  The dynamic shared-memory limit is a
// property of the kernel, shared by every run in the process: it only ever
// grows (to the largest NZ seen), so a run with a smaller NZ never lowers it
// under a larger resident run.  Above kColumnSmemMax (NZ > 6400) nothing is
// set: such runs use the coalesced kernels, and a stage that would need a
// staged kernel there fails at its launch.
size_t column_smem(int nz) { return (size_t)nz * (ZM_CX > HD_CX ? ZM_CX : HD_CX) * sizeof(double); }

cudaError_t prepare_column(int nz) {
  static std::mutex mu;
  static size_t granted[64];  // per device
  const size_t smem = column_smem(nz);
  if (smem > kColumnSmemMax) return cudaSuccess;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (smem > 48 * 1024 && smem > granted[dev]) {
    cudaError_t e = cudaFuncSetAttribute(zmean_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(hyperdiff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    granted[dev] = smem;
  }
  return cudaSuccess;
}

// ------------------------------------------------------------- band filter
// The FP64 band filter in the reference's own summation order, so that a
// filtered step is bit-identical to the reference's kernels built with
// -fmad=false (YM_Physics.cu:349-455 for the 15 EM/colour arrays, :461-584
// for pz, px and n).  Two dense contractions per band and array, each
// blocked over (mode, column) or (z, column) tiles:
//
//   coefficients  C[j][x] = inv2 * S_j(x),
//     S_j(x) = sum over warps w, in order from 0.0, of the warp's lane-0
//     shuffle tree of the 32 products v[32w + i][x] * tw[j][32w + i]
//     (YM_Physics.cu:396-426);
//   apply         v[z][x] -= delta, delta = sum over modes m in order from
//     0.0 of (A_m * cos_m(z) + B_m * sin_m(z)) (YM_Physics.cu:429-450).
//
// Products and sums are rounded separately (no fused multiply-add), as the
// reference's -fmad=false build rounds them.

// The reference's warp reduction (shfl_down by 16, 8, 4, 2, 1) leaves lane 0
// with root = T4(0) + T4(1), T4(i) = T3(i) + T3(i+2), T3(i) = T2(i) + T2(i+4),
// T2(i) = T1(i) + T1(i+8), T1(i) = a_i + a_{i+16} (every sum is commutative,
// so only the grouping matters).  Visited in bit-reversed order (0, 8, 4,
// 12, 2, ...), the sixteen T1 nodes form a balanced pairwise tree over
// consecutive visits, which a stack of four partial sums evaluates.
__host__ __device__ constexpr int bitrev4(int k) {
  return ((k & 1) << 3) | ((k & 2) << 1) | ((k & 4) >> 1) | ((k & 8) >> 3);
}

constexpr int BC_TJ = 32, BC_TX = 64, BC_CH = 32;  // coefficient tile: 32 j (16 modes) x 64 columns, z chunks of 32
constexpr int BC_RJ = 2, BC_RX = 4;                // per thread: one mode's (cos, sin) x 4 columns
constexpr int BC_THREADS = (BC_TJ / BC_RJ) * (BC_TX / BC_RX);  // 256

__global__ void __launch_bounds__(BC_THREADS, 2)
    band_coef_kernel(const __grid_constant__ ArrayList arrs, const double* __restrict__ W, int ldw, int J,
                     double* __restrict__ C, int nx, int nz, double inv2) {
  __shared__ __align__(16) double sW[2][BC_CH][BC_TJ];  // [z][j]
  __shared__ __align__(16) double sF[2][BC_CH][BC_TX];  // [z][x]
  const int j0 = blockIdx.x * BC_TJ, x0 = blockIdx.y * BC_TX, k = blockIdx.z;
  const double* G = arrs.p[k];
  double* Ck = C + (size_t)k * J * nx;
  const int tj = threadIdx.x % (BC_TJ / BC_RJ);  // mode of the tile
  const int tx = threadIdx.x / (BC_TJ / BC_RJ);  // group of 4 columns
  const int nch = (nz + BC_CH - 1) / BC_CH;

  auto stage = [&](int buf, int ch) {
    // 32 z rows of W (32 j) and of the array (64 x), asynchronously (8-byte
    // cp.async; zero padding past the edges written directly), one commit
    // group per chunk
    for (int i = threadIdx.x; i < BC_CH * BC_TJ; i += BC_THREADS) {
      const int zz = i / BC_TJ, c = i - zz * BC_TJ, z = ch * BC_CH + zz;
      if (z < nz && j0 + c < J) cp_async8(&sW[buf][zz][c], W + (size_t)z * ldw + j0 + c);
      else sW[buf][zz][c] = 0.0;
    }
    for (int i = threadIdx.x; i < BC_CH * BC_TX; i += BC_THREADS) {
      const int zz = i / BC_TX, c = i - zz * BC_TX, z = ch * BC_CH + zz;
      if (z < nz && x0 + c < nx) cp_async8(&sF[buf][zz][c], G + idx2(x0 + c, z, nx));
      else sF[buf][zz][c] = 0.0;
    }
    cp_async_commit();
  };

  double S[BC_RJ][BC_RX];
#pragma unroll
  for (int a = 0; a < BC_RJ; ++a)
#pragma unroll
    for (int b = 0; b < BC_RX; ++b) S[a][b] = 0.0;

  stage(0, 0);
  for (int ch = 0; ch < nch; ++ch) {
    const int buf = ch & 1;
    // the next chunk goes to the other buffer, released by the barrier at
    // the end of the previous chunk; then this chunk's copies are awaited
    if (ch + 1 < nch) stage(buf ^ 1, ch + 1);
    else cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    double st[4][BC_RJ][BC_RX];  // pending tree nodes of heights 1..4 (T2..T4 partial sums)
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      const int i = bitrev4(kk);
      double w0[BC_RJ], w1[BC_RJ], f0[BC_RX], f1[BC_RX];
#pragma unroll
      for (int a = 0; a < BC_RJ; ++a) {
        w0[a] = sW[buf][i][tj * BC_RJ + a];
        w1[a] = sW[buf][i + 16][tj * BC_RJ + a];
      }
#pragma unroll
      for (int b = 0; b < BC_RX; ++b) {
        f0[b] = sF[buf][i][tx * BC_RX + b];
        f1[b] = sF[buf][i + 16][tx * BC_RX + b];
      }
#pragma unroll
      for (int a = 0; a < BC_RJ; ++a)
#pragma unroll
        for (int b = 0; b < BC_RX; ++b) {
          const double p0 = f0[b] * w0[a];  // YM_Physics.cu:394 ar = v * cz (rounded)
          const double p1 = f1[b] * w1[a];
          double x = p0 + p1;  // T1(i)
          // merge with the pending nodes: one level per trailing one bit of kk
          int lvl = 0;
#pragma unroll
          for (int L = 0; L < 4; ++L) {
            if (((kk >> L) & 1) && lvl == L) {
              x = st[L][a][b] + x;
              ++lvl;
            }
          }
          if (lvl < 4) st[lvl][a][b] = x;
          else S[a][b] = S[a][b] + x;  // warp sums added in warp order from 0.0
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < BC_RJ; ++a)
#pragma unroll
    for (int b = 0; b < BC_RX; ++b) {
      const int j = j0 + tj * BC_RJ + a, x = x0 + tx * BC_RX + b;
      if (j < J && x < nx) Ck[(size_t)j * nx + x] = S[a][b] * inv2;
    }
}

constexpr int BA_TZ = 64, BA_TX = 64, BA_KM = 8;  // apply tile: 64 z x 64 columns, 8 modes staged at a time
constexpr int BA_THREADS = 256;                     // 4 x 4 outputs per thread

// v[z][x] -= sum over the band's modes in order of (A_m cos_m(z) + B_m sin_m(z))
__global__ void __launch_bounds__(BA_THREADS, 2)
    band_apply_kernel(const __grid_constant__ ArrayList arrs, const double* __restrict__ W, int ldw, int J,
                      const double* __restrict__ C, int nx, int nz) {
  __shared__ __align__(16) double sW[2][2 * BA_KM][BA_TZ + 1];  // [buffer][j][z]
  __shared__ __align__(16) double sC[2][2 * BA_KM][BA_TX + 1];  // [buffer][j][x]
  const int z0 = blockIdx.x * BA_TZ, x0 = blockIdx.y * BA_TX, k = blockIdx.z;
  double* G = arrs.p[k];
  const double* Ck = C + (size_t)k * J * nx;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // ty -> z, tx -> x
  double delta[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) delta[a][b] = 0.0;
  auto stage = [&](int buf, int jb) {  // 8 modes (16 j) of W and of the coefficients, asynchronously
    for (int i = threadIdx.x; i < 2 * BA_KM * BA_TZ; i += BA_THREADS) {
      const int jj = i / BA_TZ, c = i - jj * BA_TZ;
      const int j = jb + jj;
      if (j < J && z0 + c < nz) cp_async8(&sW[buf][jj][c], W + (size_t)(z0 + c) * ldw + j);
      else sW[buf][jj][c] = 0.0;
      if (j < J && x0 + c < nx) cp_async8(&sC[buf][jj][c], Ck + (size_t)j * nx + x0 + c);
      else sC[buf][jj][c] = 0.0;
    }
    cp_async_commit();
  };
  const int nblk = (J + 2 * BA_KM - 1) / (2 * BA_KM);
  stage(0, 0);
  for (int blk = 0; blk < nblk; ++blk) {
    const int buf = blk & 1, jb = blk * 2 * BA_KM;
    if (blk + 1 < nblk) stage(buf ^ 1, jb + 2 * BA_KM);
    else cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int mend = min(BA_KM, (J - jb) / 2);
    for (int mm = 0; mm < mend; ++mm) {
      double wc[4], ws[4], ca[4], cb[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        wc[a] = sW[buf][2 * mm][ty + 16 * a];
        ws[a] = sW[buf][2 * mm + 1][ty + 16 * a];
      }
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        ca[b] = sC[buf][2 * mm][tx + 16 * b];
        cb[b] = sC[buf][2 * mm + 1][tx + 16 * b];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const double t = ca[b] * wc[a] + cb[b] * ws[a];  // YM_Physics.cu:433 A_m cz + B_m sz
          delta[a][b] = delta[a][b] + t;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int z = z0 + ty + 16 * a, x = x0 + tx + 16 * b;
      if (z < nz && x < nx) {
        const size_t gi = idx2(x, z, nx);
        G[gi] = G[gi] - delta[a][b];
      }
    }
}

cudaError_t launch_band(const ArrayList& arrs, int narr, const double* W, int ldw, int J, double* C, int nx, int nz,
                        double inv2, cudaStream_t s) {
  dim3 g1((J + BC_TJ - 1) / BC_TJ, (nx + BC_TX - 1) / BC_TX, narr);
  band_coef_kernel<<<g1, BC_THREADS, 0, s>>>(arrs, W, ldw, J, C, nx, nz, inv2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 g2((nz + BA_TZ - 1) / BA_TZ, (nx + BA_TX - 1) / BA_TX, narr);
  band_apply_kernel<<<g2, BA_THREADS, 0, s>>>(arrs, W, ldw, J, C, nx, nz);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- energy
// Per-cell energy of YM_Energy.cu:3-21, summed with Neumaier compensation in
// a fixed order: each CTA reduces a contiguous block of cells, a second
// single-CTA pass reduces the CTA partials in index order.
constexpr int EN_THREADS = 256;
constexpr int EN_PER_THREAD = 16;

__global__ void __launch_bounds__(EN_THREADS)
    energy_partial_kernel(const __grid_constant__ State st, size_t N, double* __restrict__ part) {
  const size_t base = (size_t)blockIdx.x * EN_THREADS * EN_PER_THREAD;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < EN_PER_THREAD; ++k) {
    const size_t i = base + (size_t)k * EN_THREADS + threadIdx.x;
    if (i >= N) break;
    const double nA = fmax(st.a[FN][i], 1e-10);
    const double nB = fmax(st.b[FN][i], 1e-10);
    const double pxA = st.a[FPX][i], pzA = st.a[FPZ][i], pxB = st.b[FPX][i], pzB = st.b[FPZ][i];
    const double keA = 0.5 * (pxA * pxA + pzA * pzA) / nA;
    const double keB = 0.5 * (pxB * pxB + pzB * pzB) / nB;
    double em2 = 0.0;
    em2 = st.f[EX1][i] * st.f[EX1][i];
    em2 = em2 + st.f[EX2][i] * st.f[EX2][i];
    em2 = em2 + st.f[EX3][i] * st.f[EX3][i];
    em2 = em2 + st.f[EZ1][i] * st.f[EZ1][i];
    em2 = em2 + st.f[EZ2][i] * st.f[EZ2][i];
    em2 = em2 + st.f[EZ3][i] * st.f[EZ3][i];
    em2 = em2 + st.f[BY1][i] * st.f[BY1][i];
    em2 = em2 + st.f[BY2][i] * st.f[BY2][i];
    em2 = em2 + st.f[BY3][i] * st.f[BY3][i];
    const double e = keA + keB + 0.5 * em2;
    neumaier_add(s, c, e);
  }
  __shared__ double ss[EN_THREADS], sc[EN_THREADS];
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  for (int w = EN_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      double a = ss[threadIdx.x], ca = sc[threadIdx.x] + sc[threadIdx.x + w];
      neumaier_add(a, ca, ss[threadIdx.x + w]);
      ss[threadIdx.x] = a;
      sc[threadIdx.x] = ca;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ss[0];
    part[2 * blockIdx.x + 1] = sc[0];
  }
}

__global__ void energy_final_kernel(const double* __restrict__ part, int nparts, double* out) {
  __shared__ double ss[256], sc[256];
  double s = 0.0, c = 0.0;
  // thread t reduces a contiguous slice of the partials, in order
  const int per = (nparts + 255) / 256;
  for (int k = 0; k < per; ++k) {
    const int i = threadIdx.x * per + k;
    if (i >= nparts) break;
    c += part[2 * i + 1];
    neumaier_add(s, c, part[2 * i]);
  }
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, ca = 0.0;
    for (int t = 0; t < 256; ++t) {
      ca += sc[t];
      neumaier_add(a, ca, ss[t]);
    }
    *out = a + ca;
  }
}

int energy_nparts(size_t N) { return (int)((N + EN_THREADS * EN_PER_THREAD - 1) / (EN_THREADS * EN_PER_THREAD)); }

cudaError_t launch_energy(const State& st, size_t N, double* part, double* out, cudaStream_t s) {
  const int np = energy_nparts(N);
  energy_partial_kernel<<<np, EN_THREADS, 0, s>>>(st, N, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  energy_final_kernel<<<1, 256, 0, s>>>(part, np, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------ mode amplitude
// Per column x, F = sum_z (re + i im) e^{-2 pi i k z/nz} and Fc for re - i im
// (ymgpu2d/analysis/remote_timeseries.py:62-77 for re, im = Az2, Az3;
// ymgpu2d/analysis/resolution_convergence.py:83-86 for By2, By3).
__global__ void mode_amp_kernel(const double* __restrict__ re, const double* __restrict__ im, int nx, int nz,
                                int k, double* __restrict__ colbuf) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nx) return;
  double fr = 0, fi = 0, cr = 0, ci = 0;
  for (int z = 0; z < nz; ++z) {
    double sn, cs;
    sincospi(-2.0 * (double)k * (double)z / (double)nz, &sn, &cs);
    const double a = re[idx2(x, z, nx)], b = im[idx2(x, z, nx)];
    // (a + i b)(cs + i sn)
    fr += a * cs - b * sn;
    fi += a * sn + b * cs;
    // (a - i b)(cs + i sn)
    cr += a * cs + b * sn;
    ci += a * sn - b * cs;
  }
  colbuf[2 * x] = hypot(fr, fi);
  colbuf[2 * x + 1] = hypot(cr, ci);
}

// Without a weight: (mean_x |F| / nz, mean_x |Fc| / nz), remote_timeseries.py:72-74.
// With one: (sum_x w[x] |F| / nz, sum_x w[x] |Fc| / nz), the shear-layer
// weighted average of resolution_convergence.py:83-86.
__global__ void mode_amp_final_kernel(const double* __restrict__ colbuf, const double* __restrict__ w, int nx, int nz,
                                      double* out) {
  if (threadIdx.x != 0) return;
  double s0 = 0, s1 = 0;
  if (w == nullptr) {
    for (int x = 0; x < nx; ++x) {
      s0 += colbuf[2 * x];
      s1 += colbuf[2 * x + 1];
    }
    out[0] = s0 / nx / nz;
    out[1] = s1 / nx / nz;
  } else {
    for (int x = 0; x < nx; ++x) {
      s0 += w[x] * (colbuf[2 * x] / nz);
      s1 += w[x] * (colbuf[2 * x + 1] / nz);
    }
    out[0] = s0;
    out[1] = s1;
  }
}

cudaError_t launch_mode_amp(const double* re, const double* im, int nx, int nz, int k, double* colbuf,
                            const double* weight, double* out, cudaStream_t s) {
  mode_amp_kernel<<<(nx + 127) / 128, 128, 0, s>>>(re, im, nx, nz, k, colbuf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  mode_amp_final_kernel<<<1, 32, 0, s>>>(colbuf, weight, nx, nz, out);
  return cudaGetLastError();
}

}  // namespace ymkh
