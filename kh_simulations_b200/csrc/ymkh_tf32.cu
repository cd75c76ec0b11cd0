// ymkh_tf32.cu — the DFT band filter on the 5th-generation tensor cores:
// split-precision 3-pass TF32 with FP32 accumulation in tensor memory.
//
// The band filter of ymgpu2d/YM_Physics.cu:349-584 (per column x, for each
// subtracted mode m: A_m = inv2 sum_z v cos, B_m = inv2 sum_z v sin, then
// v -= sum_m (A_m cos + B_m sin)) is, over all 21 filtered arrays, two
// contractions per array k with the twiddle matrix W[z, j] (j = 2(m-lo) for
// cos, +1 for sin; the reference's FP32-phase twiddles):
//   GEMM 1:  C[j, x] = inv2 * sum_z W[z, j] G[z, x]      M = J, N = NX, K = NZ
//   GEMM 2:  G[z, x] -= sum_j W[z, j] C[j, x]            M = NZ, N = NX, K = J
// Here both run as tcgen05.mma kind::tf32 (M = N = 128 tiles, K = 8 per
// instruction) with every FP32/FP64 operand split as x ~ hi + lo, hi and lo
// TF32 (round to nearest), and the product formed as
//   lo_a*hi_b + hi_a*lo_b + hi_a*hi_b        (three passes, FP32 accumulate)
// which keeps ~2^-22 relative error per product against 2^-11 for one pass.
// The FP64 state is only read and written in FP64; the precision change is
// confined to the subtracted band content.
//
// Operand layout.  Every operand tile is 128 rows x 32 TF32 (K) = 16 KB, in
// the K-major 128-byte-swizzled layout the tensor core reads (8-row groups
// of 1024 B; 16-byte chunk index XOR row % 8).  The split kernels write
// whole tile images to global memory, so the GEMM stages each tile with one
// 16 KB TMA bulk copy (cp.async.bulk) and no tensor map:
//   W images  (built once per band):  A1 [mt = j/128][kt = z/32]   A2 [mt = z/128][kt = j/32]
//   G image   (per step, per array):   [array][nt = x/128][kt = z/32]      (B of GEMM 1)
//   C^T image (GEMM 1's epilogue):     [array][nt = x/128][kt = j/32]      (B of GEMM 2)
// z is padded to a multiple of 128 (Zp) and j to a multiple of 128 (Jp)
// in the images; rows and k-columns beyond NZ, J or NX are zero, and GEMM 2
// writes only z < NZ.
//
// The GEMM kernel is persistent and warp-specialised (see tf32x3_gemm_ws):
// a producer lane streams operand tiles through a 3-stage ring of "full" /
// "empty" mbarriers, an MMA lane issues 12 MMAs per stage into one of two
// TMEM accumulators, and four epilogue warps drain the other one, so the
// epilogue of a tile overlaps the main loop of the next.  Every mbarrier
// wait is bounded and reports through the device error word.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

constexpr int TT_M = 128;                 // tile rows (UMMA M)
constexpr int TT_IMG_N = 128;             // rows of a B tile image (x)
constexpr int TT_K = 32;                  // K per tile: one 128-byte swizzle row of TF32
constexpr int TT_BYTES = TT_M * TT_K * 4; // 16 KB tile image
constexpr int TT_FLOATS = TT_BYTES / 4;

// instruction descriptor, kind::tf32 (WS_IDESC below): D F32 (bits 4-5 =
// 1), A and B TF32 (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0),
// N >> 3 at bit 17, M >> 4 at bit 24

// byte offset of element (row r, k-column c) in a 128 x 32 TF32 tile image
__host__ __device__ __forceinline__ unsigned tile_off(int r, int c) {
  return (unsigned)((r >> 3) * 1024 + (r & 7) * 128 + ((((c >> 2) ^ (r & 7)) & 7) << 4) + (c & 3) * 4);
}

__device__ __forceinline__ float tf32_rna(float v) {
  unsigned u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
  return __uint_as_float(u);
}

__device__ __forceinline__ void split_f32(float f, float& hi, float& lo) {
  hi = tf32_rna(f);
  lo = tf32_rna(f - hi);  // exact difference: hi is f rounded at mantissa bit 13
}

__device__ __forceinline__ void split_f64(double g, float& hi, float& lo) {
  hi = tf32_rna((float)g);
  lo = tf32_rna((float)(g - (double)hi));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, 128-byte swizzle; start >> 4 in
// bits 0-13, leading byte offset 16 B (unused for this layout) in 16-29,
// stride byte offset 1024 B (next 8-row group) in 32-45, descriptor version
// 1 in 46-47, swizzle mode 2 (128 B) in 61-63
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- split kernels ------------------------------------------------------

// W[z * ldw + j] (FP64 holding the FP32 twiddles) -> A1 (rows j, k = z) and
// A2 (rows z, k = j) tile images, hi and lo, over z < Zp and j < Jp; the
// padding (z >= nz or j >= J) is zero.
__global__ void w_image_kernel(const double* __restrict__ W, int ldw, int J, int Jp, int nz, int Zp,
                               float* __restrict__ a1h, float* __restrict__ a1l, float* __restrict__ a2h,
                               float* __restrict__ a2l) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y;
  if (j >= Jp || z >= Zp) return;
  const float w = (j < J && z < nz) ? (float)W[(size_t)z * ldw + j] : 0.0f;
  float hi, lo;
  split_f32(w, hi, lo);
  const int kt1 = Zp / TT_K, kt2 = Jp / TT_K;
  const size_t t1 = ((size_t)(j / TT_M) * kt1 + z / TT_K) * TT_FLOATS + (tile_off(j % TT_M, z % TT_K) >> 2);
  const size_t t2 = ((size_t)(z / TT_M) * kt2 + j / TT_K) * TT_FLOATS + (tile_off(z % TT_M, j % TT_K) >> 2);
  a1h[t1] = hi;
  a1l[t1] = lo;
  a2h[t2] = hi;
  a2l[t2] = lo;
}

// G_k[z, x] (FP64) -> B image of GEMM 1, tile (nt, kt) of array k: rows x,
// k = z.  Thread (x, z-quad): four loads along z (each coalesced across the
// warp's consecutive x), split, and one 16-byte store per hi/lo chunk into
// the swizzled tile (the 8 rows of a wavefront hit 8 different chunks:
// conflict-free); the tile is then written out linearly.
__global__ void __launch_bounds__(256)
    g_image_kernel(const __grid_constant__ ArrayList arrs, int nx, int nz, int NT, int KT, float* __restrict__ gh,
                   float* __restrict__ gl) {
  __shared__ __align__(16) float sh[TT_FLOATS];
  __shared__ __align__(16) float sl[TT_FLOATS];
  const int nt = blockIdx.x, kt = blockIdx.y, k = blockIdx.z;
  const double* G = arrs.p[k];
  const int xx = threadIdx.x % TT_IMG_N, qh = threadIdx.x / TT_IMG_N;  // 2 halves of the 8 z-quads
  const int x = nt * TT_IMG_N + xx;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int q = qh * 4 + j;  // 16-byte chunk (4 consecutive z) of the tile row
    const int z = kt * TT_K + 4 * q;
    double g[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) g[c] = (x < nx && z + c < nz) ? G[(size_t)(z + c) * nx + x] : 0.0;
    float4 h, l;
    split_f64(g[0], h.x, l.x);
    split_f64(g[1], h.y, l.y);
    split_f64(g[2], h.z, l.z);
    split_f64(g[3], h.w, l.w);
    const unsigned o = tile_off(xx, 4 * q) >> 2;
    *reinterpret_cast<float4*>(sh + o) = h;
    *reinterpret_cast<float4*>(sl + o) = l;
  }
  __syncthreads();
  const size_t t = (((size_t)k * NT + nt) * KT + kt) * TT_FLOATS;
  float4* dh = reinterpret_cast<float4*>(gh + t);
  float4* dl = reinterpret_cast<float4*>(gl + t);
  for (int i = threadIdx.x; i < TT_FLOATS / 4; i += 256) {
    dh[i] = reinterpret_cast<const float4*>(sh)[i];
    dl[i] = reinterpret_cast<const float4*>(sl)[i];
  }
}

// ---- the GEMM -----------------------------------------------------------
//
// Persistent and warp-specialised: one CTA per SM walks a list of 128x128
// output tiles.  Warp 0 (one lane) streams operand tiles through a 3-stage
// shared-memory ring; warp 1 owns tensor memory and (one lane) issues the
// MMAs into one of two accumulators; warps 2-5 drain the other accumulator
// (tcgen05.ld; warp w reads TMEM lanes 32*(w%4)..+31), so the epilogue of a
// tile overlaps the main loop of the next.
//
//   EPI_COEF  (GEMM 1)  D[j, x] = sum_z Wt[j, z] G[z, x]; tiles (array, x-tile,
//                       j-tile), j fastest; epilogue: C = inv2 * D, split,
//                       into the C^T image (a warp covers one 128-byte row).
//   EPI_APPLY (GEMM 2)  D[x, z] = sum_j C^T[x, j] W[z, j] (the transposed
//                       product, so a thread owns one x); tiles (array, x-tile,
//                       z-tile), z fastest; epilogue: G[z, x] -= D, 32
//                       coalesced FP64 rows per chunk straight from registers.

struct Tf32GemmArgs {
  const float* a_hi;  // A tile images
  const float* a_lo;
  const float* b_hi;  // B tile images
  const float* b_lo;
  int KT;             // K tiles
  int NT;             // x tile images (128 rows of x) per array
  int MT;             // tiles of the other output dimension (j or z)
  int NB_TILES;       // real 128-row tiles along N: x tiles (GEMM 1) or z tiles (GEMM 2)
  int narr;
  // EPI_COEF: C^T image out, [array][x-tile][KT2] tiles (rows x, k = j)
  float* c_hi;
  float* c_lo;
  int KT2;
  float scale;
  // EPI_APPLY: G_k[z, x] -= D[x, z]
  ArrayList arrs;
  int nx;
  int nz;
  unsigned* err;
};

constexpr int EPI_COEF = 0, EPI_APPLY = 1;
constexpr int WS_THREADS = 192;                  // producer, MMA, 4 epilogue warps

// Output tiles are 128 x BN: BN = 256 takes two consecutive 128-row B tile
// images per stage (the N dimension: x for GEMM 1, z for GEMM 2), so every
// byte of A staged in shared memory feeds twice the MMA work.  Per stage:
// A hi, A lo (16 KB each), B hi, B lo (BN/128 images each); the ring has as
// many stages as fit (3 at BN = 128, 2 at 256); two BN-column FP32
// accumulators in tensor memory.
template <int BN>
struct WsCfg {
  static constexpr int NB = BN / TT_IMG_N;                  // B images per stage operand
  static constexpr int STAGE = 2 * TT_BYTES + 2 * NB * TT_BYTES;
  static constexpr int NS = BN == 128 ? 3 : 2;
  static constexpr uint32_t TMEM_COLS = 2 * BN;
  static constexpr size_t SMEM = (size_t)NS * STAGE + 1024;
  static constexpr uint32_t IDESC =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TT_M >> 4) << 24);
};

// Tile t of a GEMM: array k, M tile (j-tile of GEMM 1 or x tile of GEMM 2)
// and N group (x tiles or z tiles nb0 .. nb0 + NB - 1; those past the last
// real tile repeat it and their columns are skipped).
//   GEMM 1: N group fastest-varying after the j-tile: (k, N group, j-tile)
//   GEMM 2: (k, x tile, N group), N group fastest
template <int EPI, int NB>
__device__ __forceinline__ void ws_tile(const Tf32GemmArgs& g, int t, int& k, int& mt, int& nb0) {
  const int ngroups = (g.NB_TILES + NB - 1) / NB;
  if (EPI == EPI_COEF) {
    mt = t % g.MT;                   // j-tile, fastest
    nb0 = ((t / g.MT) % ngroups) * NB;  // first x tile image of the group
    k = t / (g.MT * ngroups);
  } else {
    nb0 = (t % ngroups) * NB;        // first z tile of the group, fastest
    mt = (t / ngroups) % g.NT;       // x tile image
    k = t / (ngroups * g.NT);
  }
}

template <int EPI, int BN>
__global__ void __launch_bounds__(WS_THREADS, 1) tf32x3_gemm_ws(const __grid_constant__ Tf32GemmArgs g) {
  using Cfg = WsCfg<BN>;
  constexpr int WS_NS = Cfg::NS, WS_STAGE = Cfg::STAGE, NB = Cfg::NB;
  constexpr uint32_t WS_TMEM_COLS = Cfg::TMEM_COLS, WS_IDESC = Cfg::IDESC;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* const smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full[WS_NS];
  __shared__ __align__(8) uint64_t empty[WS_NS];
  __shared__ __align__(8) uint64_t acc_full[2];
  __shared__ __align__(8) uint64_t acc_empty[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KT = g.KT;
  const int ntiles = EPI == EPI_COEF ? g.narr * g.MT * ((g.NB_TILES + NB - 1) / NB)
                                     : g.narr * g.NT * ((g.NB_TILES + NB - 1) / NB);

  if (tid == 0) {
    for (int s = 0; s < WS_NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(WS_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      // producer: the operand tiles of every tile of this CTA, in order
      int q = 0;  // k-tiles issued so far
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int k, mt, nb0;
        ws_tile<EPI, NB>(g, t, k, mt, nb0);
        size_t a_off, b_off[NB];
        for (int i = 0; i < NB; ++i) {
          const int nb = min(nb0 + i, g.NB_TILES - 1);  // past the last tile: repeat it (columns skipped)
          b_off[i] = EPI == EPI_COEF ? ((size_t)k * g.NT + nb) * KT * TT_FLOATS   // G image [array][x-tile]
                                     : (size_t)nb * KT * TT_FLOATS;                // W image [z-tile]
        }
        a_off = EPI == EPI_COEF ? (size_t)mt * KT * TT_FLOATS                     // Wt image [j-tile]
                                : ((size_t)k * g.NT + mt) * KT * TT_FLOATS;       // C^T image [array][x-tile]
        for (int kt = 0; kt < KT; ++kt, ++q) {
          const int s = q % WS_NS, u = q / WS_NS;
          if (u > 0) mbar_wait(&empty[s], (unsigned)((u - 1) & 1), g.err);
          unsigned char* const st = smem + (size_t)s * WS_STAGE;
          mbar_expect_tx(&full[s], (unsigned)WS_STAGE);
          const size_t o = (size_t)kt * TT_FLOATS;
          bulk_g2s(st, g.a_hi + a_off + o, TT_BYTES, &full[s]);
          bulk_g2s(st + TT_BYTES, g.a_lo + a_off + o, TT_BYTES, &full[s]);
          for (int i = 0; i < NB; ++i) {  // B hi images, then B lo images, each NB x 128 rows in a row
            bulk_g2s(st + (2 + i) * TT_BYTES, g.b_hi + b_off[i] + o, TT_BYTES, &full[s]);
            bulk_g2s(st + (2 + NB + i) * TT_BYTES, g.b_lo + b_off[i] + o, TT_BYTES, &full[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer: tile i accumulates into accumulator i % 2 once the
      // epilogue has drained that accumulator's previous tile
      int q = 0, i = 0;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int a = i & 1;
        if (i >= 2) mbar_wait(&acc_empty[a], (unsigned)(((i >> 1) - 1) & 1), g.err);
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(a * BN);
        for (int kt = 0; kt < KT; ++kt, ++q) {
          const int s = q % WS_NS, u = q / WS_NS;
          mbar_wait(&full[s], (unsigned)(u & 1), g.err);
          tc_fence_after();
          const uint32_t st = smem_u32(smem + (size_t)s * WS_STAGE);
#pragma unroll
          for (int kk = 0; kk < TT_K / 8; ++kk) {
            const uint32_t off = (uint32_t)kk * 32u;  // 8 TF32 = 32 bytes along the swizzled row
            const uint64_t ah = sw128_desc(st + off), al = sw128_desc(st + TT_BYTES + off);
            const uint64_t bh = sw128_desc(st + 2 * TT_BYTES + off), bl = sw128_desc(st + (2 + NB) * TT_BYTES + off);
            umma_tf32(d, al, bh, WS_IDESC, (kt | kk) != 0 ? 1u : 0u);
            umma_tf32(d, ah, bl, WS_IDESC, 1u);
            umma_tf32(d, ah, bh, WS_IDESC, 1u);
          }
          umma_commit(&empty[s]);  // stage s free once these MMAs have read it
        }
        umma_commit(&acc_full[a]);  // accumulator a holds tile i
      }
    }
  } else {
    // epilogue warps 2..5: TMEM lane quadrant w % 4, tile row = 32*(w%4) + lane
    const int quad = warp & 3;
    const int r = 32 * quad + lane;
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
      int k, mt, nb0;
      ws_tile<EPI, NB>(g, t, k, mt, nb0);
      const int a = i & 1;
      mbar_wait(&acc_full[a], (unsigned)((i >> 1) & 1), g.err);
      __syncwarp();
      tc_fence_after();
      const uint32_t src = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(a * BN);
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        const int nb = nb0 + c0 / TT_IMG_N;  // the N tile these 32 columns belong to
        if (nb >= g.NB_TILES) break;         // a repeated tile past the end: skipped
        const int cc = c0 % TT_IMG_N;        // columns within that tile
        uint32_t v[32];
        tmem_ld32(src + (uint32_t)c0, v);
        if (EPI == EPI_COEF) {
          // row j = mt*128 + r; columns x = nb*128 + cc + c -> C^T image tile
          // (nb, j/32), tile row cc + c, k-column j % 32 = lane
          const int xt = nb, ot = mt;
          const int j = ot * TT_M + r;
          const size_t tb = (((size_t)k * g.NT + xt) * g.KT2 + (j >> 5)) * TT_FLOATS;
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            float hi, lo;
            split_f32(__uint_as_float(v[c]) * g.scale, hi, lo);
            const unsigned o = tile_off(cc + c, lane) >> 2;
            g.c_hi[tb + o] = hi;
            g.c_lo[tb + o] = lo;
          }
        } else {
          // row x = mt*128 + r; columns z = nb*128 + cc + c: G_k[z, x] -= D
          // (z < nz; the padded rows of a last partial z tile are skipped)
          const int xt = mt, ot = nb;
          const int x = xt * TT_IMG_N + r;
          const int z0 = ot * TT_M + cc;
          if (x < g.nx && z0 < g.nz) {
            double* const G = g.arrs.p[k] + (size_t)z0 * g.nx + x;
            const size_t ld = (size_t)g.nx;
            if (z0 + 32 <= g.nz) {
              double gv[32];
#pragma unroll
              for (int c = 0; c < 32; ++c) gv[c] = G[(size_t)c * ld];
#pragma unroll
              for (int c = 0; c < 32; ++c) G[(size_t)c * ld] = gv[c] - (double)__uint_as_float(v[c]);
            } else {
#pragma unroll
              for (int c = 0; c < 32; ++c)
                if (z0 + c < g.nz) G[(size_t)c * ld] = G[(size_t)c * ld] - (double)__uint_as_float(v[c]);
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        unsigned aa = smem_u32(&acc_empty[a]);
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(aa) : "memory");
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(WS_TMEM_COLS));
  }
}

}  // namespace

int tf32_ntiles(int nx) { return (nx + TT_IMG_N - 1) / TT_IMG_N; }
int tf32_jpad(int J) { return ((J + TT_M - 1) / TT_M) * TT_M; }
int tf32_zpad(int nz) { return ((nz + TT_M - 1) / TT_M) * TT_M; }
size_t tf32_tile_floats() { return TT_FLOATS; }

cudaError_t prepare_tf32() {
  cudaError_t e = cudaFuncSetAttribute(tf32x3_gemm_ws<EPI_COEF, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)WsCfg<128>::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tf32x3_gemm_ws<EPI_APPLY, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)WsCfg<128>::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tf32x3_gemm_ws<EPI_COEF, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)WsCfg<256>::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tf32x3_gemm_ws<EPI_APPLY, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)WsCfg<256>::SMEM);
  return e;
}

// 128 x 256 tiles halve the A operand traffic per MMA but halve the tile
// count too; they are used when the GEMM still has at least 10 waves of
// tiles over the SMs.  Measured on B200, TF32 band stage: 2.58 against 2.90
// ms at 2048 x 4096 and 16.6 against 19.7 ms at 4096 x 8192, but 0.485
// against 0.464 ms at 1024 x 2048, where the wider tiles leave GEMM 1 3.4
// waves and GEMM 2 9.1.  Both widths give the same bits: each output's MMAs
// and their order are the same.
template <int EPI>
static cudaError_t launch_gemm(const Tf32GemmArgs& g, int ntiles_m_side, int sms, cudaStream_t s) {
  const int n256 = g.narr * ntiles_m_side * ((g.NB_TILES + 1) / 2);
  if (n256 >= 10 * sms) {
    tf32x3_gemm_ws<EPI, 256><<<std::min(n256, sms), WS_THREADS, WsCfg<256>::SMEM, s>>>(g);
  } else {
    const int n128 = g.narr * ntiles_m_side * g.NB_TILES;
    tf32x3_gemm_ws<EPI, 128><<<std::min(n128, sms), WS_THREADS, WsCfg<128>::SMEM, s>>>(g);
  }
  return cudaGetLastError();
}

cudaError_t launch_tf32_w_images(const double* W, int ldw, int J, int nz, const Tf32BandImages& b, cudaStream_t s) {
  const int Zp = tf32_zpad(nz);
  dim3 grid((b.Jp + 127) / 128, Zp);
  w_image_kernel<<<grid, 128, 0, s>>>(W, ldw, J, b.Jp, nz, Zp, b.a1h, b.a1l, b.a2h, b.a2l);
  return cudaGetLastError();
}

cudaError_t launch_band_tf32(const ArrayList& arrs, int narr, const Tf32BandImages& b, const Tf32Scratch& w, int nx,
                             int nz, float inv2, unsigned* err, cudaStream_t s) {
  if (narr < 1) return cudaErrorInvalidValue;
  const int Zp = tf32_zpad(nz);
  const int NT = tf32_ntiles(nx), KT1 = Zp / TT_K, MT1 = b.Jp / TT_M, KT2 = b.Jp / TT_K, MT2 = Zp / TT_M;
  g_image_kernel<<<dim3(NT, KT1, narr), 256, 0, s>>>(arrs, nx, nz, NT, KT1, w.gh, w.gl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  Tf32GemmArgs g1{};
  g1.a_hi = b.a1h;  // Wt image [j-tile][KT1]
  g1.a_lo = b.a1l;
  g1.b_hi = w.gh;   // G image [array][x-tile][KT1]
  g1.b_lo = w.gl;
  g1.KT = KT1;
  g1.NT = NT;
  g1.MT = MT1;
  g1.NB_TILES = NT;  // N = x
  g1.narr = narr;
  g1.c_hi = w.ch;
  g1.c_lo = w.cl;
  g1.KT2 = KT2;
  g1.scale = inv2;
  g1.arrs = arrs;
  g1.nx = nx;
  g1.nz = nz;
  g1.err = err;
  e = launch_gemm<EPI_COEF>(g1, MT1, sms, s);
  if (e != cudaSuccess) return e;
  Tf32GemmArgs g2 = g1;
  g2.a_hi = w.ch;   // C^T image [array][x-tile][KT2]
  g2.a_lo = w.cl;
  g2.b_hi = b.a2h;  // W image [z-tile][KT2]
  g2.b_lo = b.a2l;
  g2.KT = KT2;
  g2.MT = MT2;
  g2.NB_TILES = MT2;  // N = z
  return launch_gemm<EPI_APPLY>(g2, NT, sms, s);
}

}  // namespace ymkh
