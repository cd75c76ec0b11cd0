// ymkh_maxwell.cu — fused non-Abelian Maxwell update.
//
// One launch replaces stages 5-6 of the reference step
// (ymgpu2d/main_ym.cu:357-363): colour currents (YM_Physics.cu:9-60),
// Ampère (YM_Physics.cu:70-113), potential (YM_Physics.cu:589-599) and
// Faraday (YM_Physics.cu:120-151).  The currents are never stored.
//
// Layout: work items are (x-strip of TX columns, z-segment) pairs handed to
// persistent CTAs round-robin; a CTA streams along z with the rows it needs
// staged in shared memory NST-2 rows ahead (TMA bulk row copies, one per
// thread spread over all warps, completing on a per-stage mbarrier; wall
// boundaries use per-element cp.async with clamped indices).  When row q arrives
// it forms, for every column, the per-cell velocities px/n and pz/n of both
// beams (each division done once), then Ex(q) (Jx needs row q only) and
// Ez(q-1) (Jz needs rows q-1, q), and finally the potential and Faraday on
// row q-1, which need Ex at rows q-1, q and Ez at columns x, x+1.
//
// Reads the new fluid and the start-of-step fields from `in_*` and writes
// E, By, Az to `out`, a different buffer (neighbouring CTAs still read the
// old values).  HBM per cell: 24 arrays read, 12 written.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

// 126 output columns per strip: with 256 threads every phase is at most one
// item per thread (127 velocity columns per beam = 254 items, 126 Ex columns
// beside 127 Ez columns, Faraday's stores split over both halves), and the
// strip origin stays even, so staged rows start on 16-byte boundaries.
// The shape can be set at build time (YMKH_MX_TX/NT/NST/MINB) for sweeps;
// NT/2 >= TX + 1 keeps one item per thread per phase.  Measured at
// 4096 x 8192 on B200 (Maxwell ms): 126/256/3 1.895, 62/128/3 1.934,
// 30/64/3 2.207, 62/128/4 2.387.
#ifndef YMKH_MX_TX
#define YMKH_MX_TX 126
#define YMKH_MX_NT 256
#define YMKH_MX_NST 3
#define YMKH_MX_MINB 2
#endif
constexpr int MX_TX = YMKH_MX_TX;    // output columns per strip
constexpr int MX_NV = MX_TX + 1;     // velocity / Ez columns (one right neighbour)
constexpr int MX_NT = YMKH_MX_NT;    // threads per CTA: [0,NT/2) Ex / By half, [NT/2,NT) Ez / store half
constexpr int MX_NST = YMKH_MX_NST;  // stage ring depth: rows q-1, q in use, NST-2 rows in flight
constexpr int MX_W = MX_TX + 4;  // stage row: position s <-> x = x0 - 2 + s (66: even)

// stage offsets in rows of MX_W doubles (every array staged over the full row)
constexpr int MS_FL = 0;   // 12 fluid arrays
constexpr int MS_BY = 12;  // By1..3
constexpr int MS_AZ = 15;  // Az1..3
constexpr int MS_EX = 18;  // Ex1..3
constexpr int MS_EZ = 21;  // Ez1..3
constexpr int MS_SIZE = 24;

// work rows: per-cell velocities [2 rows][beam][px/n, pz/n], new Ex [2 rows][3], new Ez [3]
constexpr int MW_V = 0;
constexpr int MW_EX = 8;
constexpr int MW_EZ = 14;
constexpr int MW_SIZE = 17;

}  // namespace

constexpr size_t maxwell_smem_bytes() {
  return (size_t)MX_W * sizeof(double) * (MX_NST * MS_SIZE + MW_SIZE) + (size_t)MX_W * sizeof(int) +
         (size_t)8 * MX_NST + 16;
}

__global__ void __launch_bounds__(MX_NT, YMKH_MX_MINB)
    maxwell_fused_kernel(const __grid_constant__ RunTable T) {
  constexpr int TX = MX_TX, NV = MX_NV, W = MX_W, NST = MX_NST, NT = MX_NT;
  static_assert(2 * NV <= NT && TX <= NT / 2 && NV <= NT / 2, "one item per thread per phase");
  static_assert(W % 2 == 0 && TX % 2 == 0, "even strip origin and row length for 16-byte row copies");
  extern __shared__ __align__(16) double smem[];
  double* const stage = smem;
  double* const wk = smem + (size_t)NST * MS_SIZE * W;
  int* const xtab = reinterpret_cast<int*>(wk + (size_t)MW_SIZE * W);
  uint64_t* const bars = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(xtab + W) + 15) & ~static_cast<uintptr_t>(15));

  __shared__ RunDesc rd;
  __shared__ int s_run;
  // Reads the new fluid (the run's `out` fluid, written by the FCT) and the
  // start-of-step fields (`in`), writes the new fields to `out`.
  const State& fluid_new = rd.out;
  const State& fields_old = rd.in;
  const State& out = rd.out;
  const StepParams& p = rd.p;
  const int tid = threadIdx.x;

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned issued = 0, consumed = 0;
  unsigned phase_bits = 0;  // per-stage mbarrier phase of the bulk path

  for (int item = blockIdx.x; item < T.mx_items; item += gridDim.x) {
    __syncthreads();
    if (tid == 0) s_run = find_run(T.runs, T.nruns, item, true);
    __syncthreads();
    load_desc(&rd, &T.runs[s_run]);
    __syncthreads();
    const int nx = p.nx, nz = p.nz;
    const bool wall = !p.periodic_x;
    const bool bulk = rd.mx_bulk == LOAD_BULK_ALL;  // TMA bulk rows on mbarriers (else per-element cp.async)
    const double dt = p.dt, c2 = p.c2, al = p.alpha, e0 = p.eps0;
    // c = eps_0 = 1 (ymgpu2d/main_ym.cu:69): 1*x and x/1 are exact, so the
    // products and quotients by them can be skipped without changing a bit
    const bool unit = (c2 == 1.0 && e0 == 1.0);
    const int local = item - rd.mx_item0;
    const int x0 = (local % rd.mx_nstrips) * TX;
    const int zs = (local / rd.mx_nstrips) * rd.mx_seg;
    const int ze = min(nz, zs + rd.mx_seg);

    for (int i = tid; i < W; i += NT) xtab[i] = xmap(x0 - 2 + i, nx, p.periodic_x);
    __syncthreads();

    auto issue_row = [&](int q) {
      const int s = (int)(issued % NST);
      double* sb = stage + (size_t)s * MS_SIZE * W;
      const size_t ro = (size_t)zwrap(q, nz) * nx;
      auto arr = [&](int a) -> const double* {
        if (a < 12) return (a < 6) ? fluid_new.a[a] : fluid_new.b[a - 6];
        const int kind = (a - 12) / 3, c = (a - 12) % 3;
        return (kind == 0) ? fields_old.f[BY1 + c]
               : (kind == 1) ? fields_old.f[AZ1 + c]
               : (kind == 2) ? fields_old.f[EX1 + c]
                             : fields_old.f[EZ1 + c];
      };
      if (bulk) {
        // one row copy per thread, spread over the warps (lane-major); early
        // completions only drive the transaction count negative before
        // thread 0's arrival arms the phase
        if (tid == 0) mbar_expect_tx(&bars[s], (unsigned)(MS_SIZE * W * 8));
        const int a = (tid & 31) * (NT / 32) + (tid >> 5);
        if (a < MS_SIZE && dbg_ok(zwrap(q, nz) >= 0 && zwrap(q, nz) < nz && W <= nx && (x0 - 2) % 2 == 0, T.err))
          bulk_row_periodic(sb + a * W, arr(a) + ro, x0 - 2, W, nx, &bars[s]);
      } else {
        for (int i = tid; i < MS_SIZE * W; i += NT) {
          const int a = i / W, k = i - a * W;
          if (dbg_ok(zwrap(q, nz) >= 0 && zwrap(q, nz) < nz && xtab[k] >= 0 && xtab[k] < nx, T.err))
            cp_async8(sb + a * W + k, arr(a) + ro + xtab[k]);
        }
        cp_async_commit();
      }
      ++issued;
    };

    // Rows q-1 and q are read in the same iteration, so NST-2 rows are in
    // flight and the refill goes to the stage of row q-2.
    const int q_first = zs - 1, q_last = ze;
    for (int k = 0; k < NST - 2; ++k)
      if (q_first + k <= q_last) issue_row(q_first + k);
      else if (!bulk) cp_async_commit();

    for (int q = q_first; q <= q_last; ++q) {
      const int s = (int)(consumed % NST);
      const int sprev = (int)((consumed + NST - 1) % NST);
      if (bulk) {  // one thread polls the stage's mbarrier; the CTA barrier below
        // releases the others after it (no spinning by every thread)
        if (tid == 0) mbar_wait(&bars[s], (phase_bits >> s) & 1u, T.err);
        phase_bits ^= 1u << s;
      }
      else
        cp_async_wait<NST - 3>();
      __syncthreads();  // row q staged by every thread; row q-2's stage is free
      ++consumed;
      if (q + NST - 2 <= q_last) issue_row(q + NST - 2);
      else if (!bulk) cp_async_commit();
      const double* sb = stage + (size_t)s * MS_SIZE * W;      // row q
      const double* sp = stage + (size_t)sprev * MS_SIZE * W;  // row q-1
      const int rq = q & 1, rp = (q - 1) & 1;

      // ---- 1: per-cell velocities of row q at x in [x0, x0+TX] (YM_Physics.cu:22-25, 38-41)
      if (tid < 2 * NV) {
        const int b = tid / NV, k = 2 + (tid - b * NV);
        const double* fl = sb + (size_t)(MS_FL + 6 * b) * W;
        const double n = fmax(fl[FN * W + k], 1e-10);
        wk[(MW_V + rq * 4 + b * 2 + 0) * W + k] = fl[FPX * W + k] / n;
        wk[(MW_V + rq * 4 + b * 2 + 1) * W + k] = fl[FPZ * W + k] / n;
      }
      __syncthreads();

      if (tid < TX) {
        // ---- 2a: Ampère for Ex on row q, column x0+tid
        const int k = 2 + tid;
        double nq[2][3], vxr[2];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const double* fl = sb + (size_t)(MS_FL + 6 * b) * W;
          const double n0 = fl[FN * W + k], n1 = fl[FN * W + k + 1];
          vxr[b] = 0.5 * (wk[(MW_V + rq * 4 + b * 2) * W + k] + wk[(MW_V + rq * 4 + b * 2) * W + k + 1]);
#pragma unroll
          for (int a = 0; a < 3; ++a) nq[b][a] = 0.5 * (n0 * fl[(FQ1 + a) * W + k] + n1 * fl[(FQ1 + a) * W + k + 1]);
        }
        const double by1 = sb[(MS_BY + 0) * W + k], by2 = sb[(MS_BY + 1) * W + k], by3 = sb[(MS_BY + 2) * W + k];
        const double dz3[3] = {div_rn(by1 - sp[(MS_BY + 0) * W + k], p.dz, p.rdz), div_rn(by2 - sp[(MS_BY + 1) * W + k], p.dz, p.rdz),
                               div_rn(by3 - sp[(MS_BY + 2) * W + k], p.dz, p.rdz)};
        const double a1 = sb[(MS_AZ + 0) * W + k], a2 = sb[(MS_AZ + 1) * W + k], a3 = sb[(MS_AZ + 2) * W + k];
        const double kx[3] = {a2 * by3 - a3 * by2, a3 * by1 - a1 * by3, a1 * by2 - a2 * by1};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double jx = -(nq[0][a] * vxr[0] + nq[1][a] * vxr[1]);
          const double rhs = unit ? (-dz3[a] - al * kx[a]) - jx : c2 * (-dz3[a] - al * kx[a]) - jx / e0;
          wk[(MW_EX + rq * 3 + a) * W + k] = sb[(MS_EX + a) * W + k] + dt * rhs;
        }
      } else {
        // ---- 2b: Ampère for Ez on row q-1, columns [x0, x0+TX]
        const int i = tid - NT / 2;
        if (i >= 0 && i < NV) {
          const int k = 2 + i;
          double nqz[2][3], vzt[2];
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const double* f0 = sp + (size_t)(MS_FL + 6 * b) * W;
            const double* f1 = sb + (size_t)(MS_FL + 6 * b) * W;
            const double n0 = f0[FN * W + k], n1 = f1[FN * W + k];
            vzt[b] = 0.5 * (wk[(MW_V + rp * 4 + b * 2 + 1) * W + k] + wk[(MW_V + rq * 4 + b * 2 + 1) * W + k]);
#pragma unroll
            for (int a = 0; a < 3; ++a) nqz[b][a] = 0.5 * (n0 * f0[(FQ1 + a) * W + k] + n1 * f1[(FQ1 + a) * W + k]);
          }
          const int gx = xtab[k];
          const bool wz = wall && (gx == 0 || gx == nx - 1);  // YM_Fluid.cu:25-29
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const double jz = -(nqz[0][a] * vzt[0] + nqz[1][a] * vzt[1]);
            const double by = sp[(MS_BY + a) * W + k];
            const double dbx = div_rn(by - sp[(MS_BY + a) * W + k - 1], p.dx, p.rdx);
            const double ez0 = wz ? 0.0 : sp[(MS_EZ + a) * W + k];
            wk[(MW_EZ + a) * W + k] = ez0 + dt * (unit ? dbx - jz : c2 * dbx - jz / e0);
          }
        }
      }
      __syncthreads();
      // At a wall the right neighbour of the last column is the column itself
      // (YM_Physics.cu:127): its Ez is that column's new Ez.
      if (wall && x0 + TX >= nx) {
        if (tid < 3) {
          const int kl = 2 + (nx - 1 - x0);
          wk[(MW_EZ + tid) * W + kl + 1] = wk[(MW_EZ + tid) * W + kl];
        }
        __syncthreads();
      }

      // ---- 3: potential and Faraday on row q-1.  Threads [0, TX) form and
      // store By and Az of column x0+tid; threads [64, 64+TX) store the new
      // Ex and Ez of column x0+tid-64.
      const int o = q - 1;
      const int c3 = tid < NT / 2 ? tid : tid - NT / 2;
      if (c3 < TX && o >= zs && o < ze && x0 + c3 < nx &&
          dbg_ok(x0 + c3 >= 0 && o >= 0 && o < nz && 2 + c3 + 1 < W, T.err)) {
        const int k = 2 + c3;
        const size_t gi = idx2(x0 + c3, o, nx);
        double ex[3], ez[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          ex[a] = wk[(MW_EX + rp * 3 + a) * W + k];
          ez[a] = wk[(MW_EZ + a) * W + k];
        }
        if (tid < NT / 2) {
          double az[3];
#pragma unroll
          for (int a = 0; a < 3; ++a) az[a] = sp[(MS_AZ + a) * W + k];
          if (!p.freeze_az1) az[0] = az[0] - dt * ez[0];
          az[1] = az[1] - dt * ez[1];
          az[2] = az[2] - dt * ez[2];
          const double kk[3] = {az[1] * ex[2] - az[2] * ex[1], az[2] * ex[0] - az[0] * ex[2],
                                az[0] * ex[1] - az[1] * ex[0]};
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const double dex = div_rn(wk[(MW_EX + rq * 3 + a) * W + k] - ex[a], p.dz, p.rdz);
            const double dez = div_rn(wk[(MW_EZ + a) * W + k + 1] - ez[a], p.dx, p.rdx);
            out.f[BY1 + a][gi] = sp[(MS_BY + a) * W + k] - dt * (dex - dez - al * kk[a]);
            out.f[AZ1 + a][gi] = az[a];
          }
        } else {
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            out.f[EX1 + a][gi] = ex[a];
            out.f[EZ1 + a][gi] = ez[a];
          }
        }
      }
    }
    if (!bulk) cp_async_wait<0>();
  }
}

cudaError_t prepare_maxwell() {
  return cudaFuncSetAttribute(maxwell_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)maxwell_smem_bytes());
}

int maxwell_ctas_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, maxwell_fused_kernel, MX_NT, maxwell_smem_bytes());
  return n;
}

int maxwell_nstrips(int nx) { return (nx + MX_TX - 1) / MX_TX; }

int maxwell_bulk_ok(const StepParams& p) { return (p.periodic_x && (p.nx % 2) == 0 && p.nx >= MX_W) ? 1 : 0; }

cudaError_t launch_maxwell_table(const RunTable& T, int grid_ctas, cudaStream_t s) {
  const int grid = std::max(1, std::min(T.mx_items, grid_ctas));
  maxwell_fused_kernel<<<grid, MX_NT, maxwell_smem_bytes(), s>>>(T);
  return cudaGetLastError();
}

}  // namespace ymkh
