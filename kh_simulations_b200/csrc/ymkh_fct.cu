// ymkh_fct.cu — fused flux-corrected transport of both beams.
//
// One launch replaces, per time step, the reference's stages 1-4
// (ymgpu2d/main_ym.cu:324-355): velocities (YM_Fluid.cu:3-11), the four D2D
// state copies (YM_Fluid.cu:134-143), the periodic x-sweep with ghost padding
// (YM_FCT.cu:47-91) or the wall x-sweep (YM_FCT.cu:30-45), the transposed
// z-sweep (YM_FCT.cu:93-135, FCT_Sweeps.cu:12-177) and the density floor /
// wall boundary (YM_Fluid.cu:13-30), for all six swept variables
// (n, px, pz, Q1..Q3) of both beams.  The momentum and colour sources the
// reference stores at the end of the previous step (kernel_ym_lorentz,
// kernel_ym_precession, YM_Fluid.cu:32-108) are recomputed here from the
// start-of-step state, which is what they are a function of.
//
// Layout: work items are (x-strip, z-segment) pairs; for a lone run each
// persistent CTA takes a contiguous block of them and runs each strip's part
// as one piece, for batches the CTAs take them round-robin.  A strip emits TB-6 columns; thread t of a beam owns
// stage position t+1 (shear index x0-3+t), and every x-sweep phase is at
// most one position or interface per thread: interface quantities (eps, nu,
// mu, low-order fluxes) are formed once per interface.  Threads [0,TB)
// handle beam A, [TB,2TB) beam B; the beams synchronise only through their
// own named barriers.  Row data (12 fluid arrays plus the field rows the
// sources need) is staged in shared memory NST-1 rows ahead: TMA bulk row
// copies (cp.async.bulk, split at the periodic wrap), one per thread spread
// over all warps, complete on a per-stage mbarrier; wall boundaries use
// per-element cp.async with clamped indices.  For each row the x-sweep
// (FCT_Sweeps.cu:88-162) runs across the strip in shared memory; its result
// for the thread's own column feeds a register pipeline that performs the
// z-sweep along the stream, emitting row r-3 once row r arrives (halo 3,
// zero-gradient clamped z ends as FCT_Sweeps.cu:68-81).
//
// HBM traffic per cell: 24 arrays read (12 fluid + 12 fields), 12 written;
// row and column halos come from L2/shared memory.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

// Stage layout (units of W doubles); stage position sp holds shear index
// x = x0 - 4 + sp, sp in [0, W) with W = TB + 2.
constexpr int ST_FL = 0;     // fluid: (beam*6 + var)
constexpr int ST_EX = 12;    // Ex1..3 row zr
constexpr int ST_BY = 15;    // By1..3 row zr
constexpr int ST_BYM = 18;   // By1..3 row zm
constexpr int ST_EZ = 21;    // Ez1..3 row zr
constexpr int ST_EZM = 24;   // Ez1..3 row zm
constexpr int ST_AZ = 27;    // Az1..3 row zr
constexpr int ST_AZM = 30;   // Az1..3 row zm
constexpr int ST_NZP = 33;   // n (beam A, B) row zp (warm_T only)
constexpr int ST_NZM = 35;   // n (beam A, B) row zm (warm_T only)
constexpr int ST_SIZE = 37;

// Per-beam work arrays (units of W), by stage position / interface index
// (interface j+1/2 stored at j).  Fluxes F, D are dead after phase B, so the
// limited fluxes reuse their space.  WB_SZ holds the pz z-source of the last
// two rows (slot r & 1): the Q group forms it, the n/px/pz group uses it one
// row later, which keeps the two groups' work per row about equal.
constexpr int WB_F = 1, WB_D = 7, WB_FLIM = 1, WB_LOR = 13, WB_LNR = 19, WB_SZ = 25, WB_SIZE = 27;

// Named barrier of one (beam, half) thread group (ids 1..4; 0 is __syncthreads).
__device__ __forceinline__ void beam_bar(int group, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(nthreads) : "memory");
}

// apply_fct_limiter (FCT_DeviceMath.cuh:108-125) with the products by
// copysign(1, d0) written as flips of the sign bit: multiplying by -1 is an
// exact negation, i.e. the same bits.  The inner minima may differ from
// fmin's only in the sign of a zero, which max_sel(+0, .) removes.
__device__ __forceinline__ double flip_sign(double x, unsigned long long m) {
  return __longlong_as_double(__double_as_longlong(x) ^ m);
}
__device__ __forceinline__ double fct_limit_sel(double f, double dm1, double d0, double dp1) {
  const unsigned long long m = (unsigned long long)__double_as_longlong(d0) & 0x8000000000000000ull;
  const double r = max_sel(0.0, min_sel(flip_sign(dm1, m), min_sel(fabs(f), flip_sign(dp1, m))));
  return flip_sign(r, m);
}

}  // namespace

template <int TB>
constexpr size_t fct_smem_bytes(int nst) {
  return (size_t)(TB + 2) * sizeof(double) * (nst * ST_SIZE + 2 * WB_SIZE) + (size_t)(TB + 2) * sizeof(int) +
         (size_t)8 * nst + 16;
}


// The half of a thread group as a compile-time constant: the row loop is
// compiled once per half, with the swept variables' shared-memory offsets,
// which variables carry z-sources and which source each half forms fixed
// (1.0% faster at 4096 x 8192 than one loop that branches on the half).
template <int V>
struct HalfC {
  static constexpr int value = V;
};

// One TMA bulk row copy of a stage (the table in fct_fused_kernel).
struct RowCopy {
  const double* base;
  const double* base0;
  int dst, kind, len1, pad_;
};

// Per-thread z-pipeline state for the three swept variables of one half
// (H = 0: n, px, pz; H = 1: Q1, Q2, Q3) of one beam.
struct ZPipe {
  double V1[3], f1[3], d1[3], L2[3], N4[3], N3[3], N2[3], A2[3], F3[3], S1[3];
  double U1, mu1;
};

template <int TB, int NST>
__global__ void __launch_bounds__(4 * TB, (TB >= 128 ? 1 : 2))
    fct_fused_kernel(const __grid_constant__ RunTable T) {
  constexpr int W = TB + 2;
  constexpr int NT = 4 * TB;
  constexpr int TO = TB - 6;  // output columns per strip
  extern __shared__ __align__(16) double smem[];
  double* const stage = smem;
  double* const wk = smem + (size_t)NST * ST_SIZE * W;
  int* const xtab = reinterpret_cast<int*>(wk + (size_t)2 * WB_SIZE * W);
  uint64_t* const bars = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(xtab + W) + 15) & ~static_cast<uintptr_t>(15));

  __shared__ RunDesc rd;
  __shared__ int s_run;
  __shared__ RowCopy cpt[40];
  const State& st = rd.in;
  const State& out = rd.out;
  const StepParams& p = rd.p;
  const int tid = threadIdx.x;
  const int grp = tid / TB;     // (beam, half) group, 0..3
  const int beam = grp >> 1;
  const int half = grp & 1;     // 0: n, px, pz   1: Q1, Q2, Q3
  const int t = tid - grp * TB;
  const int sp = t + 1;         // this thread's stage position
  double* const wb = wk + (size_t)beam * WB_SIZE * W;

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned issued = 0, consumed = 0;  // rows issued / consumed by this CTA (all items)
  unsigned phase_bits = 0;            // per-stage mbarrier phase of the bulk path

  // Lone run (T.fct_contig): each CTA takes one contiguous block of the
  // flattened items.  Within a run the items are strip-major (a strip's
  // z-segments consecutive), and consecutive segments of one strip form one
  // piece: the z pipeline warms up (6 rows) once per piece instead of once
  // per segment, and the blocks differ by at most one segment.  Batches
  // take segment-major items round-robin, so the CTAs running at once work
  // on neighbouring strips of the same rows and share halos through L2
  // (3.5% faster on an uneven 64-run sweep).
  const bool contig = T.fct_contig != 0;
  const int per = contig ? (T.fct_items + (int)gridDim.x - 1) / (int)gridDim.x : 0;
  const int i_beg = contig ? (int)blockIdx.x * per : (int)blockIdx.x;
  const int i_end = contig ? min(T.fct_items, i_beg + per) : T.fct_items;
  int next = i_beg;
  for (int item = i_beg; item < i_end; item = next) {
    __syncthreads();  // previous piece fully consumed
    if (tid == 0) s_run = find_run(T.runs, T.nruns, item, false);
    __syncthreads();
    load_desc(&rd, &T.runs[s_run]);
    __syncthreads();
    const int nx = p.nx, nz = p.nz;
    const bool warm = p.warm_T > 0.0;
    const bool wall = !p.periodic_x;
    const bool bulk = rd.fct_bulk == LOAD_BULK_ALL;  // TMA bulk rows on mbarriers (else per-element cp.async)
    const double dt = p.dt;
    const double dtdx = p.dt / p.dx;
    const double dtdz = p.dt / p.dz;
    const int nseg = (nz + rd.fct_seg - 1) / rd.fct_seg;
    const int local = item - rd.fct_item0;
    int strip, zs, ze;
    if (contig) {
      strip = local / nseg;
      const int seg0 = local - strip * nseg;
      next = min(i_end, rd.fct_item0 + (strip + 1) * nseg);  // past this piece's last segment
      zs = seg0 * rd.fct_seg;
      ze = min(nz, (seg0 + (next - item)) * rd.fct_seg);
    } else {
      strip = local % rd.fct_nstrips;
      zs = (local / rd.fct_nstrips) * rd.fct_seg;
      ze = min(nz, zs + rd.fct_seg);
      next = item + (int)gridDim.x;
    }
    const int x0 = strip * TO;

    if (!bulk)
      for (int i = tid; i < W; i += NT) xtab[i] = xmap(x0 - 4 + i, nx, p.periodic_x);
    // the pz source before the first row is zero, as the pipeline's start
    for (int i = tid; i < 2 * 2 * W; i += NT) wk[(size_t)(i / (2 * W)) * WB_SIZE * W + WB_SZ * W + i % (2 * W)] = 0.0;
    __syncthreads();

    // bulk rows: the row copies of the item, one per array of the stage
    // (source array at the strip's first column and at column 0 for the part
    // past the periodic wrap, stage slot offset, which row, length before the
    // wrap) in a shared table read by the issuing thread
    if (bulk && tid < 33 + (warm ? 4 : 0)) {
      const int a = tid;
      const double* base;
      int dst, kind_row = 0;
      if (a < 12) {
        base = a < 6 ? st.a[a] : st.b[a - 6];
        dst = ST_FL + a;
      } else if (a < 33) {
        const int kind = (a - 12) / 3, c = (a - 12) - kind * 3;  // EX, BY, BYM, EZ, EZM, AZ, AZM
        base = (kind == 0) ? st.f[EX1 + c] : (kind <= 2) ? st.f[BY1 + c] : (kind <= 4) ? st.f[EZ1 + c] : st.f[AZ1 + c];
        dst = ST_EX + (a - 12);
        kind_row = (kind == 2 || kind == 4 || kind == 6) ? 1 : 0;
      } else {
        const int w = a - 33;  // NZP A, NZP B, NZM A, NZM B
        base = (w & 1) ? st.b[FN] : st.a[FN];
        dst = ST_NZP + w;
        kind_row = (w >> 1) ? 1 : 2;
      }
      int x = (x0 - 4) % nx;
      x = x < 0 ? x + nx : x;
      cpt[a].base = base + x;
      cpt[a].base0 = base;
      cpt[a].dst = dst;
      cpt[a].kind = kind_row;
      cpt[a].len1 = min(W, nx - x);
    }
    __syncthreads();

    auto issue_row = [&](int r) {
      const int s = (int)(issued % NST);
      double* sb = stage + (size_t)s * ST_SIZE * W;
      const int zr = zclamp(r, nz);
      const int zm = (zr == 0) ? nz - 1 : zr - 1;
      const int zp = (zr == nz - 1) ? 0 : zr + 1;
      const size_t ro = (size_t)zr * nx, rom = (size_t)zm * nx, rop = (size_t)zp * nx;
      const int narr = 33 + (warm ? 4 : 0);
      if (bulk) {
        // one row copy per thread, spread over the warps (lane-major) so no
        // single warp serialises the issue; completions that land before
        // thread 0 arms the stage only drive its transaction count negative,
        // and the phase cannot complete before that arrival.  The copy's
        // array, slot and wrap split are fixed per item (cp_*).
        if (tid == 0) mbar_expect_tx(&bars[s], (unsigned)(narr * W * 8));
        const int ca = (tid & 31) * (NT / 32) + (tid >> 5);  // lane-major over the warps
        if (ca < narr) {
          const RowCopy& c = cpt[ca];
          const int len1 = c.len1;
          if (dbg_ok(zr >= 0 && zr < nz && zm >= 0 && zm < nz && zp >= 0 && zp < nz && len1 > 0 && W - len1 <= nx &&
                         c.dst >= 0 && c.dst < ST_SIZE, T.err)) {
            const size_t off = c.kind == 0 ? ro : (c.kind == 1 ? rom : rop);
            double* const dst = sb + c.dst * W;
            bulk_g2s(dst, c.base + off, (unsigned)len1 * 8u, &bars[s]);
            if (len1 < W) bulk_g2s(dst + len1, c.base0 + off, (unsigned)(W - len1) * 8u, &bars[s]);
          }
        }
      } else {
        const bool rows_ok = dbg_ok(zr >= 0 && zr < nz && zm >= 0 && zm < nz && zp >= 0 && zp < nz, T.err);
        for (int i = tid; i < 12 * (W - 1); i += NT) {
          const int a = i / (W - 1), q = 1 + (i - a * (W - 1));
          if (rows_ok && dbg_ok(xtab[q] >= 0 && xtab[q] < nx, T.err))
            cp_async8(sb + (ST_FL + a) * W + q, (a < 6 ? st.a[a] : st.b[a - 6]) + ro + xtab[q]);
        }
        for (int i = tid; i < 21 * (W - 1); i += NT) {
          const int a = i / (W - 1), q = 1 + (i - a * (W - 1));
          const int kind = a / 3, c = a - kind * 3;  // EX, BY, BYM, EZ, EZM, AZ, AZM
          const double* base = (kind == 0) ? st.f[EX1 + c]
                               : (kind <= 2) ? st.f[BY1 + c]
                               : (kind <= 4) ? st.f[EZ1 + c]
                                             : st.f[AZ1 + c];
          const size_t off = (kind == 2 || kind == 4 || kind == 6) ? rom : ro;
          if (rows_ok && dbg_ok(xtab[q] >= 0 && xtab[q] < nx, T.err))
            cp_async8(sb + (ST_EX + a) * W + q, base + off + xtab[q]);
        }
        if (warm) {
          for (int i = tid; i < 4 * (W - 1); i += NT) {
            const int a = i / (W - 1), q = 1 + (i - a * (W - 1));
            const double* base = (a & 1) ? st.b[FN] : st.a[FN];
            if (rows_ok && dbg_ok(xtab[q] >= 0 && xtab[q] < nx, T.err))
              cp_async8(sb + (ST_NZP + a) * W + q, base + ((a >> 1) ? rom : rop) + xtab[q]);
          }
        }
        cp_async_commit();
      }
      ++issued;
    };

    const int r_first = zs - 3, r_last = ze + 2;
    for (int k = 0; k < NST - 1; ++k)
      if (r_first + k <= r_last) issue_row(r_first + k);
      else if (!bulk) cp_async_commit();

    // the piece's rows, for this thread's half (a compile-time constant here)
    auto rows = [&](auto HC) {
      constexpr int half = decltype(HC)::value;
      constexpr int k0 = 3 * half;  // first swept variable of this half
      ZPipe zp;
#pragma unroll
      for (int j = 0; j < 3; ++j)
        zp.V1[j] = zp.f1[j] = zp.d1[j] = zp.L2[j] = zp.N4[j] = zp.N3[j] = zp.N2[j] = zp.A2[j] = zp.F3[j] = zp.S1[j] = 0.0;
      zp.U1 = zp.mu1 = 0.0;
      const int x_own = x0 - 4 + sp;
      const bool zthread = (t >= 3) && (t < TB - 3);  // owns an output column
      const bool owner = zthread && (x_own < nx);

      for (int r = r_first; r <= r_last; ++r) {
        const int s = (int)(consumed % NST);
        if (bulk) {  // one thread polls the stage's mbarrier; the CTA barrier below
          // releases the others after it (no spinning by every thread)
          if (tid == 0) mbar_wait(&bars[s], (phase_bits >> s) & 1u, T.err);
          phase_bits ^= 1u << s;
        } else {
          cp_async_wait<NST - 2>();
        }
        __syncthreads();  // row r staged for everyone; the previous row's stage is free
        ++consumed;
        if (r + NST - 1 <= r_last) issue_row(r + NST - 1);
        else if (!bulk) cp_async_commit();
        const double* sb = stage + (size_t)s * ST_SIZE * W;
        const double* fl = sb + (size_t)(ST_FL + beam * 6) * W;

        // ---- A: velocities at sp, sp+1 (YM_Fluid.cu:3-11); interface sp+1/2:
        // eps, nu, mu and the low-order fluxes of this half's variables
        // (FCT_Sweeps.cu:88-98); half 0 also forms the px source at sp
        // (YM_Fluid.cu:43-66, 71-80).
        double vz_own, ux_own, mu_if = 0.0, sx = 0.0;
        double Fo[3] = {0.0, 0.0, 0.0}, Do[3] = {0.0, 0.0, 0.0};  // this thread's interface fluxes
        {
          const double n0 = max_sel(fl[FN * W + sp], 0.05);
          ux_own = fl[FPX * W + sp] / n0;
          vz_own = fl[FPZ * W + sp] / n0;
          if (t < TB - 1) {
            const double n1 = max_sel(fl[FN * W + sp + 1], 0.05);
            const double u1 = fl[FPX * W + sp + 1] / n1;
            const double e = fct_eps(ux_own, u1, dtdx);
            double nu;
            fct_nu_mu(e, nu, mu_if);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const int k = k0 + j;
              const double v0 = fl[k * W + sp], v1 = fl[k * W + sp + 1];
              Fo[j] = 0.5 * e * (v0 + v1);
              Do[j] = nu * (v1 - v0);
              wb[(WB_F + k) * W + sp] = Fo[j];
              wb[(WB_D + k) * W + sp] = Do[j];
            }
          }
          if (half == 0 && t >= 1 && t < TB - 1) {
            int ps = sp;  // at a wall the clamped ghost cells carry the edge cell's source
            if (wall) {
              const int xg = x0 - 4 + sp;
              ps = (xg < 0 ? 0 : (xg >= nx ? nx - 1 : xg)) - (x0 - 4);
            }
            const double vz = (ps == sp) ? vz_own : fl[FPZ * W + ps] / max_sel(fl[FN * W + ps], 0.05);
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const double ex = 0.5 * (sb[(ST_EX + c) * W + ps] + sb[(ST_EX + c) * W + ps - 1]);
              const double by = 0.25 * (sb[(ST_BY + c) * W + ps] + sb[(ST_BY + c) * W + ps - 1] +
                                        sb[(ST_BYM + c) * W + ps] + sb[(ST_BYM + c) * W + ps - 1]);
              const double term = fl[(FQ1 + c) * W + ps] * (ex + vz * by);
              acc = (c == 0) ? term : acc + term;
            }
            sx = -acc;
            if (warm) {
              const double dndx = (fl[FN * W + ps + 1] - fl[FN * W + ps - 1]) / (2.0 * p.dx);
              sx -= p.warm_T * dndx;
            }
          }
        }
        beam_bar(grp, TB);

        // ---- B: lorhot / lnrhot at sp (FCT_Sweeps.cu:102-103), t in [1, TB-1).
        double Lo[3] = {0.0, 0.0, 0.0}, Ln[3] = {0.0, 0.0, 0.0};  // this thread's lorhot, lnrhot
        if (t >= 1 && t < TB - 1) {
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int k = k0 + j;
            const double v0 = fl[k * W + sp];
            const double fd = Fo[j] - wb[(WB_F + k) * W + sp - 1];
            const double dd = Do[j] - wb[(WB_D + k) * W + sp - 1];
            const double lo = (k == FPX) ? v0 + dt * sx - fd : v0 - fd;
            Lo[j] = lo;
            Ln[j] = lo + dd;
            wb[(WB_LOR + k) * W + sp] = lo;
            wb[(WB_LNR + k) * W + sp] = Ln[j];
          }
        }
        beam_bar(grp, TB);

        // ---- C: antidiffusive flux and limiter at interface sp+1/2
        // (FCT_Sweeps.cu:139-160), t in [2, TB-3).
        double Fl[3] = {0.0, 0.0, 0.0};  // this thread's limited flux
        if (t >= 2 && t < TB - 3) {
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int k = k0 + j;
            const double* lor = wb + (WB_LOR + k) * W;
            const double* lnr = wb + (WB_LNR + k) * W;
            const double l1 = lnr[sp + 1];
            const double fad = mu_if * (lor[sp + 1] - Lo[j]);
            Fl[j] = fct_limit_sel(fad, Ln[j] - lnr[sp - 1], l1 - Ln[j], lnr[sp + 2] - l1);
            wb[(WB_FLIM + k) * W + sp] = Fl[j];
          }
        }
        beam_bar(grp, TB);

        // ---- D: x-swept values of the own column, z-sources, z-pipeline.
        if (zthread) {
          double Vx[3], S[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int k = k0 + j;
            Vx[j] = Ln[j] - (Fl[j] - wb[(WB_FLIM + k) * W + sp - 1]);
          }
          const double vz = vz_own;
          const double q1 = fl[FQ1 * W + sp], q2 = fl[FQ2 * W + sp], q3 = fl[FQ3 * W + sp];
          if (half == 0) {
            // the pz source of row r-1, formed by the Q group last row
            S[0] = 0.0;
            S[1] = 0.0;
            S[2] = 0.0;
            zp.S1[2] = wb[(WB_SZ + ((r - 1) & 1)) * W + sp];
          } else {
            // YM_Fluid.cu:67 (src.pz) and :76-79 (warm closure), for the other group
            const double vx = ux_own;
            double by[3], ezn[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              by[c] = 0.25 * (sb[(ST_BY + c) * W + sp] + sb[(ST_BY + c) * W + sp - 1] + sb[(ST_BYM + c) * W + sp] +
                              sb[(ST_BYM + c) * W + sp - 1]);
              ezn[c] = 0.5 * (sb[(ST_EZ + c) * W + sp] + sb[(ST_EZM + c) * W + sp]);
            }
            double sz = -(q1 * (ezn[0] - vx * by[0]) + q2 * (ezn[1] - vx * by[1]) + q3 * (ezn[2] - vx * by[2]));
            if (warm) {
              const double dndz = (sb[(ST_NZP + beam) * W + sp] - sb[(ST_NZM + beam) * W + sp]) / (2.0 * p.dz);
              sz -= p.warm_T * dndz;
            }
            wb[(WB_SZ + (r & 1)) * W + sp] = sz;
            // YM_Fluid.cu:99-107 (colour precession)
            double azn[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) azn[c] = 0.5 * (sb[(ST_AZ + c) * W + sp] + sb[(ST_AZM + c) * W + sp]);
            S[0] = p.alpha * vz * (q2 * azn[2] - q3 * azn[1]);
            S[1] = p.alpha * vz * (q3 * azn[0] - q1 * azn[2]);
            S[2] = p.alpha * vz * (q1 * azn[1] - q2 * azn[0]);
          }

          const double e = fct_eps(zp.U1, vz, dtdz);
          double nu, mu;
          fct_nu_mu(e, nu, mu);
          double outv[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const bool has_src = (half == 1) || (j == 2);  // pz and Q1..Q3 carry z-sources
            const double fR = 0.5 * e * (zp.V1[j] + Vx[j]);
            const double dR = nu * (Vx[j] - zp.V1[j]);
            const double lo = has_src ? zp.V1[j] + dt * zp.S1[j] - (fR - zp.f1[j]) : zp.V1[j] - (fR - zp.f1[j]);
            const double ln = lo + (dR - zp.d1[j]);
            const double fad = zp.mu1 * (lo - zp.L2[j]);
            const double flim = fct_limit_sel(zp.A2[j], zp.N3[j] - zp.N4[j], zp.N2[j] - zp.N3[j], ln - zp.N2[j]);
            outv[j] = zp.N3[j] - (flim - zp.F3[j]);
            zp.V1[j] = Vx[j];
            zp.S1[j] = S[j];
            zp.f1[j] = fR;
            zp.d1[j] = dR;
            zp.L2[j] = lo;
            zp.N4[j] = zp.N3[j];
            zp.N3[j] = zp.N2[j];
            zp.N2[j] = ln;
            zp.A2[j] = fad;
            zp.F3[j] = flim;
          }
          zp.U1 = vz;
          zp.mu1 = mu;
          const int o = r - 3;
          if (owner && o >= zs && o < ze) {
            // YM_Fluid.cu:20-29 (density floor, wall momentum)
            if (half == 0) {
              if (outv[0] < 0.05) outv[0] = 0.05;
              if (wall && (x_own == 0 || x_own == nx - 1)) outv[1] = 0.0;
            }
            double* const* dst = beam ? out.b : out.a;
            const size_t gi = idx2(x_own, o, nx);
            if (dbg_ok(x_own >= 0 && x_own < nx && o >= 0 && o < nz && sp >= 1 && sp + 2 < W, T.err)) {
#pragma unroll
              for (int j = 0; j < 3; ++j) dst[k0 + j][gi] = outv[j];
            }
          }
        }
      }
    };
    if (half == 0) rows(HalfC<0>{});
    else rows(HalfC<1>{});
    if (!bulk) cp_async_wait<0>();
  }
}

template <int TB, int NST>
static cudaError_t prepare_fct_t() {
  return cudaFuncSetAttribute(fct_fused_kernel<TB, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fct_smem_bytes<TB>(NST));
}

// Stage ring depth (rows in flight = NST - 1).  Measured on B200 with
// 128-wide strips, step ms at 4096 x 8192 / 1024 x 2048: 7.38 / 0.522 with
// 2 stages, 7.18 / 0.505 with 3, 7.06 / 0.497 with 4 (206 KB of shared
// memory; 5 stages do not fit).  64-wide strips run 2 CTAs of 4 stages per SM.
template <int TB>
constexpr int fct_nst() {
  return 4;
}

int fct_nstrips(int nx, int tb) { return (nx + (tb - 6) - 1) / (tb - 6); }

int fct_bulk_ok(const StepParams& p, int tb) { return (p.periodic_x && (p.nx % 2) == 0 && p.nx >= tb + 2) ? 1 : 0; }

// The kernel reads start-of-step values across strip and segment halos while
// other CTAs write theirs, so each run's fluid goes to its second buffer
// (`out`); fields are only read.  grid_ctas persistent CTAs take contiguous
// blocks of the flattened (run, strip, segment) items.
cudaError_t launch_fct_table(const RunTable& T, int tb, int grid_ctas, cudaStream_t s) {
  const int grid = std::max(1, std::min(T.fct_items, grid_ctas));
  switch (tb) {
    case 32: fct_fused_kernel<32, fct_nst<32>()><<<grid, 128, fct_smem_bytes<32>(fct_nst<32>()), s>>>(T); break;
    case 64: fct_fused_kernel<64, fct_nst<64>()><<<grid, 256, fct_smem_bytes<64>(fct_nst<64>()), s>>>(T); break;
    case 128: fct_fused_kernel<128, fct_nst<128>()><<<grid, 512, fct_smem_bytes<128>(fct_nst<128>()), s>>>(T); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t prepare_fct(int tb) {
  switch (tb) {
    case 32: return prepare_fct_t<32, fct_nst<32>()>();
    case 64: return prepare_fct_t<64, fct_nst<64>()>();
    case 128: return prepare_fct_t<128, fct_nst<128>()>();
    default: return cudaErrorInvalidValue;
  }
}

int fct_ctas_per_sm(int tb) {
  int n = 0;
  switch (tb) {
    case 32: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fct_fused_kernel<32, fct_nst<32>()>, 128, fct_smem_bytes<32>(fct_nst<32>())); break;
    case 64: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fct_fused_kernel<64, fct_nst<64>()>, 256, fct_smem_bytes<64>(fct_nst<64>())); break;
    case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fct_fused_kernel<128, fct_nst<128>()>, 512, fct_smem_bytes<128>(fct_nst<128>())); break;
    default: break;
  }
  return n;
}

}  // namespace ymkh
