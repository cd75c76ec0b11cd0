// ymkh_fct_split.cu — the flux-corrected transport as two coalesced passes.
//
// Same arithmetic as fct_fused_kernel (ymkh_fct.cu; reference:
// ymgpu2d/FCT_Sweeps.cu:39-177, YM_FCT.cu:30-135, YM_Fluid.cu:3-108), but
// split at the x-swept intermediate, which goes to a 12-array scratch:
//
//  fct_x_kernel  one CTA per (run, x-strip of XB columns, row, beam): every
//                thread loads its own cells with plain coalesced loads, the
//                x-sweep phases exchange neighbours through shared memory,
//                and the x-swept values of the 6 variables are stored.
//  fct_z_kernel  one thread per (run, column, beam, variable half, z-segment)
//                streaming along z: no shared memory and no barriers; each
//                row's inputs are read straight from global memory one row
//                ahead, the z-sweep runs in registers (halo 3, clamped ends).
//
// HBM per cell: x pass 21 arrays read (12 fluid + Ex, By at two rows),
// 12 written; z pass 33 read (12 x-swept, 12 start-of-step fluid, Ez, By,
// Az), 12 written.  More bytes than the fused single pass, but every access
// is a full-warp coalesced stream, which keeps many loads in flight.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

constexpr int XT = 64;        // x-sweep positions per CTA (per beam)
constexpr int XO = XT - 6;    // x-swept columns produced per CTA

// apply_fct_limiter (FCT_DeviceMath.cuh:108-125); the products by
// copysign(1, d0) are sign-bit flips (multiplying by -1 negates exactly)
__device__ __forceinline__ double flip_sign2(double x, unsigned long long m) {
  return __longlong_as_double(__double_as_longlong(x) ^ m);
}
__device__ __forceinline__ double fct_limit_sel2(double f, double dm1, double d0, double dp1) {
  const unsigned long long m = (unsigned long long)__double_as_longlong(d0) & 0x8000000000000000ull;
  const double r = max_sel(0.0, min_sel(flip_sign2(dm1, m), min_sel(fabs(f), flip_sign2(dp1, m))));
  return flip_sign2(r, m);
}

}  // namespace

int fctx_nstrips(int nx) { return (nx + XO - 1) / XO; }

// Items of the x pass: (strip, row, beam); of the z pass: (column block of
// 32, segment, beam, half) — both flattened per run via RunDesc.fx_item0 /
// fz_item0 (stored in the split fields of the descriptor).

// ------------------------------------------------------------------ x pass
// 2*XT threads: thread t of half h handles position x0-3+t for the
// variables 3h..3h+2 of the CTA's beam.
__global__ void __launch_bounds__(2 * XT)
    fct_x_kernel(const __grid_constant__ RunTable T) {
  __shared__ RunDesc rd;
  __shared__ double sF[6][XT], sD[6][XT], sLor[6][XT], sLnr[6][XT];
  const int tid = threadIdx.x;
  const int half = tid / XT;
  const int t = tid - half * XT;
  const int k0 = 3 * half;
  int cur_run = -1;

  for (int item = blockIdx.x; item < T.fx_items; item += gridDim.x) {
    const int r = find_run_split(T.runs, T.nruns, item, 0);
    if (r != cur_run) {
      __syncthreads();
      load_desc(&rd, &T.runs[r]);
      __syncthreads();
      cur_run = r;
    }
    const StepParams& p = rd.p;
    const State& st = rd.in;
    const int nx = p.nx, nz = p.nz;
    const int local = item - rd.fx_item0;
    const int beam = local & 1;
    const int rest = local >> 1;
    const int strip = rest % rd.fx_nstrips;
    const int z = rest / rd.fx_nstrips;
    const int x0 = strip * XO;
    const bool wall = !p.periodic_x;
    const double dt = p.dt, dtdx = p.dt / p.dx;
    const int xs = x0 - 3 + t;  // this thread's position (shear index)
    const int xm = xmap(xs, nx, p.periodic_x);
    const int xp = xmap(xs + 1, nx, p.periodic_x);
    const size_t row = (size_t)z * nx;
    double* const* fl = beam ? st.b : st.a;

    // ---- A: velocities at x and x+1, interface x+1/2, px source at x
    const double n0 = max_sel(fl[FN][row + xm], 0.05);
    const double u0 = fl[FPX][row + xm] / n0;
    const double n1 = max_sel(fl[FN][row + xp], 0.05);
    const double u1 = fl[FPX][row + xp] / n1;
    const double e = fct_eps(u0, u1, dtdx);
    double nu, mu;
    fct_nu_mu(e, nu, mu);
    double v0[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      v0[j] = fl[k0 + j][row + xm];
      const double v1 = fl[k0 + j][row + xp];
      sF[k0 + j][t] = 0.5 * e * (v0[j] + v1);
      sD[k0 + j][t] = nu * (v1 - v0[j]);
    }
    double sx = 0.0;
    if (half == 0) {
      // source of the clamped ghost cells is the edge cell's (wall case)
      const int xc = wall ? xm : xm;
      const int xcm = xmap(wall ? (xc == 0 ? 0 : xc - 1) : xs - 1, nx, p.periodic_x);
      const int zm = (z == 0) ? nz - 1 : z - 1;
      const size_t rowm = (size_t)zm * nx;
      const double vz = fl[FPZ][row + xc] / max_sel(fl[FN][row + xc], 0.05);
      double acc = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double* Ex = st.f[EX1 + c];
        const double* By = st.f[BY1 + c];
        const double ex = 0.5 * (Ex[row + xc] + Ex[row + xcm]);
        const double by = 0.25 * (By[row + xc] + By[row + xcm] + By[rowm + xc] + By[rowm + xcm]);
        const double term = fl[FQ1 + c][row + xc] * (ex + vz * by);
        acc = (c == 0) ? term : acc + term;
      }
      sx = -acc;
      if (p.warm_T > 0.0) {
        const int xcp = xmap(wall ? (xc == nx - 1 ? nx - 1 : xc + 1) : xs + 1, nx, p.periodic_x);
        const double dndx = (fl[FN][row + xcp] - fl[FN][row + xcm]) / (2.0 * p.dx);
        sx -= p.warm_T * dndx;
      }
    }
    __syncthreads();
    // ---- B: lorhot / lnrhot at x (positions 1..XT-2)
    if (t >= 1 && t < XT - 1) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int k = k0 + j;
        const double fd = sF[k][t] - sF[k][t - 1];
        const double dd = sD[k][t] - sD[k][t - 1];
        const double lo = (k == FPX) ? v0[j] + dt * sx - fd : v0[j] - fd;
        sLor[k][t] = lo;
        sLnr[k][t] = lo + dd;
      }
    }
    __syncthreads();
    // ---- C: limited antidiffusive flux at x+1/2 (positions 2..XT-4)
    double flim[3] = {0.0, 0.0, 0.0};
    if (t >= 2 && t < XT - 3) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int k = k0 + j;
        const double fad = mu * (sLor[k][t + 1] - sLor[k][t]);
        flim[j] = fct_limit_sel2(fad, sLnr[k][t] - sLnr[k][t - 1], sLnr[k][t + 1] - sLnr[k][t],
                                 sLnr[k][t + 2] - sLnr[k][t + 1]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 3; ++j) sF[k0 + j][t] = flim[j];  // F is dead: reuse for the limited flux
    __syncthreads();
    // ---- D: x-swept value at x (positions 3..XT-4), stored to scratch
    if (t >= 3 && t < XT - 3 && xs < nx) {
      double* const* xo = beam ? rd.xsw.b : rd.xsw.a;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int k = k0 + j;
        xo[k][row + xs] = sLnr[k][t] - (sF[k][t] - sF[k][t - 1]);
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ z pass
// One thread per (column, beam, half) streams a z-segment.  Each lane stages
// its own inputs for the next ZNST-1 rows in a per-warp shared-memory ring
// with 8-byte cp.async (no registers held by loads in flight), so every warp
// keeps ~2 rows of loads in flight while its z-pipeline (the registers of
// the fused kernel) consumes the current row.
constexpr int ZB = 32;    // columns per warp
constexpr int ZNST = 3;   // ring depth (rows)
constexpr int ZNV = 30;   // staged values per lane per row

// slot layout per lane and row
enum {
  ZV_X = 0,          // x-swept values of the half's 3 variables
  ZV_N = 3, ZV_PZ = 4, ZV_Q = 5,  // n, pz, Q1..Q3 (start of step)
  ZV_PX = 8,         // half 0: px
  ZV_BY = 9,         // half 0: By[c] at (x, zr), (xm, zr), (x, zm), (xm, zm): 9 + 4c + j
  ZV_EZ = 21,        // half 0: Ez[c] at zr, zm: 21 + 2c + j
  ZV_NZP = 27, ZV_NZM = 28,  // half 0, warm_T: n at zp, zm
  ZV_AZ = 9          // half 1: Az[c] at zr, zm: 9 + 2c + j
};

__global__ void __launch_bounds__(128)
    fct_z_kernel(const __grid_constant__ RunTable T) {
  __shared__ RunDesc rd;
  extern __shared__ __align__(16) double zring[];  // [4 warps][ZNST][ZNV][ZB]
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;  // 4 warps: (beam, half)
  const int beam = warp >> 1;
  const int half = warp & 1;
  const int k0 = 3 * half;
  double (*rg)[ZNV][ZB] = reinterpret_cast<double (*)[ZNV][ZB]>(zring + (size_t)warp * ZNST * ZNV * ZB);
  int cur_run = -1;

  for (int item = blockIdx.x; item < T.fz_items; item += gridDim.x) {
    const int r = find_run_split(T.runs, T.nruns, item, 1);
    if (r != cur_run) {
      __syncthreads();
      load_desc(&rd, &T.runs[r]);
      __syncthreads();
      cur_run = r;
    }
    const StepParams& p = rd.p;
    const int nx = p.nx, nz = p.nz;
    const int local = item - rd.fz_item0;
    const int cb = local % rd.fz_ncols;
    const int seg = local / rd.fz_ncols;
    const int x = cb * ZB + lane;
    const int zs = seg * rd.fz_seg;
    const int ze = min(nz, zs + rd.fz_seg);
    const bool active = x < nx;
    const int xc = active ? x : nx - 1;  // inactive lanes read a valid cell and emit nothing
    const int xcm = p.periodic_x ? (xc == 0 ? nx - 1 : xc - 1) : (xc == 0 ? 0 : xc - 1);
    const bool wall = !p.periodic_x;
    const bool warm = p.warm_T > 0.0;
    const double dt = p.dt, dtdz = p.dt / p.dz;
    const State& st = rd.in;
    double* const* fl = beam ? st.b : st.a;
    double* const* xsw = beam ? rd.xsw.b : rd.xsw.a;
    double* const* dst = beam ? rd.out.b : rd.out.a;

    auto issue = [&](int rr, int s) {
      const int zr = zclamp(rr, nz);
      const int zm = (zr == 0) ? nz - 1 : zr - 1;
      const size_t row = (size_t)zr * nx, rowm = (size_t)zm * nx;
      double (*sl)[ZB] = rg[s];
#pragma unroll
      for (int j = 0; j < 3; ++j) cp_async8(&sl[ZV_X + j][lane], xsw[k0 + j] + row + xc);
      cp_async8(&sl[ZV_N][lane], fl[FN] + row + xc);
      cp_async8(&sl[ZV_PZ][lane], fl[FPZ] + row + xc);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async8(&sl[ZV_Q + c][lane], fl[FQ1 + c] + row + xc);
      if (half == 0) {
        cp_async8(&sl[ZV_PX][lane], fl[FPX] + row + xc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double* By = st.f[BY1 + c];
          cp_async8(&sl[ZV_BY + 4 * c + 0][lane], By + row + xc);
          cp_async8(&sl[ZV_BY + 4 * c + 1][lane], By + row + xcm);
          cp_async8(&sl[ZV_BY + 4 * c + 2][lane], By + rowm + xc);
          cp_async8(&sl[ZV_BY + 4 * c + 3][lane], By + rowm + xcm);
          cp_async8(&sl[ZV_EZ + 2 * c + 0][lane], st.f[EZ1 + c] + row + xc);
          cp_async8(&sl[ZV_EZ + 2 * c + 1][lane], st.f[EZ1 + c] + rowm + xc);
        }
        if (warm) {
          const int zp = (zr == nz - 1) ? 0 : zr + 1;
          cp_async8(&sl[ZV_NZP][lane], fl[FN] + (size_t)zp * nx + xc);
          cp_async8(&sl[ZV_NZM][lane], fl[FN] + rowm + xc);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cp_async8(&sl[ZV_AZ + 2 * c + 0][lane], st.f[AZ1 + c] + row + xc);
          cp_async8(&sl[ZV_AZ + 2 * c + 1][lane], st.f[AZ1 + c] + rowm + xc);
        }
      }
    };

    const int r_first = zs - 3, r_last = ze + 2;
#pragma unroll
    for (int k = 0; k < ZNST - 1; ++k) {
      if (r_first + k <= r_last) issue(r_first + k, k);
      cp_async_commit();
    }

    double V1[3], f1[3], d1[3], L2[3], N4[3], N3[3], N2[3], A2[3], F3[3], S1[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) V1[j] = f1[j] = d1[j] = L2[j] = N4[j] = N3[j] = N2[j] = A2[j] = F3[j] = S1[j] = 0.0;
    double U1 = 0.0, mu1 = 0.0;

    for (int rr = r_first, it = 0; rr <= r_last; ++rr, ++it) {
      cp_async_wait<ZNST - 2>();
      __syncwarp();
      const double (*sl)[ZB] = rg[it % ZNST];
      double Vx[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) Vx[j] = sl[ZV_X + j][lane];
      const double n0 = max_sel(sl[ZV_N][lane], 0.05);
      const double vz = sl[ZV_PZ][lane] / n0;
      const double q1 = sl[ZV_Q + 0][lane], q2 = sl[ZV_Q + 1][lane], q3 = sl[ZV_Q + 2][lane];
      double S[3];
      if (half == 0) {
        // YM_Fluid.cu:44, 52-67 (src.pz) and :76-79 (warm closure)
        const double vx = sl[ZV_PX][lane] / n0;
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double by = 0.25 * (sl[ZV_BY + 4 * c + 0][lane] + sl[ZV_BY + 4 * c + 1][lane] +
                                    sl[ZV_BY + 4 * c + 2][lane] + sl[ZV_BY + 4 * c + 3][lane]);
          const double ez = 0.5 * (sl[ZV_EZ + 2 * c + 0][lane] + sl[ZV_EZ + 2 * c + 1][lane]);
          const double qa = (c == 0) ? q1 : (c == 1) ? q2 : q3;
          const double term = qa * (ez - vx * by);
          acc = (c == 0) ? term : acc + term;
        }
        double sz = -acc;
        if (warm) {
          const double dndz = (sl[ZV_NZP][lane] - sl[ZV_NZM][lane]) / (2.0 * p.dz);
          sz -= p.warm_T * dndz;
        }
        S[0] = 0.0;
        S[1] = 0.0;
        S[2] = sz;
      } else {
        // YM_Fluid.cu:99-107 (colour precession)
        double azn[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) azn[c] = 0.5 * (sl[ZV_AZ + 2 * c + 0][lane] + sl[ZV_AZ + 2 * c + 1][lane]);
        S[0] = p.alpha * vz * (q2 * azn[2] - q3 * azn[1]);
        S[1] = p.alpha * vz * (q3 * azn[0] - q1 * azn[2]);
        S[2] = p.alpha * vz * (q1 * azn[1] - q2 * azn[0]);
      }
      __syncwarp();
      // refill the slot consumed last iteration (row rr + ZNST - 1)
      {
        const int rn = rr + ZNST - 1;
        if (rn <= r_last) issue(rn, (it + ZNST - 1) % ZNST);
        cp_async_commit();
      }
      const double e = fct_eps(U1, vz, dtdz);
      double nu, mu;
      fct_nu_mu(e, nu, mu);
      double outv[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const bool has_src = (half == 1) || (j == 2);
        const double fR = 0.5 * e * (V1[j] + Vx[j]);
        const double dR = nu * (Vx[j] - V1[j]);
        const double lo = has_src ? V1[j] + dt * S1[j] - (fR - f1[j]) : V1[j] - (fR - f1[j]);
        const double ln = lo + (dR - d1[j]);
        const double fad = mu1 * (lo - L2[j]);
        const double flim = fct_limit_sel2(A2[j], N3[j] - N4[j], N2[j] - N3[j], ln - N2[j]);
        outv[j] = N3[j] - (flim - F3[j]);
        V1[j] = Vx[j];
        S1[j] = S[j];
        f1[j] = fR;
        d1[j] = dR;
        L2[j] = lo;
        N4[j] = N3[j];
        N3[j] = N2[j];
        N2[j] = ln;
        A2[j] = fad;
        F3[j] = flim;
      }
      U1 = vz;
      mu1 = mu;
      const int o = rr - 3;
      if (active && o >= zs && o < ze) {
        // YM_Fluid.cu:20-29 (density floor, wall momentum)
        if (half == 0) {
          if (outv[0] < 0.05) outv[0] = 0.05;
          if (wall && (x == 0 || x == nx - 1)) outv[1] = 0.0;
        }
        const size_t gi = (size_t)o * nx + x;
#pragma unroll
        for (int j = 0; j < 3; ++j) dst[k0 + j][gi] = outv[j];
      }
    }
    cp_async_wait<0>();
    __syncwarp();
  }
}

int fctz_ncols(int nx) { return (nx + ZB - 1) / ZB; }

constexpr size_t fctz_smem_bytes() { return (size_t)4 * ZNST * ZNV * ZB * sizeof(double); }

cudaError_t prepare_fct_split() {
  return cudaFuncSetAttribute(fct_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fctz_smem_bytes());
}

cudaError_t launch_fct_split_table(const RunTable& T, int grid_x, int grid_z, cudaStream_t s) {
  fct_x_kernel<<<std::max(1, std::min(T.fx_items, grid_x)), 2 * XT, 0, s>>>(T);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  fct_z_kernel<<<std::max(1, std::min(T.fz_items, grid_z)), 128, fctz_smem_bytes(), s>>>(T);
  return cudaGetLastError();
}

int fct_split_ctas_per_sm(int which) {
  int n = 0;
  if (which == 0)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fct_x_kernel, 2 * XT, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fct_z_kernel, 128, fctz_smem_bytes());
  return n;
}

}  // namespace ymkh
