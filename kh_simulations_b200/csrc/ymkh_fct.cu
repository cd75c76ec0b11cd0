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
// Layout: a CTA owns an x-strip [x0, x0+TX) and a z-segment [zs, ze) and
// streams along z.  Threads [0,TX) handle beam A, [TX,2TX) beam B.  Row data
// (12 fluid arrays plus the field rows the sources need) is staged into
// shared memory with cp.async NST-1 rows ahead.  For each row the x-sweep
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

// Offsets (in units of W doubles) inside one stage buffer.
constexpr int ST_FL = 0;     // fluid: (beam*6 + var)
constexpr int ST_EX = 12;    // Ex1..3, row zr
constexpr int ST_BY = 15;    // By1..3, row zr
constexpr int ST_BYM = 18;   // By1..3, row zm
constexpr int ST_EZ = 21;    // Ez1..3, row zr
constexpr int ST_EZM = 24;   // Ez1..3, row zm
constexpr int ST_AZ = 27;    // Az1..3, row zr
constexpr int ST_AZM = 30;   // Az1..3, row zm
constexpr int ST_NZP = 33;   // n (beam A, B), row zp (warm_T only)
constexpr int ST_NZM = 35;   // n (beam A, B), row zm (warm_T only)
constexpr int ST_SIZE = 37;

// Work arrays (units of W): beam-shared node fields, then per beam.
constexpr int WK_EXN = 0, WK_BYN = 3, WK_EZN = 6, WK_AZN = 9, WK_SHARED = 12;
constexpr int WB_U = 0, WB_VZ = 1, WB_S = 2, WB_LOR = 3, WB_LNR = 9, WB_FLIM = 15, WB_SIZE = 21;

}  // namespace

template <int TX>
constexpr size_t fct_smem_bytes(int nst) {
  return (size_t)(TX + 8) * sizeof(double) * (nst * ST_SIZE + WK_SHARED + 2 * WB_SIZE) +
         (size_t)(TX + 8) * sizeof(int);
}

template <int TX, int NST>
__global__ void __launch_bounds__(2 * TX)
    fct_fused_kernel(const __grid_constant__ State st, const __grid_constant__ State out,
                     const __grid_constant__ StepParams p, int seg_len) {
  constexpr int W = TX + 8;
  constexpr int NT = 2 * TX;
  extern __shared__ __align__(16) double smem[];
  double* stage = smem;
  double* wk = smem + (size_t)NST * ST_SIZE * W;
  int* xtab = reinterpret_cast<int*>(wk + (size_t)(WK_SHARED + 2 * WB_SIZE) * W);

  const int nx = p.nx, nz = p.nz;
  const int tid = threadIdx.x;
  const int beam = tid / TX;
  const int t = tid - beam * TX;
  const int x0 = blockIdx.x * TX;
  const int zs = blockIdx.y * seg_len;
  const int ze = min(nz, zs + seg_len);
  if (zs >= nz) return;
  const bool warm = p.warm_T > 0.0;
  const double dt = p.dt;
  const double dtdx = p.dt / p.dx;
  const double dtdz = p.dt / p.dz;

  // Mapped shear index of every stage position p <-> x = x0 - 4 + p.
  for (int i = tid; i < W; i += NT) xtab[i] = xmap(x0 - 4 + i, nx, p.periodic_x);
  __syncthreads();

  auto issue_row = [&](int r, int s) {
    double* sb = stage + (size_t)s * ST_SIZE * W;
    const int zr = zclamp(r, nz);
    const int zm = (zr == 0) ? nz - 1 : zr - 1;
    const int zp = (zr == nz - 1) ? 0 : zr + 1;
    const size_t ro = (size_t)zr * nx, rom = (size_t)zm * nx, rop = (size_t)zp * nx;
    // 12 fluid rows, positions [1, TX+7)
    for (int i = tid; i < 12 * (TX + 6); i += NT) {
      const int a = i / (TX + 6), q = i - a * (TX + 6);
      const double* src = (a < 6 ? st.a[a] : st.b[a - 6]) + ro + xtab[1 + q];
      cp_async8(sb + (ST_FL + a) * W + 1 + q, src);
    }
    // Ex (zr), By (zr), By (zm), positions [1, TX+6)
    for (int i = tid; i < 9 * (TX + 5); i += NT) {
      const int a = i / (TX + 5), q = i - a * (TX + 5);
      const int c = a % 3;
      const double* base = (a < 3) ? st.f[EX1 + c] : st.f[BY1 + c];
      const double* src = base + (a < 6 ? ro : rom) + xtab[1 + q];
      cp_async8(sb + (ST_EX + a) * W + 1 + q, src);
    }
    // Ez (zr, zm), Az (zr, zm), positions [4, TX+4)
    for (int i = tid; i < 12 * TX; i += NT) {
      const int a = i / TX, q = i - a * TX;
      const int c = a % 3, kind = a / 3;
      const double* base = (kind < 2) ? st.f[EZ1 + c] : st.f[AZ1 + c];
      const double* src = base + ((kind & 1) ? rom : ro) + xtab[4 + q];
      cp_async8(sb + (ST_EZ + a) * W + 4 + q, src);
    }
    if (warm) {
      for (int i = tid; i < 4 * TX; i += NT) {
        const int a = i / TX, q = i - a * TX;
        const double* base = (a & 1) ? st.b[FN] : st.a[FN];
        const double* src = base + ((a >> 1) ? rom : rop) + xtab[4 + q];
        cp_async8(sb + (ST_NZP + a) * W + 4 + q, src);
      }
    }
  };

  const int r_first = zs - 3, r_last = ze + 2;
  // prologue: NST-1 rows in flight
#pragma unroll
  for (int k = 0; k < NST - 1; ++k) {
    if (r_first + k <= r_last) issue_row(r_first + k, k);
    cp_async_commit();
  }

  // z-pipeline registers (see header comment); index k = swept variable.
  double V1[6], f1[6], d1[6], L2[6], N4[6], N3[6], N2[6], A2[6], F3[6], S1[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    V1[k] = f1[k] = d1[k] = L2[k] = N4[k] = N3[k] = N2[k] = A2[k] = F3[k] = S1[k] = 0.0;
  }
  double U1 = 0.0, mu1 = 0.0;

  double* const xn = wk;                                   // beam-shared node fields
  double* const wb = wk + (size_t)(WK_SHARED + beam * WB_SIZE) * W;  // this beam
  const int x_own = x0 + t;
  const bool wall = !p.periodic_x;

  for (int r = r_first, it = 0; r <= r_last; ++r, ++it) {
    __syncthreads();  // every thread is done with the stage about to be refilled
    {
      const int rn = r + NST - 1;
      if (rn <= r_last) issue_row(rn, (it + NST - 1) % NST);
      cp_async_commit();
    }
    cp_async_wait<NST - 1>();
    __syncthreads();
    const double* sb = stage + (size_t)(it % NST) * ST_SIZE * W;
    const double* fl = sb + (size_t)(ST_FL + beam * 6) * W;

    // ---- Phase A: velocities (YM_Fluid.cu:3-11) and node-centred fields.
    for (int q = t; q < TX + 6; q += TX) {
      const int pp = 1 + q;
      const double ns = fmax(fl[FN * W + pp], 0.05);
      wb[WB_U * W + pp] = fl[FPX * W + pp] / ns;
      wb[WB_VZ * W + pp] = fl[FPZ * W + pp] / ns;
    }
    for (int i = tid; i < (TX + 4) + TX; i += NT) {
      if (i < TX + 4) {
        const int pp = 2 + i;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double* ex = sb + (ST_EX + c) * W;
          const double* by = sb + (ST_BY + c) * W;
          const double* bym = sb + (ST_BYM + c) * W;
          // YM_Fluid.cu:48-62
          xn[(WK_EXN + c) * W + pp] = 0.5 * (ex[pp] + ex[pp - 1]);
          xn[(WK_BYN + c) * W + pp] = 0.25 * (by[pp] + by[pp - 1] + bym[pp] + bym[pp - 1]);
        }
      } else {
        const int pp = 4 + (i - (TX + 4));
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          xn[(WK_EZN + c) * W + pp] = 0.5 * (sb[(ST_EZ + c) * W + pp] + sb[(ST_EZM + c) * W + pp]);
          xn[(WK_AZN + c) * W + pp] = 0.5 * (sb[(ST_AZ + c) * W + pp] + sb[(ST_AZM + c) * W + pp]);
        }
      }
    }
    __syncthreads();

    // ---- Phase B: x-sweep low-order solution (FCT_Sweeps.cu:88-133) at
    // positions [2, TX+6); the px source is kernel_ym_lorentz's src.px.
    for (int q = t; q < TX + 4; q += TX) {
      const int pp = 2 + q;
      int ps = pp;  // source cell: clamped ends evaluate the edge cell's source
      if (wall) {
        const int xg = x0 - 4 + pp;
        const int xc = xg < 0 ? 0 : (xg >= nx ? nx - 1 : xg);
        ps = xc - (x0 - 4);
      }
      const double vz = wb[WB_VZ * W + ps];
      double sx = -(fl[FQ1 * W + ps] * (xn[(WK_EXN + 0) * W + ps] + vz * xn[(WK_BYN + 0) * W + ps]) +
                    fl[FQ2 * W + ps] * (xn[(WK_EXN + 1) * W + ps] + vz * xn[(WK_BYN + 1) * W + ps]) +
                    fl[FQ3 * W + ps] * (xn[(WK_EXN + 2) * W + ps] + vz * xn[(WK_BYN + 2) * W + ps]));
      if (warm) {
        const double dndx = (fl[FN * W + ps + 1] - fl[FN * W + ps - 1]) / (2.0 * p.dx);
        sx -= p.warm_T * dndx;
      }
      wb[WB_S * W + pp] = sx;
      const double um = wb[WB_U * W + pp - 1], u0 = wb[WB_U * W + pp], up = wb[WB_U * W + pp + 1];
      const double eL = fct_eps(um, u0, dtdx), eR = fct_eps(u0, up, dtdx);
      double nuL, muL, nuR, muR;
      fct_nu_mu(eL, nuL, muL);
      fct_nu_mu(eR, nuR, muR);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double vm = fl[k * W + pp - 1], v0 = fl[k * W + pp], vp = fl[k * W + pp + 1];
        const double fL = 0.5 * eL * (vm + v0);
        const double fR = 0.5 * eR * (v0 + vp);
        const double dL = nuL * (v0 - vm);
        const double dR = nuR * (vp - v0);
        double lo;
        if (k == FPX)
          lo = v0 + dt * sx - (fR - fL);
        else
          lo = v0 - (fR - fL);
        wb[(WB_LOR + k) * W + pp] = lo;
        wb[(WB_LNR + k) * W + pp] = lo + (dR - dL);
      }
    }
    __syncthreads();

    // ---- Phase C: antidiffusive fluxes and limiter at interfaces p+1/2,
    // p in [3, TX+4) (FCT_Sweeps.cu:139-160).
    for (int q = t; q < TX + 1; q += TX) {
      const int pp = 3 + q;
      const double e = fct_eps(wb[WB_U * W + pp], wb[WB_U * W + pp + 1], dtdx);
      double nu, mu;
      fct_nu_mu(e, nu, mu);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double* lor = wb + (WB_LOR + k) * W;
        const double* lnr = wb + (WB_LNR + k) * W;
        const double fad = mu * (lor[pp + 1] - lor[pp]);
        wb[(WB_FLIM + k) * W + pp] =
            fct_limit(fad, lnr[pp] - lnr[pp - 1], lnr[pp + 1] - lnr[pp], lnr[pp + 2] - lnr[pp + 1]);
      }
    }
    __syncthreads();

    // ---- Phase D: x-swept value of the own column, z-sources, z-pipeline.
    {
      const int pp = 4 + t;
      double Vx[6];
#pragma unroll
      for (int k = 0; k < 6; ++k)
        Vx[k] = wb[(WB_LNR + k) * W + pp] - (wb[(WB_FLIM + k) * W + pp] - wb[(WB_FLIM + k) * W + pp - 1]);
      const double vx = wb[WB_U * W + pp];
      const double vz = wb[WB_VZ * W + pp];
      const double q1 = fl[FQ1 * W + pp], q2 = fl[FQ2 * W + pp], q3 = fl[FQ3 * W + pp];
      const double by1 = xn[(WK_BYN + 0) * W + pp], by2 = xn[(WK_BYN + 1) * W + pp],
                   by3 = xn[(WK_BYN + 2) * W + pp];
      // YM_Fluid.cu:67 (src.pz) and :76-79 (warm closure)
      double sz = -(q1 * (xn[(WK_EZN + 0) * W + pp] - vx * by1) + q2 * (xn[(WK_EZN + 1) * W + pp] - vx * by2) +
                    q3 * (xn[(WK_EZN + 2) * W + pp] - vx * by3));
      if (warm) {
        const double dndz = (sb[(ST_NZP + beam) * W + pp] - sb[(ST_NZM + beam) * W + pp]) / (2.0 * p.dz);
        sz -= p.warm_T * dndz;
      }
      // YM_Fluid.cu:99-107 (colour precession)
      const double a1 = xn[(WK_AZN + 0) * W + pp], a2 = xn[(WK_AZN + 1) * W + pp], a3 = xn[(WK_AZN + 2) * W + pp];
      double S[6];
      S[FN] = 0.0;
      S[FPX] = 0.0;
      S[FPZ] = sz;
      S[FQ1] = p.alpha * vz * (q2 * a3 - q3 * a2);
      S[FQ2] = p.alpha * vz * (q3 * a1 - q1 * a3);
      S[FQ3] = p.alpha * vz * (q1 * a2 - q2 * a1);

      // z-sweep pipeline: interface r-1/2 now known.
      const double e = fct_eps(U1, vz, dtdz);
      double nu, mu;
      fct_nu_mu(e, nu, mu);
      const int o = r - 3;
      const bool emit = (o >= zs) && (o < ze) && (x_own < nx);
      double outv[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double fR = 0.5 * e * (V1[k] + Vx[k]);
        const double dR = nu * (Vx[k] - V1[k]);
        double lo;
        if (k >= FPZ)
          lo = V1[k] + dt * S1[k] - (fR - f1[k]);
        else
          lo = V1[k] - (fR - f1[k]);
        const double ln = lo + (dR - d1[k]);
        const double fad = mu1 * (lo - L2[k]);
        const double flim = fct_limit(A2[k], N3[k] - N4[k], N2[k] - N3[k], ln - N2[k]);
        outv[k] = N3[k] - (flim - F3[k]);
        V1[k] = Vx[k];
        S1[k] = S[k];
        f1[k] = fR;
        d1[k] = dR;
        L2[k] = lo;
        N4[k] = N3[k];
        N3[k] = N2[k];
        N2[k] = ln;
        A2[k] = fad;
        F3[k] = flim;
      }
      U1 = vz;
      mu1 = mu;
      if (emit) {
        // YM_Fluid.cu:20-29 (density floor, wall momentum)
        if (outv[FN] < 0.05) outv[FN] = 0.05;
        if (wall && (x_own == 0 || x_own == nx - 1)) outv[FPX] = 0.0;
        double* const* dst = beam ? out.b : out.a;
        const size_t gi = idx2(x_own, o, nx);
#pragma unroll
        for (int k = 0; k < 6; ++k) dst[k][gi] = outv[k];
      }
    }
  }
  cp_async_wait<0>();
}

// The kernel reads start-of-step values across strip and segment halos while
// other CTAs write theirs, so the fluid it writes goes to a second state
// buffer (`out`); fields are only read.
template <int TX, int NST>
static cudaError_t prepare_fct_t() {
  return cudaFuncSetAttribute(fct_fused_kernel<TX, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fct_smem_bytes<TX>(NST));
}

template <int TX, int NST>
static cudaError_t launch_fct_t(const State& in, const State& out, const StepParams& p, int seg_len,
                                cudaStream_t s) {
  const size_t smem = fct_smem_bytes<TX>(NST);
  dim3 grid((p.nx + TX - 1) / TX, (p.nz + seg_len - 1) / seg_len);
  fct_fused_kernel<TX, NST><<<grid, 2 * TX, smem, s>>>(in, out, p, seg_len);
  return cudaGetLastError();
}

cudaError_t prepare_fct(int tx) {
  switch (tx) {
    case 32: return prepare_fct_t<32, 3>();
    case 64: return prepare_fct_t<64, 3>();
    case 128: return prepare_fct_t<128, 3>();
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fct(const State& in, const State& out, const StepParams& p, int tx, int seg_len,
                       cudaStream_t s) {
  switch (tx) {
    case 32: return launch_fct_t<32, 3>(in, out, p, seg_len, s);
    case 64: return launch_fct_t<64, 3>(in, out, p, seg_len, s);
    case 128: return launch_fct_t<128, 3>(in, out, p, seg_len, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ymkh
