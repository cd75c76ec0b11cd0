// ymkh_maxwell.cu — fused non-Abelian Maxwell update.
//
// One launch replaces stages 5-6 of the reference step
// (ymgpu2d/main_ym.cu:357-363): colour currents (YM_Physics.cu:9-60),
// Ampère (YM_Physics.cu:70-113), potential (YM_Physics.cu:589-599) and
// Faraday (YM_Physics.cu:120-151).  The currents are never stored: each CTA
// forms them from the new fluid for its tile plus a one-cell halo, updates E
// on the tile plus the halo Faraday needs, then Az and By on the tile.
//
// Reads the new fluid and the start-of-step fields from `in_*`, writes the
// new E, By, Az to `out` (a different buffer: neighbouring tiles still read
// the old values).  HBM per cell: 12 fluid + 12 field arrays read, 12 written.

#include "ymkh_common.cuh"

namespace ymkh {

namespace {
constexpr int MX_TX = 32;
constexpr int MX_TZ = 6;  // keeps the static shared tiles under 48 KB
}  // namespace

__global__ void __launch_bounds__(MX_TX* MX_TZ)
    maxwell_fused_kernel(const __grid_constant__ State fluid_new, const __grid_constant__ State fields_old,
                         const __grid_constant__ State out, const __grid_constant__ StepParams p) {
  constexpr int TX = MX_TX, TZ = MX_TZ;
  constexpr int FW = TX + 1, FH = TZ + 1;  // fluid tile   x in [x0, x0+TX], z in [z0, z0+TZ]
  constexpr int BW = TX + 2, BH = TZ + 2;  // By tile      x in [x0-1, x0+TX], z in [z0-1, z0+TZ]
  constexpr int AW = TX, AH = TZ + 1;      // Az, Ex tile  x in [x0, x0+TX), z in [z0, z0+TZ]
  constexpr int EW = TX + 1, EH = TZ;      // Ez tile      x in [x0, x0+TX], z in [z0, z0+TZ)
  __shared__ double s_fl[12][FH][FW];
  __shared__ double s_by[3][BH][BW];
  __shared__ double s_az[3][AH][AW];
  __shared__ double s_ex[3][AH][AW];  // old, then new Ex
  __shared__ double s_ez[3][EH][EW];  // old, then new Ez

  const int nx = p.nx, nz = p.nz;
  const int x0 = blockIdx.x * TX, z0 = blockIdx.y * TZ;
  const int tid = threadIdx.x;
  constexpr int NT = TX * TZ;
  const bool wall = !p.periodic_x;

  for (int i = tid; i < 12 * FH * FW; i += NT) {
    const int a = i / (FH * FW), r = i - a * FH * FW, zz = r / FW, xx = r - zz * FW;
    const int gx = xmap(x0 + xx, nx, p.periodic_x), gz = zwrap(z0 + zz, nz);
    const double* src = (a < 6) ? fluid_new.a[a] : fluid_new.b[a - 6];
    s_fl[a][zz][xx] = src[idx2(gx, gz, nx)];
  }
  for (int i = tid; i < 3 * BH * BW; i += NT) {
    const int c = i / (BH * BW), r = i - c * BH * BW, zz = r / BW, xx = r - zz * BW;
    const int gx = xmap(x0 - 1 + xx, nx, p.periodic_x), gz = zwrap(z0 - 1 + zz, nz);
    s_by[c][zz][xx] = fields_old.f[BY1 + c][idx2(gx, gz, nx)];
  }
  for (int i = tid; i < 3 * AH * AW; i += NT) {
    const int c = i / (AH * AW), r = i - c * AH * AW, zz = r / AW, xx = r - zz * AW;
    const int gx = xmap(x0 + xx, nx, p.periodic_x), gz = zwrap(z0 + zz, nz);
    s_az[c][zz][xx] = fields_old.f[AZ1 + c][idx2(gx, gz, nx)];
    s_ex[c][zz][xx] = fields_old.f[EX1 + c][idx2(gx, gz, nx)];
  }
  for (int i = tid; i < 3 * EH * EW; i += NT) {
    const int c = i / (EH * EW), r = i - c * EH * EW, zz = r / EW, xx = r - zz * EW;
    const int gx = xmap(x0 + xx, nx, p.periodic_x), gz = zwrap(z0 + zz, nz);
    // YM_Fluid.cu:25-29: the wall boundary zeroes Ez before Ampère
    const bool wz = wall && (gx == 0 || gx == nx - 1);
    s_ez[c][zz][xx] = wz ? 0.0 : fields_old.f[EZ1 + c][idx2(gx, gz, nx)];
  }
  __syncthreads();

  const double dt = p.dt, c2 = p.c2, al = p.alpha, e0 = p.eps0;
  // ---- Ampère for Ex on x in [x0, x0+TX), z in [z0, z0+TZ] (needs Jx).
  double exn[3][2];
#pragma unroll
  for (int nex = 0; nex < 2; ++nex) {
    const int i = tid + nex * NT;
    if (i >= AW * AH) break;
    const int zz = i / AW, xx = i - zz * AW;  // fluid (xx, zz) and (xx+1, zz)
    double jx[3];
    double nq[2][3], vxr[2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const double n0 = s_fl[b * 6 + FN][zz][xx], np = s_fl[b * 6 + FN][zz][xx + 1];
      vxr[b] = 0.5 * (s_fl[b * 6 + FPX][zz][xx] / fmax(n0, 1e-10) + s_fl[b * 6 + FPX][zz][xx + 1] / fmax(np, 1e-10));
#pragma unroll
      for (int a = 0; a < 3; ++a)
        nq[b][a] = 0.5 * (n0 * s_fl[b * 6 + FQ1 + a][zz][xx] + np * s_fl[b * 6 + FQ1 + a][zz][xx + 1]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) jx[a] = -(nq[0][a] * vxr[0] + nq[1][a] * vxr[1]);
    // By at (x, z) is s_by[zz+1][xx+1]; (x, zm) is s_by[zz][xx+1]
    const double by1 = s_by[0][zz + 1][xx + 1], by2 = s_by[1][zz + 1][xx + 1], by3 = s_by[2][zz + 1][xx + 1];
    const double d1 = (by1 - s_by[0][zz][xx + 1]) / p.dz;
    const double d2 = (by2 - s_by[1][zz][xx + 1]) / p.dz;
    const double d3 = (by3 - s_by[2][zz][xx + 1]) / p.dz;
    const double a1 = s_az[0][zz][xx], a2 = s_az[1][zz][xx], a3 = s_az[2][zz][xx];
    const double k1 = a2 * by3 - a3 * by2;
    const double k2 = a3 * by1 - a1 * by3;
    const double k3 = a1 * by2 - a2 * by1;
    exn[0][nex] = s_ex[0][zz][xx] + dt * (c2 * (-d1 - al * k1) - jx[0] / e0);
    exn[1][nex] = s_ex[1][zz][xx] + dt * (c2 * (-d2 - al * k2) - jx[1] / e0);
    exn[2][nex] = s_ex[2][zz][xx] + dt * (c2 * (-d3 - al * k3) - jx[2] / e0);
  }
  // ---- Ampère for Ez on x in [x0, x0+TX], z in [z0, z0+TZ) (needs Jz).
  double ezn[3][2];
#pragma unroll
  for (int nez = 0; nez < 2; ++nez) {
    const int i = tid + nez * NT;
    if (i >= EW * EH) break;
    const int zz = i / EW, xx = i - zz * EW;  // fluid (xx, zz) and (xx, zz+1)
    double nqz[2][3], vzt[2];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const double n0 = s_fl[b * 6 + FN][zz][xx], nzp = s_fl[b * 6 + FN][zz + 1][xx];
      vzt[b] = 0.5 * (s_fl[b * 6 + FPZ][zz][xx] / fmax(n0, 1e-10) + s_fl[b * 6 + FPZ][zz + 1][xx] / fmax(nzp, 1e-10));
#pragma unroll
      for (int a = 0; a < 3; ++a)
        nqz[b][a] = 0.5 * (n0 * s_fl[b * 6 + FQ1 + a][zz][xx] + nzp * s_fl[b * 6 + FQ1 + a][zz + 1][xx]);
    }
    const double by[3] = {s_by[0][zz + 1][xx + 1], s_by[1][zz + 1][xx + 1], s_by[2][zz + 1][xx + 1]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double jz = -(nqz[0][a] * vzt[0] + nqz[1][a] * vzt[1]);
      const double dbx = (by[a] - s_by[a][zz + 1][xx]) / p.dx;
      ezn[a][nez] = s_ez[a][zz][xx] + dt * (c2 * dbx - jz / e0);
    }
  }
  __syncthreads();  // all old Ex/Ez reads done
#pragma unroll
  for (int nex = 0; nex < 2; ++nex) {
    const int i = tid + nex * NT;
    if (i >= AW * AH) break;
    const int zz = i / AW, xx = i - zz * AW;
#pragma unroll
    for (int a = 0; a < 3; ++a) s_ex[a][zz][xx] = exn[a][nex];
  }
#pragma unroll
  for (int nez = 0; nez < 2; ++nez) {
    const int i = tid + nez * NT;
    if (i >= EW * EH) break;
    const int zz = i / EW, xx = i - zz * EW;
#pragma unroll
    for (int a = 0; a < 3; ++a) s_ez[a][zz][xx] = ezn[a][nez];
  }
  __syncthreads();
  // At a wall the right neighbour of the last column is the column itself
  // (YM_Physics.cu:127), so the halo Ez is that column's new Ez.
  if (wall && x0 + TX >= nx) {
    for (int i = tid; i < 3 * EH; i += NT) {
      const int a = i / EH, zz = i - a * EH;
      const int xl = nx - 1 - x0;  // local index of the last real column
      s_ez[a][zz][xl + 1] = s_ez[a][zz][xl];
    }
    __syncthreads();
  }

  // ---- Potential and Faraday on the tile.
  {
    const int zz = tid / TX, xx = tid - zz * TX;
    const int gx = x0 + xx, gz = z0 + zz;
    if (gx < nx && gz < nz) {
      const size_t gi = idx2(gx, gz, nx);
      double az[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) az[a] = s_az[a][zz][xx];
      if (!p.freeze_az1) az[0] = az[0] - dt * s_ez[0][zz][xx];
      az[1] = az[1] - dt * s_ez[1][zz][xx];
      az[2] = az[2] - dt * s_ez[2][zz][xx];
      const double e1 = s_ex[0][zz][xx], e2 = s_ex[1][zz][xx], e3 = s_ex[2][zz][xx];
      const double k[3] = {az[1] * e3 - az[2] * e2, az[2] * e1 - az[0] * e3, az[0] * e2 - az[1] * e1};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double dex = (s_ex[a][zz + 1][xx] - s_ex[a][zz][xx]) / p.dz;
        const double dez = (s_ez[a][zz][xx + 1] - s_ez[a][zz][xx]) / p.dx;
        const double byo = s_by[a][zz + 1][xx + 1];
        out.f[BY1 + a][gi] = byo - dt * (dex - dez - al * k[a]);
        out.f[EX1 + a][gi] = s_ex[a][zz][xx];
        out.f[EZ1 + a][gi] = s_ez[a][zz][xx];
        out.f[AZ1 + a][gi] = az[a];
      }
    }
  }
}

cudaError_t launch_maxwell(const State& fluid_new, const State& fields_old, const State& out, const StepParams& p,
                           cudaStream_t s) {
  dim3 grid((p.nx + MX_TX - 1) / MX_TX, (p.nz + MX_TZ - 1) / MX_TZ);
  maxwell_fused_kernel<<<grid, MX_TX * MX_TZ, 0, s>>>(fluid_new, fields_old, out, p);
  return cudaGetLastError();
}

}  // namespace ymkh
