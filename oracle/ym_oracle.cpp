// ym_oracle.cpp — FP64 CPU restatement of the ymgpu2d Kelvin–Helmholtz step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path of
// kh_simulations_b200: only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs load it.  The product never links it.
//
// It restates, stage by stage and in the reference's operation order, the
// body of the time loop ymgpu2d/main_ym.cu:322-479 with the kernels of
// ymgpu2d/YM_Fluid.cu, YM_FCT.cu, FCT_Sweeps.cu, FCT_DeviceMath.cuh,
// YM_Physics.cu and YM_Energy.cu.  Built with -ffp-contract=off so that every
// product and sum is rounded as written, it reproduces the reference kernels
// built with nvcc -fmad=false bit for bit, except where a transcendental
// function is evaluated (the FP32 filter twiddles, which the caller may pass
// in as a table produced on the GPU; the sponge's exp; the initial state).
//
// Reductions follow the reference's order exactly: the z-mean uses the
// shared-memory halving tree of YM_Physics.cu:301-308, the DFT filter the
// warp-shuffle tree plus sequential warp sum of YM_Physics.cu:398-428, and the
// energy the sequential host sum of YM_Energy.cu:29-31.
//
// Parallelism: OpenMP over independent lines / cells; results do not depend
// on the thread count.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <complex>
#include <omp.h>

#include "../include/ymkh.h"

namespace {

// State order (include/ymkh.h): fields 0..11, fluid A 12..17, fluid B 18..23.
enum { EX1, EX2, EX3, EZ1, EZ2, EZ3, BY1, BY2, BY3, AZ1, AZ2, AZ3 };
enum { FN = 0, FPX, FPZ, FQ1, FQ2, FQ3 };

inline size_t IDX(int x, int z, int nx) { return (size_t)x + (size_t)z * (size_t)nx; }

// ---------------------------------------------------------------------------
// FCT_DeviceMath.cuh:38-46 compute_eps
inline double fct_eps(double uL, double uR, double dt, double dx) {
  double v = 0.5 * (uL + uR);
  return v * (dt / dx);
}
// FCT_DeviceMath.cuh:52-63 compute_nu_mu
inline void fct_nu_mu(double eps, double& nu, double& mu) {
  double scrh = std::fmin(1.0 / 6.0, std::fabs(eps));
  scrh = (1.0 / 3.0) * scrh * scrh;
  nu = (1.0 / 6.0) + (1.0 / 3.0) * (eps * eps - scrh * scrh);
  mu = 0.25 - 0.5 * nu;
}
// FCT_DeviceMath.cuh:108-125 apply_fct_limiter
inline double fct_limit(double f, double dm1, double d0, double dp1) {
  double s = std::copysign(1.0, d0);
  double term = s * dm1, terp = s * dp1, fa = std::fabs(f);
  double lim = std::fmax(0.0, std::fmin(term, std::fmin(fa, terp)));
  return s * lim;
}

// FCT_Sweeps.cu:39-177 restated for one line of n cells read through an
// index map: periodic (the padded periodic x-sweep of YM_FCT.cu:47-91, whose
// real outputs only touch the 3 ghost cells on each side) or clamped (the
// zero-gradient ends of the kernel's own halo loads, used by the z-sweep of
// YM_FCT.cu:93-135 and the wall x-sweep of YM_FCT.cu:30-45).
struct Line {
  int n;
  bool periodic;
  const double* u;  // velocity along the line (start-of-step)
  const double* v;  // swept variable (old)
  const double* s;  // source or nullptr
  ptrdiff_t stride;
};

inline int line_map(const Line& L, int i) {
  if (L.periodic) { int r = i % L.n; return r < 0 ? r + L.n : r; }
  return i < 0 ? 0 : (i >= L.n ? L.n - 1 : i);
}

void sweep_line(const Line& L, double* out, double dx, double dt, std::vector<double>& wk) {
  const int n = L.n;
  wk.resize(3 * (size_t)(n + 6));
  double* lor = wk.data() + 2;               // indices -2 .. n+1
  double* lnr = wk.data() + (n + 6) + 2;     // indices -2 .. n+1
  double* fad = wk.data() + 2 * (n + 6) + 1; // interfaces j+1/2, j = -1 .. n-1
  auto U = [&](int i) { return L.u[(ptrdiff_t)line_map(L, i) * L.stride]; };
  auto V = [&](int i) { return L.v[(ptrdiff_t)line_map(L, i) * L.stride]; };
  auto S = [&](int i) { return L.s ? L.s[(ptrdiff_t)line_map(L, i) * L.stride] : 0.0; };
  // Phase B (FCT_Sweeps.cu:88-133)
  for (int i = -2; i <= n + 1; ++i) {
    double eL = fct_eps(U(i - 1), U(i), dt, dx);
    double eR = fct_eps(U(i), U(i + 1), dt, dx);
    double nuL, muL, nuR, muR;
    fct_nu_mu(eL, nuL, muL);
    fct_nu_mu(eR, nuR, muR);
    double vm = V(i - 1), v0 = V(i), vp = V(i + 1);
    double fL = 0.5 * eL * (vm + v0);
    double fR = 0.5 * eR * (v0 + vp);
    double dL = nuL * (v0 - vm);
    double dR = nuR * (vp - v0);
    lor[i] = v0 + dt * S(i) - (fR - fL);
    lnr[i] = lor[i] + (dR - dL);
  }
  // Phase C antidiffusive fluxes (FCT_Sweeps.cu:139-152)
  for (int j = -1; j <= n - 1; ++j) {
    double e = fct_eps(U(j), U(j + 1), dt, dx);
    double nu, mu;
    fct_nu_mu(e, nu, mu);
    fad[j] = mu * (lor[j + 1] - lor[j]);
  }
  // Limiter and update (FCT_Sweeps.cu:155-162)
  for (int i = 0; i < n; ++i) {
    double dm1 = lnr[i] - lnr[i - 1];
    double d0 = lnr[i + 1] - lnr[i];
    double dp1 = lnr[i + 2] - lnr[i + 1];
    double fl = fct_limit(fad[i - 1], lnr[i - 1] - lnr[i - 2], dm1, d0);
    double fr = fct_limit(fad[i], dm1, d0, dp1);
    out[(ptrdiff_t)i * L.stride] = lnr[i] - (fr - fl);
  }
}

struct Sim {
  int nx, nz;
  size_t N;
  ymkh_params p;
  double* st[YMKH_NSTATE];
  const float* tw_cos;  // optional [mtab+1][nz] table, mode-major
  const float* tw_sin;
  int tw_mmax;          // highest mode present in the table (-1 = none)

  double* F(int i) { return st[i]; }
  double* A(int k) { return st[12 + k]; }
  double* B(int k) { return st[18 + k]; }
};

// ---------------------------------------------------------------------------
// YM_Fluid.cu:3-11 kernel_update_velocities
void velocities(const Sim& s, const double* n, const double* px, const double* pz,
                double* ux, double* uz) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)s.N; ++i) {
    double sn = std::fmax(n[i], 0.05);
    ux[i] = px[i] / sn;
    uz[i] = pz[i] / sn;
  }
}

// YM_Fluid.cu:32-84 kernel_ym_lorentz
void lorentz(Sim& s, double* const fl[6], double* spx, double* spz) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      int xm = p.periodic_x ? (x + nx - 1) % nx : std::max(0, x - 1);
      int zm = (z == 0) ? nz - 1 : z - 1;
      double ns = std::fmax(fl[FN][idx], 0.05);
      double vx = fl[FPX][idx] / ns;
      double vz = fl[FPZ][idx] / ns;
      double ex[3], ez[3], by[3];
      for (int a = 0; a < 3; ++a) {
        const double* Ex = s.st[EX1 + a];
        const double* Ez = s.st[EZ1 + a];
        const double* By = s.st[BY1 + a];
        ex[a] = 0.5 * (Ex[idx] + Ex[IDX(xm, z, nx)]);
        ez[a] = 0.5 * (Ez[idx] + Ez[IDX(x, zm, nx)]);
        by[a] = 0.25 * (By[idx] + By[IDX(xm, z, nx)] + By[IDX(x, zm, nx)] + By[IDX(xm, zm, nx)]);
      }
      double q1 = fl[FQ1][idx], q2 = fl[FQ2][idx], q3 = fl[FQ3][idx];
      double sx = -(q1 * (ex[0] + vz * by[0]) + q2 * (ex[1] + vz * by[1]) + q3 * (ex[2] + vz * by[2]));
      double sz = -(q1 * (ez[0] - vx * by[0]) + q2 * (ez[1] - vx * by[1]) + q3 * (ez[2] - vx * by[2]));
      if (p.warm_T > 0.0) {
        int xp = p.periodic_x ? (x + 1) % nx : std::min(nx - 1, x + 1);
        int xm2 = p.periodic_x ? (x + nx - 1) % nx : std::max(0, x - 1);
        int zp = (z == nz - 1) ? 0 : z + 1;
        int zm2 = (z == 0) ? nz - 1 : z - 1;
        const double* n = fl[FN];
        double dndx = (n[IDX(xp, z, nx)] - n[IDX(xm2, z, nx)]) / (2.0 * p.dx);
        double dndz = (n[IDX(x, zp, nx)] - n[IDX(x, zm2, nx)]) / (2.0 * p.dz);
        sx -= p.warm_T * dndx;
        sz -= p.warm_T * dndz;
      }
      spx[idx] = sx;
      spz[idx] = sz;
    }
}

// YM_Fluid.cu:86-108 kernel_ym_precession
void precession(Sim& s, double* const fl[6], double* sq1, double* sq2, double* sq3) {
  const int nx = s.nx, nz = s.nz;
  const double al = s.p.alpha_YM;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      int zm = (z == 0) ? nz - 1 : z - 1;
      double ns = std::fmax(fl[FN][idx], 0.05);
      double vz = fl[FPZ][idx] / ns;
      double a1 = 0.5 * (s.st[AZ1][idx] + s.st[AZ1][IDX(x, zm, nx)]);
      double a2 = 0.5 * (s.st[AZ2][idx] + s.st[AZ2][IDX(x, zm, nx)]);
      double a3 = 0.5 * (s.st[AZ3][idx] + s.st[AZ3][IDX(x, zm, nx)]);
      double q1 = fl[FQ1][idx], q2 = fl[FQ2][idx], q3 = fl[FQ3][idx];
      sq1[idx] = al * vz * (q2 * a3 - q3 * a2);
      sq2[idx] = al * vz * (q3 * a1 - q1 * a3);
      sq3[idx] = al * vz * (q1 * a2 - q2 * a1);
    }
}

// YM_FCT.cu:30-91 (x-sweep, periodic or wall) and :93-135 (z-sweep): the
// reference sweeps n, px, pz, Q1..Q3 of one beam with the start-of-step
// velocity; the x-sweep adds dt*src_px to px, the z-sweep dt*src_pz to pz and
// dt*sQ^a to Q^a.
void fct_beam(Sim& s, double* const fl[6], const double* ux, const double* uz,
              const double* spx, const double* spz, const double* const sq[3]) {
  const int nx = s.nx, nz = s.nz;
  const double dt = s.p.dt_step;
  std::vector<double> old((size_t)6 * s.N);
  for (int k = 0; k < 6; ++k) std::memcpy(old.data() + k * s.N, fl[k], s.N * sizeof(double));
  // x-sweep
  const double* xsrc[6] = {nullptr, spx, nullptr, nullptr, nullptr, nullptr};
#pragma omp parallel
  {
    std::vector<double> wk;
#pragma omp for schedule(static) collapse(2)
    for (int k = 0; k < 6; ++k)
      for (int z = 0; z < nz; ++z) {
        size_t b = (size_t)z * nx;
        Line L{nx, s.p.periodic_x != 0, ux + b, old.data() + k * s.N + b,
               xsrc[k] ? xsrc[k] + b : nullptr, 1};
        sweep_line(L, fl[k] + b, s.p.dx, dt, wk);
      }
  }
  // z-sweep on the x-swept values, clamped ends
  for (int k = 0; k < 6; ++k) std::memcpy(old.data() + k * s.N, fl[k], s.N * sizeof(double));
  const double* zsrc[6] = {nullptr, nullptr, spz, sq[0], sq[1], sq[2]};
#pragma omp parallel
  {
    std::vector<double> wk;
#pragma omp for schedule(static) collapse(2)
    for (int k = 0; k < 6; ++k)
      for (int x = 0; x < nx; ++x) {
        Line L{nz, false, uz + x, old.data() + k * s.N + x, zsrc[k] ? zsrc[k] + x : nullptr,
               (ptrdiff_t)nx};
        sweep_line(L, fl[k] + x, s.p.dz, dt, wk);
      }
  }
}

// YM_Fluid.cu:13-30 kernel_enforce_boundaries
void boundaries(Sim& s) {
  const int nx = s.nx, nz = s.nz;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      if (s.A(FN)[idx] < 0.05) s.A(FN)[idx] = 0.05;
      if (s.B(FN)[idx] < 0.05) s.B(FN)[idx] = 0.05;
      if (!s.p.periodic_x && (x == 0 || x == nx - 1)) {
        s.A(FPX)[idx] = 0.0;
        s.B(FPX)[idx] = 0.0;
        s.st[EZ1][idx] = s.st[EZ2][idx] = s.st[EZ3][idx] = 0.0;
      }
    }
}

// YM_Physics.cu:9-60 kernel_ym_currents
void currents(Sim& s, double* jx[3], double* jz[3]) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      int xp = p.periodic_x ? (x + 1) % nx : std::min(nx - 1, x + 1);
      int zp = (z == nz - 1) ? 0 : z + 1;
      size_t ixp = IDX(xp, z, nx), izp = IDX(x, zp, nx);
      double nq[2][3], nqz[2][3], vxr[2], vzt[2];
      for (int b = 0; b < 2; ++b) {
        double* const* fl = b == 0 ? &s.st[12] : &s.st[18];
        double n0 = fl[FN][idx], np = fl[FN][ixp], nzp = fl[FN][izp];
        vxr[b] = 0.5 * (fl[FPX][idx] / std::fmax(n0, 1e-10) + fl[FPX][ixp] / std::fmax(np, 1e-10));
        vzt[b] = 0.5 * (fl[FPZ][idx] / std::fmax(n0, 1e-10) + fl[FPZ][izp] / std::fmax(nzp, 1e-10));
        for (int a = 0; a < 3; ++a) {
          const double* Q = fl[FQ1 + a];
          nq[b][a] = 0.5 * (n0 * Q[idx] + np * Q[ixp]);
          nqz[b][a] = 0.5 * (n0 * Q[idx] + nzp * Q[izp]);
        }
      }
      for (int a = 0; a < 3; ++a) {
        jx[a][idx] = -(nq[0][a] * vxr[0] + nq[1][a] * vxr[1]);
        jz[a][idx] = -(nqz[0][a] * vzt[0] + nqz[1][a] * vzt[1]);
      }
    }
}

// YM_Physics.cu:70-113 kernel_ym_ampere
void ampere(Sim& s, double* jx[3], double* jz[3]) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
  const double c2 = p.c * p.c, dt = p.dt_step, a = p.alpha_YM;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      int zm = (z == 0) ? nz - 1 : z - 1;
      int xm = p.periodic_x ? (x + nx - 1) % nx : (x == 0 ? 0 : x - 1);
      double by1 = s.st[BY1][idx], by2 = s.st[BY2][idx], by3 = s.st[BY3][idx];
      double d1z = (by1 - s.st[BY1][IDX(x, zm, nx)]) / p.dz;
      double d2z = (by2 - s.st[BY2][IDX(x, zm, nx)]) / p.dz;
      double d3z = (by3 - s.st[BY3][IDX(x, zm, nx)]) / p.dz;
      double a1 = s.st[AZ1][idx], a2 = s.st[AZ2][idx], a3 = s.st[AZ3][idx];
      double c1 = a2 * by3 - a3 * by2;
      double cc2 = a3 * by1 - a1 * by3;
      double c3 = a1 * by2 - a2 * by1;
      s.st[EX1][idx] += dt * (c2 * (-d1z - a * c1) - jx[0][idx] / p.eps_0);
      s.st[EX2][idx] += dt * (c2 * (-d2z - a * cc2) - jx[1][idx] / p.eps_0);
      s.st[EX3][idx] += dt * (c2 * (-d3z - a * c3) - jx[2][idx] / p.eps_0);
      double d1x = (by1 - s.st[BY1][IDX(xm, z, nx)]) / p.dx;
      double d2x = (by2 - s.st[BY2][IDX(xm, z, nx)]) / p.dx;
      double d3x = (by3 - s.st[BY3][IDX(xm, z, nx)]) / p.dx;
      s.st[EZ1][idx] += dt * (c2 * d1x - jz[0][idx] / p.eps_0);
      s.st[EZ2][idx] += dt * (c2 * d2x - jz[1][idx] / p.eps_0);
      s.st[EZ3][idx] += dt * (c2 * d3x - jz[2][idx] / p.eps_0);
    }
}

// YM_Physics.cu:589-599 kernel_ym_potential
void potential(Sim& s) {
  const double dt = s.p.dt_step;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)s.N; ++i) {
    if (!s.p.freeze_az1) s.st[AZ1][i] -= dt * s.st[EZ1][i];
    s.st[AZ2][i] -= dt * s.st[EZ2][i];
    s.st[AZ3][i] -= dt * s.st[EZ3][i];
  }
}

// YM_Physics.cu:120-151 kernel_ym_faraday
void faraday(Sim& s) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
  const double dt = p.dt_step, a = p.alpha_YM;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      size_t idx = IDX(x, z, nx);
      int zp = (z == nz - 1) ? 0 : z + 1;
      int xp = p.periodic_x ? (x + 1) % nx : std::min(nx - 1, x + 1);
      double dex[3], dez[3];
      for (int c = 0; c < 3; ++c) {
        dex[c] = (s.st[EX1 + c][IDX(x, zp, nx)] - s.st[EX1 + c][idx]) / p.dz;
        dez[c] = (s.st[EZ1 + c][IDX(xp, z, nx)] - s.st[EZ1 + c][idx]) / p.dx;
      }
      double a1 = s.st[AZ1][idx], a2 = s.st[AZ2][idx], a3 = s.st[AZ3][idx];
      double e1 = s.st[EX1][idx], e2 = s.st[EX2][idx], e3 = s.st[EX3][idx];
      double c1 = a2 * e3 - a3 * e2;
      double c2 = a3 * e1 - a1 * e3;
      double c3 = a1 * e2 - a2 * e1;
      s.st[BY1][idx] -= dt * (dex[0] - dez[0] - a * c1);
      s.st[BY2][idx] -= dt * (dex[1] - dez[1] - a * c2);
      s.st[BY3][idx] -= dt * (dex[2] - dez[2] - a * c3);
    }
}

// The 12 colour-2/3 arrays touched by the sponge, xi_cut and hyperdiffusion
// (YM_Physics.cu:175-181, 203-209, 251-256).
void colour23(Sim& s, double* out[12]) {
  double* v[12] = {s.st[BY2], s.st[BY3], s.st[EX2], s.st[EX3], s.st[EZ2], s.st[EZ3],
                   s.st[AZ2], s.st[AZ3], s.A(FQ2), s.A(FQ3), s.B(FQ2), s.B(FQ3)};
  for (int i = 0; i < 12; ++i) out[i] = v[i];
}

// YM_Physics.cu:161-182 kernel_ym_sponge
void sponge(Sim& s) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
  double* v[12];
  colour23(s, v);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      double xc = (nx * p.dx) * 0.5;
      double xi = std::fabs((x * p.dx - xc) / p.epsilon);
      if (xi <= p.xi_sponge) continue;
      double sig = p.sigma_sponge * (xi - p.xi_sponge);
      double dec = std::exp(-sig * p.dt_step);
      size_t idx = IDX(x, z, nx);
      for (int k = 0; k < 12; ++k) v[k][idx] *= dec;
    }
}

// YM_Physics.cu:192-210 kernel_ym_xicut
void xicut(Sim& s) {
  const int nx = s.nx, nz = s.nz;
  const ymkh_params& p = s.p;
  double* v[12];
  colour23(s, v);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      double xc = (nx * p.dx) * 0.5;
      double xi = std::fabs((x * p.dx - xc) / p.epsilon);
      if (xi <= p.xi_cut) continue;
      size_t idx = IDX(x, z, nx);
      for (int k = 0; k < 12; ++k) v[k][idx] = 0.0;
    }
}

// The 15 arrays of the z-mean and EM band filters, in the reference's order
// (YM_Physics.cu:284-298 and :373-379).
void filter15(Sim& s, double* out[15]) {
  double* v[15] = {s.st[BY1], s.st[EX1], s.st[EZ1], s.st[BY2], s.st[BY3],
                   s.st[EX2], s.st[EX3], s.st[EZ2], s.st[EZ3], s.st[AZ2],
                   s.st[AZ3], s.A(FQ2), s.A(FQ3), s.B(FQ2), s.B(FQ3)};
  for (int i = 0; i < 15; ++i) out[i] = v[i];
}

// YM_Physics.cu:272-327 kernel_ym_subtract_zmean (nz a power of two)
void zmean(Sim& s) {
  const int nx = s.nx, nz = s.nz;
  double* v[15];
  filter15(s, v);
#pragma omp parallel
  {
    std::vector<double> t(nz);
#pragma omp for schedule(static) collapse(2)
    for (int k = 0; k < 15; ++k)
      for (int x = 0; x < nx; ++x) {
        for (int z = 0; z < nz; ++z) t[z] = v[k][IDX(x, z, nx)];
        for (int st = nz >> 1; st > 0; st >>= 1)
          for (int z = 0; z < st; ++z) t[z] += t[z + st];
        double inv = 1.0 / (double)nz;
        double m = t[0] * inv;
        for (int z = 0; z < nz; ++z) v[k][IDX(x, z, nx)] -= m;
      }
  }
}

// YM_Physics.cu:387-388: the FP32 phase and twiddles of mode m at row z.
inline void twiddle(const Sim& s, int m, int z, float& c, float& sn) {
  if (s.tw_cos && m <= s.tw_mmax) {
    c = s.tw_cos[(size_t)m * s.nz + z];
    sn = s.tw_sin[(size_t)m * s.nz + z];
    return;
  }
  float phase = 2.0f * (float)M_PI * m * z / (float)s.nz;
  c = cosf(phase);
  sn = sinf(phase);
}

// YM_Physics.cu:349-455 (and the identical per-array arithmetic of
// :461-519, :526-584): subtract modes [lo, hi] from one column of one array.
// a[] holds the column (nz values); all coefficients use the original column.
void dft_band_column(const Sim& s, double* col, int lo, int hi, std::vector<double>& wk) {
  const int nz = s.nz, nw = nz / 32;
  wk.assign((size_t)nz, 0.0);
  double* delta = wk.data();
  double ar[32], br[32];
  std::vector<double> wa(nw), wb(nw);
  for (int m = lo; m <= hi; ++m) {
    for (int w = 0; w < nw; ++w) {
      for (int l = 0; l < 32; ++l) {
        float c, sn;
        twiddle(s, m, w * 32 + l, c, sn);
        ar[l] = col[w * 32 + l] * (double)c;
        br[l] = col[w * 32 + l] * (double)sn;
      }
      // __shfl_down_sync tree seen from lane 0 (YM_Physics.cu:399-406)
      for (int off = 16; off > 0; off >>= 1)
        for (int l = 0; l < off; ++l) { ar[l] += ar[l + off]; br[l] += br[l + off]; }
      wa[w] = ar[0];
      wb[w] = br[0];
    }
    double sc = 0, ss = 0;
    for (int w = 0; w < nw; ++w) { sc += wa[w]; ss += wb[w]; }
    float inv2 = 2.0f / (float)nz;
    double Am = sc * (double)inv2, Bm = ss * (double)inv2;
    for (int z = 0; z < nz; ++z) {
      float c, sn;
      twiddle(s, m, z, c, sn);
      delta[z] += Am * (double)c + Bm * (double)sn;
    }
  }
  for (int z = 0; z < nz; ++z) col[z] = col[z] - delta[z];
}

void dft_band(Sim& s, double* const* arrs, int narr, int lo, int hi) {
  const int nx = s.nx, nz = s.nz;
#pragma omp parallel
  {
    std::vector<double> col(nz), wk;
#pragma omp for schedule(static) collapse(2)
    for (int k = 0; k < narr; ++k)
      for (int x = 0; x < nx; ++x) {
        for (int z = 0; z < nz; ++z) col[z] = arrs[k][IDX(x, z, nx)];
        dft_band_column(s, col.data(), lo, hi, wk);
        for (int z = 0; z < nz; ++z) arrs[k][IDX(x, z, nx)] = col[z];
      }
  }
}

// Band list of ymgpu2d/main_ym.cu:392-430 plus the extension bands.
int bands(const ymkh_params& p, int lo[], int hi[]) {
  int n = 0;
  if (p.kz_suppress_max >= 1) { lo[n] = 1; hi[n] = p.kz_suppress_max; ++n; }
  if (p.kz_suppress_hi > p.kz_suppress_max + 1) {
    lo[n] = p.kz_suppress_max + 2; hi[n] = p.kz_suppress_hi; ++n;
  }
  for (int i = 0; i < p.n_extra_bands && i < YMKH_MAX_EXTRA_BANDS; ++i) {
    lo[n] = p.extra_band_lo[i]; hi[n] = p.extra_band_hi[i]; ++n;
  }
  return n;
}

// YM_Physics.cu:228-259 kernel_ym_hyperdiffuse_z.  The reference updates in
// place while neighbours read (a race it documents); this restatement uses the
// race-free reading in which every stencil reads the pre-update values.
void hyperdiffuse(Sim& s) {
  const int nx = s.nx, nz = s.nz;
  const double mu = s.p.hyp_diff_coeff;
  double* v[12];
  colour23(s, v);
#pragma omp parallel
  {
    std::vector<double> col(nz);
#pragma omp for schedule(static) collapse(2)
    for (int k = 0; k < 12; ++k)
      for (int x = 0; x < nx; ++x) {
        for (int z = 0; z < nz; ++z) col[z] = v[k][IDX(x, z, nx)];
        for (int z = 0; z < nz; ++z) {
          int zm1 = (z == 0) ? nz - 1 : z - 1;
          int zm2 = (z <= 1) ? z - 2 + nz : z - 2;
          int zp1 = (z == nz - 1) ? 0 : z + 1;
          int zp2 = (z >= nz - 2) ? z + 2 - nz : z + 2;
          double d4 = col[zm2] - 4.0 * col[zm1] + 6.0 * col[z] - 4.0 * col[zp1] + col[zp2];
          v[k][IDX(x, z, nx)] = col[z] - mu * d4;
        }
      }
  }
}

// One iteration of ymgpu2d/main_ym.cu:324-455.  The sources that the
// reference carries from the end of the previous iteration (or from the
// initial precompute at :228-237) are pure functions of the state at the
// start of this iteration and are recomputed here.
void step_once(Sim& s) {
  const size_t N = s.N;
  std::vector<double> buf(N * 16);
  double* uxA = &buf[0 * N]; double* uzA = &buf[1 * N];
  double* uxB = &buf[2 * N]; double* uzB = &buf[3 * N];
  double* spxA = &buf[4 * N]; double* spzA = &buf[5 * N];
  double* spxB = &buf[6 * N]; double* spzB = &buf[7 * N];
  double* sqA[3] = {&buf[8 * N], &buf[9 * N], &buf[10 * N]};
  double* sqB[3] = {&buf[11 * N], &buf[12 * N], &buf[13 * N]};
  double* flA[6]; double* flB[6];
  for (int k = 0; k < 6; ++k) { flA[k] = s.A(k); flB[k] = s.B(k); }
  // 7 (previous iteration) / init precompute: sources
  lorentz(s, flA, spxA, spzA);
  lorentz(s, flB, spxB, spzB);
  precession(s, flA, sqA[0], sqA[1], sqA[2]);
  precession(s, flB, sqB[0], sqB[1], sqB[2]);
  // 1. velocities
  velocities(s, flA[FN], flA[FPX], flA[FPZ], uxA, uzA);
  velocities(s, flB[FN], flB[FPX], flB[FPZ], uxB, uzB);
  // 2-3. FCT x then z sweeps (the reference does x A, x B, z A, z B; the
  // beams are independent so the order between them is immaterial)
  fct_beam(s, flA, uxA, uzA, spxA, spzA, sqA);
  fct_beam(s, flB, uxB, uzB, spxB, spzB, sqB);
  // 4. boundaries
  boundaries(s);
  // 5-6. currents, Ampère, potential, Faraday
  double* jx[3] = {&buf[0 * N], &buf[1 * N], &buf[2 * N]};
  double* jz[3] = {&buf[3 * N], &buf[4 * N], &buf[5 * N]};
  currents(s, jx, jz);
  ampere(s, jx, jz);
  potential(s);
  faraday(s);
  // 6b, 6b2
  if (s.p.xi_sponge > 0.0) sponge(s);
  if (s.p.xi_cut > 0.0) xicut(s);
  // 6c
  if (s.p.suppress_kz0) zmean(s);
  // 6c2 / 6c3
  int lo[2 + YMKH_MAX_EXTRA_BANDS], hi[2 + YMKH_MAX_EXTRA_BANDS];
  int nb = bands(s.p, lo, hi);
  double* em[15];
  filter15(s, em);
  double* flu[6] = {s.A(FPZ), s.B(FPZ), s.A(FPX), s.B(FPX), s.A(FN), s.B(FN)};
  for (int b = 0; b < nb; ++b) dft_band(s, em, 15, lo[b], hi[b]);
  for (int b = 0; b < nb; ++b) dft_band(s, flu, 6, lo[b], hi[b]);
  // 6d
  if (s.p.hyp_diff_coeff > 0.0) hyperdiffuse(s);
  // 6e
  if (s.p.suppress_kz0) {
    std::memset(s.st[BY1], 0, N * sizeof(double));
    std::memset(s.st[EX1], 0, N * sizeof(double));
    std::memset(s.st[EZ1], 0, N * sizeof(double));
  }
}

}  // namespace

extern "C" {

// nsteps iterations in place on the 24 host arrays.  tw_cos/tw_sin: optional
// FP32 twiddle table [(tw_mmax+1) * nz], mode-major, as produced on the GPU.
int orc_step(const ymkh_grid* g, const ymkh_params* p, double* const* state, int nsteps,
             const float* tw_cos, const float* tw_sin, int tw_mmax) {
  if (!g || !p || !state || g->nx < 4 || g->nz < 4) return YMKH_EINVAL;
  Sim s;
  s.nx = g->nx; s.nz = g->nz; s.N = (size_t)g->nx * g->nz; s.p = *p;
  for (int i = 0; i < YMKH_NSTATE; ++i) s.st[i] = state[i];
  s.tw_cos = tw_cos; s.tw_sin = tw_sin; s.tw_mmax = (tw_cos && tw_sin) ? tw_mmax : -1;
  for (int k = 0; k < nsteps; ++k) step_once(s);
  return 0;
}

// YM_Energy.cu:3-32: per-cell energy, sequential host sum in index order.
double orc_energy(const ymkh_grid* g, double* const* st) {
  const size_t N = (size_t)g->nx * g->nz;
  std::vector<double> e(N);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)N; ++i) {
    double nA = std::fmax(st[12 + FN][i], 1e-10);
    double nB = std::fmax(st[18 + FN][i], 1e-10);
    double pxA = st[12 + FPX][i], pzA = st[12 + FPZ][i];
    double pxB = st[18 + FPX][i], pzB = st[18 + FPZ][i];
    double keA = 0.5 * (pxA * pxA + pzA * pzA) / nA;
    double keB = 0.5 * (pxB * pxB + pzB * pzB) / nB;
    double em = 0.5 * (st[EX1][i] * st[EX1][i] + st[EX2][i] * st[EX2][i] + st[EX3][i] * st[EX3][i] +
                       st[EZ1][i] * st[EZ1][i] + st[EZ2][i] * st[EZ2][i] + st[EZ3][i] * st[EZ3][i] +
                       st[BY1][i] * st[BY1][i] + st[BY2][i] * st[BY2][i] + st[BY3][i] * st[BY3][i]);
    e[i] = keA + keB + em;
  }
  double total = 0.0;
  for (size_t i = 0; i < N; ++i) total += e[i];
  return total;
}

// ymgpu2d/analysis/remote_timeseries.py:62-77 (numpy fast path): amplitude of
// mode k of Az2 + i Az3 along z, averaged over x; out[1] for the conjugate.
int orc_mode_amp(const ymkh_grid* g, double* const* st, int k, double* out) {
  const int nx = g->nx, nz = g->nz;
  double sa = 0.0, sc = 0.0;
  for (int x = 0; x < nx; ++x) {
    std::complex<double> F(0, 0), Fc(0, 0);
    for (int z = 0; z < nz; ++z) {
      double ang = -2.0 * M_PI * k * (double)z / (double)nz;
      std::complex<double> ker(std::cos(ang), std::sin(ang));
      std::complex<double> sig(st[AZ2][IDX(x, z, nx)], st[AZ3][IDX(x, z, nx)]);
      F += ker * sig;
      Fc += ker * std::conj(sig);
    }
    sa += std::abs(F);
    sc += std::abs(Fc);
  }
  out[0] = sa / nx / nz;
  out[1] = sc / nx / nz;
  return 0;
}

// Host evaluation of the FP32 twiddles (YM_Physics.cu:387-388) with the C
// library's cosf/sinf; the GPU table from ymkh_twiddles is authoritative.
int orc_twiddles(int nz, int m_lo, int m_hi, float* c, float* sn) {
  for (int m = m_lo; m <= m_hi; ++m)
    for (int z = 0; z < nz; ++z) {
      float ph = 2.0f * (float)M_PI * m * z / (float)nz;
      c[(size_t)(m - m_lo) * nz + z] = cosf(ph);
      sn[(size_t)(m - m_lo) * nz + z] = sinf(ph);
    }
  return 0;
}

int orc_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
