// ymkh_init.cu — initial KH equilibrium and seed (ymgpu2d/YM_Init.cu:32-257).
//
// The reference builds its initial state with a mix of FP32 transcendentals
// (coshf, tanhf, logf, expf, sinf, cosf, sqrtf) and FP64 arithmetic.  The
// expressions below keep the same operand types and order (the FP32 calls
// are made on the same float arguments), so that with -fmad=false the state
// is bit-identical to the reference's kernel_ym_init on the same GPU.  Every
// run_mode 0..6 is supported, with the optional eigenmode seed profiles
// (YM_Init.cuh:10-17), init_by1_eq and vz_edge_taper.

#include "ymkh_common.cuh"

namespace ymkh {


// YM_Init.cu:11-18
__device__ __forceinline__ double log_cosh_stable(double xi) {
  const double SAFE_XI = 80.0;
  if (fabs(xi) < SAFE_XI) return (double)logf(coshf((float)xi));
  const double ax = fabs(xi);
  return ax - 0.6931471805599453 + log1p(exp(-2.0 * ax));
}

__global__ void init_kernel(const __grid_constant__ State st, const __grid_constant__ InitArgs A) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= A.nx || z >= A.nz) return;
  const size_t idx = idx2(x, z, A.nx);
  const int nx = A.nx, nz = A.nz;
  const double dx = A.dx, dz = A.dz, V0 = A.V0, epsilon = A.epsilon, perturb_amp = A.perturb_amp;

  const double k_z = A.k_mode * 2.0f * (double)M_PI / (nz * dz);
  const double x_c = (nx * dx) * 0.5f;
  const double xi = (x * dx - x_c) / epsilon;
  const double z_val = z * dz;
  const double sech_xi = 1.0f / coshf(xi);
  const double xi_seed_cutoff = 3.0f;
  const double seed_win = (fabsf(xi) < xi_seed_cutoff) ? 1.0f : 0.0f;
  const double base_seed = perturb_amp * V0 * sech_xi * seed_win;
  const double az1_eq = -V0 * log_cosh_stable(xi);

  double by1_init = 0.0f, by2_init = 0.0f, by3_init = 0.0f;
  double az1_init = 0.0f, az2_init = 0.0f, az3_init = 0.0f;
  double vz_A = +V0 * tanhf(xi);
  double qA_amp = 0.0f, qB_amp = 0.0f;
  const int run_mode = A.run_mode;

  if (run_mode == 0) {
    by2_init = base_seed * sinf(k_z * z_val);
    az1_init = az1_eq;
  } else if (run_mode == 1) {
    by2_init = base_seed * cosf(k_z * z_val);
    by3_init = base_seed * sinf(k_z * z_val);
    az1_init = az1_eq;
  } else if (run_mode == 6) {
    az1_init = az1_eq;
    double az_amp = 0.0f;
    if (A.az) {
      az_amp = perturb_amp * V0 * A.az[x];
      if (A.by) by2_init = perturb_amp * V0 * A.by[x] * cosf(k_z * z_val);
      if (A.by) by3_init = perturb_amp * V0 * A.by[x] * sinf(k_z * z_val);
      if (A.qA) qA_amp = perturb_amp * V0 * A.qA[x];
      if (A.qB) qB_amp = perturb_amp * V0 * A.qB[x];
    } else {
      const double xi_char = 1.0f / sqrtf(A.alpha_YM * k_z * V0 + 1e-12f);
      az_amp = perturb_amp * V0 * expf(-0.5f * xi * xi / (xi_char * xi_char));
    }
    az2_init = az_amp * cosf(k_z * z_val);
    az3_init = az_amp * sinf(k_z * z_val);
    if (A.init_by1_eq) {
      const double mean_lc = (nx * dx) / (4.0f * epsilon) - 0.693147f;
      by1_init = -2.0f * V0 * epsilon * (logf(coshf(xi)) - mean_lc);
    }
  } else if (run_mode == 2) {
    by1_init = base_seed * sinf(k_z * z_val);
    az1_init = 0.0f;
  } else if (run_mode == 4) {
    const double Lx = nx * dx;
    const double x_phys = x * dx;
    const double s = (x_phys < Lx * (1.0f / 3.0f) || x_phys >= Lx * (2.0f / 3.0f)) ? 1.0f : -1.0f;
    vz_A = V0 * s;
    const double kx_az1 = 3.0f * 2.0f * (double)M_PI / Lx;
    az1_init = -V0 * cosf(kx_az1 * x_phys);
    by2_init = perturb_amp * V0 * sinf(k_z * z_val);
  } else if (run_mode == 5) {
    const double Lx = nx * dx;
    const double x_ph = x * dx;
    const double xi5 = (x_ph - 0.5f * Lx) / epsilon;
    vz_A = V0 * tanhf(xi5);
    const double kx_cos = 2.0f * (double)M_PI / Lx;
    az1_init = -V0 * cosf(kx_cos * x_ph);
    by1_init = -V0 * kx_cos * sinf(kx_cos * x_ph);
    const double sech5 = 1.0f / coshf(xi5);
    const double bs5 = perturb_amp * V0 * sech5;
    by2_init = bs5 * cosf(k_z * z_val);
    by3_init = bs5 * sinf(k_z * z_val);
  } else {
    const double L = nx * dx;
    const double xi1 = (x * dx - L * 0.25f) / epsilon;
    const double xi2 = (x * dx - L * 0.75f) / epsilon;
    const double shear = tanhf(xi1) - tanhf(xi2) - 1.0f;
    vz_A = V0 * shear;
    az1_init = -V0 * (log_cosh_stable(xi1) - log_cosh_stable(xi2));
    by1_init = V0 * (tanhf(xi1) - tanhf(xi2)) / epsilon;
    const double sech1 = 1.0f / coshf(xi1);
    const double sech2 = 1.0f / coshf(xi2);
    const double base_dt = perturb_amp * V0 * (sech1 + sech2);
    by2_init = base_dt * cosf(k_z * z_val);
    by3_init = base_dt * sinf(k_z * z_val);
  }

  if (A.vz_edge_taper > 0.0f && (run_mode == 1 || run_mode == 6)) {
    const double dt_tap = 3.0f;
    const double axi = fabsf(xi);
    const double w = 0.5f * (1.0f - tanhf((axi - A.vz_edge_taper) / dt_tap));
    vz_A *= w;
    if (A.init_by1_eq) {
      const double axi_h = fabsf(xi + 0.5f * dx / epsilon);
      const double u = (axi_h - A.vz_edge_taper) / dt_tap;
      const double I = logf(coshf(axi_h)) - 0.5f * dt_tap * (u + logf(coshf(u)) + 0.693147f);
      const double Lxi = (nx * dx) * 0.5f / epsilon;
      const double mean_I = (0.5f * A.vz_edge_taper * A.vz_edge_taper - A.vz_edge_taper * 0.693147f +
                             (Lxi - A.vz_edge_taper) * (A.vz_edge_taper - 0.693147f)) /
                            Lxi;
      by1_init = -2.0f * V0 * epsilon * (I - mean_I);
    }
  }

  st.f[BY1][idx] = by1_init;
  st.f[BY2][idx] = by2_init;
  st.f[BY3][idx] = by3_init;
  st.f[AZ1][idx] = az1_init;
  st.f[AZ2][idx] = az2_init;
  st.f[AZ3][idx] = az3_init;
  st.f[EX1][idx] = st.f[EX2][idx] = st.f[EX3][idx] = 0.0;
  st.f[EZ1][idx] = st.f[EZ2][idx] = st.f[EZ3][idx] = 0.0;
  st.a[FN][idx] = 1.0f;
  st.a[FPX][idx] = 0.0f;
  st.a[FPZ][idx] = vz_A;
  st.a[FQ1][idx] = +1.0f;
  st.a[FQ2][idx] = qA_amp * cosf(k_z * z_val);
  st.a[FQ3][idx] = qA_amp * sinf(k_z * z_val);
  st.b[FN][idx] = 1.0f;
  st.b[FPX][idx] = 0.0f;
  st.b[FPZ][idx] = -vz_A;
  st.b[FQ1][idx] = -1.0f;
  st.b[FQ2][idx] = qB_amp * cosf(k_z * z_val);
  st.b[FQ3][idx] = qB_amp * sinf(k_z * z_val);
}

cudaError_t launch_init(const State& st, const InitArgs& a, cudaStream_t s) {
  dim3 th(32, 8);
  dim3 bl((a.nx + 31) / 32, (a.nz + 7) / 8);
  init_kernel<<<bl, th, 0, s>>>(st, a);
  return cudaGetLastError();
}

}  // namespace ymkh
