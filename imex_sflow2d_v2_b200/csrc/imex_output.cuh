// Device side of output_solution (src/inpout_2d.f90:5683-6180): the values
// the .q_2d / .p_2d / ESRI writers print, computed from the device state, and
// the in-place changes the reference makes while writing them (|q| < 1e-20
// set to 0 in q for .q_2d, :5807-5813; DEPOSIT and EROSION below 1e-20 set
// to 0 for .p_2d, :6115-6122).  The host copies the planes and formats them.
#pragma once

#include "imex_kernels.cuh"

namespace imex {

// Columns of one .p_2d line after x_comp, y_comp (the WRITE at :6142-6148)
// for the physics this library runs (no additional gas, liquid, stochastic
// or pore-pressure variables):
//   h, u, v, B_out, h+B_out, alphas(ns), T, rho_m, red_grav, DEPOSIT(ns),
//   EROSION(ns), SUM(ERODIBLE)/(1-porosity), alphal, shear_vel, Ri,
//   Rouse_no(ns), mu_eff, hmax, pdynmax, mod_vel_max, inertial_number
__host__ __device__ constexpr int p2d_cols(int ns) { return 17 + 4 * ns; }

struct OutputArgs {
  double* q;              // pitched state planes (zeroed in place when cons)
  double* deposit;        // pitched (ns planes) or null
  double* erosion;        // pitched (ns planes) or null
  const double* erodible; // pitched (ns planes) or null
  const double* Bcent;    // pitched or null
  const double* Bx;       // B_prime_x, B_prime_y
  const double* By;
  PostPlanes post;        // hmax/pdynmax/mod_vel_max when post_on
  int post_on, cons, phys, esri;
  double* p2d;            // p2d_cols(ns) compact planes of nx*ny
  double* esr;            // 2 compact planes: qp(1), qp(4) of the module qp
};

__device__ __forceinline__ double tiny0(double v) { return (fabs(v) < 1.0e-20) ? 0.0 : v; }

template <int NS>
__global__ void __launch_bounds__(128)
    k_output_prep(const __grid_constant__ DevParams Pp, OutputArgs A) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const long long n = (long long)P.nx * P.ny;
  const size_t N = (size_t)P.plane;
  for (long long cc = (long long)blockIdx.x * blockDim.x + threadIdx.x; cc < n;
       cc += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(cc % P.nx), k = (int)(cc / P.nx);
    const size_t c = (size_t)k * P.pitch + j;
    double qc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = A.q[c + i * N];
    if (A.esri) {   // the driver's qp (before the .q_2d zeroing)
      double qp[NP];
      qc_to_qp<NS>(P, qc, qp);
      A.esr[cc] = qp[0];
      A.esr[n + cc] = qp[3];
    }
    if (A.cons) {
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        if (fabs(qc[i]) < 1.0e-20) {
          qc[i] = 0.0;
          A.q[c + i * N] = 0.0;
        }
      }
    }
    if (!A.phys) continue;
    double qp[NP], p_dyn = 0.0;
    qc_to_qp<NS>(P, qc, qp, &p_dyn);
    const Mixt m = mixt_var<NS>(P, qp);
    double r_h = qp[0], r_u = qp[NV], r_v = qp[NV + 1], r_T = qp[3];
    double r_rho_m = m.rho_m, r_red_grav = m.red_grav;
    const double r_Ri = m.Ri;
    double al[NS], mu_eff = 0.0, inertial = 0.0, r_alphal = 0.0;
    const double shear_vel = 0.0;   // rheology_model 8 only
    if (r_h > 0.0) {
#pragma unroll
      for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qp[4 + i] : qp[4 + i] / r_h;
      if (P.rheology_flag && P.rheology_model == 1) {
        // no pore-pressure variable: the excess pore pressure is 0
        const double dp = fmax_f(0.0, 0.0);
        mu_eff = P.mu * fmax_f(0.0, 1.0 - dp / (r_rho_m * r_h * r_red_grav));
      }
    } else {
#pragma unroll
      for (int i = 0; i < NS; ++i) al[i] = 0.0;
    }
    r_h = tiny0(r_h);
    r_u = tiny0(r_u);
    r_v = tiny0(r_v);
    const double B = A.Bcent ? A.Bcent[c] : 0.0;
    const double B_out = tiny0(B);
    double dep[NS], ers[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      al[i] = tiny0(al[i]);
      dep[i] = A.deposit ? A.deposit[c + i * N] : 0.0;
      ers[i] = A.erosion ? A.erosion[c + i * N] : 0.0;
      if (fabs(dep[i]) < 1.0e-20) {
        dep[i] = 0.0;
        if (A.deposit) A.deposit[c + i * N] = 0.0;
      }
      if (fabs(ers[i]) < 1.0e-20) {
        ers[i] = 0.0;
        if (A.erosion) A.erosion[c + i * N] = 0.0;
      }
    }
    r_T = tiny0(r_T);
    r_rho_m = tiny0(r_rho_m);
    r_red_grav = tiny0(r_red_grav);
    r_alphal = tiny0(r_alphal);
    mu_eff = tiny0(mu_eff);
    inertial = tiny0(inertial);
    double esum = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) esum = esum + (A.erodible ? A.erodible[c + i * N] : 0.0);
    const double etot = esum / (1.0 - P.erodible_porosity);
    double* o = A.p2d + cc;
    int col = 0;
    auto put = [&](double v) {
      o[(size_t)col * n] = v;
      ++col;
    };
    put(r_h);
    put(r_u);
    put(r_v);
    put(B_out);
    put(r_h + B_out);
#pragma unroll
    for (int i = 0; i < NS; ++i) put(al[i]);
    put(r_T);
    put(r_rho_m);
    put(r_red_grav);
#pragma unroll
    for (int i = 0; i < NS; ++i) put(dep[i]);
#pragma unroll
    for (int i = 0; i < NS; ++i) put(ers[i]);
    put(etot);
    put(r_alphal);
    put(shear_vel);
    put(r_Ri);
#pragma unroll
    for (int i = 0; i < NS; ++i) put(0.0);   // Rouse_no
    put(mu_eff);
    put(A.post_on ? A.post.hmax[c] : 0.0);
    put(A.post_on ? A.post.pdynmax[c] : 0.0);
    put(A.post_on ? A.post.mvmax[c] : 0.0);
    put(inertial);
  }
}

}  // namespace imex
