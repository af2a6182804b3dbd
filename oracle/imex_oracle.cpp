// TEST INFRASTRUCTURE ONLY -- the oracle.
//
// A CPU restatement, in C++17, of the IMEX_SfloW2D time step as written in
// the reference Fortran (demichie/IMEX_SfloW2D_v2).  Every routine below
// names the reference routine and the file:line range it follows.  The
// operation order of every floating-point expression follows the Fortran
// source (left-to-right, parentheses kept, no contraction: build with
// -ffp-contract=off), so the oracle is a faithful specification of the
// reference's numbers, including its quirks:
//   * module work arrays (face states, speeds, fluxes, RK stage arrays) are
//     never cleared between steps, so cells outside the solve mask keep the
//     values of the last step that touched them (allocated arrays start at 0
//     here; the Fortran leaves them uninitialised);
//   * the "dry cell" face assignments in reconstruction are overwritten by the
//     unconditional qp_to_qc just after them (src/solver_2d.f90:3677-3734);
//   * the x_stencil(3)=y_stag(k+1) typo (src/solver_2d.f90:3616) leaks into the
//     v-component x-slope of inlet cells with sourceN;
//   * DOT_PRODUCT of a COMPLEX first argument conjugates it (Fortran rule), so
//     the complex-step derivative carries a conjugated term in c_phys_var;
//   * complex arithmetic follows the Fortran compiler rules: plain products,
//     Smith's range-reduced quotient, products with a REAL operand scale both
//     parts.
// Nothing in the product links this file.
//
// Parity status: unpinned against the reference binary (no Fortran compiler
// in this image and no golden outputs in the reference); pinned by analytic
// known-answer tests in tests/.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "imex_oracle.h"
#include "../imex_sflow2d_v2_b200/csrc/ipow_tables.h"

namespace {

constexpr double EPS = 2.220446049250313e-16;  // EPSILON(1.0_wp)
constexpr int MAXV = IMEX_MAX_VARS;
constexpr int MAXP = IMEX_MAX_VARS + 2;
constexpr int MAXS = IMEX_MAX_SOLID;
constexpr int LNSRCH_MAX_TRIALS = 4096;

// MIN/MAX with a defined answer for NaN operands (the non-NaN one).
inline double fmin_f(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return (b < a) ? b : a;
}
inline double fmax_f(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return (b > a) ? b : a;
}

// x**y for the non-integer exponents of the mass-exchange closures
// (settling drag, hindered settling, entrainment, inlet ramps).  Both the CPU
// oracle and the CUDA path evaluate it with this same sequence of IEEE
// operations and the same tables (ipow_tables.h), so the two agree bit for
// bit; the sequence is
//   log x = e*ln2 - log(invc_i) + log1p(r): m in [1,2), i its top 7 fraction
//           bits, r = m*invc_i - 1 by one fused multiply-add (|r| < 2^-8),
//           log1p(r) by its Taylor series to r^7, -log(invc_i) tabulated as a
//           sum of two doubles,
//   z = y*log x carried as an unevaluated sum of two doubles (exact product
//       error by one fused multiply-add, Knuth's two-sum),
//   exp z = 2^(k/64) * exp(r), r = z - k*ln2/64 (ln2/64 split in two),
//           exp(r) - 1 by its Taylor series to r^6, 2^(j/64) tabulated.
// Every fused multiply-add is the IEEE single-rounding operation on both
// sides (CUDA fma, C++ std::fma).
// Accuracy against the exact power: within 0.52 ulp (tested); the reference's
// libm pow is within 1 ulp, so results differ from it at that level only.
inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
inline void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = std::fma(a, b, -p);
}
double ipow(double x, double y) {
  if (std::isnan(x) || std::isnan(y)) return x + y;
  if (x == 0.0 && y != 0.0) return (y > 0.0) ? 0.0 : HUGE_VAL;
  if (x < 0.0 && y != 0.0) return std::nan("");
  if (std::isinf(x) && y != 0.0) return (y > 0.0) ? x : 0.0;
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  const double LN2_HI = 0x1.62e42fee00000p-1, LN2_LO = 0x1.a39ef35793c76p-33;
  const double LN2_64_HI = 0x1.62e42fee00000p-7, LN2_64_LO = 0x1.a39ef35793c76p-39;
  const double INV_LN2_64 = 0x1.71547652b82fep+6;
  // log x = e*ln2 - log(invc_i) + log1p(r), m*invc_i = 1 + r, |r| < 2^-8
  int e;
  double m = std::frexp(x, &e);          // m in [1/2, 1)
  m = m * 2.0;
  e = e - 1;
  const int i = (int)((m - 1.0) * 128.0);
  const double r = std::fma(m, IPOW_INVC[i], -1.0);
  double P = std::fma(r, 0x1.2492492492492p-3, -0x1.5555555555555p-3);   // 1/7, -1/6
  P = std::fma(r, P, 0x1.999999999999ap-3);                               // 1/5
  P = std::fma(r, P, -0x1.0000000000000p-2);                              // -1/4
  P = std::fma(r, P, 0x1.5555555555555p-2);                               // 1/3
  P = std::fma(r, P, -0x1.0000000000000p-1);                              // -1/2
  const double l1p = std::fma(r * r, P, r);
  double a, b, hi, c;
  two_sum((double)e * LN2_HI, IPOW_LOGC_HI[i], a, b);
  two_sum(a, l1p, hi, c);
  double lo = ((b + c) + IPOW_LOGC_LO[i]) + (double)e * LN2_LO;
  // z = y*log x in double-double
  double p, pe;
  two_prod(y, hi, p, pe);
  pe = std::fma(y, lo, pe);
  double zh, zl;
  two_sum(p, pe, zh, zl);
  if (zh > 709.78) return HUGE_VAL;
  if (zh < -745.1) return 0.0;
  // exp z = 2^(k/64) exp(rr), |rr| < ln2/128
  const double kf = std::nearbyint(zh * INV_LN2_64);
  const long long k = (long long)kf;
  const int j = (int)(k & 63);
  const int me = (int)((k - j) / 64);
  double rh, rl;
  two_sum(zh, -(kf * LN2_64_HI), rh, rl);
  const double rr = rh + (rl + std::fma(-kf, LN2_64_LO, zl));
  double E = std::fma(rr, 0x1.6c16c16c16c17p-10, 0x1.1111111111111p-7);  // 1/720, 1/120
  E = std::fma(rr, E, 0x1.5555555555555p-5);                              // 1/24
  E = std::fma(rr, E, 0x1.5555555555555p-3);                              // 1/6
  E = std::fma(rr, E, 0x1.0000000000000p-1);                              // 1/2
  const double em1 = std::fma(rr * rr, E, rr);
  const double th = IPOW_EXP2_HI[j];
  return std::ldexp(th + std::fma(th, em1, IPOW_EXP2_LO[j]), me);
}

// ---------------------------------------------------------------- complex
struct cplx {
  double re, im;
};
inline cplx C(double r, double i = 0.0) { return {r, i}; }
inline cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// COMPLEX op REAL: the REAL operand is promoted to (r,0) and the compiler's
// complex lowering drops the products with the known-zero imaginary part.
inline cplx mulr(cplx a, double r) { return {a.re * r, a.im * r}; }
inline cplx divr(cplx a, double r) { return {a.re / r, a.im / r}; }
inline cplx addr(cplx a, double r) { return {a.re + r, a.im}; }
inline cplx subr(cplx a, double r) { return {a.re - r, a.im}; }
inline cplx rsub(double r, cplx a) { return {r - a.re, -a.im}; }
inline cplx conj(cplx a) { return {a.re, -a.im}; }
// Smith (1962) range-reduced complex division.
inline cplx operator/(cplx a, cplx b) {
  if (std::fabs(b.re) < std::fabs(b.im)) {
    double ratio = b.re / b.im;
    double div = (b.re * ratio) + b.im;
    double tr = (a.re * ratio) + a.im;
    double ti = (a.im * ratio) - a.re;
    return {tr / div, ti / div};
  } else {
    double ratio = b.im / b.re;
    double div = (b.im * ratio) + b.re;
    double tr = (a.im * ratio) + a.re;
    double ti = a.im - (a.re * ratio);
    return {tr / div, ti / div};
  }
}
inline cplx rdiv(double r, cplx b) { return C(r, 0.0) / b; }
// Principal square root by the half-angle formulas.
inline cplx csqrt_(cplx z) {
  if (z.im == 0.0) {
    if (z.re < 0.0) return {0.0, std::copysign(std::sqrt(-z.re), z.im)};
    return {std::fabs(std::sqrt(z.re)), z.im};
  }
  if (z.re == 0.0) {
    double r = std::sqrt(0.5 * std::fabs(z.im));
    return {r, std::copysign(r, z.im)};
  }
  double d = std::sqrt(z.re * z.re + z.im * z.im);
  if (z.re > 0.0) {
    double r = std::sqrt(0.5 * (d + z.re));
    double s = 0.5 * (z.im / r);
    return {r, s};
  } else {
    double s = std::sqrt(0.5 * (d - z.re));
    double r = std::fabs(0.5 * (z.im / s));
    return {r, std::copysign(s, z.im)};
  }
}

}  // namespace

// ====================================================================== ctx
struct OracleCtx {
  ImexParams p;
  int nx, ny, nv, np, ns, neq, nrk;
  int idx_u, idx_v;  // 0-based positions n_vars, n_vars+1
  double dx, dy, dx2, dy2, one_by_dx, one_by_dy;
  double eps_sing, eps_sing4, h, one_by_h;
  double rho_a_amb, inv_pres;
  double inv_rho_s[MAXS];
  bool implicit_flag[MAXV];
  int n_nh;
  double a_tilde_ij[4][4], a_dirk_ij[4][4], omega_tilde[4], omega[4];
  std::vector<double> x_comp, x_stag, y_comp, y_stag;

  // static planes (Fortran layout)
  std::vector<double> B_cent, Bx, By, Bxx, Bxy, Byy, gc, dgc_dx, gc_sx, gc_sy;
  std::vector<int32_t> source_cell;
  std::vector<int8_t> sE, sW, sS, sN, B_nodata;
  std::vector<double> sEx, sEy, sWx, sWy, sSx, sSy, sNx, sNy;
  std::vector<double> cell_source_fractions, solve_mask_time, source_xy;
  std::vector<double> erodible, deposit, erosion;

  // state and module work arrays
  std::vector<double> q, q0, q_fv, qp;
  std::vector<double> q_rk, qp_rk, divFlux, NH, SI_NH, expl_terms;
  std::vector<double> qL, qR, qB, qT, qpL, qpR, qpB, qpT;
  std::vector<double> axNeg, axPos, ayNeg, ayPos, ax_max, ay_max;
  std::vector<double> Hx, Hy;
  std::vector<uint8_t> mask, mask_temp, mask_x, mask_y;
  std::vector<int> j_cent, k_cent, j_stag_x, k_stag_x, j_stag_y, k_stag_y;
  int64_t solve_cells = 0, solve_interfaces_x = 0, solve_interfaces_y = 0;
  // face "wetness" at the time of writing, for the stale-read instrument
  std::vector<int32_t> epL, epR, epB, epT;  // reconstruction epoch of the last write
  int32_t recon_epoch = 0;
  std::atomic<int64_t> stale_wet_reads{0};
  // mass budget (test instrument): cumulative changes of SUM(q(1,:,:)) by
  // cause since set_state, in units of q(1) (multiply by dx*dy for mass):
  // [0] fluxes through faces with exactly one solved side (domain border,
  // inlet ring), from the face fluxes alone; [1] assembly fixes; [2] the
  // erosion/deposition update; [3] term [0] of the last step only
  long double mass_budget[4] = {0.0L, 0.0L, 0.0L, 0.0L};
  long double stage_face_flux[4] = {0.0L, 0.0L, 0.0L, 0.0L};

  double t = 0.0, dt = 0.0, dt_old = 0.0, dt_old_old = 0.0, t_end = 1e300,
         t_output = -1.0;
  int64_t steps = 0;
  // statistics
  std::atomic<int64_t> newton_cells{0}, newton_iters{0}, lnsrch_trials{0},
      newton_maxit{0};
  std::atomic<int64_t> hist[16];
  uint32_t error_mask = 0;
  int first_err_code = 0;
  int64_t first_err_index = -1;

  // index helpers (1-based j,k as in Fortran)
  inline size_t c2(int j, int k) const { return (size_t)(j - 1) + (size_t)nx * (k - 1); }
  inline size_t sx2(int j, int k) const { return (size_t)(j - 1) + (size_t)(nx + 1) * (k - 1); }
  inline size_t sy2(int j, int k) const { return (size_t)(j - 1) + (size_t)nx * (k - 1); }
  inline double* Q(std::vector<double>& a, int j, int k) { return &a[(size_t)nv * c2(j, k)]; }
  inline double* QP(std::vector<double>& a, int j, int k) { return &a[(size_t)np * c2(j, k)]; }
  inline double* QRK(std::vector<double>& a, int n, int j, int k, int r) {
    return &a[(size_t)n * (c2(j, k) + (size_t)nx * ny * (r - 1))];
  }
  inline double* FX(std::vector<double>& a, int n, int j, int k) { return &a[(size_t)n * sx2(j, k)]; }
  inline double* FY(std::vector<double>& a, int n, int j, int k) { return &a[(size_t)n * sy2(j, k)]; }

  // may be called from parallel loops: the result (OR of codes, lowest
  // cell index and code) does not depend on the order of the calls
  void record_error(int code, int j, int k) {
    int64_t idx = (int64_t)c2(j, k);
#pragma omp critical(oracle_record_error)
    {
      error_mask |= IMEX_ERRBIT(code);
      if (first_err_index < 0 || idx < first_err_index ||
          (idx == first_err_index && code < first_err_code)) {
        first_err_index = idx;
        first_err_code = code;
      }
    }
  }

  // ------------------------------------------------------------- physics
  void mixt_var(const double* qpj, double& r_Ri, double& r_rho_m, double& r_rho_c,
                double& r_red_grav, bool sp_heat_flag, double& r_sp_heat_c,
                double& r_sp_heat_mix) const;
  void eval_sp_heat(const double* r_alphas, double r_inv_rhom, double& spc,
                    double& spm) const;
  void r_phys_var(const double* r_qj, double& r_h, double& r_u, double& r_v,
                  double* r_alphas, double& r_rho_m, double& r_T,
                  double& r_red_grav, double& p_dyn) const;
  void qc_to_qp(const double* qc, double* qpo, double& p_dyn) const;
  void qp_to_qc(const double* qpi, double* qc) const;
  void qp_to_qp2(const double* qpj, double Bj, double* qp2) const;
  void eval_local_speeds_x(const double* qpj, double gcf, double& vmin, double& vmax) const;
  void eval_local_speeds_y(const double* qpj, double gcf, double& vmin, double& vmax) const;
  void eval_fluxes(const double* qcj, const double* qpj, double gcf, int dir, double* flux) const;
  void eval_expl_terms(double bx, double by, double bxx, double bxy, double byy,
                       double gcf, double dgcx, double dgcy, const double* qpj,
                       double* expl, double csf) const;
  void c_phys_var(const cplx* c_qj, cplx& h_, cplx& u, cplx& v, cplx& T, cplx& rho_m,
                  cplx* alphas, cplx& inv_rhom) const;
  void eval_implicit_terms(double bx, double by, const cplx* qj, cplx* nh) const;
  void eval_implicit_terms_r(double bx, double by, const double* r_qj, double* r_nh) const;
  void eval_nh_semi_impl_terms(double bx, double by, double bxx, double bxy, double byy,
                               double gcf, const double* qcj, const double* qpj,
                               double* si) const;
  double settling_velocity(double diam, double rhos, double rhoc, double ikv) const;
  void eval_mass_exchange_terms(const double* qpj, double bx, double by,
                                const double* erod, double dtl, double* ers,
                                double* dep, double& cpe, double& cpl, double* eqns,
                                double& topo, uint32_t& err) const;
  void eval_source_bdry(double time, double vx, double vy, double* sb) const;
  void kt_face(const double* qLf, const double* qpLf, const double* qRf, const double* qpRf,
               double aN, double aP, double gcf, int dir, double* H) const;
  static double minmod(double a, double b);
  static double maxmod(double a, double b);
  double limit(const double* v, const double* z, int lim) const;

  // ---------------------------------------------------------------- solver
  void check_solve(bool solve_all, double tt);
  void reconstruction(const double* q_expl, const double* qp_expl, bool stage_arrays);
  // A face written in an earlier step matters only if it carries a thickness
  // or a normal velocity (otherwise its speeds, flux and state are all zero).
  bool face_wet(const double* qpf, int iu) const { return qpf[0] > EPS || qpf[iu] != 0.0; }
  // A stage value of a cell outside the mask, compared with the value a fresh
  // evaluation from the current q would give.
  void note_stage_read(int jj, int kk);
  void eval_speeds();
  void eval_flux_KT();
  void eval_hyperbolic_terms(int irk);
  double timestep();
  void eval_f(const double* qj, const double* qj_old, double a_diag, const double* coeff_f,
              const double* Rj_not_impl, double bx, double by, double dtl, double* f_nl,
              double& scal_f) const;
  void eval_jacobian(const double* qj_rel, const double* qj_org, const double* coeff_f,
                     double bx, double by, double dtl, double a_diag, double* left) const;
  void lnsrch(const double* x_old, const double* qj_org, const double* qj_old,
              double scal_f_old, const double* grad_f, double* desc_dir,
              const double* coeff_f, double* qj_rel, double& scal_f, double* right_term,
              double stpmax, bool& check, const double* Rj_not_impl, double bx, double by,
              double dtl, double a_diag, int64_t& trials) const;
  int solve_rk_step(double* qj, const double* qj_old, double a_diag, const double* Rj_not_impl,
                    double bx, double by, double dtl, int64_t& trials) const;
  uint32_t imex_RK_solver(double dtl);
  uint32_t update_erosion_deposition_cell(double dtl);
  void post_step_sweep();
  void initial_sweep();
  // driver output sweep (src/IMEX_SfloW2D.f90:253-309, 391-442)
  bool post_on = false;
  int n_thk = 0, n_pdyn = 0;
  double thk_lev[10], pdyn_lev[10];
  std::vector<double> hmax, pdynmax, mvmax;
  std::vector<uint8_t> vuln;  // (n_thk*n_pdyn, cell)
  void post_cell(int j, int k, bool init);
  void topography_reconstruction();
};

// ------------------------------------------------------------------ mixt_var
// src/constitutive_2d.f90:1333-1483 (gas carrier, no liquid, no add. gas)
void OracleCtx::mixt_var(const double* qpj, double& r_Ri, double& r_rho_m,
                         double& r_rho_c, double& r_red_grav, bool sp_heat_flag,
                         double& r_sp_heat_c, double& r_sp_heat_mix) const {
  double r_h = qpj[0];
  if (qpj[0] <= EPS) {
    r_red_grav = 0.0;
    r_rho_m = rho_a_amb;
    r_rho_c = rho_a_amb;
    r_sp_heat_c = p.sp_heat_a;
    r_sp_heat_mix = p.sp_heat_a;
    r_Ri = 0.0;
    return;
  }
  double r_u = qpj[idx_u], r_v = qpj[idx_v], r_T = qpj[3];
  double r_alphas[MAXS];
  for (int i = 0; i < ns; ++i)
    r_alphas[i] = p.alpha_flag ? qpj[4 + i] : qpj[4 + i] / qpj[0];
  double alphas_tot = 0.0;
  for (int i = 0; i < ns; ++i) alphas_tot += r_alphas[i];
  double r_alphal = 0.0;
  double sum_alphag = 0.0, dot_alphag_rhog = 0.0;  // n_add_gas = 0
  double r_rho_a = p.pres / (p.sp_gas_const_a * r_T);
  r_rho_c = ((((1.0 - r_alphal) - alphas_tot) - sum_alphag) * r_rho_a + dot_alphag_rhog) /
            ((1.0 - r_alphal) - alphas_tot);
  double dot = 0.0;
  for (int i = 0; i < ns; ++i) dot += r_alphas[i] * p.rho_s[i];
  r_rho_m = (1.0 - alphas_tot) * r_rho_c + dot;
  double r_inv_rhom = 1.0 / r_rho_m;
  r_red_grav = (r_rho_m - rho_a_amb) / r_rho_m * p.grav;
  double vel2 = r_u * r_u + r_v * r_v;
  if (vel2 > 0.0)
    r_Ri = fmin_f(1.0e15, r_red_grav * r_h / vel2);
  else
    r_Ri = 0.0;
  if (sp_heat_flag) eval_sp_heat(r_alphas, r_inv_rhom, r_sp_heat_c, r_sp_heat_mix);
}

// src/constitutive_2d.f90:1503-1597 (gas, no liquid)
void OracleCtx::eval_sp_heat(const double* r_alphas, double r_inv_rhom, double& spc,
                             double& spm) const {
  double r_xs[MAXS];
  for (int i = 0; i < ns; ++i) r_xs[i] = r_alphas[i] * p.rho_s[i] * r_inv_rhom;
  double sxs = 0.0;
  for (int i = 0; i < ns; ++i) sxs += r_xs[i];
  double r_xc = 1.0 - sxs;
  spc = 0.0;
  if (r_xc > EPS)
    spc = ((r_xc - 0.0) * p.sp_heat_a + 0.0) / r_xc;
  else
    spc = p.sp_heat_a;
  double dot = 0.0;
  for (int i = 0; i < ns; ++i) dot += r_xs[i] * p.sp_heat_s[i];
  spm = dot + r_xc * spc;
}

// ------------------------------------------------------------- r_phys_var
// src/constitutive_2d.f90:541-967 (vertical-profile branch off)
void OracleCtx::r_phys_var(const double* r_qj, double& r_h, double& r_u, double& r_v,
                           double* r_alphas, double& r_rho_m, double& r_T,
                           double& r_red_grav, double& p_dyn) const {
  double inv_qj1, r_xs[MAXS];
  if (r_qj[0] > EPS) {
    inv_qj1 = 1.0 / r_qj[0];
    for (int i = 0; i < ns; ++i) r_xs[i] = r_qj[4 + i] * inv_qj1;
    double sq = 0.0;
    for (int i = 0; i < ns; ++i) sq += r_qj[4 + i];
    if (sq == r_qj[0]) {
      double sx = 0.0;
      for (int i = 0; i < ns; ++i) sx += r_xs[i];
      for (int i = 0; i < ns; ++i) r_xs[i] = r_xs[i] / sx;
    }
  } else {
    r_h = 0.0;
    r_u = 0.0;
    r_v = 0.0;
    for (int i = 0; i < ns; ++i) r_alphas[i] = 0.0;
    r_rho_m = rho_a_amb;
    r_T = p.T_ambient;
    r_red_grav = 0.0;
    p_dyn = 0.0;
    return;
  }
  double r_xs_tot = 0.0;
  for (int i = 0; i < ns; ++i) r_xs_tot += r_xs[i];
  double r_xc = 1.0 - r_xs_tot;
  double r_sp_heat_c_by_xc = ((r_xc - 0.0) * p.sp_heat_a + 0.0);
  double dot = 0.0;
  for (int i = 0; i < ns; ++i) dot += r_xs[i] * p.sp_heat_s[i];
  double r_sp_heat_mix = dot + r_sp_heat_c_by_xc;
  if (r_qj[0] > eps_sing) {
    if (p.energy_flag)
      r_T = (r_qj[3] - 0.5 * (r_qj[1] * r_qj[1] + r_qj[2] * r_qj[2]) * inv_qj1) /
            (r_qj[0] * r_sp_heat_mix);
    else
      r_T = r_qj[3] / (r_qj[0] * r_sp_heat_mix);
    if (r_T <= 0.0) r_T = p.T_ambient;
  } else {
    r_T = p.T_ambient;
  }
  double r_sp_gas_const_c;
  if (r_xc > EPS)
    r_sp_gas_const_c = ((r_xc - 0.0) * p.sp_gas_const_a + 0.0) / r_xc;
  else
    r_sp_gas_const_c = p.sp_gas_const_a;
  double r_inv_rho_c = r_sp_gas_const_c * r_T * inv_pres;
  double dot2 = 0.0;
  for (int i = 0; i < ns; ++i) dot2 += r_xs[i] * inv_rho_s[i];
  double r_inv_rhom = dot2 + r_xc * r_inv_rho_c;
  r_rho_m = 1.0 / r_inv_rhom;
  for (int i = 0; i < ns; ++i) r_alphas[i] = r_xs[i] * r_rho_m * inv_rho_s[i];
  r_h = r_qj[0] * r_inv_rhom;
  r_red_grav = (r_rho_m - rho_a_amb) * r_inv_rhom * p.grav;
  if (r_qj[0] > eps_sing) {
    r_u = r_qj[1] * inv_qj1;
    r_v = r_qj[2] * inv_qj1;
  } else {
    double q1 = r_qj[0];
    double q14 = (q1 * q1) * (q1 * q1);
    r_u = std::sqrt(2.0) * r_qj[0] * r_qj[1] / std::sqrt(q14 + eps_sing4);
    r_v = std::sqrt(2.0) * r_qj[0] * r_qj[2] / std::sqrt(q14 + eps_sing4);
  }
  p_dyn = 0.5 * r_rho_m * (r_u * r_u + r_v * r_v);
}

// src/constitutive_2d.f90:1628-1681
void OracleCtx::qc_to_qp(const double* qc, double* qpo, double& p_dyn) const {
  double r_h, r_u, r_v, r_alphas[MAXS], r_rho_m, r_T, r_red_grav;
  r_phys_var(qc, r_h, r_u, r_v, r_alphas, r_rho_m, r_T, r_red_grav, p_dyn);
  qpo[0] = r_h;
  qpo[1] = r_h * r_u;
  qpo[2] = r_h * r_v;
  qpo[3] = r_T;
  for (int i = 0; i < ns; ++i) qpo[4 + i] = p.alpha_flag ? r_alphas[i] : r_alphas[i] * r_h;
  qpo[idx_u] = r_u;
  qpo[idx_v] = r_v;
}

// src/constitutive_2d.f90:1709-2140 (vertical-profile branch off, gas carrier)
void OracleCtx::qp_to_qc(const double* qpi, double* qc) const {
  double r_h = qpi[0];
  double r_hu, r_hv, r_u, r_v;
  if (r_h > EPS) {
    r_hu = qpi[1];
    r_hv = qpi[2];
    r_u = qpi[idx_u];
    r_v = qpi[idx_v];
  } else {
    for (int i = 0; i < nv; ++i) qc[i] = 0.0;
    return;
  }
  double r_T = qpi[3];
  double r_alphas[MAXS], r_alphas_rhos[MAXS];
  for (int i = 0; i < ns; ++i)
    r_alphas[i] = p.alpha_flag ? qpi[4 + i] : qpi[4 + i] / qpi[0];
  double alphas_tot = 0.0;
  for (int i = 0; i < ns; ++i) alphas_tot += r_alphas[i];
  for (int i = 0; i < ns; ++i) r_alphas_rhos[i] = r_alphas[i] * p.rho_s[i];
  double r_alphal = 0.0;
  double r_rho_a = p.pres / (p.sp_gas_const_a * r_T);
  double r_rho_c = ((((1.0 - r_alphal) - alphas_tot) - 0.0) * r_rho_a + 0.0) /
                   ((1.0 - r_alphal) - alphas_tot);
  // the correction of r_alphas at src/constitutive_2d.f90:1924-1932 does not
  // reach any output (r_alphas_rhos and alphas_tot were taken before it)
  double r_alphac = 1.0 - alphas_tot;
  double sar = 0.0;
  for (int i = 0; i < ns; ++i) sar += r_alphas_rhos[i];
  double r_rho_m = r_alphac * r_rho_c + sar;
  double r_inv_rhom = 1.0 / r_rho_m;
  double r_xs[MAXS];
  for (int i = 0; i < ns; ++i) r_xs[i] = r_alphas_rhos[i] * r_inv_rhom;
  double r_xc = r_alphac * r_rho_c * r_inv_rhom;
  double r_sp_heat_c;
  if (r_xc > EPS)
    r_sp_heat_c = ((r_xc - 0.0) * p.sp_heat_a + 0.0) / r_xc;
  else
    r_sp_heat_c = p.sp_heat_a;
  double dot = 0.0;
  for (int i = 0; i < ns; ++i) dot += r_xs[i] * p.sp_heat_s[i];
  double r_sp_heat_mix = dot + r_xc * r_sp_heat_c;
  qc[0] = r_rho_m * r_h;
  qc[1] = r_rho_m * r_hu;
  qc[2] = r_rho_m * r_hv;
  if (p.energy_flag) {
    if (r_h > 0.0)
      qc[3] = r_h * r_rho_m * (r_sp_heat_mix * r_T + 0.5 * (r_u * r_u + r_v * r_v));
    else
      qc[3] = 0.0;
  } else {
    qc[3] = r_h * r_rho_m * r_sp_heat_mix * r_T;
  }
  for (int i = 0; i < ns; ++i) qc[4 + i] = r_xs[i] * qc[0];
}

// src/constitutive_2d.f90:2155-2179
void OracleCtx::qp_to_qp2(const double* qpj, double Bj, double* qp2) const {
  qp2[0] = qpj[0] + Bj;
  if (qpj[0] <= 0.0) {
    qp2[1] = 0.0;
    qp2[2] = 0.0;
  } else {
    qp2[1] = qpj[1] / qpj[0];
    qp2[2] = qpj[2] / qpj[0];
  }
}

// src/constitutive_2d.f90:2194-2240
void OracleCtx::eval_local_speeds_x(const double* qpj, double gcf, double& vmin,
                                    double& vmax) const {
  double Ri, rho_m, rho_c, red_grav, spc, spm;
  mixt_var(qpj, Ri, rho_m, rho_c, red_grav, false, spc, spm);
  double r_h = qpj[0], r_u = qpj[idx_u];
  if (red_grav * r_h < 0.0) {
    vmin = r_u;
    vmax = r_u;
  } else {
    double c = std::sqrt(red_grav * r_h * gcf);
    vmin = r_u - c;
    vmax = r_u + c;
  }
}

// src/constitutive_2d.f90:2254-2298
void OracleCtx::eval_local_speeds_y(const double* qpj, double gcf, double& vmin,
                                    double& vmax) const {
  double Ri, rho_m, rho_c, red_grav, spc, spm;
  mixt_var(qpj, Ri, rho_m, rho_c, red_grav, false, spc, spm);
  double r_h = qpj[0], r_v = qpj[idx_v];
  if (red_grav * r_h < 0.0) {
    vmin = r_v;
    vmax = r_v;
  } else {
    double c = std::sqrt(gcf * red_grav * r_h);
    vmin = r_v - c;
    vmax = r_v + c;
  }
}

// src/constitutive_2d.f90:2316-2509 (shape_coeff = 1)
void OracleCtx::eval_fluxes(const double* qcj, const double* qpj, double gcf, int dir,
                            double* flux) const {
  if (qpj[0] > EPS) {
    double r_h = qpj[0], r_u = qpj[idx_u], r_v = qpj[idx_v];
    double Ri, rho_m, rho_c, red_grav, spc, spm;
    mixt_var(qpj, Ri, rho_m, rho_c, red_grav, false, spc, spm);
    double pres_term = 0.5 * rho_m * gcf * red_grav * (r_h * r_h);
    double vel = (dir == 1) ? r_u : r_v;
    flux[0] = vel * qcj[0];
    if (dir == 1) {
      flux[1] = r_u * qcj[1] + pres_term;
      flux[2] = r_u * qcj[2];
    } else {
      flux[1] = r_v * qcj[1];
      flux[2] = r_v * qcj[2] + pres_term;
    }
    if (p.energy_flag)
      flux[3] = vel * (qcj[3] + pres_term);
    else
      flux[3] = vel * qcj[3];
    for (int i = 0; i < ns; ++i) flux[4 + i] = vel * qcj[4 + i];
    if (flux[0] > 0.0) {
      double s = 0.0;
      for (int i = 0; i < ns; ++i) s += flux[4 + i];
      if (s / flux[0] > 1.0)
        for (int i = 0; i < ns; ++i) flux[4 + i] = flux[4 + i] / s * flux[0];
    }
  } else {
    for (int i = 0; i < nv; ++i) flux[i] = 0.0;
  }
}

// src/constitutive_2d.f90:3015-3245 (bottom radial source off)
void OracleCtx::eval_expl_terms(double bx, double by, double bxx, double bxy, double byy,
                                double gcf, double dgcx, double dgcy, const double* qpj,
                                double* expl, double csf) const {
  for (int i = 0; i < nv; ++i) expl[i] = 0.0;
  if (qpj[0] <= EPS && csf == 0.0) return;
  double r_h = qpj[0], r_u = qpj[idx_u], r_v = qpj[idx_v];
  double Ri, rho_m, rho_c, red_grav, spc, spm;
  mixt_var(qpj, Ri, rho_m, rho_c, red_grav, true, spc, spm);
  double centr = 0.0;
  if (p.curvature_term_flag)
    centr = bxx * (r_u * r_u) + 2.0 * bxy * r_u * r_v + byy * (r_v * r_v);
  double tg = red_grav + centr;
  expl[1] = -(gcf * rho_m * tg * r_h * bx) + 0.5 * rho_m * red_grav * (r_h * r_h) * dgcx;
  expl[2] = -(gcf * rho_m * tg * r_h * by) + 0.5 * rho_m * red_grav * (r_h * r_h) * dgcy;
  if (p.energy_flag)
    expl[3] = expl[1] * r_u + expl[2] * r_v;
  else
    expl[3] = 0.0;
}

// ------------------------------------------------------------ c_phys_var
// src/constitutive_2d.f90:1145-1313 (gas carrier, no liquid, no add. gas)
void OracleCtx::c_phys_var(const cplx* c_qj, cplx& h_, cplx& u, cplx& v, cplx& T,
                           cplx& rho_m, cplx* alphas, cplx& inv_rhom) const {
  cplx inv_cqj1, xs[MAXS];
  if (c_qj[0].re > EPS) {
    inv_cqj1 = rdiv(1.0, c_qj[0]);
    for (int i = 0; i < ns; ++i) xs[i] = c_qj[4 + i] * inv_cqj1;
  } else {
    h_ = C(0.0);
    u = C(0.0);
    v = C(0.0);
    T = C(p.T_ambient);
    rho_m = C(rho_a_amb);
    for (int i = 0; i < ns; ++i) alphas[i] = C(0.0);
    inv_rhom = rdiv(1.0, rho_m);
    return;
  }
  cplx xs_tot = C(0.0);
  for (int i = 0; i < ns; ++i) xs_tot = xs_tot + xs[i];
  cplx xc = rsub(1.0, xs_tot);
  cplx sum_xg = C(0.0), dot_xg = C(0.0);  // n_add_gas = 0
  cplx sp_heat_c = (mulr(xc - sum_xg, p.sp_heat_a) + dot_xg) / xc;
  // DOT_PRODUCT(complex, real) = SUM(CONJG(a)*b)
  cplx dot = C(0.0);
  for (int i = 0; i < ns; ++i) dot = dot + mulr(conj(xs[i]), p.sp_heat_s[i]);
  cplx sp_heat_mix = dot + xc * sp_heat_c;
  if (c_qj[0].re > eps_sing) {
    if (p.energy_flag)
      T = (c_qj[3] - mulr(c_qj[1] * c_qj[1] + c_qj[2] * c_qj[2], 0.5) * inv_cqj1) /
          (c_qj[0] * sp_heat_mix);
    else
      T = c_qj[3] / (c_qj[0] * sp_heat_mix);
    if (T.re <= 0.0) T = C(p.T_ambient);
  } else {
    T = C(p.T_ambient);
  }
  cplx sp_gas_const_c = (mulr(xc - sum_xg, p.sp_gas_const_a) + dot_xg) / xc;
  cplx inv_rho_c = mulr(sp_gas_const_c * T, inv_pres);
  // DOT_PRODUCT(complex, complex) = SUM(CONJG(a)*b); c_inv_rho_s is COMPLEX
  cplx dot2 = C(0.0);
  for (int i = 0; i < ns; ++i) dot2 = dot2 + conj(xs[i]) * C(inv_rho_s[i], 0.0);
  inv_rhom = dot2 + xc * inv_rho_c;
  rho_m = rdiv(1.0, inv_rhom);
  for (int i = 0; i < ns; ++i) alphas[i] = rho_m * xs[i] * C(inv_rho_s[i], 0.0);
  h_ = c_qj[0] * inv_rhom;
  if (c_qj[0].re > eps_sing) {
    u = c_qj[1] * inv_cqj1;
    v = c_qj[2] * inv_cqj1;
  } else {
    cplx q1 = c_qj[0];
    cplx q12 = q1 * q1;
    cplx den = csqrt_(addr(q12 * q12, eps_sing4));
    u = mulr(c_qj[0], std::sqrt(2.0));
    u = (u * c_qj[1]) / den;
    v = mulr(c_qj[0], std::sqrt(2.0));
    v = (v * c_qj[2]) / den;
  }
}

// src/constitutive_2d.f90:3327-3823 (rheology models 0, 1, 6; no pore pressure)
void OracleCtx::eval_implicit_terms(double bx, double by, const cplx* qj, cplx* nh) const {
  for (int i = 0; i < nv; ++i) nh[i] = C(0.0, 0.0);
  if (!p.rheology_flag) return;
  cplx h_, u, v, T, rho_m, alphas[MAXS], inv_rho_m;
  c_phys_var(qj, h_, u, v, T, rho_m, alphas, inv_rho_m);
  cplx red_grav = mulr(subr(rho_m, rho_a_amb) / rho_m, p.grav);
  cplx w;
  if (p.slope_correction_flag)
    w = mulr(u, bx) + mulr(v, by);
  else
    w = C(0.0, 0.0);
  cplx mod_vel2 = u * u + v * v + w * w;
  cplx mod_vel = csqrt_(mod_vel2);
  cplx mod_vel_hor = csqrt_(u * u + v * v);
  if (p.rheology_model == 1) {
    if (mod_vel.re != 0.0) {
      cplx turb_stress = divr(rho_m * red_grav, p.xi) * mod_vel2;
      nh[1] = nh[1] - turb_stress * (u / mod_vel);
      nh[2] = nh[2] - turb_stress * (v / mod_vel);
    }
  } else if (p.rheology_model == 6) {
    if (mod_vel.re != 0.0) {
      nh[1] = nh[1] - mulr(rho_m * (u / mod_vel_hor), p.friction_factor) * mod_vel2;
      nh[2] = nh[2] - mulr(rho_m * (v / mod_vel_hor), p.friction_factor) * mod_vel2;
    }
  }
}

// The real path of eval_implicit_terms: CMPLX(r_qj,0) through the complex code,
// REAL() of the result (src/constitutive_2d.f90:3425-3441, 3812-3818).
void OracleCtx::eval_implicit_terms_r(double bx, double by, const double* r_qj,
                                      double* r_nh) const {
  cplx qj[MAXV], nh[MAXV];
  for (int i = 0; i < nv; ++i) qj[i] = C(r_qj[i], 0.0);
  eval_implicit_terms(bx, by, qj, nh);
  for (int i = 0; i < nv; ++i) r_nh[i] = nh[i].re;
}

// src/constitutive_2d.f90:3841-4397 (Voellmy-Salm Coulomb part; others zero)
void OracleCtx::eval_nh_semi_impl_terms(double bx, double by, double bxx, double bxy,
                                        double byy, double gcf, const double* qcj,
                                        const double* qpj, double* si) const {
  (void)qcj;
  for (int i = 0; i < nv; ++i) si[i] = 0.0;
  if (!p.rheology_flag) return;
  double r_h = qpj[0], r_u = qpj[idx_u], r_v = qpj[idx_v];
  double Ri, rho_m, rho_c, red_grav, spc, spm;
  mixt_var(qpj, Ri, rho_m, rho_c, red_grav, false, spc, spm);
  double r_w = p.slope_correction_flag ? (r_u * bx + r_v * by) : 0.0;
  double mod_vel = std::sqrt(r_u * r_u + r_v * r_v + r_w * r_w);
  if (p.rheology_model == 1) {
    if (mod_vel > 0.0) {
      double centr = 0.0;
      if (p.curvature_term_flag)
        centr = bxx * (r_u * r_u) + 2.0 * bxy * r_u * r_v + byy * (r_v * r_v);
      double temp = p.mu * rho_m * (red_grav + centr) * r_h * std::sqrt(gcf);
      temp = fmax_f(0.0, temp);
      temp = fmax_f(0.0, temp);
      si[1] = si[1] - temp * r_u / mod_vel;
      si[2] = si[2] - temp * r_v / mod_vel;
    }
  }
}

// src/constitutive_2d.f90:5148-5214
static double settling_velocity_g(double diam, double rhos, double rhoc, double ikv,
                                  double grav) {
  double inv_sqrt_C_D = 1.0;
  if (rhos <= rhoc) return 0.0;
  double const_part = std::sqrt(0.75 * (rhos / rhoc - 1.0) * diam * grav);
  double sv = const_part * inv_sqrt_C_D;
  double Rey = diam * sv * ikv;
  if (Rey <= 1000.0) {
    for (int i = 1; i <= 20; ++i) {
      double sv_old = sv;
      inv_sqrt_C_D = std::sqrt(Rey / (24.0 * (1.0 + 0.15 * ipow(Rey, 0.687))));
      sv = const_part * inv_sqrt_C_D;
      if (std::fabs(sv_old - sv) / sv_old < 1.0e-6) return sv;
      Rey = diam * sv * ikv;
    }
  }
  return sv;
}
double OracleCtx::settling_velocity(double diam, double rhos, double rhoc,
                                    double ikv) const {
  return settling_velocity_g(diam, rhos, rhoc, ikv, p.grav);
}

// src/constitutive_2d.f90:4424-5003 (no liquid, no pore pressure, no profiles)
void OracleCtx::eval_mass_exchange_terms(const double* qpj, double bx, double by,
                                         const double* erod, double dtl, double* ers,
                                         double* dep, double& cpe, double& cpl,
                                         double* eqns, double& topo,
                                         uint32_t& err) const {
  for (int i = 0; i < ns; ++i) {
    ers[i] = 0.0;
    dep[i] = 0.0;
  }
  cpe = 0.0;
  cpl = 0.0;
  for (int i = 0; i < nv; ++i) eqns[i] = 0.0;
  topo = 0.0;
  if (qpj[0] <= EPS) return;
  const double alpha_max = 0.6, hind_exp = 4.65;
  double r_h = qpj[0], r_u = qpj[idx_u], r_v = qpj[idx_v];
  double r_alphas[MAXS];
  for (int i = 0; i < ns; ++i)
    r_alphas[i] = p.alpha_flag ? qpj[4 + i] : qpj[4 + i] / qpj[0];
  double alphas_tot = 0.0;
  for (int i = 0; i < ns; ++i) alphas_tot += r_alphas[i];
  double r_w = p.slope_correction_flag ? (r_u * bx + r_v * by) : 0.0;
  double mod_vel2 = r_u * r_u + r_v * r_v + r_w * r_w;
  double mod_vel = std::sqrt(mod_vel2);
  double tot_solid_erosion;
  if (p.erosion_coeff > 0.0) {
    double tot_erosion = p.erosion_coeff * mod_vel * r_h * (1.0 - alphas_tot);
    tot_solid_erosion = tot_erosion * (1.0 - p.erodible_porosity);
    for (int i = 0; i < ns; ++i) ers[i] = p.erodible_fract[i] * tot_solid_erosion;
  } else {
    tot_solid_erosion = 0.0;
    for (int i = 0; i < ns; ++i) ers[i] = 0.0;
  }
  for (int i = 0; i < ns; ++i) ers[i] = fmax_f(0.0, fmin_f(ers[i], erod[i] / dtl));
  tot_solid_erosion = 0.0;
  for (int i = 0; i < ns; ++i) tot_solid_erosion += ers[i];
  double tot_erosion = tot_solid_erosion / (1.0 - p.erodible_porosity);
  cpe = tot_erosion * p.erodible_porosity;
  if (alphas_tot <= p.alphastot_min) return;
  double r_T = qpj[3];
  double r_Ri, r_rho_m, r_rho_c, r_red_grav, r_sp_heat_c, r_sp_heat_mix;
  mixt_var(qpj, r_Ri, r_rho_m, r_rho_c, r_red_grav, true, r_sp_heat_c, r_sp_heat_mix);
  double inv_kin_visc = 1.0 / p.kin_visc_c;
  double rhoc = r_rho_c;
  for (int i = 0; i < ns; ++i) {
    if (r_alphas[i] > 0.0 && p.settling_flag) {
      double sv = settling_velocity(p.diam_s[i], p.rho_s[i], rhoc, inv_kin_visc);
      dep[i] = r_alphas[i] * sv * 1.0;
      dep[i] = dep[i] * ipow(1.0 - fmin_f(1.0, alphas_tot / alpha_max), hind_exp);
      dep[i] = fmin_f(dep[i], r_h * r_alphas[i] / dtl);
      if (dep[i] < 0.0) err |= IMEX_ERRBIT(IMEX_EEROSION);
    }
  }
  cpl = 0.0;
  double sdep = 0.0;
  for (int i = 0; i < ns; ++i) sdep += dep[i];
  cpl = cpl + p.coeff_porosity * sdep;
  double sal = 0.0;
  for (int i = 0; i < ns; ++i) sal += r_alphas[i];
  cpl = fmin_f(cpl, r_h * fmax_f(0.0, p.maximum_solid_packing - sal) / dtl);
  cpl = fmin_f(cpl, (r_h * (1.0 - sal) - p.coeff_porosity * (r_h * sal - dtl * sdep)) / dtl);
  double T_erodible = p.erodible_deposit_flag ? r_T : p.T_erodible;
  double air_entr;
  if (p.entrainment_flag && r_h > 0.0 && r_Ri > 0.0) {
    double entr_coeff = 0.075 / std::sqrt(1.0 + 718.0 * ipow(r_Ri, 2.4));
    air_entr = entr_coeff * std::sqrt(mod_vel2);
  } else {
    air_entr = 0.0;
  }
  for (int i = 0; i < nv; ++i) eqns[i] = 0.0;
  double dep_tot = 0.0, ers_tot = 0.0, rho_dep_tot = 0.0, rho_ers_tot = 0.0;
  for (int i = 0; i < ns; ++i) dep_tot += dep[i];
  for (int i = 0; i < ns; ++i) ers_tot += ers[i];
  for (int i = 0; i < ns; ++i) rho_dep_tot += p.rho_s[i] * dep[i];
  for (int i = 0; i < ns; ++i) rho_ers_tot += p.rho_s[i] * ers[i];
  eqns[0] = rho_a_amb * air_entr + rho_ers_tot - rho_dep_tot + p.rho_c_sub * cpe -
            r_rho_c * cpl;
  eqns[1] = -(r_u * (rho_dep_tot + r_rho_c * cpl));
  eqns[2] = -(r_v * (rho_dep_tot + r_rho_c * cpl));
  double sdh = 0.0, seh = 0.0;
  for (int i = 0; i < ns; ++i) sdh += p.rho_s[i] * p.sp_heat_s[i] * dep[i];
  for (int i = 0; i < ns; ++i) seh += p.rho_s[i] * p.sp_heat_s[i] * ers[i];
  if (p.energy_flag)
    eqns[3] = -(r_T * (sdh + r_rho_c * r_sp_heat_c * cpl)) -
              0.5 * mod_vel2 * (rho_dep_tot + r_rho_c * cpl) +
              T_erodible * (seh + p.rho_c_sub * r_sp_heat_c * cpe) +
              p.T_ambient * p.sp_heat_a * rho_a_amb * air_entr;
  else
    eqns[3] = -(r_T * (sdh + r_rho_c * r_sp_heat_c * cpl)) +
              T_erodible * (seh + p.rho_c_sub * r_sp_heat_c * cpe) +
              p.T_ambient * p.sp_heat_a * rho_a_amb * air_entr;
  for (int i = 0; i < ns; ++i) eqns[4 + i] = p.rho_s[i] * (ers[i] - dep[i]);
  topo = (dep_tot - ers_tot) / (1.0 - p.erodible_porosity);
}

// src/constitutive_2d.f90:5024-5130
void OracleCtx::eval_source_bdry(double time, double vx, double vy, double* sb) const {
  const double* tp = p.time_param;
  if (time >= tp[3]) {
    sb[0] = 0.0;
    sb[1] = 0.0;
    sb[2] = 0.0;
    sb[3] = p.T_source;
    for (int i = 0; i < ns; ++i) sb[4 + i] = 0.0;
    sb[idx_u] = 0.0;
    sb[idx_v] = 0.0;
    return;
  }
  double t_rem = std::fmod(time, tp[0]);
  double t_coeff = 0.0;
  const double pi_g = 4.0 * std::atan(1.0);
  if (tp[2] == 0.0) {
    if (t_rem <= tp[1]) t_coeff = 1.0;
  } else {
    if (t_rem < tp[2])
      t_coeff = 0.5 * (1.0 - std::cos(pi_g * t_rem / tp[2]));
    else if (t_rem <= (tp[1] - tp[2]))
      t_coeff = 1.0;
    else if (t_rem <= tp[1])
      t_coeff = 0.5 * (1.0 + std::cos(pi_g * ((t_rem - tp[1]) / tp[2] + 1.0)));
  }
  double tc15 = ipow(t_coeff, 1.5), tc05 = ipow(t_coeff, 0.5);
  sb[0] = t_coeff * p.h_source;
  sb[1] = tc15 * p.h_source * p.vel_source * vx;
  sb[2] = tc15 * p.h_source * p.vel_source * vy;
  sb[3] = p.T_source;
  for (int i = 0; i < ns; ++i)
    sb[4 + i] = p.alpha_flag ? p.alphas_source[i] : t_coeff * p.h_source * p.alphas_source[i];
  sb[idx_u] = tc05 * p.vel_source * vx;
  sb[idx_v] = tc05 * p.vel_source * vy;
}

// ------------------------------------------------------------- limiters
// src/geometry_2d.f90:1634-1676
double OracleCtx::minmod(double a, double b) {
  if (fmin_f(std::fabs(a), std::fabs(b)) <= 0.0) return 0.0;
  double sa = a / std::fabs(a), sb = b / std::fabs(b);
  return 0.5 * (sa + sb) * fmin_f(std::fabs(a), std::fabs(b));
}
double OracleCtx::maxmod(double a, double b) {
  if (std::fabs(a * b) <= 0.0) return 0.0;
  double sa = a / std::fabs(a), sb = b / std::fabs(b);
  return 0.5 * (sa + sb) * fmax_f(std::fabs(a), std::fabs(b));
}
// src/geometry_2d.f90:1555-1620
double OracleCtx::limit(const double* v, const double* z, int lim) const {
  double a = (v[2] - v[1]) / (z[2] - z[1]);
  double b = (v[1] - v[0]) / (z[1] - z[0]);
  double c = (v[2] - v[0]) / (z[2] - z[0]);
  switch (lim) {
    case 0: return 0.0;
    case 1: return minmod(a, b);
    case 2: return maxmod(minmod(a, 2.0 * b), minmod(2.0 * a, b));
    case 3: return minmod(c, p.theta * minmod(a, b));
    case 4: return minmod(c, 2.0 * minmod(a, b));
    case 5: return c;
    case 6: return a;
    case 7: return b;
  }
  return 0.0;
}

// ---------------------------------------------------------- check_solve
// src/solver_2d.f90:666-857
void OracleCtx::check_solve(bool solve_all, double tt) {
  for (int k = 2; k <= ny - 1; ++k)
    for (int j = 2; j <= nx - 1; ++j) mask[c2(j, k)] = solve_all ? 1 : 0;
  for (int k = 2; k <= ny - 1; ++k)
    for (int j = 2; j <= nx - 1; ++j)
      if (Q(q, j, k)[0] > 0.0 && solve_mask_time[c2(j, k)] <= tt) mask[c2(j, k)] = 1;
  if (p.bottom_radial_source_flag)
    for (size_t c = 0; c < mask.size(); ++c)
      if (cell_source_fractions[c] > 0.0) mask[c] = 1;
  if (p.radial_source_flag)
    for (int k = 2; k <= ny - 1; ++k)
      for (int j = 2; j <= nx - 1; ++j)
        if (source_cell[c2(j, k)] == 2) mask[c2(j, k)] = 1;
  for (int i = 1; i <= nrk; ++i) {
    mask_temp = mask;
    for (int k = 2; k <= ny - 1; ++k)
      for (int j = 2; j <= nx - 1; ++j) {
        uint8_t m = mask[c2(j, k)];
        m = m | mask_temp[c2(j - 1, k)];
        m = m | mask_temp[c2(j + 1, k)];
        m = m | mask_temp[c2(j, k - 1)];
        m = m | mask_temp[c2(j, k + 1)];
        mask[c2(j, k)] = m;
      }
  }
  if (p.radial_source_flag)
    for (size_t c = 0; c < mask.size(); ++c)
      if (source_cell[c] == 1) mask[c] = 0;
  std::fill(mask_x.begin(), mask_x.end(), 0);
  std::fill(mask_y.begin(), mask_y.end(), 0);
  int64_t i = 0;
  for (int k = 1; k <= ny; ++k)
    for (int j = 1; j <= nx; ++j)
      if (mask[c2(j, k)]) {
        j_cent[i] = j;
        k_cent[i] = k;
        ++i;
        mask_x[sx2(j, k)] = 1;
        mask_x[sx2(j + 1, k)] = 1;
        mask_y[sy2(j, k)] = 1;
        mask_y[sy2(j, k + 1)] = 1;
      }
  solve_cells = i;
  i = 0;
  for (int k = 1; k <= ny; ++k)
    for (int j = 1; j <= nx + 1; ++j)
      if (mask_x[sx2(j, k)]) {
        j_stag_x[i] = j;
        k_stag_x[i] = k;
        ++i;
      }
  solve_interfaces_x = i;
  i = 0;
  for (int k = 1; k <= ny + 1; ++k)
    for (int j = 1; j <= nx; ++j)
      if (mask_y[sy2(j, k)]) {
        j_stag_y[i] = j;
        k_stag_y[i] = k;
        ++i;
      }
  solve_interfaces_y = i;
}

// ------------------------------------------------------- reconstruction
// src/solver_2d.f90:3093-3918.  `stage_arrays` marks the stage-1 call, whose
// neighbour values come from q_rk/qp_rk (for the stale-read instrument).
void OracleCtx::reconstruction(const double* q_expl, const double* qp_expl,
                               bool stage_arrays) {
  const bool src_any = p.lateral_source_flag || p.radial_source_flag;
  ++recon_epoch;
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < solve_cells; ++l) {
    const int j = j_cent[l], k = k_cent[l];
    double qrecW[MAXP], qrecE[MAXP], qrecS[MAXP], qrecN[MAXP];
    double source_bdry[MAXP] = {0};
    double qrec_prime_x[MAXP] = {0}, qrec_prime_y[MAXP] = {0};
    double qp2recW[3], qp2recE[3], qp2recS[3], qp2recN[3];
    double qrec_stencil[3] = {0, 0, 0}, x_stencil[3] = {0, 0, 0}, y_stencil[3] = {0, 0, 0};
    auto QPC = [&](int jj, int kk) -> const double* { return qp_expl + (size_t)np * c2(jj, kk); };
    auto QPE = [&](int i, int jj, int kk) -> double {
#ifndef ORACLE_TIMING
      if (stage_arrays && !mask[c2(jj, kk)]) note_stage_read(jj, kk);
#endif
      return QPC(jj, kk)[i - 1];
    };
    const size_t cc = c2(j, k);
    for (int i = 0; i < np; ++i) qrecW[i] = qrecE[i] = qrecS[i] = qrecN[i] = QPC(j, k)[i];
    x_stencil[1] = x_comp[j - 1];
    y_stencil[1] = y_comp[k - 1];
    const int scell = (src_any ? source_cell[cc] : 0);
    if (src_any && scell == 2) {
      if (sE[cc])
        eval_source_bdry(t, sEx[cc], sEy[cc], source_bdry);
      else if (sW[cc])
        eval_source_bdry(t, sWx[cc], sWy[cc], source_bdry);
      else if (sS[cc])
        eval_source_bdry(t, sSx[cc], sSy[cc], source_bdry);
      else if (sN[cc])
        eval_source_bdry(t, sNx[cc], sNy[cc], source_bdry);
    }
    const bool rad = p.radial_source_flag != 0;
    for (int i = 1; i <= nv; ++i) {
      qrec_stencil[1] = QPC(j, k)[i - 1];
      if (nx > 1) {
        if (j == 1) {
          x_stencil[0] = x_stag[0];
          x_stencil[2] = x_comp[j];
          if (scell == 2) {
            qrec_stencil[0] = source_bdry[i - 1];
            qrec_stencil[2] = QPE(i, j + 1, k);
            qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
          } else {
            const ImexBC& b = p.bcW[i - 1];
            if (b.flag == 0) {
              qrec_stencil[0] = b.value;
              qrec_stencil[2] = QPE(i, j + 1, k);
              qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
            } else if (b.flag == 1) {
              qrec_prime_x[i - 1] = b.value;
            } else if (b.flag == 2) {
              qrec_prime_x[i - 1] = (QPE(i, 2, k) - QPE(i, 1, k)) * one_by_dx;
            }
          }
        } else if (j == nx) {
          x_stencil[2] = x_stag[nx];
          x_stencil[0] = x_comp[j - 2];
          if (scell == 2) {
            qrec_stencil[2] = source_bdry[i - 1];
            qrec_stencil[0] = QPE(i, j - 1, k);
            qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
          } else {
            const ImexBC& b = p.bcE[i - 1];
            if (b.flag == 0) {
              qrec_stencil[2] = b.value;
              qrec_stencil[0] = QPE(i, j - 1, k);
              qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
            } else if (b.flag == 1) {
              qrec_prime_x[i - 1] = b.value;
            } else if (b.flag == 2) {
              qrec_prime_x[i - 1] = (QPE(i, nx, k) - QPE(i, nx - 1, k)) * one_by_dx;
            }
          }
        } else {
          x_stencil[0] = x_comp[j - 2];
          x_stencil[2] = x_comp[j];
          qrec_stencil[0] = QPE(i, j - 1, k);
          qrec_stencil[2] = QPE(i, j + 1, k);
          if (rad && scell == 2) {
            if (sE[cc]) {
              x_stencil[2] = x_stag[j];
              qrec_stencil[2] = source_bdry[i - 1];
            } else if (sW[cc]) {
              x_stencil[0] = x_stag[j - 1];
              qrec_stencil[0] = source_bdry[i - 1];
            }
          }
          qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
        }
        double dq = p.reconstr_coeff * dx2 * qrec_prime_x[i - 1];
        qrecW[i - 1] = qrec_stencil[1] - dq;
        qrecE[i - 1] = qrec_stencil[1] + dq;
        if (j == 1) {
          if (scell == 2)
            qrecW[i - 1] = source_bdry[i - 1];
          else if (p.bcW[i - 1].flag == 0)
            qrecW[i - 1] = p.bcW[i - 1].value;
          else if (i == 2)
            qrecW[i - 1] = fmin_f(qrecW[i - 1], 0.0);
        }
        if (j == nx) {
          if (scell == 2)
            qrecE[i - 1] = source_bdry[i - 1];
          else if (p.bcE[i - 1].flag == 0)
            qrecE[i - 1] = p.bcE[i - 1].value;
          else if (i == 2)
            qrecE[i - 1] = fmax_f(qrecE[i - 1], 0.0);
        }
      }
      if (ny > 1) {
        if (k == 1) {
          y_stencil[0] = y_stag[0];
          y_stencil[2] = y_comp[k];
          const ImexBC& b = p.bcS[i - 1];
          if (b.flag == 0) {
            qrec_stencil[0] = b.value;
            qrec_stencil[2] = QPE(i, j, k + 1);
            qrec_prime_y[i - 1] = limit(qrec_stencil, y_stencil, p.limiter[i - 1]);
          } else if (b.flag == 1) {
            qrec_prime_y[i - 1] = b.value;
          } else if (b.flag == 2) {
            qrec_prime_y[i - 1] = (QPE(i, j, 2) - QPE(i, j, 1)) * one_by_dy;
          }
        } else if (k == ny) {
          y_stencil[0] = y_comp[k - 2];
          y_stencil[2] = y_stag[ny];
          const ImexBC& b = p.bcN[i - 1];
          if (b.flag == 0) {
            qrec_stencil[0] = QPE(i, j, k - 1);
            qrec_stencil[2] = b.value;
            qrec_prime_y[i - 1] = limit(qrec_stencil, y_stencil, p.limiter[i - 1]);
          } else if (b.flag == 1) {
            qrec_prime_y[i - 1] = b.value;
          } else if (b.flag == 2) {
            qrec_prime_y[i - 1] = (QPE(i, j, ny) - QPE(i, j, ny - 1)) * one_by_dy;
          }
        } else {
          y_stencil[0] = y_comp[k - 2];
          y_stencil[2] = y_comp[k];
          qrec_stencil[0] = QPE(i, j, k - 1);
          qrec_stencil[2] = QPE(i, j, k + 1);
          if (rad && scell == 2) {
            if (sS[cc]) {
              y_stencil[0] = y_stag[k - 1];
              qrec_stencil[0] = source_bdry[i - 1];
            } else if (sN[cc]) {
              y_stencil[2] = y_stag[k];
              qrec_stencil[2] = source_bdry[i - 1];
            }
          }
          qrec_prime_y[i - 1] = limit(qrec_stencil, y_stencil, p.limiter[i - 1]);
        }
        double dq = p.reconstr_coeff * dy2 * qrec_prime_y[i - 1];
        qrecS[i - 1] = qrec_stencil[1] - dq;
        qrecN[i - 1] = qrec_stencil[1] + dq;
        if (k == 1) {
          if (p.bcS[i - 1].flag == 0)
            qrecS[i - 1] = p.bcS[i - 1].value;
          else if (i == 3)
            qrecS[i - 1] = fmin_f(qrecS[i - 1], 0.0);
        }
        if (k == ny) {
          if (p.bcN[i - 1].flag == 0)
            qrecN[i - 1] = p.bcN[i - 1].value;
          else if (i == 3)
            qrecN[i - 1] = fmax_f(qrecN[i - 1], 0.0);
        }
      }
    }
    // u and v with the limiters of hu and hv
    for (int i = nv + 1; i <= nv + 2; ++i) {
      if (nx > 1) {
        qrec_stencil[1] = QPC(j, k)[i - 1];
        if (j == 1) {
          qp_to_qp2(qrecW, B_cent[cc], qp2recW);
          qrec_stencil[0] = qp2recW[i - nv];
          qrec_stencil[2] = QPE(i, j + 1, k);
        } else if (j == nx) {
          qp_to_qp2(qrecE, B_cent[cc], qp2recE);
          qrec_stencil[0] = QPE(i, j - 1, k);
          qrec_stencil[2] = qp2recE[i - nv];
        } else {
          qrec_stencil[0] = QPE(i, j - 1, k);
          qrec_stencil[2] = QPE(i, j + 1, k);
          if (rad && scell == 2) {
            if (sE[cc]) {
              x_stencil[2] = x_stag[j];
              qrec_stencil[2] = source_bdry[i - 1];
            } else if (sW[cc]) {
              x_stencil[0] = x_stag[j - 1];
              qrec_stencil[0] = source_bdry[i - 1];
            }
          }
        }
        qrec_prime_x[i - 1] = limit(qrec_stencil, x_stencil, p.limiter[i - 1]);
        double dq = p.reconstr_coeff * dx2 * qrec_prime_x[i - 1];
        qrecW[i - 1] = qrec_stencil[1] - dq;
        qrecE[i - 1] = qrec_stencil[1] + dq;
        if (j == 1) {
          qp_to_qp2(qrecW, B_cent[cc], qp2recW);
          qrecW[i - 1] = qp2recW[i - nv];
        } else if (j == nx) {
          qp_to_qp2(qrecE, B_cent[cc], qp2recE);
          qrecE[i - 1] = qp2recE[i - nv];
        } else if (rad && scell == 2) {
          if (sE[cc]) {
            for (int m = 0; m < np; ++m) qrecE[m] = source_bdry[m];
          } else if (sW[cc]) {
            for (int m = 0; m < np; ++m) qrecW[m] = source_bdry[m];
          }
        }
      }
      if (ny > 1) {
        qrec_stencil[1] = QPC(j, k)[i - 1];
        if (k == 1) {
          qp_to_qp2(qrecS, B_cent[cc], qp2recS);
          qrec_stencil[0] = qp2recS[i - nv];
          qrec_stencil[2] = QPE(i, j, k + 1);
        } else if (k == ny) {
          qp_to_qp2(qrecN, B_cent[cc], qp2recN);
          qrec_stencil[0] = QPE(i, j, k - 1);
          qrec_stencil[2] = qp2recN[i - nv];
        } else {
          qrec_stencil[0] = QPE(i, j, k - 1);
          qrec_stencil[2] = QPE(i, j, k + 1);
          if (rad && scell == 2) {
            if (sS[cc]) {
              y_stencil[0] = y_stag[k - 1];
              qrec_stencil[0] = source_bdry[i - 1];
            } else if (sN[cc]) {
              x_stencil[2] = y_stag[k];  // src/solver_2d.f90:3616 writes x_stencil here
              qrec_stencil[2] = source_bdry[i - 1];
            }
          }
        }
        qrec_prime_y[i - 1] = limit(qrec_stencil, y_stencil, p.limiter[i - 1]);
        double dq = p.reconstr_coeff * dy2 * qrec_prime_y[i - 1];
        qrecS[i - 1] = qrec_stencil[1] - dq;
        qrecN[i - 1] = qrec_stencil[1] + dq;
        if (k == 1) {
          qp_to_qp2(qrecS, B_cent[cc], qp2recS);
          qrecS[i - 1] = qp2recS[i - nv];
        } else if (k == ny) {
          qp_to_qp2(qrecN, B_cent[cc], qp2recN);
          qrecN[i - 1] = qp2recN[i - nv];
        } else if (rad && scell == 2) {
          if (sS[cc]) {
            for (int m = 0; m < np; ++m) qrecS[m] = source_bdry[m];
          } else if (sN[cc]) {
            for (int m = 0; m < np; ++m) qrecN[m] = source_bdry[m];
          }
        }
      }
    }
    // the dry-cell face assignments (src/solver_2d.f90:3675-3705, 3795-3826)
    // are overwritten by the unconditional lines that follow them, so only
    // those lines are written here.
    if (nx > 1) {
      qp_to_qc(qrecW, FX(qR, nv, j, k));
      qp_to_qc(qrecE, FX(qL, nv, j + 1, k));
      std::memcpy(FX(qpR, np, j, k), qrecW, sizeof(double) * np);
      std::memcpy(FX(qpL, np, j + 1, k), qrecE, sizeof(double) * np);
      epR[sx2(j, k)] = recon_epoch;
      epL[sx2(j + 1, k)] = recon_epoch;
      if (j == 1) {
        std::memcpy(FX(qL, nv, j, k), FX(qR, nv, j, k), sizeof(double) * nv);
        std::memcpy(FX(qpL, np, j, k), FX(qpR, np, j, k), sizeof(double) * np);
        epL[sx2(j, k)] = recon_epoch;
      } else if (j == nx) {
        std::memcpy(FX(qR, nv, j + 1, k), FX(qL, nv, j + 1, k), sizeof(double) * nv);
        std::memcpy(FX(qpR, np, j + 1, k), FX(qpL, np, j + 1, k), sizeof(double) * np);
        epR[sx2(j + 1, k)] = recon_epoch;
      } else if (rad && scell == 2) {
        if (sE[cc]) {
          std::memcpy(FX(qR, nv, j + 1, k), FX(qL, nv, j + 1, k), sizeof(double) * nv);
          std::memcpy(FX(qpR, np, j + 1, k), FX(qpL, np, j + 1, k), sizeof(double) * np);
          epR[sx2(j + 1, k)] = recon_epoch;
        } else if (sW[cc]) {
          std::memcpy(FX(qL, nv, j, k), FX(qR, nv, j, k), sizeof(double) * nv);
          std::memcpy(FX(qpL, np, j, k), FX(qpR, np, j, k), sizeof(double) * np);
          epL[sx2(j, k)] = recon_epoch;
        }
      }
    } else {
      std::memcpy(FX(qR, nv, j, k), (q_expl + (size_t)nv * c2(j, k)), sizeof(double) * nv);
      std::memcpy(FX(qL, nv, j + 1, k), (q_expl + (size_t)nv * c2(j, k)), sizeof(double) * nv);
      std::memcpy(FX(qpR, np, j, k), QPC(j, k), sizeof(double) * np);
      std::memcpy(FX(qpL, np, j + 1, k), QPC(j, k), sizeof(double) * np);
    }
    if (ny > 1) {
      qp_to_qc(qrecS, FY(qT, nv, j, k));
      qp_to_qc(qrecN, FY(qB, nv, j, k + 1));
      std::memcpy(FY(qpT, np, j, k), qrecS, sizeof(double) * np);
      std::memcpy(FY(qpB, np, j, k + 1), qrecN, sizeof(double) * np);
      epT[sy2(j, k)] = recon_epoch;
      epB[sy2(j, k + 1)] = recon_epoch;
      if (k == 1) {
        std::memcpy(FY(qB, nv, j, k), FY(qT, nv, j, k), sizeof(double) * nv);
        std::memcpy(FY(qpB, np, j, k), FY(qpT, np, j, k), sizeof(double) * np);
        epB[sy2(j, k)] = recon_epoch;
      } else if (k == ny) {
        std::memcpy(FY(qT, nv, j, k + 1), FY(qB, nv, j, k + 1), sizeof(double) * nv);
        std::memcpy(FY(qpT, np, j, k + 1), FY(qpB, np, j, k + 1), sizeof(double) * np);
        epT[sy2(j, k + 1)] = recon_epoch;
      } else if (rad && scell == 2) {
        if (sS[cc]) {
          std::memcpy(FY(qB, nv, j, k), FY(qT, nv, j, k), sizeof(double) * nv);
          std::memcpy(FY(qpB, np, j, k), FY(qpT, np, j, k), sizeof(double) * np);
          epB[sy2(j, k)] = recon_epoch;
        } else if (sN[cc]) {
          std::memcpy(FY(qT, nv, j, k + 1), FY(qB, nv, j, k + 1), sizeof(double) * nv);
          std::memcpy(FY(qpT, np, j, k + 1), FY(qpB, np, j, k + 1), sizeof(double) * np);
          epT[sy2(j, k + 1)] = recon_epoch;
        }
      }
    } else {
      for (int kk = k; kk <= k + 1; ++kk) {
        std::memcpy(FY(qB, nv, j, kk), (q_expl + (size_t)nv * c2(j, k)), sizeof(double) * nv);
        std::memcpy(FY(qT, nv, j, kk), (q_expl + (size_t)nv * c2(j, k)), sizeof(double) * nv);
        std::memcpy(FY(qpB, np, j, kk), QPC(j, k), sizeof(double) * np);
        std::memcpy(FY(qpT, np, j, kk), QPC(j, k), sizeof(double) * np);
      }
    }
  }
}

// src/solver_2d.f90:3931-4008 (one speed per interface: the reference stores
// the same value in all n_eqns entries)
void OracleCtx::eval_speeds() {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < solve_interfaces_x; ++l) {
      int j = j_stag_x[l], k = k_stag_x[l];
      size_t f = sx2(j, k);
#ifndef ORACLE_TIMING
      if (epL[f] != recon_epoch && face_wet(FX(qpL, np, j, k), idx_u)) ++stale_wet_reads;
#endif
#ifndef ORACLE_TIMING
      if (epR[f] != recon_epoch && face_wet(FX(qpR, np, j, k), idx_u)) ++stale_wet_reads;
#endif
      double lmin, lmax, rmin, rmax;
      eval_local_speeds_x(FX(qpL, np, j, k), gc_sx[f], lmin, lmax);
      eval_local_speeds_x(FX(qpR, np, j, k), gc_sx[f], rmin, rmax);
      axNeg[f] = fmin_f(fmin_f(lmin, rmin), 0.0);
      axPos[f] = fmax_f(fmax_f(lmax, rmax), 0.0);
    }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < solve_interfaces_y; ++l) {
      int j = j_stag_y[l], k = k_stag_y[l];
      size_t f = sy2(j, k);
#ifndef ORACLE_TIMING
      if (epB[f] != recon_epoch && face_wet(FY(qpB, np, j, k), idx_v)) ++stale_wet_reads;
#endif
#ifndef ORACLE_TIMING
      if (epT[f] != recon_epoch && face_wet(FY(qpT, np, j, k), idx_v)) ++stale_wet_reads;
#endif
      double bmin, bmax, tmin, tmax;
      eval_local_speeds_y(FY(qpB, np, j, k), gc_sy[f], bmin, bmax);
      eval_local_speeds_y(FY(qpT, np, j, k), gc_sy[f], tmin, tmax);
      ayNeg[f] = fmin_f(fmin_f(bmin, tmin), 0.0);
      ayPos[f] = fmax_f(fmax_f(bmax, tmax), 0.0);
    }
  }
}

// One interface of eval_flux_KT (src/solver_2d.f90:2862-2923 for x, dir 1;
// :2932-2990 for y, dir 2) + average_KT (:3017-3047): the physical fluxes of
// both face states, the KT combination, the solid-flux cap (x: .GE., y: .GT.)
// and the zero-velocity rule (x: qp(2) of both faces; y: q(3) of both faces).
void OracleCtx::kt_face(const double* qLf, const double* qpLf, const double* qRf,
                        const double* qpRf, double aN, double aP, double gcf, int dir,
                        double* H) const {
  double fluxL[MAXV], fluxR[MAXV], avg[MAXV];
  eval_fluxes(qLf, qpLf, gcf, dir, fluxL);
  eval_fluxes(qRf, qpRf, gcf, dir, fluxR);
  for (int i = 0; i < nv; ++i)
    avg[i] = (aN == aP) ? 0.0 : (aP * fluxL[i] - aN * fluxR[i]) / (aP - aN);
  for (int i = 0; i < nv; ++i) {
    if (aN == aP)
      H[i] = 0.0;
    else
      H[i] = avg[i] + (aP * aN) / (aP - aN) * (qRf[i] - qLf[i]);
  }
  double s = 0.0;
  for (int i = 0; i < ns; ++i) s += H[4 + i];
  if (dir == 1) {
    if (s / H[0] >= 1.0) {
      double r = 0.0;
      for (int i = 0; i < ns; ++i) r += H[4 + i] / H[0];
      for (int i = 0; i < ns; ++i) H[4 + i] = H[4 + i] / r;
    }
    if (qpLf[1] == 0.0 && qpRf[1] == 0.0) {
      H[0] = 0.0;
      for (int i = 3; i < nv; ++i) H[i] = 0.0;
    }
  } else {
    if (s / H[0] > 1.0) {
      double r = s / H[0];
      for (int i = 0; i < ns; ++i) H[4 + i] = H[4 + i] / r;
    }
    if (qLf[2] == 0.0 && qRf[2] == 0.0) {
      H[0] = 0.0;
      for (int i = 3; i < nv; ++i) H[i] = 0.0;
    }
  }
}

// src/solver_2d.f90:2832-3000
void OracleCtx::eval_flux_KT() {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < solve_interfaces_x; ++l) {
      int j = j_stag_x[l], k = k_stag_x[l];
      size_t f = sx2(j, k);
      kt_face(FX(qL, nv, j, k), FX(qpL, np, j, k), FX(qR, nv, j, k), FX(qpR, np, j, k),
              axNeg[f], axPos[f], gc_sx[f], 1, FX(Hx, nv, j, k));
    }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < solve_interfaces_y; ++l) {
      int j = j_stag_y[l], k = k_stag_y[l];
      size_t f = sy2(j, k);
      kt_face(FY(qB, nv, j, k), FY(qpB, np, j, k), FY(qT, nv, j, k), FY(qpT, np, j, k),
              ayNeg[f], ayPos[f], gc_sy[f], 2, FY(Hy, nv, j, k));
    }
  }
}

void OracleCtx::note_stage_read(int jj, int kk) {
  // inlet-interior cells are never solved; their stage values stay at their
  // initial (zero) contents, which the CUDA path reproduces
  if (p.radial_source_flag && source_cell[c2(jj, kk)] == 1) return;
  // fresh value: q as it stands, qp = f(q) as in the driver's sweeps
  const double* qs = Q(q_rk, jj, kk);  // q_rk(:,jj,kk,1)
  const double* qc = Q(q, jj, kk);
  bool differs = std::memcmp(qs, qc, sizeof(double) * nv) != 0;
  if (!differs) {
    double fresh[MAXP], pd;
    if (qc[0] > 0.0) {
      qc_to_qp(qc, fresh, pd);
    } else {
      for (int i = 0; i < np; ++i) fresh[i] = 0.0;
      fresh[3] = p.T_ambient;
    }
    differs = std::memcmp(fresh, QP(qp_rk, jj, kk), sizeof(double) * np) != 0;
  }
  // dry on both sides: the neighbour only feeds temperature / fraction slopes
  // of faces whose thickness is zero, which reach no output
  if (differs && (qs[0] > 0.0 || qc[0] > 0.0)) ++stale_wet_reads;
}

// src/solver_2d.f90:2614-2691 for stage irk (stage arrays are contiguous per stage)
void OracleCtx::eval_hyperbolic_terms(int irk) {
  const size_t N = (size_t)nx * ny;
  const double* qe = &q_rk[(size_t)nv * N * (irk - 1)];
  const double* qpe = &qp_rk[(size_t)np * N * (irk - 1)];
  reconstruction(qe, qpe, true);
  eval_speeds();
  eval_flux_KT();
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    double* d = QRK(divFlux, nv, j, k, irk);
    for (int i = 0; i < nv; ++i) {
      d[i] = 0.0;
      if (nx > 1) d[i] = d[i] + (FX(Hx, nv, j + 1, k)[i] - FX(Hx, nv, j, k)[i]) * one_by_dx;
      if (ny > 1) d[i] = d[i] + (FY(Hy, nv, j, k + 1)[i] - FY(Hy, nv, j, k)[i]) * one_by_dy;
    }
  }
  // mass budget: SUM over solved cells of divFlux(1) written as the flux
  // through the faces that have exactly one solved side (interior faces
  // cancel); a cell outside the domain counts as not solved
  auto solved = [&](int jj, int kk) {
    return jj >= 1 && jj <= nx && kk >= 1 && kk <= ny && mask[c2(jj, kk)] != 0;
  };
  long double f = 0.0L;
  if (nx > 1)
    for (int64_t l = 0; l < solve_interfaces_x; ++l) {
      int j = j_stag_x[l], k = k_stag_x[l];
      int w = (int)solved(j - 1, k) - (int)solved(j, k);
      if (w) f += (long double)w * FX(Hx, nv, j, k)[0] * (long double)one_by_dx;
    }
  if (ny > 1)
    for (int64_t l = 0; l < solve_interfaces_y; ++l) {
      int j = j_stag_y[l], k = k_stag_y[l];
      int w = (int)solved(j, k - 1) - (int)solved(j, k);
      if (w) f += (long double)w * FY(Hy, nv, j, k)[0] * (long double)one_by_dy;
    }
  stage_face_flux[irk - 1] = f;
}

// src/solver_2d.f90:872-1005
double OracleCtx::timestep() {
  double dtl = p.max_dt;
  if (p.cfl != -1.0) {
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < solve_cells; ++l) {
      int j = j_cent[l], k = k_cent[l];
      double pd;
      if (Q(q, j, k)[0] > 0.0) {
        qc_to_qp(Q(q, j, k), QP(qp, j, k), pd);
      } else {
        double* o = QP(qp, j, k);
        for (int i = 0; i < np; ++i) o[i] = 0.0;
        o[3] = p.T_ambient;
      }
    }
    reconstruction(q.data(), qp.data(), false);
    eval_speeds();
    for (int64_t l = 0; l < solve_interfaces_x; ++l) {
      size_t f = sx2(j_stag_x[l], k_stag_x[l]);
      ax_max[f] = fmax_f(axPos[f], -axNeg[f]);
    }
    for (int64_t l = 0; l < solve_interfaces_y; ++l) {
      size_t f = sy2(j_stag_y[l], k_stag_y[l]);
      ay_max[f] = fmax_f(ayPos[f], -ayNeg[f]);
    }
    // dt_interface = dt when max_a <= 0: the running minimum, whose value
    // never lowers the final minimum (the reference reads it racily).
    for (int64_t l = 0; l < solve_cells; ++l) {
      int j = j_cent[l], k = k_cent[l];
      double max_a = fmax_f(ax_max[sx2(j, k)], ax_max[sx2(j + 1, k)]);
      double dtx = (max_a > 0.0) ? p.cfl * dx / max_a : dtl;
      max_a = fmax_f(ay_max[sy2(j, k)], ay_max[sy2(j, k + 1)]);
      double dty = (max_a > 0.0) ? p.cfl * dy / max_a : dtl;
      double dt_cfl = fmin_f(dtx, dty);
      dtl = fmin_f(dtl, dt_cfl);
    }
  }
  return dtl;
}

// src/solver_2d.f90:2243-2282
void OracleCtx::eval_f(const double* qj, const double* qj_old, double a_diag,
                       const double* coeff_f, const double* Rj_not_impl, double bx,
                       double by, double dtl, double* f_nl, double& scal_f) const {
  double nh[MAXV];
  eval_implicit_terms_r(bx, by, qj, nh);
  for (int i = 0; i < nv; ++i) {
    double Rj = Rj_not_impl[i] - a_diag * nh[i];
    f_nl[i] = qj[i] - qj_old[i] + dtl * Rj;
    f_nl[i] = coeff_f[i] * f_nl[i];
  }
  double d = 0.0;
  for (int i = 0; i < nv; ++i) d += f_nl[i] * f_nl[i];
  scal_f = 0.5 * d;
}

// src/solver_2d.f90:2300-2365; left is (n_eqns,n_vars) column-major
void OracleCtx::eval_jacobian(const double* qj_rel, const double* qj_org,
                              const double* coeff_f, double bx, double by, double dtl,
                              double a_diag, double* left) const {
  for (int i = 0; i < nv * nv; ++i) left[i] = 0.0;
  cplx init[MAXV], rel[MAXV], qc[MAXV], nh[MAXV];
  for (int i = 0; i < nv; ++i) init[i] = C(qj_rel[i], 0.0);
  for (int i = 0; i < nv; ++i) {
    left[i + nv * i] = coeff_f[i] * qj_org[i];
    if (implicit_flag[i]) {
      for (int m = 0; m < nv; ++m) rel[m] = init[m];
      rel[i] = C(qj_rel[i], h);
      for (int m = 0; m < nv; ++m) qc[m] = mulr(rel[m], qj_org[m]);
      eval_implicit_terms(bx, by, qc, nh);
      for (int r = 0; r < nv; ++r) {
        double jac = coeff_f[i] * nh[r].im * one_by_h;
        left[r + nv * i] = left[r + nv * i] - dtl * a_diag * jac;
      }
    }
  }
}

// src/solver_2d.f90:2019-2224
void OracleCtx::lnsrch(const double* x_old, const double* qj_org, const double* qj_old,
                       double scal_f_old, const double* grad_f, double* desc_dir,
                       const double* coeff_f, double* qj_rel, double& scal_f,
                       double* right_term, double stpmax, bool& check,
                       const double* Rj_not_impl, double bx, double by, double dtl,
                       double a_diag, int64_t& trials) const {
  const double TOLX = EPS;
  check = false;
  // NORM2 with the scaled sum of squares
  double scale = 0.0, ssq = 0.0;
  for (int i = 0; i < nv; ++i) {
    if (desc_dir[i] != 0.0) {
      double ax = std::fabs(desc_dir[i]);
      if (scale < ax) {
        double val = scale / ax;
        ssq = 1.0 + ssq * val * val;
        scale = ax;
      } else {
        double val = ax / scale;
        ssq = ssq + val * val;
      }
    }
  }
  double desc_dir_abs = scale * std::sqrt(ssq);
  if (desc_dir_abs > stpmax)
    for (int i = 0; i < nv; ++i) desc_dir[i] = desc_dir[i] * stpmax / desc_dir_abs;
  double slope = 0.0;
  for (int i = 0; i < nv; ++i) slope += grad_f[i] * desc_dir[i];
  double mx = 0.0;
  for (int i = 0; i < nv; ++i) {
    double r = std::fabs(desc_dir[i]) / fmax_f(std::fabs(x_old[i]), 1.0);
    mx = (i == 0) ? r : fmax_f(mx, r);
  }
  double alamin = TOLX / mx;
  if (alamin == 0.0) {
    for (int i = 0; i < nv; ++i) qj_rel[i] = x_old[i];
    return;
  }
  double alam = 1.0, alam2 = 0.0, scal_f2 = 0.0, tmplam = 0.0;
  double qj[MAXV];
  // the reference loop ends only through the two exits below; a non-finite
  // first backtrack would keep alam from shrinking, so the trials are capped
  // (the CUDA path uses the same cap) and the cap exits like alam < alamin
  for (int ntrial = 0;; ++ntrial) {
    if (ntrial == LNSRCH_MAX_TRIALS) {
      for (int i = 0; i < nv; ++i) qj_rel[i] = x_old[i];
      scal_f = scal_f_old;
      check = true;
      break;
    }
    for (int i = 0; i < nv; ++i) qj_rel[i] = x_old[i] + alam * desc_dir[i];
    for (int i = 0; i < nv; ++i) qj[i] = qj_rel[i] * qj_org[i];
    eval_f(qj, qj_old, a_diag, coeff_f, Rj_not_impl, bx, by, dtl, right_term, scal_f);
    ++trials;
    if (scal_f <= 0.9 * scal_f_old) {
      break;
    } else if (alam < alamin) {
      for (int i = 0; i < nv; ++i) qj_rel[i] = x_old[i];
      scal_f = scal_f_old;
      check = true;
      break;
    } else {
      if (alam == 1.0) {
        tmplam = -slope / (2.0 * (scal_f - scal_f_old - slope));
      } else {
        double rhs1 = scal_f - scal_f_old - alam * slope;
        double rhs2 = scal_f2 - scal_f_old - alam2 * slope;
        double a = (rhs1 / (alam * alam) - rhs2 / (alam2 * alam2)) / (alam - alam2);
        double b = (-alam2 * rhs1 / (alam * alam) + alam * rhs2 / (alam2 * alam2)) /
                   (alam - alam2);
        if (a == 0.0) {
          tmplam = -slope / (2.0 * b);
        } else {
          double disc = b * b - 3.0 * a * slope;
          if (disc < 0.0)
            tmplam = 0.5 * alam;
          else if (b <= 0.0)
            tmplam = (-b + std::sqrt(disc)) / (3.0 * a);
          else
            tmplam = -slope / (b + std::sqrt(disc));
        }
        if (tmplam > 0.5 * alam) tmplam = 0.5 * alam;
      }
    }
    alam2 = alam;
    scal_f2 = scal_f;
    alam = fmax_f(tmplam, 0.5 * alam);
  }
}

// src/solver_2d.f90:1660-1994 (normalize_q = T, normalize_f = F, opt_search_NL = T)
int OracleCtx::solve_rk_step(double* qj, const double* qj_old, double a_diag,
                             const double* Rj_not_impl, double bx, double by, double dtl,
                             int64_t& trials) const {
  const double STPMX = 100.0, TOLF = 1.0e-10, TOLMIN = 1.0e-6;
  double coeff_f[MAXV], grad_f[MAXV], qj_org[MAXV], qj_rel[MAXV], right_term[MAXV];
  double left[MAXV * MAXV], desc_dir[MAXV], x_old[MAXV];
  double scal_f = 0.0, scal_f_old;
  bool check = false;
  for (int i = 0; i < nv; ++i) coeff_f[i] = 1.0;
  for (int i = 0; i < nv; ++i) grad_f[i] = 0.0;
  for (int i = 0; i < nv; ++i) qj_org[i] = fmax_f(std::fabs(qj[i]), 1.0e-3);
  for (int i = 0; i < nv; ++i) qj_rel[i] = qj[i] / qj_org[i];
  // explicit / implicit index lists (implicit_flag(2:3) only)
  int ex[MAXV], ne = 0, im[2] = {1, 2};
  for (int i = 0; i < nv; ++i)
    if (!implicit_flag[i]) ex[ne++] = i;
  int nl_iter;
  for (nl_iter = 1; nl_iter <= 100; ++nl_iter) {
    const double TOLXn = EPS;
    eval_f(qj, qj_old, a_diag, coeff_f, Rj_not_impl, bx, by, dtl, right_term, scal_f);
    double mx = std::fabs(right_term[0]);
    for (int i = 1; i < nv; ++i) mx = fmax_f(mx, std::fabs(right_term[i]));
    if (mx < TOLF) break;
    eval_jacobian(qj_rel, qj_org, coeff_f, bx, by, dtl, a_diag, left);
    // block elimination with the explicit diagonal, 2x2 Cramer on rows/cols 2,3
    double d1[MAXV], d2[2];
    for (int a = 0; a < ne; ++a) d1[a] = right_term[ex[a]];
    for (int a = 0; a < 2; ++a) d2[a] = right_term[im[a]];
    for (int a = 0; a < ne; ++a) d1[a] = d1[a] / left[ex[a] + nv * ex[a]];
    // MATMUL(desc_dir_small1, left_matrix_small21): small21 holds the packed
    // entries left(im, ex) (column-major pack), reshaped (n_e, 2)
    {
      double packed[2 * MAXV];
      int pp = 0;
      for (int a = 0; a < ne; ++a)
        for (int b = 0; b < 2; ++b) packed[pp++] = left[im[b] + nv * ex[a]];
      for (int b = 0; b < 2; ++b) {
        double s = 0.0;
        for (int a = 0; a < ne; ++a) s += d1[a] * packed[a + ne * b];
        d2[b] = d2[b] - s;
      }
    }
    double s11 = left[im[0] + nv * im[0]], s12 = left[im[0] + nv * im[1]];
    double s21 = left[im[1] + nv * im[0]], s22 = left[im[1] + nv * im[1]];
    double inv_det = 1.0 / (s11 * s22 - s21 * s12);
    double sol0 = (d2[0] * s22 - d2[1] * s12) * inv_det;
    double sol1 = (s11 * d2[1] - s21 * d2[0]) * inv_det;
    for (int i = 0; i < nv; ++i) desc_dir[i] = 0.0;
    // unpack(-small2, implicit, 0) + unpack(-small1, .not.implicit, 0)
    double u2[MAXV], u1[MAXV];
    for (int i = 0; i < nv; ++i) u2[i] = u1[i] = 0.0;
    u2[im[0]] = -sol0;
    u2[im[1]] = -sol1;
    for (int a = 0; a < ne; ++a) u1[ex[a]] = -d1[a];
    for (int i = 0; i < nv; ++i) desc_dir[i] = u2[i] + u1[i];
    for (int i = 0; i < nv; ++i) x_old[i] = qj_rel[i];
    scal_f_old = scal_f;
    if (nl_iter > 1) {
      double dd = 0.0;
      for (int i = 0; i < nv; ++i) dd += qj_rel[i] * qj_rel[i];
      double stpmax = STPMX * fmax_f(std::sqrt(dd), (double)nv);
      for (int c = 0; c < nv; ++c) {
        double s = 0.0;
        for (int r = 0; r < nv; ++r) s += right_term[r] * left[r + nv * c];
        grad_f[c] = s;
      }
      lnsrch(x_old, qj_org, qj_old, scal_f_old, grad_f, desc_dir, coeff_f, qj_rel, scal_f,
             right_term, stpmax, check, Rj_not_impl, bx, by, dtl, a_diag, trials);
    } else {
      for (int i = 0; i < nv; ++i) qj_rel[i] = x_old[i] + desc_dir[i];
      for (int i = 0; i < nv; ++i) qj[i] = qj_rel[i] * qj_org[i];
      eval_f(qj, qj_old, a_diag, coeff_f, Rj_not_impl, bx, by, dtl, right_term, scal_f);
    }
    for (int i = 0; i < nv; ++i) qj[i] = qj_rel[i] * qj_org[i];
    mx = std::fabs(right_term[0]);
    for (int i = 1; i < nv; ++i) mx = fmax_f(mx, std::fabs(right_term[i]));
    if (mx < TOLF) {
      check = false;
      break;
    }
    if (check) {
      double m2 = 0.0;
      for (int i = 0; i < nv; ++i) {
        double r = std::fabs(grad_f[i]) * fmax_f(std::fabs(qj_rel[i]), 1.0) /
                   fmax_f(scal_f, 0.5 * nv);
        m2 = (i == 0) ? r : fmax_f(m2, r);
      }
      check = (m2 < TOLMIN);
    }
    double m3 = 0.0;
    for (int i = 0; i < nv; ++i) {
      double r = std::fabs(qj_rel[i] - x_old[i]) / fmax_f(std::fabs(qj_rel[i]), 1.0);
      m3 = (i == 0) ? r : fmax_f(m3, r);
    }
    if (m3 < TOLXn) break;
  }
  return nl_iter > 100 ? 100 : nl_iter;
}

// src/solver_2d.f90:1021-1632
uint32_t OracleCtx::imex_RK_solver(double dtl) {
  const double T_amb = p.T_ambient;
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    std::memcpy(Q(q0, j, k), Q(q, j, k), sizeof(double) * nv);
    for (int r = 1; r <= nrk; ++r) {
      double* a = QRK(q_rk, nv, j, k, r);
      double* b = QRK(qp_rk, np, j, k, r);
      for (int i = 0; i < nv; ++i) a[i] = 0.0;
      for (int i = 0; i < np; ++i) b[i] = 0.0;
      b[3] = T_amb;
      double* d = QRK(divFlux, nv, j, k, r);
      double* n = QRK(NH, nv, j, k, r);
      double* s = QRK(SI_NH, nv, j, k, r);
      double* e = QRK(expl_terms, nv, j, k, r);
      for (int i = 0; i < nv; ++i) d[i] = n[i] = s[i] = e[i] = 0.0;
    }
  }
  for (int i_RK = 1; i_RK <= nrk; ++i_RK) {
    double a_tilde[4] = {0, 0, 0, 0}, a_dirk[4] = {0, 0, 0, 0};
    for (int m = 1; m <= i_RK - 1; ++m) {
      a_tilde[m - 1] = a_tilde_ij[i_RK - 1][m - 1];
      a_dirk[m - 1] = a_dirk_ij[i_RK - 1][m - 1];
    }
    const double a_diag = a_dirk_ij[i_RK - 1][i_RK - 1];
    int64_t local_newton = 0, local_iters = 0, local_trials = 0, local_maxit = 0;
    int64_t local_hist[16] = {0};
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : local_newton, local_iters, local_trials, local_maxit)
    for (int64_t l = 0; l < solve_cells; ++l) {
      int j = j_cent[l], k = k_cent[l];
      size_t cc = c2(j, k);
      double q_guess[MAXV], q_si[MAXV], Rj_not_impl[MAXV];
      const double* q0c = Q(q0, j, k);
      double* qfv = Q(q_fv, j, k);
      if (i_RK == 1)
        for (int i = 0; i < nv; ++i) q_guess[i] = q0c[i];
      for (int i = 0; i < nv; ++i) {
        double sa = 0.0, sb = 0.0;
        for (int m = 1; m <= i_RK; ++m)
          sa += (QRK(divFlux, nv, j, k, m)[i] - QRK(expl_terms, nv, j, k, m)[i]) * a_tilde[m - 1];
        for (int m = 1; m <= i_RK; ++m)
          sb += (QRK(NH, nv, j, k, m)[i] + QRK(SI_NH, nv, j, k, m)[i]) * a_dirk[m - 1];
        qfv[i] = q0c[i] - dtl * (sa - sb);
      }
      double pd;
      qc_to_qp(qfv, QP(qp, j, k), pd);
      double* SIc = QRK(SI_NH, nv, j, k, i_RK);
      double* NHc = QRK(NH, nv, j, k, i_RK);
      if (a_diag != 0.0) {
        if (qfv[0] > 0.0) {
          double bxx = Bxx.empty() ? 0.0 : Bxx[cc];
          double bxy = Bxy.empty() ? 0.0 : Bxy[cc];
          double byy = Byy.empty() ? 0.0 : Byy[cc];
          eval_nh_semi_impl_terms(Bx[cc], By[cc], bxx, bxy, byy, gc[cc], qfv, QP(qp, j, k), SIc);
          for (int i = 0; i < nv; ++i) q_si[i] = qfv[i] + dtl * a_diag * SIc[i];
          if (qfv[1] * qfv[1] + qfv[2] * qfv[2] == 0.0) {
            q_si[1] = 0.0;
            q_si[2] = 0.0;
          } else if (q_si[1] * qfv[1] < 0.0 || q_si[2] * qfv[2] < 0.0) {
            q_si[1] = 0.0;
            q_si[2] = 0.0;
          } else {
            double S = std::sqrt(q_si[1] * q_si[1] + q_si[2] * q_si[2]);
            double F = std::sqrt(qfv[1] * qfv[1] + qfv[2] * qfv[2]);
            q_si[1] = S * qfv[1] / F;
            q_si[2] = S * qfv[2] / F;
          }
          for (int i = 0; i < nv; ++i) SIc[i] = (q_si[i] - qfv[i]) / (dtl * a_diag);
          for (int i = 0; i < nv; ++i) q_guess[i] = q_si[i];
          for (int i = 0; i < nv; ++i) {
            double sa = 0.0, sb = 0.0;
            for (int m = 1; m <= i_RK - 1; ++m)
              sa += (QRK(divFlux, nv, j, k, m)[i] - QRK(expl_terms, nv, j, k, m)[i]) *
                    a_tilde[m - 1];
            for (int m = 1; m <= i_RK - 1; ++m)
              sb += (QRK(NH, nv, j, k, m)[i] + QRK(SI_NH, nv, j, k, m)[i]) * a_dirk[m - 1];
            Rj_not_impl[i] = (sa - sb) - a_diag * SIc[i];
          }
          int64_t trials = 0;
          int it = solve_rk_step(q_guess, q0c, a_diag, Rj_not_impl, Bx[cc], By[cc], dtl, trials);
          local_newton += 1;
          local_iters += it;
          local_trials += trials;
          if (it >= 100) local_maxit += 1;
#pragma omp atomic
          local_hist[it < 16 ? it - 1 + (it == 0) : 15] += 1;
          if (ny == 1) q_guess[2] = 0.0;
          if (nx == 1) q_guess[1] = 0.0;
          eval_implicit_terms_r(Bx[cc], By[cc], q_guess, NHc);
          if (q_si[1] * q_si[1] + q_si[2] * q_si[2] == 0.0) {
            q_guess[1] = 0.0;
            q_guess[2] = 0.0;
          } else if (q_guess[1] * q_si[1] <= 0.0 && q_guess[2] * q_si[2] <= 0.0) {
            q_guess[1] = 0.0;
            q_guess[2] = 0.0;
          } else {
            double S = std::sqrt(q_guess[1] * q_guess[1] + q_guess[2] * q_guess[2]);
            double F = std::sqrt(q_si[1] * q_si[1] + q_si[2] * q_si[2]);
            q_guess[1] = S * q_si[1] / F;
            q_guess[2] = S * q_si[2] / F;
          }
        } else {
          for (int i = 0; i < nv; ++i) q_guess[i] = qfv[i];
          for (int i = 0; i < nv; ++i) q_si[i] = qfv[i];
          for (int i = 0; i < nv; ++i) SIc[i] = 0.0;
          for (int i = 0; i < nv; ++i) NHc[i] = 0.0;
        }
      }
      if (a_diag != 0.0)
        for (int i = 0; i < nv; ++i) NHc[i] = (q_guess[i] - q_si[i]) / (dtl * a_diag);
      double* qrk = QRK(q_rk, nv, j, k, i_RK);
      for (int i = 0; i < nv; ++i) qrk[i] = q_guess[i];
      if (omega_tilde[i_RK - 1] > 0.0) {
        double* qprk = QRK(qp_rk, np, j, k, i_RK);
        if (qrk[0] > 0.0) {
          qc_to_qp(qrk, qprk, pd);
        } else {
          for (int i = 0; i < np; ++i) qprk[i] = 0.0;
          qprk[3] = T_amb;
        }
        double bxx = Bxx.empty() ? 0.0 : Bxx[cc];
        double bxy = Bxy.empty() ? 0.0 : Bxy[cc];
        double byy = Byy.empty() ? 0.0 : Byy[cc];
        eval_expl_terms(Bx[cc], By[cc], bxx, bxy, byy, gc[cc], dgc_dx[cc], dgc_dx[cc], qprk,
                        QRK(expl_terms, nv, j, k, i_RK), cell_source_fractions[cc]);
      }
    }
    newton_cells += local_newton;
    newton_iters += local_iters;
    lnsrch_trials += local_trials;
    newton_maxit += local_maxit;
    for (int b = 0; b < 16; ++b) hist[b] += local_hist[b];
    if (omega_tilde[i_RK - 1] > 0.0) eval_hyperbolic_terms(i_RK);
  }
  // assemble_sol
  double s1 = 0.0, s2 = 0.0;
  for (int m = 0; m < nrk; ++m) s1 += std::fabs(omega_tilde[m] - a_tilde_ij[nrk - 1][m]);
  for (int m = 0; m < nrk; ++m) s2 += std::fabs(omega[m] - a_dirk_ij[nrk - 1][m]);
  const bool last_stage = (s1 == 0.0 && s2 == 0.0);
  uint32_t err = 0;
  {
    // mass budget: q(1) changes by -dt * SUM_m w_m * (face flux of stage m)
    long double fl = 0.0L;
    for (int m = 1; m <= nrk; ++m) {
      const double w = last_stage ? a_tilde_ij[nrk - 1][m - 1] : omega_tilde[m - 1];
      if (w != 0.0) fl += (long double)w * stage_face_flux[m - 1];
    }
    mass_budget[3] = -(long double)dtl * fl;
    mass_budget[0] += mass_budget[3];
  }
  long double fix_before = 0.0L, fix_after = 0.0L;
#pragma omp parallel for schedule(static) reduction(+ : fix_before, fix_after)
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    size_t cc = c2(j, k);
    double* qc = Q(q, j, k);
    const double* q0c = Q(q0, j, k);
    double pd;
    if (last_stage) {
      std::memcpy(qc, QRK(q_rk, nv, j, k, nrk), sizeof(double) * nv);
    } else {
      for (int i = 0; i < nv; ++i) {
        double sa = 0.0, sb = 0.0;
        for (int m = 1; m <= nrk; ++m)
          sa += (QRK(divFlux, nv, j, k, m)[i] - QRK(expl_terms, nv, j, k, m)[i]) * omega_tilde[m - 1];
        for (int m = 1; m <= nrk; ++m)
          sb += (QRK(NH, nv, j, k, m)[i] + QRK(SI_NH, nv, j, k, m)[i]) * omega[m - 1];
        qc[i] = q0c[i] - dtl * (sa - sb);
      }
    }
    fix_before += qc[0];
    bool anynan = false;
    for (int i = 0; i < nv; ++i) anynan |= std::isnan(qc[i]);
    if (anynan) record_error(IMEX_ENAN, j, k);
    if (qc[0] < EPS) {
      if (qc[0] > -1.0e-7) {
        qc[0] = 0.0;
        for (int i = 1; i < nv; ++i) qc[i] = 0.0;
      } else {
        record_error(IMEX_ENEGH, j, k);
        if (q0c[0] > 0.0) qc_to_qp(q0c, QP(qp, j, k), pd);
      }
    }
    bool anyneg = false, anybad = false;
    for (int i = 0; i < ns; ++i) anyneg |= (qc[4 + i] < 0.0);
    if (anyneg) {
      for (int i = 0; i < ns; ++i) anybad |= (qc[4 + i] <= -1.0e-7);
      if (anybad) {
        record_error(IMEX_ENEGSOLID, j, k);
        if (q0c[0] > 0.0) qc_to_qp(q0c, QP(qp, j, k), pd);
      } else {
        for (int i = 0; i < ns; ++i)
          if (qc[4 + i] > -1.0e-7) qc[4 + i] = 0.0;
      }
    }
    qc_to_qp(qc, QP(qp, j, k), pd);
    if (QP(qp, j, k)[3] < 273.0) {
      record_error(IMEX_ELOWT, j, k);
      qc_to_qp(q0c, QP(qp, j, k), pd);
    }
    double ssum = 0.0;
    for (int i = 0; i < ns; ++i) ssum += qc[4 + i];
    if (ssum > qc[0]) {
      if ((ssum - qc[0]) / qc[0] < 1.0e-10 || qc[0] < EPS) {
        qc_to_qp(q0c, QP(qp, j, k), pd);
        double s = 0.0;
        for (int i = 0; i < ns; ++i) s += qc[4 + i];
        for (int i = 0; i < ns; ++i) qc[4 + i] = qc[4 + i] / s * qc[0];
      } else {
        record_error(IMEX_ESOLIDSUM, j, k);
        if (q0c[0] > 0.0) qc_to_qp(q0c, QP(qp, j, k), pd);
        if (qc[0] > 0.0) qc_to_qp(qc, QP(qp, j, k), pd);
      }
    }
    if (!B_nodata.empty() && B_nodata[cc])
      for (int i = 0; i < nv; ++i) qc[i] = 0.0;
    fix_after += qc[0];
  }
  mass_budget[1] += fix_after - fix_before;
  (void)err;
  return error_mask;
}

// src/solver_2d.f90:2380-2595
uint32_t OracleCtx::update_erosion_deposition_cell(double dtl) {
  if (p.erosion_coeff == 0.0 && !p.settling_flag && !p.entrainment_flag) return 0;
  uint32_t err_all = 0;
  long double ex_before = 0.0L, ex_after = 0.0L;
#pragma omp parallel for schedule(static) reduction(+ : ex_before, ex_after) reduction(| : err_all)
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    size_t cc = c2(j, k);
    double* qc = Q(q, j, k);
    double* qpc = QP(qp, j, k);
    double pd;
    ex_before += qc[0];
    if (qc[0] > 0.0) {
      qc_to_qp(qc, qpc, pd);
    } else {
      for (int i = 0; i < np; ++i) qpc[i] = 0.0;
      qpc[3] = p.T_ambient;
    }
    double ers[MAXS], dep[MAXS], cpe, cpl, eqns[MAXV], topo;
    uint32_t err = 0;
    double erod[MAXS];
    for (int i = 0; i < ns; ++i) erod[i] = erodible[(size_t)i + ns * cc];
    eval_mass_exchange_terms(qpc, Bx[cc], By[cc], erod, dtl, ers, dep, cpe, cpl, eqns, topo, err);
    if (p.bottom_radial_source_flag) {
      double oos = 1.0 - cell_source_fractions[cc];
      for (int i = 0; i < ns; ++i) dep[i] = dep[i] * oos;
      for (int i = 0; i < ns; ++i) ers[i] = ers[i] * oos;
      for (int i = 0; i < nv; ++i) eqns[i] = eqns[i] * oos;
      topo = topo * oos;
    }
    for (int i = 0; i < nv; ++i) qc[i] = qc[i] + dtl * eqns[i];
    for (int i = 0; i < ns; ++i) qc[4 + i] = fmax_f(0.0, qc[4 + i]);
    const size_t N = (size_t)nx * ny;
    for (int i = 0; i < ns; ++i) deposit[cc + N * i] = deposit[cc + N * i] + dtl * dep[i];
    for (int i = 0; i < ns; ++i) erosion[cc + N * i] = erosion[cc + N * i] + dtl * ers[i];
    for (int i = 0; i < ns; ++i)
      erodible[(size_t)i + ns * cc] = erodible[(size_t)i + ns * cc] - dtl * ers[i];
    if (p.erodible_deposit_flag)
      for (int i = 0; i < ns; ++i)
        erodible[(size_t)i + ns * cc] = erodible[(size_t)i + ns * cc] + dtl * dep[i];
    if (p.topo_change_flag) B_cent[cc] = B_cent[cc] + dtl * topo;
    bool anyneg = false;
    for (int i = 0; i < ns; ++i) anyneg |= (qc[4 + i] < 0.0);
    if (anyneg) err |= IMEX_ERRBIT(IMEX_EEROSION);
    if (qc[0] <= 0.0) {
      if (qc[0] > -1.0e-10) {
        for (int i = 0; i < nv; ++i) qc[i] = 0.0;
      } else {
        err |= IMEX_ERRBIT(IMEX_EEROSION);
        qc_to_qp(qc, qpc, pd);
      }
    }
    double s = 0.0;
    for (int i = 0; i < ns; ++i) s += qc[4 + i];
    if (s > qc[0]) {
      if (qc[0] < 1.0e-10) {
        double s2 = 0.0;
        for (int i = 0; i < ns; ++i) s2 += qc[4 + i];
        for (int i = 0; i < ns; ++i) qc[4 + i] = qc[4 + i] / s2 * qc[0];
      } else {
        err |= IMEX_ERRBIT(IMEX_EEROSION);
        qc_to_qp(qc, qpc, pd);
      }
    }
    double r_red_grav;
    if (qc[0] > 0.0) {
      qc_to_qp(qc, qpc, pd);
      double Ri, rho_m, rho_c, spc, spm;
      mixt_var(qpc, Ri, rho_m, rho_c, r_red_grav, false, spc, spm);
    } else {
      for (int i = 0; i < np; ++i) qpc[i] = 0.0;
      qpc[3] = p.T_ambient;
      r_red_grav = 0.0;
    }
    if (r_red_grav <= 0.0)
      for (int i = 0; i < nv; ++i) qc[i] = 0.0;
    if (err) record_error(IMEX_EEROSION, j, k);
    err_all |= err;
    ex_after += qc[0];
  }
  mass_budget[2] += ex_after - ex_before;
  return err_all;
}

// src/IMEX_SfloW2D.f90:391-447 (qp part; max tables are outside the step)
void OracleCtx::post_step_sweep() {
  if (post_on) {
    for (int64_t l = 0; l < solve_cells; ++l) post_cell(j_cent[l], k_cent[l], false);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    double pd;
    if (Q(q, j, k)[0] > 0.0) {
      qc_to_qp(Q(q, j, k), QP(qp, j, k), pd);
    } else {
      double* o = QP(qp, j, k);
      for (int i = 0; i < np; ++i) o[i] = 0.0;
      o[3] = p.T_ambient;
    }
  }
}

// src/geometry_2d.f90:683-860: the *_geom derivatives of B_cent (5-point
// stencils on cells 3..n-2 in the reference's summation order, then the
// border copies, columns before rows) and, with slope correction, grav_coeff,
// d_grav_coeff_dx and the staggered grav_coeff.
void OracleCtx::topography_reconstruction() {
  const double cf1[5] = {-2.0, -1.0, 0.0, 1.0, 2.0};
  const double cf2[5] = {2.0, -1.0, -2.0, -1.0, 2.0};
  const double norm1_x = 10.0 * dx, norm1_y = 10.0 * dy;
  const double norm2_x = 7.0 * (dx * dx), norm2_y = 7.0 * (dy * dy);
  const double norm_xy = (10.0 * dx) * (10.0 * dy);
  const size_t N = (size_t)nx * ny;
  if (Bxx.empty()) Bxx.assign(N, 0.0);
  if (Bxy.empty()) Bxy.assign(N, 0.0);
  if (Byy.empty()) Byy.assign(N, 0.0);
  auto B = [&](int j, int k) { return B_cent[c2(j, k)]; };
  for (int k = 3; k <= ny - 2; ++k)
    for (int j = 3; j <= nx - 2; ++j) {
      double px = 0.0, sxx = 0.0, py = 0.0, syy = 0.0;
      for (int kj = 1; kj <= 5; ++kj) {
        px = px + cf1[kj - 1] * B(j + kj - 3, k);
        sxx = sxx + cf2[kj - 1] * B(j + kj - 3, k);
      }
      for (int kk = 1; kk <= 5; ++kk) {
        py = py + cf1[kk - 1] * B(j, k + kk - 3);
        syy = syy + cf2[kk - 1] * B(j, k + kk - 3);
      }
      const size_t c = c2(j, k);
      Bx[c] = px / norm1_x;
      By[c] = py / norm1_y;
      Bxx[c] = sxx / norm2_x;
      Byy[c] = syy / norm2_y;
      double ws = 0.0;
      for (int kk = 1; kk <= 5; ++kk)
        for (int kj = 1; kj <= 5; ++kj) ws = ws + cf1[kj - 1] * cf1[kk - 1] * B(j + kj - 3, k + kk - 3);
      Bxy[c] = ws / norm_xy;
    }
  std::vector<double>* planes[5] = {&Bx, &By, &Bxx, &Byy, &Bxy};
  for (auto* pl : planes) {
    std::vector<double>& a = *pl;
    for (int k = 1; k <= ny; ++k) {
      a[c2(1, k)] = a[c2(3, k)];
      a[c2(2, k)] = a[c2(3, k)];
      a[c2(nx - 1, k)] = a[c2(nx - 2, k)];
      a[c2(nx, k)] = a[c2(nx - 2, k)];
    }
    for (int j = 1; j <= nx; ++j) {
      a[c2(j, 1)] = a[c2(j, 3)];
      a[c2(j, 2)] = a[c2(j, 3)];
      a[c2(j, ny - 1)] = a[c2(j, ny - 2)];
      a[c2(j, ny)] = a[c2(j, ny - 2)];
    }
  }
  if (p.slope_correction_flag) {
    for (size_t c = 0; c < N; ++c) {
      gc[c] = 1.0 / (1.0 + Bx[c] * Bx[c] + By[c] * By[c]);
      dgc_dx[c] = -(2.0 * (gc[c] * gc[c]) * (Bx[c] * Bxx[c] + By[c] * Bxy[c]));
    }
    for (int k = 1; k <= ny; ++k) {
      gc_sx[sx2(1, k)] = gc[c2(1, k)];
      for (int j = 2; j <= nx; ++j) gc_sx[sx2(j, k)] = 0.5 * (gc[c2(j - 1, k)] + gc[c2(j, k)]);
      gc_sx[sx2(nx + 1, k)] = gc[c2(nx, k)];
    }
    for (int j = 1; j <= nx; ++j) {
      gc_sy[sy2(j, 1)] = gc[c2(j, 1)];
      for (int k = 2; k <= ny; ++k) gc_sy[sy2(j, k)] = 0.5 * (gc[c2(j, k - 1)] + gc[c2(j, k)]);
      gc_sy[sy2(j, ny + 1)] = gc[c2(j, ny)];
    }
  }
}

// One cell of the driver's output sweep: qp, running maxima and the
// vulnerability table (src/IMEX_SfloW2D.f90:398-440; init: :261-307).
void OracleCtx::post_cell(int j, int k, bool init) {
  const size_t c = c2(j, k);
  if (Q(q, j, k)[0] > 0.0) {
    double pd;
    double* o = QP(qp, j, k);
    qc_to_qp(Q(q, j, k), o, pd);
    hmax[c] = init ? o[0] : fmax_f(hmax[c], o[0]);
    double r_u = o[idx_u], r_v = o[idx_v];
    double mod_vel = std::sqrt(r_u * r_u + r_v * r_v);
    if (o[0] > 0.001) {
      pdynmax[c] = init ? pd : fmax_f(pdynmax[c], pd);
      mvmax[c] = init ? mod_vel : fmax_f(mvmax[c], mod_vel);
    }
    int it = 0, nt = n_thk * n_pdyn;
    for (int a = 0; a < n_thk; ++a) {
      bool thck = o[0] >= thk_lev[a];
      for (int b = 0; b < n_pdyn; ++b, ++it) {
        bool pdyn = pd >= pdyn_lev[b];
        uint8_t& v = vuln[(size_t)it + (size_t)nt * c];
        v = init ? (uint8_t)(thck && pdyn) : (uint8_t)(v || (thck && pdyn));
      }
    }
  } else {
    double* o = QP(qp, j, k);
    // the first sweep clears qp(1:n_vars), the per-step one qp(1:n_vars+2)
    for (int i = 0; i < (init ? nv : np); ++i) o[i] = 0.0;
    o[3] = p.T_ambient;
    if (init) {
      hmax[c] = 0.0;
      pdynmax[c] = 0.0;
    }
  }
}

// src/IMEX_SfloW2D.f90:237-301 (after check_solve(.TRUE.))
void OracleCtx::initial_sweep() {
  for (int64_t l = 0; l < solve_cells; ++l) {
    int j = j_cent[l], k = k_cent[l];
    double pd;
    if (Q(q, j, k)[0] > 0.0) {
      qc_to_qp(Q(q, j, k), QP(qp, j, k), pd);
    } else {
      double* o = QP(qp, j, k);
      for (int i = 0; i < nv; ++i) o[i] = 0.0;
      o[3] = p.T_ambient;
    }
  }
}

// ================================================================== C API
static std::vector<double> copy_plane(const double* src, size_t n, double fill) {
  std::vector<double> v(n, fill);
  if (src) std::memcpy(v.data(), src, n * sizeof(double));
  return v;
}
template <class T>
static std::vector<T> copy_plane_t(const T* src, size_t n) {
  std::vector<T> v(n, (T)0);
  if (src) std::memcpy(v.data(), src, n * sizeof(T));
  return v;
}

extern "C" {

OracleCtx* oracle_create(const ImexParams* pp, const ImexStatic* s) {
  OracleCtx* o = new OracleCtx();
  o->p = *pp;
  const ImexParams& p = o->p;
  o->nx = p.nx;
  o->ny = p.ny;
  o->ns = p.n_solid;
  o->nv = 4 + p.n_solid;
  o->np = o->nv + 2;
  o->neq = o->nv;
  o->nrk = p.n_rk;
  o->idx_u = o->nv;
  o->idx_v = o->nv + 1;
  const int nx = o->nx, ny = o->ny, nv = o->nv, np = o->np;
  // init_grid, src/geometry_2d.f90:240-300
  o->dx = (nx > 1) ? p.cell_size : 1.0;
  o->dy = (ny > 1) ? p.cell_size : 1.0;
  o->dx2 = o->dx / 2.0;
  o->dy2 = o->dy / 2.0;
  o->one_by_dx = 1.0 / o->dx;
  o->one_by_dy = 1.0 / o->dy;
  o->eps_sing = p.eps_sing;
  o->eps_sing4 = (p.eps_sing * p.eps_sing) * (p.eps_sing * p.eps_sing);
  o->x_stag.resize(nx + 1);
  o->y_stag.resize(ny + 1);
  o->x_comp.resize(nx);
  o->y_comp.resize(ny);
  for (int j = 1; j <= nx + 1; ++j) o->x_stag[j - 1] = p.x0 + (double)(j - 1) * o->dx;
  for (int k = 1; k <= ny + 1; ++k) o->y_stag[k - 1] = p.y0 + (double)(k - 1) * o->dy;
  for (int j = 1; j <= nx; ++j) o->x_comp[j - 1] = 0.5 * (o->x_stag[j - 1] + o->x_stag[j]);
  for (int k = 1; k <= ny; ++k) o->y_comp[k - 1] = 0.5 * (o->y_stag[k - 1] + o->y_stag[k]);
  // allocate_solver_variables, src/solver_2d.f90:273-274
  o->h = (double)nv * EPS;
  o->one_by_h = 1.0 / o->h;
  // read_param: inpout_2d.f90:1330,1353,1882
  o->inv_pres = 1.0 / p.pres;
  o->rho_a_amb = p.pres / (p.sp_gas_const_a * p.T_ambient);
  for (int i = 0; i < o->ns; ++i) o->inv_rho_s[i] = 1.0 / p.rho_s[i];
  // init_problem_param, constitutive_2d.f90:469-518
  for (int i = 0; i < nv; ++i) o->implicit_flag[i] = (i == 1 || i == 2);
  o->n_nh = 2;
  // Butcher tableau, src/solver_2d.f90:404-486
  std::memset(o->a_tilde_ij, 0, sizeof(o->a_tilde_ij));
  std::memset(o->a_dirk_ij, 0, sizeof(o->a_dirk_ij));
  std::memset(o->omega_tilde, 0, sizeof(o->omega_tilde));
  std::memset(o->omega, 0, sizeof(o->omega));
  if (o->nrk == 1) {
    o->a_tilde_ij[0][0] = 1.0;
    o->omega_tilde[0] = 1.0;
  } else if (o->nrk == 2) {
    o->a_tilde_ij[1][0] = 1.0;
    o->omega_tilde[0] = 1.0;
    o->a_dirk_ij[1][1] = 1.0;
    o->omega[1] = 1.0;
  } else if (o->nrk == 3) {
    o->a_tilde_ij[1][0] = 0.5;
    o->a_tilde_ij[2][0] = 0.5;
    o->a_tilde_ij[2][1] = 0.5;
    o->omega_tilde[0] = o->omega_tilde[1] = o->omega_tilde[2] = 1.0 / 3.0;
    o->a_dirk_ij[0][0] = 0.25;
    o->a_dirk_ij[1][1] = 0.25;
    o->a_dirk_ij[2][0] = 1.0 / 3.0;
    o->a_dirk_ij[2][1] = 1.0 / 3.0;
    o->a_dirk_ij[2][2] = 1.0 / 3.0;
    o->omega[0] = o->omega[1] = o->omega[2] = 1.0 / 3.0;
  } else if (o->nrk == 4) {
    o->a_tilde_ij[1][0] = 0.5;
    o->a_tilde_ij[2][0] = 1.0 / 3.0;
    o->a_tilde_ij[3][1] = 1.0;
    o->omega_tilde[1] = 1.0;
    o->a_dirk_ij[1][1] = 0.5;
    o->a_dirk_ij[2][2] = 1.0 / 3.0;
    o->a_dirk_ij[3][2] = 0.75;
    o->a_dirk_ij[3][3] = 0.25;
    o->omega[2] = 0.75;
    o->omega[3] = 0.25;
  }
  const size_t N = (size_t)nx * ny, NX = (size_t)(nx + 1) * ny, NY = (size_t)nx * (ny + 1);
  o->B_cent = copy_plane(s->B_cent, N, 0.0);
  o->Bx = copy_plane(s->B_prime_x_geom, N, 0.0);
  o->By = copy_plane(s->B_prime_y_geom, N, 0.0);
  if (s->B_second_xx_geom) o->Bxx = copy_plane(s->B_second_xx_geom, N, 0.0);
  if (s->B_second_xy_geom) o->Bxy = copy_plane(s->B_second_xy_geom, N, 0.0);
  if (s->B_second_yy_geom) o->Byy = copy_plane(s->B_second_yy_geom, N, 0.0);
  o->gc = copy_plane(s->grav_coeff, N, 1.0);
  o->dgc_dx = copy_plane(s->d_grav_coeff_dx, N, 0.0);
  o->gc_sx = copy_plane(s->grav_coeff_stag_x, NX, 1.0);
  o->gc_sy = copy_plane(s->grav_coeff_stag_y, NY, 1.0);
  o->source_cell = copy_plane_t<int32_t>(s->source_cell, N);
  o->sE = copy_plane_t<int8_t>(s->sourceE, N);
  o->sW = copy_plane_t<int8_t>(s->sourceW, N);
  o->sS = copy_plane_t<int8_t>(s->sourceS, N);
  o->sN = copy_plane_t<int8_t>(s->sourceN, N);
  o->sEx = copy_plane(s->sourceE_vect_x, N, 0.0);
  o->sEy = copy_plane(s->sourceE_vect_y, N, 0.0);
  o->sWx = copy_plane(s->sourceW_vect_x, N, 0.0);
  o->sWy = copy_plane(s->sourceW_vect_y, N, 0.0);
  o->sSx = copy_plane(s->sourceS_vect_x, N, 0.0);
  o->sSy = copy_plane(s->sourceS_vect_y, N, 0.0);
  o->sNx = copy_plane(s->sourceN_vect_x, N, 0.0);
  o->sNy = copy_plane(s->sourceN_vect_y, N, 0.0);
  if (s->B_nodata) o->B_nodata = copy_plane_t<int8_t>(s->B_nodata, N);
  o->solve_mask_time = copy_plane(s->solve_mask_time, N, 0.0);
  o->cell_source_fractions.assign(N, 0.0);
  o->erodible = copy_plane(s->erodible, N * o->ns, 0.0);
  o->deposit = copy_plane(s->deposit, N * o->ns, 0.0);
  o->erosion = copy_plane(s->erosion, N * o->ns, 0.0);
  // work arrays (zero: the reference leaves them uninitialised)
  o->q.assign(N * nv, 0.0);
  o->q0.assign(N * nv, 0.0);
  o->q_fv.assign(N * nv, 0.0);
  o->qp.assign(N * np, 0.0);
  for (size_t c = 0; c < N; ++c) o->qp[c * np + 3] = p.T_ambient;
  o->q_rk.assign(N * nv * o->nrk, 0.0);
  o->qp_rk.assign(N * np * o->nrk, 0.0);
  o->divFlux.assign(N * nv * o->nrk, 0.0);
  o->NH.assign(N * nv * o->nrk, 0.0);
  o->SI_NH.assign(N * nv * o->nrk, 0.0);
  o->expl_terms.assign(N * nv * o->nrk, 0.0);
  o->qL.assign(NX * nv, 0.0);
  o->qR.assign(NX * nv, 0.0);
  o->qpL.assign(NX * np, 0.0);
  o->qpR.assign(NX * np, 0.0);
  o->qB.assign(NY * nv, 0.0);
  o->qT.assign(NY * nv, 0.0);
  o->qpB.assign(NY * np, 0.0);
  o->qpT.assign(NY * np, 0.0);
  o->axNeg.assign(NX, 0.0);
  o->axPos.assign(NX, 0.0);
  o->ayNeg.assign(NY, 0.0);
  o->ayPos.assign(NY, 0.0);
  o->ax_max.assign(NX, 0.0);
  o->ay_max.assign(NY, 0.0);
  o->Hx.assign(NX * nv, 0.0);
  o->Hy.assign(NY * nv, 0.0);
  o->epL.assign(NX, -1);
  o->epR.assign(NX, -1);
  o->epB.assign(NY, -1);
  o->epT.assign(NY, -1);
  o->mask.assign(N, 0);
  // border rows and columns are always solved (src/solver_2d.f90:350-353)
  for (int k = 1; k <= ny; ++k) {
    o->mask[o->c2(1, k)] = 1;
    o->mask[o->c2(nx, k)] = 1;
  }
  for (int j = 1; j <= nx; ++j) {
    o->mask[o->c2(j, 1)] = 1;
    o->mask[o->c2(j, ny)] = 1;
  }
  o->mask_temp.assign(N, 0);
  o->mask_x.assign(NX, 0);
  o->mask_y.assign(NY, 0);
  o->j_cent.assign(N, 0);
  o->k_cent.assign(N, 0);
  o->j_stag_x.assign(NX, 0);
  o->k_stag_x.assign(NX, 0);
  o->j_stag_y.assign(NY, 0);
  o->k_stag_y.assign(NY, 0);
  for (int b = 0; b < 16; ++b) o->hist[b] = 0;
  return o;
}

void oracle_destroy(OracleCtx* o) { delete o; }

void oracle_set_state(OracleCtx* o, const double* q, double t) {
  std::memcpy(o->q.data(), q, o->q.size() * sizeof(double));
  for (int i = 0; i < 4; ++i) o->mass_budget[i] = 0.0L;
  o->t = t;
  o->check_solve(true, t);
  o->initial_sweep();
}

void oracle_get_state(OracleCtx* o, double* q, double* qp) {
  if (q) std::memcpy(q, o->q.data(), o->q.size() * sizeof(double));
  if (qp) std::memcpy(qp, o->qp.data(), o->qp.size() * sizeof(double));
}

void oracle_get_exchange(OracleCtx* o, double* erodible, double* deposit, double* erosion,
                         double* B_cent) {
  if (erodible) std::memcpy(erodible, o->erodible.data(), o->erodible.size() * sizeof(double));
  if (deposit) std::memcpy(deposit, o->deposit.data(), o->deposit.size() * sizeof(double));
  if (erosion) std::memcpy(erosion, o->erosion.data(), o->erosion.size() * sizeof(double));
  if (B_cent) std::memcpy(B_cent, o->B_cent.data(), o->B_cent.size() * sizeof(double));
}

int64_t oracle_check_solve(OracleCtx* o, double t, int solve_all) {
  o->check_solve(solve_all != 0, t);
  return o->solve_cells;
}

double oracle_timestep(OracleCtx* o) { return o->timestep(); }

uint32_t oracle_rk_step(OracleCtx* o, double t, double dt) {
  o->t = t;
  o->dt = dt;
  o->newton_cells = 0;
  o->newton_iters = 0;
  o->lnsrch_trials = 0;
  o->newton_maxit = 0;
  for (int b = 0; b < 16; ++b) o->hist[b] = 0;
  return o->imex_RK_solver(dt);
}

uint32_t oracle_erosion_deposition(OracleCtx* o, double dt) {
  return o->update_erosion_deposition_cell(dt);
}

void oracle_post_step(OracleCtx* o) { o->post_step_sweep(); }

void oracle_get_masks(OracleCtx* o, int8_t* m, int8_t* mx, int8_t* my) {
  if (m)
    for (size_t i = 0; i < o->mask.size(); ++i) m[i] = (int8_t)o->mask[i];
  if (mx)
    for (size_t i = 0; i < o->mask_x.size(); ++i) mx[i] = (int8_t)o->mask_x[i];
  if (my)
    for (size_t i = 0; i < o->mask_y.size(); ++i) my[i] = (int8_t)o->mask_y[i];
}

void oracle_set_clock(OracleCtx* o, double t, double dt0, double t_end, double t_output) {
  o->t = t;
  o->dt_old = dt0;
  o->dt_old_old = dt0;
  o->t_end = t_end;
  o->t_output = t_output;
}

// src/IMEX_SfloW2D.f90:337-447 without the I/O
uint32_t oracle_advance(OracleCtx* o, int n_steps, double* t) {
  uint32_t err = 0;
  for (int s = 0; s < n_steps; ++s) {
    o->check_solve(false, o->t);
    double dt = o->timestep();
    if (o->t + dt > o->t_end) dt = o->t_end - o->t;
    if (o->t_output >= 0.0 && o->t + dt > o->t_output) dt = o->t_output - o->t;
    dt = fmin_f(dt, 1.1 * 0.5 * (o->dt_old + o->dt_old_old));
    o->dt_old_old = o->dt_old;
    o->dt_old = dt;
    o->dt = dt;
    o->newton_cells = 0;
    o->newton_iters = 0;
    o->lnsrch_trials = 0;
    o->newton_maxit = 0;
    for (int b = 0; b < 16; ++b) o->hist[b] = 0;
    err |= o->imex_RK_solver(dt);
    err |= o->update_erosion_deposition_cell(dt);
    if (o->p.topo_change_flag) o->topography_reconstruction();
    o->t = o->t + dt;
    o->post_step_sweep();
    o->steps += 1;
  }
  if (t) *t = o->t;
  return err;
}

void oracle_stats(OracleCtx* o, ImexStats* st) {
  std::memset(st, 0, sizeof(*st));
  st->solve_cells = o->solve_cells;
  st->newton_cells = o->newton_cells;
  st->newton_iters = o->newton_iters;
  st->lnsrch_trials = o->lnsrch_trials;
  st->newton_maxit_cells = o->newton_maxit;
  for (int b = 0; b < 16; ++b) st->newton_hist[b] = o->hist[b];
  st->error_mask = o->error_mask;
  st->first_error_code = o->first_err_code;
  if (o->first_err_index >= 0) {
    st->first_error_j = (int32_t)(o->first_err_index % o->nx) + 1;
    st->first_error_k = (int32_t)(o->first_err_index / o->nx) + 1;
  }
  st->dt = o->dt;
  st->t = o->t;
  st->steps = o->steps;
}

int64_t oracle_stale_wet_reads(OracleCtx* o) { return o->stale_wet_reads; }

void oracle_mass_budget(OracleCtx* o, double* out) {
  for (int i = 0; i < 4; ++i) out[i] = (double)o->mass_budget[i];
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_qc_to_qp(OracleCtx* o, const double* qc, double* qpo) {
  double pd;
  o->qc_to_qp(qc, qpo, pd);
}

void oracle_qp_to_qc(OracleCtx* o, const double* qpi, double* qc) { o->qp_to_qc(qpi, qc); }

void oracle_implicit_terms(OracleCtx* o, const double* q_re, const double* q_im, double* nh_re,
                           double* nh_im) {
  cplx qj[MAXV], nh[MAXV];
  for (int i = 0; i < o->nv; ++i) qj[i] = C(q_re[i], q_im ? q_im[i] : 0.0);
  o->eval_implicit_terms(0.0, 0.0, qj, nh);
  for (int i = 0; i < o->nv; ++i) {
    nh_re[i] = nh[i].re;
    if (nh_im) nh_im[i] = nh[i].im;
  }
}

void oracle_mixt_var(OracleCtx* o, const double* qp, double* out) {
  double Ri, rho_m, rho_c, red_grav, spc, spm;
  o->mixt_var(qp, Ri, rho_m, rho_c, red_grav, false, spc, spm);
  out[0] = Ri;
  out[1] = rho_m;
  out[2] = rho_c;
  out[3] = red_grav;
}

void oracle_local_speeds(OracleCtx* o, const double* qp, double gcf, int dir, double* out) {
  if (dir == 1)
    o->eval_local_speeds_x(qp, gcf, out[0], out[1]);
  else
    o->eval_local_speeds_y(qp, gcf, out[0], out[1]);
}

void oracle_eval_fluxes(OracleCtx* o, const double* qc, const double* qp, double gcf, int dir,
                        double* flux) {
  o->eval_fluxes(qc, qp, gcf, dir, flux);
}

void oracle_kt_interface(OracleCtx* o, const double* qcL, const double* qpL, const double* qcR,
                         const double* qpR, double gcf, int dir, double* H, double* speeds) {
  double lmin, lmax, rmin, rmax;
  if (dir == 1) {
    o->eval_local_speeds_x(qpL, gcf, lmin, lmax);
    o->eval_local_speeds_x(qpR, gcf, rmin, rmax);
  } else {
    o->eval_local_speeds_y(qpL, gcf, lmin, lmax);
    o->eval_local_speeds_y(qpR, gcf, rmin, rmax);
  }
  const double aN = fmin_f(fmin_f(lmin, rmin), 0.0), aP = fmax_f(fmax_f(lmax, rmax), 0.0);
  o->kt_face(qcL, qpL, qcR, qpR, aN, aP, gcf, dir, H);
  if (speeds) {
    speeds[0] = aN;
    speeds[1] = aP;
  }
}

int oracle_solve_rk_step(OracleCtx* o, double* qj, const double* qj_old,
                         const double* rj_not_impl, double bprime_x, double bprime_y,
                         double dt, double a_diag) {
  int64_t trials = 0;
  return o->solve_rk_step(qj, qj_old, a_diag, rj_not_impl, bprime_x, bprime_y, dt, trials);
}

double oracle_ipow(double x, double y) { return ipow(x, y); }
void oracle_ipow_n(long long n, const double* x, const double* y, double* out) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < n; ++i) out[i] = ipow(x[i], y[i]);
}
void oracle_limit_n(long long n, const double* v1, const double* v2, const double* v3,
                    const double* z1, const double* z2, const double* z3, int limiter,
                    double theta, double* out) {
  OracleCtx tmp;
  tmp.p.theta = theta;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < n; ++i) {
    const double v[3] = {v1[i], v2[i], v3[i]}, z[3] = {z1[i], z2[i], z3[i]};
    out[i] = tmp.limit(v, z, limiter);
  }
}
void oracle_settling_velocity_n(long long n, const double* diam, const double* rhos,
                                const double* rhoc, const double* ikv, double grav,
                                double* out) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < n; ++i)
    out[i] = settling_velocity_g(diam[i], rhos[i], rhoc[i], ikv[i], grav);
}

double oracle_limit(double v1, double v2, double v3, double z1, double z2, double z3,
                    int limiter, double theta) {
  OracleCtx tmp;
  tmp.p.theta = theta;
  double v[3] = {v1, v2, v3}, z[3] = {z1, z2, z3};
  return tmp.limit(v, z, limiter);
}

}  // extern "C"

// Driver output sweep and print values (test infrastructure for the GPU's
// imex_gpu_post_*): levels already normalised by the caller.
extern "C" void oracle_post_init(OracleCtx* o, int n_thk, const double* thk, int n_pdyn,
                                 const double* pdyn) {
  o->n_thk = n_thk;
  o->n_pdyn = n_pdyn;
  for (int i = 0; i < n_thk; ++i) o->thk_lev[i] = thk[i];
  for (int i = 0; i < n_pdyn; ++i) o->pdyn_lev[i] = pdyn[i];
  const size_t N = (size_t)o->nx * o->ny;
  o->hmax.assign(N, 0.0);
  o->pdynmax.assign(N, 0.0);
  o->mvmax.assign(N, 0.0);
  o->vuln.assign(N * (size_t)(n_thk * n_pdyn), 0);
  for (int64_t l = 0; l < o->solve_cells; ++l) o->post_cell(o->j_cent[l], o->k_cent[l], true);
  o->post_on = true;
}

// SUM(q(1,:,:)), SUM(qp(1,:,:)), COUNT(q(1,:,:) > 1e-7), SUM(q(5:4+n_solid,:,:))
// in array element order, times dx*dy (src/IMEX_SfloW2D.f90:476-484).
extern "C" void oracle_post_diag(OracleCtx* o, double* out) {
  const size_t N = (size_t)o->nx * o->ny;
  double m = 0.0, v = 0.0, a = 0.0, sm = 0.0;
  for (size_t c = 0; c < N; ++c) m += o->q[c * o->nv];
  for (size_t c = 0; c < N; ++c) v += o->qp[c * o->np];
  for (size_t c = 0; c < N; ++c) a += (o->q[c * o->nv] > 1.0e-7) ? 1.0 : 0.0;
  for (size_t c = 0; c < N; ++c)
    for (int i = 4; i < o->nv; ++i) sm += o->q[c * o->nv + i];
  const double cell = o->dx * o->dy;
  out[0] = cell * m;
  out[1] = cell * v;
  out[2] = cell * a;
  out[3] = cell * sm;
}

extern "C" void oracle_get_post(OracleCtx* o, double* hmax, double* pdynmax, double* mvmax,
                                int8_t* vuln) {
  const size_t N = (size_t)o->nx * o->ny;
  for (size_t c = 0; c < N; ++c) {
    if (hmax) hmax[c] = o->hmax[c];
    if (pdynmax) pdynmax[c] = o->pdynmax[c];
    if (mvmax) mvmax[c] = o->mvmax[c];
  }
  if (vuln)
    for (size_t i = 0; i < o->vuln.size(); ++i) vuln[i] = (int8_t)o->vuln[i];
}

extern "C" void oracle_topography_reconstruction(OracleCtx* o) { o->topography_reconstruction(); }

extern "C" void oracle_get_topo(OracleCtx* o, double* bx, double* by, double* bxx, double* bxy,
                                double* byy, double* gc, double* dgc) {
  const size_t N = (size_t)o->nx * o->ny;
  for (size_t c = 0; c < N; ++c) {
    if (bx) bx[c] = o->Bx[c];
    if (by) by[c] = o->By[c];
    if (bxx && !o->Bxx.empty()) bxx[c] = o->Bxx[c];
    if (bxy && !o->Bxy.empty()) bxy[c] = o->Bxy[c];
    if (byy && !o->Byy.empty()) byy[c] = o->Byy[c];
    if (gc) gc[c] = o->gc[c];
    if (dgc) dgc[c] = o->dgc_dx[c];
  }
}

// ---------------------------------------------------------------- set-up
// Restatements of init_grid's DEM sampling, compute_cell_fract and the
// restart regridding, loop for loop as the reference writes them.

// init_grid's x_stag/x_comp (src/geometry_2d.f90:250-320) for a grid of n
// cells: spacing cell_size, or 1 for a single cell.
static double setup_comp(double o, double d, int J) {   // J 1-based
  const double a = o + (double)(J - 1) * d, b = o + (double)J * d;
  return 0.5 * (a + b);
}

// src/geometry_2d.f90:320-342 with interp_2d_nodata (:1242-1296) and
// interp_2d_scalar (:1174-1226); node coordinates per src/inpout_2d.f90:
// 3579-3589.  Returns 0, or 1 when a cell centre lies west/south of the
// first node (the reference would index outside the DEM), 2 for a
// non-finite index.
extern "C" int oracle_setup_dem(int ncols, int nrows, double xll, double yll, double cs,
                                double nodata, const double* z, int nx, int ny, double x0,
                                double y0, double cell_size, double* B_cent, int8_t* B_nodata) {
  const double dx = nx > 1 ? cell_size : 1.0, dy = ny > 1 ? cell_size : 1.0;
  std::vector<double> x1(ncols), y1(nrows), zc((size_t)ncols * nrows);
  for (int j = 1; j <= ncols; ++j) x1[j - 1] = xll + ((double)j - 0.5) * cs;
  for (int k = 1; k <= nrows; ++k) y1[k - 1] = yll + ((double)k - 0.5) * cs;
  for (size_t i = 0; i < zc.size(); ++i) zc[i] = fmax_f(0.0, z[i]);   // MAX(0, z)
  auto Z = [&](const double* a, int ix, int iy) { return a[(size_t)(ix - 1) + (size_t)(iy - 1) * ncols]; };
  int status = 0;
  for (int k = 1; k <= ny; ++k) {
    for (int j = 1; j <= nx; ++j) {
      const double x2 = setup_comp(x0, dx, j), y2 = setup_comp(y0, dy, k);
      const size_t c = (size_t)(j - 1) + (size_t)(k - 1) * nx;
      int ix = 1, iy = 1;
      double ax = 0.0, ay = 0.0;
      bool ok = true;
      if (ncols > 1) {
        const double v = (x2 - x1[0]) / (x1[1] - x1[0]);
        if (!(v > -1.0e9 && v < 1.0e9)) ok = false;
        else ix = std::min((int)std::floor(v) + 1, ncols - 1);
      }
      if (nrows > 1) {
        const double v = (y2 - y1[0]) / (y1[1] - y1[0]);
        if (!(v > -1.0e9 && v < 1.0e9)) ok = false;
        else iy = std::min((int)std::floor(v) + 1, nrows - 1);
      }
      if (!ok || ix < 1 || iy < 1) {
        status |= ok ? 1 : 2;
        B_cent[c] = 0.0;
        B_nodata[c] = 0;
        continue;
      }
      if (ncols > 1) ax = (x1[ix] - x2) / (x1[ix] - x1[ix - 1]);
      if (nrows > 1) ay = (y1[iy] - y2) / (y1[iy] - y1[iy - 1]);
      bool nod;
      double f2;
      if (ncols == 1) {
        nod = (Z(z, ix, iy) == nodata) || (Z(z, ix, iy + 1) == nodata);
        f2 = ay * Z(zc.data(), ix, iy) + (1.0 - ay) * Z(zc.data(), ix, iy + 1);
      } else if (nrows == 1) {
        nod = (Z(z, ix, iy) == nodata) || (Z(z, ix + 1, iy) == nodata);
        f2 = ax * Z(zc.data(), ix, iy) + (1.0 - ax) * Z(zc.data(), ix + 1, iy);
      } else {
        nod = (Z(z, ix, iy) == nodata) || (Z(z, ix, iy + 1) == nodata) ||
              (Z(z, ix + 1, iy) == nodata) || (Z(z, ix + 1, iy + 1) == nodata);
        f2 = ax * (ay * Z(zc.data(), ix, iy) + (1.0 - ay) * Z(zc.data(), ix, iy + 1)) +
             (1.0 - ax) * (ay * Z(zc.data(), ix + 1, iy) + (1.0 - ay) * Z(zc.data(), ix + 1, iy + 1));
      }
      B_cent[c] = f2;
      B_nodata[c] = nod ? 1 : 0;
    }
  }
  return status;
}

// compute_cell_fract (src/geometry_2d.f90:1678-1773): every subgrid point of
// every cell that meets the bounding square.
extern "C" void oracle_cell_fract(int nx, int ny, double x0, double y0, double cell_size,
                                  double xs, double ys, double rs, double r2s, double angle_deg,
                                  double* cell_fract) {
  const int n = 200, n2 = n * n;
  const double dx = nx > 1 ? cell_size : 1.0, dy = ny > 1 ? cell_size : 1.0;
  const double ang_rad = ((angle_deg / 180.0) * std::atan(1.0)) * 4.0;
  const double ca = std::cos(ang_rad), sa = std::sin(ang_rad);
  std::vector<double> xsub(n2), ysub(n2);
  for (int h = 1; h <= n; ++h) {
    for (int i = h; i <= n2; i += n) xsub[i - 1] = (double)h;
    for (int i = (h - 1) * n + 1; i <= h * n; ++i) ysub[i - 1] = (double)h;
  }
  for (int i = 0; i < n2; ++i) {
    xsub[i] = (2.0 * xsub[i] - 1.0) / (2.0 * (double)n);
    ysub[i] = (2.0 * ysub[i] - 1.0) / (2.0 * (double)n);
    xsub[i] = (xsub[i] - 0.5) * dx;
    ysub[i] = (ysub[i] - 0.5) * dy;
  }
  const double R = (rs > r2s) ? rs : r2s;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 1; j <= nx; ++j) {
    const double xsj = x0 + (double)(j - 1) * dx, xsj1 = x0 + (double)j * dx;
    const double xc = 0.5 * (xsj + xsj1);
    for (int k = 1; k <= ny; ++k) {
      const double ysk = y0 + (double)(k - 1) * dy, ysk1 = y0 + (double)k * dy;
      const double yc = 0.5 * (ysk + ysk1);
      double& out = cell_fract[(size_t)(j - 1) + (size_t)(k - 1) * nx];
      if (xsj1 < (xs - R) || xsj > (xs + R) || ysk1 < (ys - R) || ysk > (ys + R)) {
        out = 0.0;
        continue;
      }
      int cnt = 0;
      for (int i = 0; i < n2; ++i) {
        const double X = (xc + xsub[i]) - xs, Y = (yc + ysub[i]) - ys;
        const double u = X * ca + Y * sa;
        const double v = -(X * sa) + Y * ca;
        if ((u * u) / (rs * rs) + (v * v) / (r2s * r2s) <= 1.0) cnt += 1;
      }
      out = (double)((float)cnt / (float)n2);
    }
  }
}

// read_solution's regridding of a restart raster (src/inpout_2d.f90:
// 5190-5246) through regrid_scalar (src/geometry_2d.f90:1491-1534).
// Returns 0, or 2 for a non-finite index.
extern "C" int oracle_regrid(int ncols, int nrows, double xll, double yll, double cs,
                             double nodata, const double* fin_raw, int nx, int ny, double x0,
                             double y0, double cell_size, double* fout) {
  std::vector<double> xin(ncols + 1), yin(nrows + 1), fin(fin_raw, fin_raw + (size_t)ncols * nrows);
  for (auto& v : fin)
    if (v == nodata) v = 0.0;
  for (int j = 1; j <= ncols + 1; ++j) xin[j - 1] = xll + (double)(j - 1) * cs;
  for (int k = 1; k <= nrows + 1; ++k) yin[k - 1] = yll + (double)(k - 1) * cs;
  const int nXin = ncols, nYin = nrows + 1;
  const double dXin = xin[1] - xin[0], dYin = yin[1] - yin[0];
  auto ceil_ok = [](double v, int& o) {
    if (!(v > -1.0e9 && v < 1.0e9)) return false;
    o = (int)std::ceil(v);
    return true;
  };
  int status = 0;
  for (int j = 1; j <= nx; ++j) {
    const double xl = x0 + (double)(j - 1) * cell_size, xr = x0 + (double)j * cell_size;
    for (int k = 1; k <= ny; ++k) {
      const double yl = y0 + (double)(k - 1) * cell_size, yr = y0 + (double)k * cell_size;
      double& f = fout[(size_t)(j - 1) + (size_t)(k - 1) * nx];
      int a, b, c, d;
      if (!ceil_ok((xl - xin[0]) / dXin, a) || !ceil_ok((xr - xin[0]) / dXin, b) ||
          !ceil_ok((yl - yin[0]) / dYin, c) || !ceil_ok((yr - yin[0]) / dYin, d)) {
        status |= 2;
        f = 0.0;
        continue;
      }
      const int ix1 = std::max(1, a), ix2 = std::min(nXin, b + 1);
      const int iy1 = std::max(1, c), iy2 = std::min(nYin, d + 1);
      f = 0.0;
      for (int ix = ix1; ix <= ix2 - 1; ++ix) {
        const double alfa_x = (fmin_f(xr, xin[ix]) - fmax_f(xl, xin[ix - 1])) / (xr - xl);
        for (int iy = iy1; iy <= iy2 - 1; ++iy) {
          const double alfa_y = (fmin_f(yr, yin[iy]) - fmax_f(yl, yin[iy - 1])) / (yr - yl);
          f = f + alfa_x * alfa_y * fin[(size_t)(ix - 1) + (size_t)(iy - 1) * ncols];
        }
      }
    }
  }
  return status;
}

// ----------------------------------------------------------- output values
// The values output_solution prints (src/inpout_2d.f90:5683-6180) and its
// in-place changes: cons sets |q| < 1e-20 to 0 in q (:5807-5813); phys
// computes the .p_2d columns from that q (:5914-6148) and sets DEPOSIT and
// EROSION below 1e-20 to 0 (:6115-6122); esri takes qp(1) and qp(4) of the
// driver's qp, i.e. of q before the .q_2d zeroing.  p2d: 17+4*ns planes of
// nx*ny (after x_comp, y_comp): h, u, v, B_out, h+B_out, alphas, T, rho_m,
// red_grav, DEPOSIT, EROSION, SUM(ERODIBLE)/(1-porosity), alphal, shear_vel,
// Ri, Rouse_no, mu_eff, hmax, pdynmax, mod_vel_max, inertial_number, for
// the physics without additional gas, liquid, stochastic or pore-pressure
// variables (the excess pore pressure of mu_eff is taken as 0).
extern "C" void oracle_output_prep(OracleCtx* o, int cons, int phys, int esri, double* p2d,
                                   double* esr) {
  const int nx = o->nx, ny = o->ny, nv = o->nv, ns = o->ns, np = o->np;
  const size_t N = (size_t)nx * ny;
  const ImexParams& p = o->p;
  auto t0 = [](double v) { return (std::fabs(v) < 1.0e-20) ? 0.0 : v; };
  for (int k = 1; k <= ny; ++k) {
    for (int j = 1; j <= nx; ++j) {
      const size_t c = o->c2(j, k);
      double* q = &o->q[(size_t)nv * c];
      double qp[MAXV], p_dyn = 0.0;
      if (esri) {
        o->qc_to_qp(q, qp, p_dyn);
        esr[c] = qp[0];
        esr[N + c] = qp[3];
      }
      if (cons)
        for (int i = 0; i < nv; ++i)
          if (std::fabs(q[i]) < 1.0e-20) q[i] = 0.0;
      if (!phys) continue;
      o->qc_to_qp(q, qp, p_dyn);
      double r_Ri, r_rho_m, r_rho_c, r_red_grav, spc, spm;
      o->mixt_var(qp, r_Ri, r_rho_m, r_rho_c, r_red_grav, false, spc, spm);
      double r_h = qp[0], r_u = qp[nv], r_v = qp[nv + 1], r_T = qp[3];
      double al[MAXS], mu_eff = 0.0, inertial = 0.0, r_alphal = 0.0;
      const double shear_vel = 0.0;
      if (r_h > 0.0) {
        for (int i = 0; i < ns; ++i) al[i] = p.alpha_flag ? qp[4 + i] : qp[4 + i] / r_h;
        if (p.rheology_flag && p.rheology_model == 1) {
          const double dp = fmax_f(0.0, 0.0);
          mu_eff = p.mu * fmax_f(0.0, 1.0 - dp / (r_rho_m * r_h * r_red_grav));
        }
      } else {
        for (int i = 0; i < ns; ++i) al[i] = 0.0;
      }
      r_h = t0(r_h);
      r_u = t0(r_u);
      r_v = t0(r_v);
      const double B = o->B_cent.empty() ? 0.0 : o->B_cent[c];
      const double B_out = t0(B);
      double dep[MAXS], ers[MAXS];
      for (int i = 0; i < ns; ++i) {
        al[i] = t0(al[i]);
        dep[i] = o->deposit.empty() ? 0.0 : o->deposit[c + N * i];
        ers[i] = o->erosion.empty() ? 0.0 : o->erosion[c + N * i];
        if (std::fabs(dep[i]) < 1.0e-20) {
          dep[i] = 0.0;
          if (!o->deposit.empty()) o->deposit[c + N * i] = 0.0;
        }
        if (std::fabs(ers[i]) < 1.0e-20) {
          ers[i] = 0.0;
          if (!o->erosion.empty()) o->erosion[c + N * i] = 0.0;
        }
      }
      r_T = t0(r_T);
      r_rho_m = t0(r_rho_m);
      r_red_grav = t0(r_red_grav);
      r_alphal = t0(r_alphal);
      mu_eff = t0(mu_eff);
      inertial = t0(inertial);
      double esum = 0.0;
      for (int i = 0; i < ns; ++i)
        esum = esum + (o->erodible.empty() ? 0.0 : o->erodible[(size_t)i + ns * c]);
      const double etot = esum / (1.0 - p.erodible_porosity);
      int col = 0;
      auto put = [&](double v) { p2d[(size_t)col++ * N + c] = v; };
      put(r_h);
      put(r_u);
      put(r_v);
      put(B_out);
      put(r_h + B_out);
      for (int i = 0; i < ns; ++i) put(al[i]);
      put(r_T);
      put(r_rho_m);
      put(r_red_grav);
      for (int i = 0; i < ns; ++i) put(dep[i]);
      for (int i = 0; i < ns; ++i) put(ers[i]);
      put(etot);
      put(r_alphal);
      put(shear_vel);
      put(r_Ri);
      for (int i = 0; i < ns; ++i) put(0.0);
      put(mu_eff);
      put(o->hmax.empty() ? 0.0 : o->hmax[c]);
      put(o->pdynmax.empty() ? 0.0 : o->pdynmax[c]);
      put(o->mvmax.empty() ? 0.0 : o->mvmax[c]);
      put(inertial);
      (void)np;
    }
  }
}
