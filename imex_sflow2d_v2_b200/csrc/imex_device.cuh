// imex_device.cuh -- device-side physics of the IMEX_SfloW2D time step (sm_100a).
//
// Point functions of the reference's constitutive module and limiter, written
// for registers: arrays are sized at compile time by the number of solid
// classes NS (n_vars = 4 + NS).  Every floating-point expression keeps the
// reference's evaluation order (left to right, parentheses kept) and the file
// is compiled with --fmad=false, so results are bit-identical to a CPU build
// of the same expressions without contraction.  MIN/MAX return the non-NaN
// operand when one is NaN.
//
// Reference routines (src/constitutive_2d.f90 unless noted):
//   mixt_var :1333-1483, eval_sp_heat :1503-1597, r_phys_var/qc_to_qp
//   :541-967,1628-1681, qp_to_qc :1709-2140, qp_to_qp2 :2155-2179,
//   eval_local_speeds_x/y :2194-2298, eval_fluxes :2316-2509,
//   eval_expl_terms :3015-3245, c_phys_var :1145-1313,
//   eval_implicit_terms :3327-3823, eval_nh_semi_impl_terms :3841-4397,
//   eval_mass_exchange_terms :4424-5003, settling_velocity :5148-5214,
//   eval_source_bdry :5024-5130; limit/minmod/maxmod src/geometry_2d.f90:1555-1676.
#pragma once

#include <cstdint>

#include "ipow_tables.h"

#ifndef IMEX_HD
#define IMEX_HD __device__ __forceinline__
#endif
// Heavy point functions are kept out of line: they are called from several
// places per kernel and inlining every copy multiplies code size (and ptxas
// time) without a measurable gain for these FP64-bound bodies.
#ifndef IMEX_NOINL
#define IMEX_NOINL __device__ __noinline__
#endif
// Per function, measured on the 4096^2 workload: x**y and the settling
// velocity stay out of line (inlined, erosion 9.3 -> 10.7 ms); the
// conserved <-> physical conversions and the limiter are inlined (flux
// 11.1 -> 10.2 ms, first Newton pass 6.1 -> 5.6, erosion 9.3 -> 8.8).
#ifndef IMEX_IPOW_FN
#define IMEX_IPOW_FN IMEX_NOINL
#endif
#ifndef IMEX_QCQP_FN
#define IMEX_QCQP_FN __device__ __forceinline__
#endif
#ifndef IMEX_LIMIT_FN
#define IMEX_LIMIT_FN __device__ __forceinline__
#endif
#ifndef IMEX_SETTLE_FN
#define IMEX_SETTLE_FN IMEX_NOINL
#endif
// Functions with one or two call sites per kernel (the Newton pieces, the
// mass-exchange terms) are inlined: their per-cell arrays then live in
// registers instead of being passed through the stack.
#ifndef IMEX_FLAT
#define IMEX_FLAT __device__ __forceinline__
#endif
// The complex fallback of the real implicit terms (non-finite values only;
// inlined it measured 1 ms per step faster than as a call at 4096^2).
#ifndef IMEX_RC_FN
#define IMEX_RC_FN __device__ __forceinline__
#endif
// Complex division and square root (the complex-step Jacobian) are called,
// not inlined: one copy each keeps the Newton kernels' hot code small enough
// for the instruction cache (2.5 ms per step less at 4096^2 than inlined).
#ifndef IMEX_CPLX_FN
#define IMEX_CPLX_FN __device__ __noinline__
#endif
// IEEE division in the real implicit terms.
#ifndef IMEX_DIV_FN
#define IMEX_DIV_FN IMEX_HD
#endif

#ifndef IMEX_TU_NS
#error "define IMEX_TU_NS (the translation unit's namespace) before including the kernels"
#endif
namespace imex {
// The library is built from more than one translation unit, each with its
// own copy of these kernels and device functions: an inline namespace named
// per unit keeps their symbols apart.
inline namespace IMEX_TU_NS {

constexpr double EPS = 2.220446049250313e-16;  // EPSILON(1.0_wp)
constexpr int MAXS = 4;

// Kernel parameter block (passed by value).
struct DevParams {
  int nx, ny, ns, nv, np;
  int64_t pitch;          // elements per row of a plane
  int64_t plane;          // elements per plane (pitch * ny)
  double x0, y0, dx, dy, dx2, dy2, one_by_dx, one_by_dy;
  double eps_sing, eps_sing4, hstep, one_by_h;
  double cfl, max_dt, reconstr_coeff, theta;
  int limiter[10];
  int bcW_flag[8], bcE_flag[8], bcS_flag[8], bcN_flag[8];
  double bcW_val[8], bcE_val[8], bcS_val[8], bcN_val[8];
  int energy_flag, alpha_flag, rheology_flag, rheology_model;
  int slope_correction_flag, curvature_term_flag, radial_source_flag;
  int settling_flag, entrainment_flag, erodible_deposit_flag, topo_change_flag;
  int has_cellinfo, has_release_time, has_exchange;
  double grav, T_ambient, pres, inv_pres, sp_heat_a, sp_gas_const_a, kin_visc_c;
  double rho_a_amb;
  double rho_s[MAXS], inv_rho_s[MAXS], diam_s[MAXS], sp_heat_s[MAXS];
  double mu, xi, friction_factor, maximum_solid_packing;
  double h_source, vel_source, T_source, alphas_source[MAXS], time_param[4];
  double erosion_coeff, erodible_porosity, T_erodible, alphastot_min;
  double erodible_fract[MAXS], rho_c_sub, coeff_porosity;
  int n_ring;             // inlet ring cells (source_cell == 2)
};
// Kernels take DevParams by value (a __grid_constant__ parameter): its
// fields are read from the constant bank, not from global memory.
static_assert(sizeof(DevParams) <= 2048, "DevParams must fit the kernel parameter space");

// cellinfo bits
constexpr uint8_t CI_SRC_MASK = 3;   // source_cell value 0/1/2
constexpr uint8_t CI_E = 4, CI_W = 8, CI_S = 16, CI_N = 32, CI_NODATA = 64;

struct RingCell {            // one inlet ring cell, sorted by linear index
  int64_t idx;               // j + nx*k (0-based)
  double vx[4], vy[4];       // E, W, S, N unit-vector components
};

IMEX_HD double fmin_f(double a, double b) {
  if (isnan(a)) return b;
  if (isnan(b)) return a;
  return (b < a) ? b : a;
}
IMEX_HD double fmax_f(double a, double b) {
  if (isnan(a)) return b;
  if (isnan(b)) return a;
  return (b > a) ? b : a;
}
IMEX_DIV_FN double ddiv(double a, double b) { return a / b; }

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
IMEX_HD void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
IMEX_HD void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}
// The body, inlined where one call site runs in a loop (the settling drag);
// `ipow` below is the called copy.  Two library calls are replaced by exact
// bit operations on their common ranges: frexp of a positive normal x (the
// exponent field and the fraction with the exponent of [1, 2)), and ldexp
// by a power of two whose product stays normal (an exact product).  The top
// seven fraction bits are (m - 1)*128 truncated, read from the bits.
IMEX_HD double ipow_body(double x, double y) {
  if (isnan(x) || isnan(y)) return x + y;
  if (x == 0.0 && y != 0.0) return (y > 0.0) ? 0.0 : __longlong_as_double(0x7ff0000000000000LL);
  if (x < 0.0 && y != 0.0) return __longlong_as_double(0x7ff8000000000000LL);
  if (isinf(x) && y != 0.0) return (y > 0.0) ? x : 0.0;
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  const double LN2_HI = 0x1.62e42fee00000p-1, LN2_LO = 0x1.a39ef35793c76p-33;
  const double LN2_64_HI = 0x1.62e42fee00000p-7, LN2_64_LO = 0x1.a39ef35793c76p-39;
  const double INV_LN2_64 = 0x1.71547652b82fep+6;
  // log x = e*ln2 - log(invc_i) + log1p(r), m*invc_i = 1 + r, |r| < 2^-8
  int e, i;
  double m;
  const long long xb = __double_as_longlong(x);
  const int ef = (int)(xb >> 52);   // x > 0 here: the sign bit is clear
  if (ef > 0) {
    // normal: m = x with the exponent of [1, 2), e the unbiased exponent
    m = __longlong_as_double((xb & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    e = ef - 1023;
    i = (int)((xb >> 45) & 127);
  } else {
    m = frexp(x, &e);               // m in [1/2, 1)
    m = m * 2.0;
    e = e - 1;
    i = (int)((m - 1.0) * 128.0);
  }
  const double r = fma(m, IPOW_INVC[i], -1.0);
  double P = fma(r, 0x1.2492492492492p-3, -0x1.5555555555555p-3);   // 1/7, -1/6
  P = fma(r, P, 0x1.999999999999ap-3);                               // 1/5
  P = fma(r, P, -0x1.0000000000000p-2);                              // -1/4
  P = fma(r, P, 0x1.5555555555555p-2);                               // 1/3
  P = fma(r, P, -0x1.0000000000000p-1);                              // -1/2
  const double l1p = fma(r * r, P, r);
  double a, b, hi, c;
  two_sum((double)e * LN2_HI, IPOW_LOGC_HI[i], a, b);
  two_sum(a, l1p, hi, c);
  double lo = ((b + c) + IPOW_LOGC_LO[i]) + (double)e * LN2_LO;
  // z = y*log x in double-double
  double p, pe;
  two_prod(y, hi, p, pe);
  pe = fma(y, lo, pe);
  double zh, zl;
  two_sum(p, pe, zh, zl);
  if (zh > 709.78) return __longlong_as_double(0x7ff0000000000000LL);
  if (zh < -745.1) return 0.0;
  // exp z = 2^(k/64) exp(rr), |rr| < ln2/128
  const double kf = rint(zh * INV_LN2_64);
  const long long k = (long long)kf;
  const int j = (int)(k & 63);
  const int me = (int)((k - j) / 64);
  double rh, rl;
  two_sum(zh, -(kf * LN2_64_HI), rh, rl);
  const double rr = rh + (rl + fma(-kf, LN2_64_LO, zl));
  double E = fma(rr, 0x1.6c16c16c16c17p-10, 0x1.1111111111111p-7);  // 1/720, 1/120
  E = fma(rr, E, 0x1.5555555555555p-5);                              // 1/24
  E = fma(rr, E, 0x1.5555555555555p-3);                              // 1/6
  E = fma(rr, E, 0x1.0000000000000p-1);                              // 1/2
  const double em1 = fma(rr * rr, E, rr);
  const double th = IPOW_EXP2_HI[j];
  const double v = th + fma(th, em1, IPOW_EXP2_LO[j]);   // in [1, 2]
  if (me >= -1000 && me <= 1000)
    return v * __longlong_as_double((long long)(me + 1023) << 52);
  return ldexp(v, me);
}
IMEX_IPOW_FN double ipow(double x, double y) { return ipow_body(x, y); }

// ------------------------------------------------------------- complex
struct cplx {
  double re, im;
};
IMEX_HD cplx C(double r, double i = 0.0) { return {r, i}; }
IMEX_HD cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
IMEX_HD cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
IMEX_HD cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
IMEX_HD cplx mulr(cplx a, double r) { return {a.re * r, a.im * r}; }
IMEX_HD cplx divr(cplx a, double r) { return {a.re / r, a.im / r}; }
IMEX_HD cplx addr(cplx a, double r) { return {a.re + r, a.im}; }
IMEX_HD cplx subr(cplx a, double r) { return {a.re - r, a.im}; }
IMEX_HD cplx rsub(double r, cplx a) { return {r - a.re, -a.im}; }
IMEX_HD cplx conj(cplx a) { return {a.re, -a.im}; }
// Smith (1962) range-reduced complex division.
IMEX_CPLX_FN cplx operator/(cplx a, cplx b) {
  if (fabs(b.re) < fabs(b.im)) {
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
IMEX_HD cplx rdiv(double r, cplx b) { return C(r, 0.0) / b; }
// Principal square root by the half-angle formulas.
IMEX_CPLX_FN cplx csqrt_(cplx z) {
  if (z.im == 0.0) {
    if (z.re < 0.0) return {0.0, copysign(sqrt(-z.re), z.im)};
    return {fabs(sqrt(z.re)), z.im};
  }
  if (z.re == 0.0) {
    double r = sqrt(0.5 * fabs(z.im));
    return {r, copysign(r, z.im)};
  }
  double d = sqrt(z.re * z.re + z.im * z.im);
  if (z.re > 0.0) {
    double r = sqrt(0.5 * (d + z.re));
    double s = 0.5 * (z.im / r);
    return {r, s};
  } else {
    double s = sqrt(0.5 * (d - z.re));
    double r = fabs(0.5 * (z.im / s));
    return {r, copysign(s, z.im)};
  }
}

// ------------------------------------------------------------- mixt_var
struct Mixt {
  double rho_m, rho_c, red_grav, Ri;
};

template <int NS>
IMEX_HD Mixt mixt_var(const DevParams& P, const double* qpj) {
  constexpr int NV = 4 + NS;
  Mixt m;
  if (qpj[0] <= EPS) {
    m.red_grav = 0.0;
    m.rho_m = P.rho_a_amb;
    m.rho_c = P.rho_a_amb;
    m.Ri = 0.0;
    return m;
  }
  double r_h = qpj[0], r_u = qpj[NV], r_v = qpj[NV + 1], r_T = qpj[3];
  double al[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qpj[4 + i] : qpj[4 + i] / qpj[0];
  double at = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) at += al[i];
  double r_rho_a = P.pres / (P.sp_gas_const_a * r_T);
  m.rho_c = ((((1.0 - 0.0) - at) - 0.0) * r_rho_a + 0.0) / ((1.0 - 0.0) - at);
  double dot = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dot += al[i] * P.rho_s[i];
  m.rho_m = (1.0 - at) * m.rho_c + dot;
  m.red_grav = (m.rho_m - P.rho_a_amb) / m.rho_m * P.grav;
  double vel2 = r_u * r_u + r_v * r_v;
  m.Ri = (vel2 > 0.0) ? fmin_f(1.0e15, m.red_grav * r_h / vel2) : 0.0;
  return m;
}

// eval_sp_heat (gas carrier): returns the carrier specific heat; alphas are
// the volume fractions of mixt_var and inv_rhom = 1/rho_m.
template <int NS>
IMEX_HD double sp_heat_c_of(const DevParams& P, const double* qpj, double rho_m) {
  double al[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qpj[4 + i] : qpj[4 + i] / qpj[0];
  double inv_rhom = 1.0 / rho_m;
  double xs[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) xs[i] = al[i] * P.rho_s[i] * inv_rhom;
  double sxs = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sxs += xs[i];
  double xc = 1.0 - sxs;
  if (xc > EPS) return ((xc - 0.0) * P.sp_heat_a + 0.0) / xc;
  return P.sp_heat_a;
}

// ----------------------------------------------------------- qc_to_qp
// r_phys_var + qc_to_qp; also returns red_grav through the out pointer.
template <int NS>
IMEX_QCQP_FN void qc_to_qp(const DevParams& P, const double* qc, double* qp,
                         double* p_dyn = nullptr) {
  constexpr int NV = 4 + NS;
  if (!(qc[0] > EPS)) {
    qp[0] = 0.0;
    qp[1] = 0.0 * 0.0;
    qp[2] = 0.0 * 0.0;
    qp[3] = P.T_ambient;
#pragma unroll
    for (int i = 0; i < NS; ++i) qp[4 + i] = P.alpha_flag ? 0.0 : 0.0 * 0.0;
    qp[NV] = 0.0;
    qp[NV + 1] = 0.0;
    if (p_dyn) *p_dyn = 0.0;
    return;
  }
  double inv_qj1 = 1.0 / qc[0];
  double xs[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) xs[i] = qc[4 + i] * inv_qj1;
  double sq = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sq += qc[4 + i];
  if (sq == qc[0]) {
    double sx = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) sx += xs[i];
#pragma unroll
    for (int i = 0; i < NS; ++i) xs[i] = xs[i] / sx;
  }
  double xs_tot = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) xs_tot += xs[i];
  double xc = 1.0 - xs_tot;
  double cpc_by_xc = ((xc - 0.0) * P.sp_heat_a + 0.0);
  double dot = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dot += xs[i] * P.sp_heat_s[i];
  double cpm = dot + cpc_by_xc;
  double T;
  if (qc[0] > P.eps_sing) {
    if (P.energy_flag)
      T = (qc[3] - 0.5 * (qc[1] * qc[1] + qc[2] * qc[2]) * inv_qj1) / (qc[0] * cpm);
    else
      T = qc[3] / (qc[0] * cpm);
    if (T <= 0.0) T = P.T_ambient;
  } else {
    T = P.T_ambient;
  }
  double sgc = (xc > EPS) ? ((xc - 0.0) * P.sp_gas_const_a + 0.0) / xc : P.sp_gas_const_a;
  double inv_rho_c = sgc * T * P.inv_pres;
  double dot2 = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dot2 += xs[i] * P.inv_rho_s[i];
  double inv_rhom = dot2 + xc * inv_rho_c;
  double rho_m = 1.0 / inv_rhom;
  double h = qc[0] * inv_rhom;
  double u, v;
  if (qc[0] > P.eps_sing) {
    u = qc[1] * inv_qj1;
    v = qc[2] * inv_qj1;
  } else {
    double q1 = qc[0];
    double q14 = (q1 * q1) * (q1 * q1);
    double den = sqrt(q14 + P.eps_sing4);
    u = 1.4142135623730951 * qc[0] * qc[1] / den;
    v = 1.4142135623730951 * qc[0] * qc[2] / den;
  }
  qp[0] = h;
  qp[1] = h * u;
  qp[2] = h * v;
  qp[3] = T;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    double al = xs[i] * rho_m * P.inv_rho_s[i];
    qp[4 + i] = P.alpha_flag ? al : al * h;
  }
  qp[NV] = u;
  qp[NV + 1] = v;
  if (p_dyn) *p_dyn = 0.5 * rho_m * (u * u + v * v);  // r_phys_var's p_dyn
}

// The driver's convention for a cell's physical state: qc_to_qp when q1 > 0,
// otherwise zeros with T = T_ambient (src/solver_2d.f90:902-911).
template <int NS>
IMEX_HD void cell_qp(const DevParams& P, const double* qc, double* qp) {
  constexpr int NP = 6 + NS;
  if (qc[0] > 0.0) {
    qc_to_qp<NS>(P, qc, qp);
  } else {
#pragma unroll
    for (int i = 0; i < NP; ++i) qp[i] = 0.0;
    qp[3] = P.T_ambient;
  }
}

// ----------------------------------------------------------- qp_to_qc
template <int NS>
IMEX_QCQP_FN void qp_to_qc(const DevParams& P, const double* qp, double* qc) {
  constexpr int NV = 4 + NS;
  double r_h = qp[0];
  if (!(r_h > EPS)) {
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = 0.0;
    return;
  }
  double r_hu = qp[1], r_hv = qp[2], r_u = qp[NV], r_v = qp[NV + 1], r_T = qp[3];
  double al[NS], alr[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qp[4 + i] : qp[4 + i] / qp[0];
  double at = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) at += al[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) alr[i] = al[i] * P.rho_s[i];
  double r_rho_a = P.pres / (P.sp_gas_const_a * r_T);
  double r_rho_c = ((((1.0 - 0.0) - at) - 0.0) * r_rho_a + 0.0) / ((1.0 - 0.0) - at);
  double r_alphac = 1.0 - at;
  double sar = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sar += alr[i];
  double r_rho_m = r_alphac * r_rho_c + sar;
  double r_inv_rhom = 1.0 / r_rho_m;
  double xs[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) xs[i] = alr[i] * r_inv_rhom;
  double r_xc = r_alphac * r_rho_c * r_inv_rhom;
  double cpc = (r_xc > EPS) ? ((r_xc - 0.0) * P.sp_heat_a + 0.0) / r_xc : P.sp_heat_a;
  double dot = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dot += xs[i] * P.sp_heat_s[i];
  double cpm = dot + r_xc * cpc;
  qc[0] = r_rho_m * r_h;
  qc[1] = r_rho_m * r_hu;
  qc[2] = r_rho_m * r_hv;
  if (P.energy_flag)
    qc[3] = (r_h > 0.0) ? r_h * r_rho_m * (cpm * r_T + 0.5 * (r_u * r_u + r_v * r_v)) : 0.0;
  else
    qc[3] = r_h * r_rho_m * cpm * r_T;
#pragma unroll
  for (int i = 0; i < NS; ++i) qc[4 + i] = xs[i] * qc[0];
}

// qp_to_qc and mixt_var of one face state in one pass: the volume fractions,
// the carrier and the mixture densities, which both compute with the same
// operations in the same order, are computed once (a state whose h is not
// above EPS goes through mixt_var itself, so that NaN and dry states keep
// both functions' own branches).
template <int NS>
IMEX_QCQP_FN void face_qc_mixt(const DevParams& P, const double* qp, double* qc, Mixt& m) {
  constexpr int NV = 4 + NS;
  double r_h = qp[0];
  if (!(r_h > EPS)) {
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = 0.0;
    m = mixt_var<NS>(P, qp);
    return;
  }
  double r_hu = qp[1], r_hv = qp[2], r_u = qp[NV], r_v = qp[NV + 1], r_T = qp[3];
  double al[NS], alr[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qp[4 + i] : qp[4 + i] / qp[0];
  double at = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) at += al[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) alr[i] = al[i] * P.rho_s[i];
  double r_rho_a = P.pres / (P.sp_gas_const_a * r_T);
  double r_rho_c = ((((1.0 - 0.0) - at) - 0.0) * r_rho_a + 0.0) / ((1.0 - 0.0) - at);
  double r_alphac = 1.0 - at;
  double sar = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sar += alr[i];
  double r_rho_m = r_alphac * r_rho_c + sar;
  // mixt_var: rho_m = (1 - at)*rho_c + SUM(al*rho_s), the same operations
  m.rho_c = r_rho_c;
  m.rho_m = r_rho_m;
  m.red_grav = (r_rho_m - P.rho_a_amb) / r_rho_m * P.grav;
  const double vel2 = r_u * r_u + r_v * r_v;
  m.Ri = (vel2 > 0.0) ? fmin_f(1.0e15, m.red_grav * r_h / vel2) : 0.0;
  double r_inv_rhom = 1.0 / r_rho_m;
  double xs[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) xs[i] = alr[i] * r_inv_rhom;
  double r_xc = r_alphac * r_rho_c * r_inv_rhom;
  double cpc = (r_xc > EPS) ? ((r_xc - 0.0) * P.sp_heat_a + 0.0) / r_xc : P.sp_heat_a;
  double dot = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dot += xs[i] * P.sp_heat_s[i];
  double cpm = dot + r_xc * cpc;
  qc[0] = r_rho_m * r_h;
  qc[1] = r_rho_m * r_hu;
  qc[2] = r_rho_m * r_hv;
  if (P.energy_flag)
    qc[3] = (r_h > 0.0) ? r_h * r_rho_m * (cpm * r_T + 0.5 * (r_u * r_u + r_v * r_v)) : 0.0;
  else
    qc[3] = r_h * r_rho_m * cpm * r_T;
#pragma unroll
  for (int i = 0; i < NS; ++i) qc[4 + i] = xs[i] * qc[0];
}

// ----------------------------------------------------------- limiters
// minmod/maxmod (src/geometry_2d.f90:1555-1676).  The signs a/|a|, b/|b| of
// finite nonzero operands are exactly +-1, so 0.5*(sa + sb) is exactly +-1
// (same signs) or +0 (opposite signs, 1 + -1 = +0): the result is then
// +-min (+-max) or +0 without the two divisions.  Infinite or NaN operands
// take the reference's expression.
IMEX_HD double minmod(double a, double b) {
  if (fmin_f(fabs(a), fabs(b)) <= 0.0) return 0.0;
  if (isfinite(a) && isfinite(b)) {
    const double m = fmin_f(fabs(a), fabs(b));
    return ((a > 0.0) == (b > 0.0)) ? ((a > 0.0) ? m : -m) : 0.0;
  }
  double sa = a / fabs(a), sb = b / fabs(b);
  return 0.5 * (sa + sb) * fmin_f(fabs(a), fabs(b));
}
IMEX_HD double maxmod(double a, double b) {
  if (fabs(a * b) <= 0.0) return 0.0;
  if (isfinite(a) && isfinite(b)) {
    const double m = fmax_f(fabs(a), fabs(b));
    return ((a > 0.0) == (b > 0.0)) ? ((a > 0.0) ? m : -m) : 0.0;
  }
  double sa = a / fabs(a), sb = b / fabs(b);
  return 0.5 * (sa + sb) * fmax_f(fabs(a), fabs(b));
}
// limit() with limiter 1 (minmod) on equally spaced centres, z3 - z2 ==
// z2 - z1 == dz > 0.  For finite differences d3, d1 of one sign the two
// slopes are d3/dz and d1/dz; rounded division by a positive dz is monotone,
// so the smaller slope magnitude is the rounded quotient of the smaller
// difference: one division instead of two.  Where a quotient could overflow
// (an infinite slope makes minmod NaN) or a difference is not finite,
// limit() itself is used.
IMEX_HD double minmod_uniform(double v1, double v2, double v3, double dz, double z1, double z2,
                              double z3, double theta);
IMEX_LIMIT_FN double limit(double v1, double v2, double v3, double z1, double z2, double z3,
                        int lim, double theta) {
  if (lim == 1) {
    // minmod(a,b) with a=(v3-v2)/(z3-z2), b=(v2-v1)/(z2-z1), z increasing:
    // when one difference is zero, or the two are finite, of opposite sign
    // and their quotients cannot overflow (an infinite quotient makes
    // minmod NaN), the result is exactly 0 and the quotients are not needed.
    double d3 = v3 - v2, d1 = v2 - v1;
    if (isfinite(d3) && isfinite(d1) && (z3 > z2) && (z2 > z1)) {
      if (d3 == 0.0 || d1 == 0.0) return 0.0;
      if ((d3 > 0.0) != (d1 > 0.0) && fmax_f(fabs(d3), fabs(d1)) <= 1e290 &&
          z3 - z2 >= 1e-10 && z2 - z1 >= 1e-10)
        return 0.0;
    }
    double a = d3 / (z3 - z2);
    double b = d1 / (z2 - z1);
    return minmod(a, b);
  }
  double a = (v3 - v2) / (z3 - z2);
  double b = (v2 - v1) / (z2 - z1);
  double c = (v3 - v1) / (z3 - z1);
  switch (lim) {
    case 0: return 0.0;
    case 2: return maxmod(minmod(a, 2.0 * b), minmod(2.0 * a, b));
    case 3: return minmod(c, theta * minmod(a, b));
    case 4: return minmod(c, 2.0 * minmod(a, b));
    case 5: return c;
    case 6: return a;
    case 7: return b;
  }
  return 0.0;
}
IMEX_HD double minmod_uniform(double v1, double v2, double v3, double dz, double z1, double z2,
                              double z3, double theta) {
  const double d3 = v3 - v2, d1 = v2 - v1;
  if (isfinite(d3) && isfinite(d1)) {
    if (d3 == 0.0 || d1 == 0.0) return 0.0;
    const double a3 = fabs(d3), a1 = fabs(d1);
    if (fmax_f(a3, a1) <= 1e290 && dz >= 1e-10) {
      if ((d3 > 0.0) != (d1 > 0.0)) return 0.0;
      const double q = fmin_f(a3, a1) / dz;
      if (q <= 0.0) return 0.0;
      return (d3 > 0.0) ? q : -q;
    }
  }
  return limit(v1, v2, v3, z1, z2, z3, 1, theta);
}

// ------------------------------------------------------ source boundary
template <int NS>
IMEX_HD void eval_source_bdry(const DevParams& P, double time, double vx, double vy,
                              double* sb) {
  constexpr int NV = 4 + NS;
  const double* tp = P.time_param;
  if (time >= tp[3]) {
    sb[0] = 0.0;
    sb[1] = 0.0;
    sb[2] = 0.0;
    sb[3] = P.T_source;
#pragma unroll
    for (int i = 0; i < NS; ++i) sb[4 + i] = 0.0;
    sb[NV] = 0.0;
    sb[NV + 1] = 0.0;
    return;
  }
  double t_rem = fmod(time, tp[0]);
  double t_coeff = 0.0;
  const double pi_g = 3.141592653589793;
  if (tp[2] == 0.0) {
    if (t_rem <= tp[1]) t_coeff = 1.0;
  } else {
    if (t_rem < tp[2])
      t_coeff = 0.5 * (1.0 - cos(pi_g * t_rem / tp[2]));
    else if (t_rem <= (tp[1] - tp[2]))
      t_coeff = 1.0;
    else if (t_rem <= tp[1])
      t_coeff = 0.5 * (1.0 + cos(pi_g * ((t_rem - tp[1]) / tp[2] + 1.0)));
  }
  double tc15 = ipow(t_coeff, 1.5), tc05 = ipow(t_coeff, 0.5);
  sb[0] = t_coeff * P.h_source;
  sb[1] = tc15 * P.h_source * P.vel_source * vx;
  sb[2] = tc15 * P.h_source * P.vel_source * vy;
  sb[3] = P.T_source;
#pragma unroll
  for (int i = 0; i < NS; ++i)
    sb[4 + i] = P.alpha_flag ? P.alphas_source[i] : t_coeff * P.h_source * P.alphas_source[i];
  sb[NV] = tc05 * P.vel_source * vx;
  sb[NV + 1] = tc05 * P.vel_source * vy;
}

// --------------------------------------------------- speeds and fluxes
// eval_local_speeds_x / _y; dir 1 = x, 2 = y.
template <int NS>
IMEX_HD void local_speeds(const DevParams& P, const double* qpj, const Mixt& m, double gcf,
                          int dir, double& vmin, double& vmax) {
  constexpr int NV = 4 + NS;
  double r_h = qpj[0];
  double vel = (dir == 1) ? qpj[NV] : qpj[NV + 1];
  if (m.red_grav * r_h < 0.0) {
    vmin = vel;
    vmax = vel;
  } else {
    double c = (dir == 1) ? sqrt(m.red_grav * r_h * gcf) : sqrt(gcf * m.red_grav * r_h);
    vmin = vel - c;
    vmax = vel + c;
  }
}

template <int NS>
IMEX_HD void eval_fluxes(const DevParams& P, const double* qcj, const double* qpj,
                         const Mixt& m, double gcf, int dir, double* flux) {
  constexpr int NV = 4 + NS;
  if (qpj[0] > EPS) {
    double r_h = qpj[0], r_u = qpj[NV], r_v = qpj[NV + 1];
    double pres_term = 0.5 * m.rho_m * gcf * m.red_grav * (r_h * r_h);
    double vel = (dir == 1) ? r_u : r_v;
    flux[0] = vel * qcj[0];
    if (dir == 1) {
      flux[1] = r_u * qcj[1] + pres_term;
      flux[2] = r_u * qcj[2];
    } else {
      flux[1] = r_v * qcj[1];
      flux[2] = r_v * qcj[2] + pres_term;
    }
    flux[3] = P.energy_flag ? vel * (qcj[3] + pres_term) : vel * qcj[3];
#pragma unroll
    for (int i = 0; i < NS; ++i) flux[4 + i] = vel * qcj[4 + i];
    if (flux[0] > 0.0) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < NS; ++i) s += flux[4 + i];
      if (s / flux[0] > 1.0) {
#pragma unroll
        for (int i = 0; i < NS; ++i) flux[4 + i] = flux[4 + i] / s * flux[0];
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < NV; ++i) flux[i] = 0.0;
  }
}

// eval_expl_terms without the bottom radial source
template <int NS>
IMEX_HD void eval_expl_terms(const DevParams& P, double bx, double by, double bxx, double bxy,
                             double byy, double gcf, double dgc, const double* qpj,
                             double* expl) {
  constexpr int NV = 4 + NS;
#pragma unroll
  for (int i = 0; i < NV; ++i) expl[i] = 0.0;
  if (qpj[0] <= EPS) return;
  double r_h = qpj[0], r_u = qpj[NV], r_v = qpj[NV + 1];
  Mixt m = mixt_var<NS>(P, qpj);
  double centr = 0.0;
  if (P.curvature_term_flag) centr = bxx * (r_u * r_u) + 2.0 * bxy * r_u * r_v + byy * (r_v * r_v);
  double tg = m.red_grav + centr;
  expl[1] = -(gcf * m.rho_m * tg * r_h * bx) + 0.5 * m.rho_m * m.red_grav * (r_h * r_h) * dgc;
  expl[2] = -(gcf * m.rho_m * tg * r_h * by) + 0.5 * m.rho_m * m.red_grav * (r_h * r_h) * dgc;
  expl[3] = P.energy_flag ? expl[1] * r_u + expl[2] * r_v : 0.0;
}

// ------------------------------------------------ implicit terms (real)
// eval_implicit_terms for real input; rows other than 2,3 are zero.  The
// reference evaluates this case through its complex routine with zero
// imaginary parts (src/constitutive_2d.f90:3435-3441).  While every operand
// is finite those imaginary parts stay zero and the real parts are exactly
// this real-arithmetic sequence; once an operand is infinite or NaN, products
// with the zero imaginary parts turn into NaN and reach the real parts.  So
// the real sequence runs while all its values are finite, and any non-finite
// value sends the evaluation to the complex routine (implicit_terms_rc).
template <int NS>
struct CPrefix;

template <int NS>
IMEX_RC_FN void implicit_terms_rc(const DevParams& P, double bx, double by, const double* q,
                                  double& nh2, double& nh3);

template <int NS>
IMEX_HD void implicit_terms_r(const DevParams& P, double bx, double by, const double* q,
                              double& nh2, double& nh3) {
  nh2 = 0.0;
  nh3 = 0.0;
  if (!P.rheology_flag) return;
  bool fin = true;
  // c_phys_var (real parts)
  double rho_m, u, v;
  if (q[0] > EPS) {
#pragma unroll
    for (int i = 0; i < 4 + NS; ++i) fin &= isfinite(q[i]);
    double inv = ddiv(1.0, q[0]);
    double xs[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) xs[i] = q[4 + i] * inv;
    double xs_tot = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) xs_tot = xs_tot + xs[i];
    double xc = 1.0 - xs_tot;
    double spc = ddiv(((xc - 0.0) * P.sp_heat_a) + 0.0, xc);
    double dot = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) dot = dot + xs[i] * P.sp_heat_s[i];
    double spm = dot + xc * spc;
    fin &= isfinite(inv) & isfinite(xs_tot) & isfinite(spc) & isfinite(spm);
    double T;
    if (q[0] > P.eps_sing) {
      double T_num, T_den;
      if (P.energy_flag) {
        double ke = ((q[1] * q[1] + q[2] * q[2]) * 0.5) * inv;
        fin &= isfinite(ke);
        T_num = q[3] - ke;
      } else {
        T_num = q[3];
      }
      T_den = q[0] * spm;
      T = ddiv(T_num, T_den);
      fin &= isfinite(T_num) & isfinite(T_den) & isfinite(T);
      if (T <= 0.0) T = P.T_ambient;
    } else {
      T = P.T_ambient;
    }
    double sgc = ddiv(((xc - 0.0) * P.sp_gas_const_a) + 0.0, xc);
    double irc = (sgc * T) * P.inv_pres;
    double dot2 = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) dot2 = dot2 + xs[i] * P.inv_rho_s[i];
    double irm = dot2 + xc * irc;
    rho_m = ddiv(1.0, irm);
    fin &= isfinite(sgc) & isfinite(irc) & isfinite(irm) & isfinite(rho_m);
    if (q[0] > P.eps_sing) {
      u = q[1] * inv;
      v = q[2] * inv;
    } else {
      double q12 = q[0] * q[0];
      double den = sqrt(q12 * q12 + P.eps_sing4);
      u = ddiv((q[0] * 1.4142135623730951) * q[1], den);
      v = ddiv((q[0] * 1.4142135623730951) * q[2], den);
      fin &= isfinite(den);
    }
  } else {
    rho_m = P.rho_a_amb;
    u = 0.0;
    v = 0.0;
  }
  double red_grav = ddiv(rho_m - P.rho_a_amb, rho_m) * P.grav;
  double w = P.slope_correction_flag ? u * bx + v * by : 0.0;
  double mv2 = u * u + v * v + w * w;
  double mv = sqrt(mv2);
  fin &= isfinite(u) & isfinite(v) & isfinite(red_grav) & isfinite(w) & isfinite(mv2);
  if (P.rheology_model == 1) {
    if (mv != 0.0) {
      double ts = ddiv(rho_m * red_grav, P.xi) * mv2;
      double ur = ddiv(u, mv), vr = ddiv(v, mv);
      nh2 = 0.0 - ts * ur;
      nh3 = 0.0 - ts * vr;
      fin &= isfinite(ts) & isfinite(ur) & isfinite(vr) & isfinite(nh2) & isfinite(nh3);
    }
  } else if (P.rheology_model == 6) {
    if (mv != 0.0) {
      double mvh = sqrt(u * u + v * v);
      double a2 = rho_m * ddiv(u, mvh), a3 = rho_m * ddiv(v, mvh);
      nh2 = 0.0 - (a2 * P.friction_factor) * mv2;
      nh3 = 0.0 - (a3 * P.friction_factor) * mv2;
      fin &= isfinite(mvh) & isfinite(a2) & isfinite(a3) & isfinite(nh2) & isfinite(nh3);
    }
  }
  if (!fin) implicit_terms_rc<NS>(P, bx, by, q, nh2, nh3);
}

// --------------------------------------------- implicit terms (complex)
// The complex-step Jacobian perturbs only q(2) or q(3), so every mixture
// quantity built from q(1) and the solid loads alone (1/q1, mass fractions,
// c_p, gas constant and 1/rho of the mixture's solid part) is the same for
// both columns.  It is evaluated once per Newton iteration (CPrefix) and
// shared; the operations, and so the values, are those of c_phys_var.
template <int NS>
struct CPrefix {
  cplx inv, xc, spm, sgc, dot2;
};

template <int NS>
IMEX_FLAT void implicit_prefix_c(const DevParams& P, const cplx* q, CPrefix<NS>& pre) {
  if (!P.rheology_flag || !(q[0].re > EPS)) return;
  cplx inv = rdiv(1.0, q[0]);
  cplx xs[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) xs[i] = q[4 + i] * inv;
  cplx xs_tot = C(0.0);
#pragma unroll
  for (int i = 0; i < NS; ++i) xs_tot = xs_tot + xs[i];
  cplx xc = rsub(1.0, xs_tot);
  cplx spc = (mulr(xc - C(0.0), P.sp_heat_a) + C(0.0)) / xc;
  cplx dot = C(0.0);
#pragma unroll
  for (int i = 0; i < NS; ++i) dot = dot + mulr(conj(xs[i]), P.sp_heat_s[i]);
  pre.spm = dot + xc * spc;
  pre.sgc = (mulr(xc - C(0.0), P.sp_gas_const_a) + C(0.0)) / xc;
  cplx dot2 = C(0.0);
#pragma unroll
  for (int i = 0; i < NS; ++i) dot2 = dot2 + conj(xs[i]) * C(P.inv_rho_s[i], 0.0);
  pre.dot2 = dot2;
  pre.inv = inv;
  pre.xc = xc;
}

template <int NS>
IMEX_FLAT void implicit_terms_c(const DevParams& P, double bx, double by, const cplx* q,
                                 const CPrefix<NS>& pre, cplx& nh2, cplx& nh3) {
  nh2 = C(0.0, 0.0);
  nh3 = C(0.0, 0.0);
  if (!P.rheology_flag) return;
  cplx rho_m, u, v;
  if (q[0].re > EPS) {
    const cplx inv = pre.inv, xc = pre.xc, spm = pre.spm;
    cplx T;
    if (q[0].re > P.eps_sing) {
      if (P.energy_flag)
        T = (q[3] - mulr(q[1] * q[1] + q[2] * q[2], 0.5) * inv) / (q[0] * spm);
      else
        T = q[3] / (q[0] * spm);
      if (T.re <= 0.0) T = C(P.T_ambient);
    } else {
      T = C(P.T_ambient);
    }
    cplx irc = mulr(pre.sgc * T, P.inv_pres);
    cplx irm = pre.dot2 + xc * irc;
    rho_m = rdiv(1.0, irm);
    if (q[0].re > P.eps_sing) {
      u = q[1] * inv;
      v = q[2] * inv;
    } else {
      cplx q12 = q[0] * q[0];
      cplx den = csqrt_(addr(q12 * q12, P.eps_sing4));
      u = (mulr(q[0], 1.4142135623730951) * q[1]) / den;
      v = (mulr(q[0], 1.4142135623730951) * q[2]) / den;
    }
  } else {
    rho_m = C(P.rho_a_amb);
    u = C(0.0);
    v = C(0.0);
  }
  cplx red_grav = mulr(subr(rho_m, P.rho_a_amb) / rho_m, P.grav);
  cplx w = P.slope_correction_flag ? mulr(u, bx) + mulr(v, by) : C(0.0, 0.0);
  cplx mv2 = u * u + v * v + w * w;
  cplx mv = csqrt_(mv2);
  if (P.rheology_model == 1) {
    if (mv.re != 0.0) {
      cplx ts = divr(rho_m * red_grav, P.xi) * mv2;
      nh2 = C(0.0, 0.0) - ts * (u / mv);
      nh3 = C(0.0, 0.0) - ts * (v / mv);
    }
  } else if (P.rheology_model == 6) {
    if (mv.re != 0.0) {
      cplx mvh = csqrt_(u * u + v * v);
      nh2 = C(0.0, 0.0) - mulr(rho_m * (u / mvh), P.friction_factor) * mv2;
      nh3 = C(0.0, 0.0) - mulr(rho_m * (v / mvh), P.friction_factor) * mv2;
    }
  }
}

// The reference's real evaluation: complex routine, zero imaginary parts.
template <int NS>
IMEX_RC_FN void implicit_terms_rc(const DevParams& P, double bx, double by, const double* q,
                                  double& nh2, double& nh3) {
  cplx qc[4 + NS];
#pragma unroll
  for (int i = 0; i < 4 + NS; ++i) qc[i] = C(q[i], 0.0);
  CPrefix<NS> pre;
  implicit_prefix_c<NS>(P, qc, pre);
  cplx c2, c3;
  implicit_terms_c<NS>(P, bx, by, qc, pre, c2, c3);
  nh2 = c2.re;
  nh3 = c3.re;
}

template <int NS>
IMEX_HD void semi_impl_terms(const DevParams& P, double bx, double by, double bxx,
                             double bxy, double byy, double gcf, const double* qpj,
                             double& si2, double& si3) {
  constexpr int NV = 4 + NS;
  si2 = 0.0;
  si3 = 0.0;
  if (!P.rheology_flag) return;
  double r_h = qpj[0], r_u = qpj[NV], r_v = qpj[NV + 1];
  Mixt m = mixt_var<NS>(P, qpj);
  double r_w = P.slope_correction_flag ? (r_u * bx + r_v * by) : 0.0;
  double mod_vel = sqrt(r_u * r_u + r_v * r_v + r_w * r_w);
  if (P.rheology_model == 1 && mod_vel > 0.0) {
    double centr = 0.0;
    if (P.curvature_term_flag) centr = bxx * (r_u * r_u) + 2.0 * bxy * r_u * r_v + byy * (r_v * r_v);
    double temp = P.mu * m.rho_m * (m.red_grav + centr) * r_h * sqrt(gcf);
    temp = fmax_f(0.0, temp);
    temp = fmax_f(0.0, temp);
    si2 = 0.0 - temp * r_u / mod_vel;
    si3 = 0.0 - temp * r_v / mod_vel;
  }
}

// ------------------------------------------------------ mass exchange
// (d / s < t) for the rounded quotient, without the division where the
// answer is certain.  With s and t positive and s*t normal, the products
// below are within 2^-52 relative of s*t*(1 -+ 2^-40): below the lower one,
// d/s < t*(1 - 2^-41), whose rounding is already below t (t's half ulp is
// t*2^-53); above the upper one, d/s > t*(1 + 2^-41) rounds above t.
// Rounding is monotone, so the quotient compares as the bounds do.  Between
// them, and outside the ranges, the quotient is taken.
IMEX_HD bool rel_change_below(double d, double s, double t) {
  if (s > 1e-200 && s < 1e200 && d <= 1e300) {
    const double st = s * t;
    if (d < st * (1.0 - 0x1p-40)) return true;
    if (d > st * (1.0 + 0x1p-40)) return false;
  }
  return d / s < t;
}

IMEX_SETTLE_FN double settling_velocity(const DevParams& P, double diam, double rhos, double rhoc,
                                 double ikv) {
  double inv_sqrt_C_D = 1.0;
  if (rhos <= rhoc) return 0.0;
  double const_part = sqrt(0.75 * (rhos / rhoc - 1.0) * diam * P.grav);
  double sv = const_part * inv_sqrt_C_D;
  double Rey = diam * sv * ikv;
  if (Rey <= 1000.0) {
    for (int i = 1; i <= 20; ++i) {
      double sv_old = sv;
      inv_sqrt_C_D = sqrt(Rey / (24.0 * (1.0 + 0.15 * ipow_body(Rey, 0.687))));
      sv = const_part * inv_sqrt_C_D;
      if (rel_change_below(fabs(sv_old - sv), sv_old, 1.0e-6)) return sv;
      Rey = diam * sv * ikv;
    }
  }
  return sv;
}

}  // namespace IMEX_TU_NS
}  // namespace imex
