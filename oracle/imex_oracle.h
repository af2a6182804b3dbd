/*
 * imex_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU oracle: a line-by-line C++ restatement of the reference
 * IMEX_SfloW2D time step (src/solver_2d.f90, src/constitutive_2d.f90,
 * src/geometry_2d.f90 limiters).  It exists to check the CUDA path; nothing
 * in the product links or calls it.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm load it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * this image, so the oracle could not be checked against the reference
 * binary; the reference ships no golden outputs (TESTS/run_tests.sh only
 * checks that output files exist).  Parity is therefore UNPINNED against the
 * reference build; the oracle is pinned by analytic known-answer tests
 * (lake at rest, mass conservation, symmetry, closed-form Voellmy relaxation,
 * complex-step vs finite differences) in tests/test_oracle_*.py.
 */
#ifndef IMEX_ORACLE_H
#define IMEX_ORACLE_H

#include <stdint.h>
#include "../include/imex_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleCtx OracleCtx;

OracleCtx* oracle_create(const ImexParams* p, const ImexStatic* s);
void oracle_destroy(OracleCtx* o);
/* q in Fortran layout; also runs check_solve(.TRUE.) and the initial qp sweep
 * of the driver (src/IMEX_SfloW2D.f90:237-301). */
void oracle_set_state(OracleCtx* o, const double* q, double t);
void oracle_get_state(OracleCtx* o, double* q, double* qp);
void oracle_get_exchange(OracleCtx* o, double* erodible, double* deposit,
                         double* erosion, double* B_cent);
int64_t oracle_check_solve(OracleCtx* o, double t, int solve_all);
double oracle_timestep(OracleCtx* o);
/* returns an error mask (IMEX_ERRBIT bits) of the reference's checks */
uint32_t oracle_rk_step(OracleCtx* o, double t, double dt);
uint32_t oracle_erosion_deposition(OracleCtx* o, double dt);
void oracle_post_step(OracleCtx* o);
void oracle_get_masks(OracleCtx* o, int8_t* m, int8_t* mx, int8_t* my);
void oracle_set_clock(OracleCtx* o, double t, double dt0, double t_end, double t_output);
/* n passes of the driver loop body; returns OR of error masks */
uint32_t oracle_advance(OracleCtx* o, int n_steps, double* t);
void oracle_stats(OracleCtx* o, ImexStats* st);
/* reads of a neighbour's face or stage values that were written in an
 * earlier step and belong to a cell that was wet then (the reference's
 * arrays are never cleared between steps) */
int64_t oracle_stale_wet_reads(OracleCtx* o);
/* Changes of SUM(q(1,:,:)) since set_state by cause (multiply by dx*dy for
 * mass): out[0] the fluxes through faces with exactly one solved side
 * (domain border and inlet ring), computed from the face fluxes alone, so
 * that SUM(q1) - SUM(q1 at set_state) - out[0] - out[1] - out[2] vanishes to
 * round-off only if every interior face flux enters both of its cells;
 * out[1] the assembly fixes (small negative h zeroed, no-data cells);
 * out[2] the erosion/deposition update; out[3] out[0] of the last step. */
void oracle_mass_budget(OracleCtx* o, double* out);
void oracle_set_threads(int n);
int oracle_max_threads(void);

/* Point functions exposed for unit tests (qc in, qp out; sizes n_vars / n_vars+2). */
void oracle_qc_to_qp(OracleCtx* o, const double* qc, double* qp);
void oracle_qp_to_qc(OracleCtx* o, const double* qp, double* qc);
/* nh(1:n_vars) from eval_implicit_terms with complex input (re, im arrays) */
void oracle_implicit_terms(OracleCtx* o, const double* q_re, const double* q_im,
                           double* nh_re, double* nh_im);
/* one solve_rk_step on a single cell: qj in/out, returns nl_iter at exit */
int oracle_solve_rk_step(OracleCtx* o, double* qj, const double* qj_old,
                         const double* rj_not_impl, double bprime_x,
                         double bprime_y, double dt, double a_diag);
/* mixt_var (Ri, rho_m, rho_c, red_grav) of one physical state */
void oracle_mixt_var(OracleCtx* o, const double* qp, double* out /* 4 */);
/* eval_local_speeds_x (dir 1) / _y (dir 2): out = (vel_min, vel_max) */
void oracle_local_speeds(OracleCtx* o, const double* qp, double gcf, int dir, double* out);
void oracle_eval_fluxes(OracleCtx* o, const double* qc, const double* qp, double gcf, int dir,
                        double* flux);
/* one KT interface from its two face states (speeds, fluxes, average_KT,
 * solid-flux cap, zero-velocity rule); speeds (may be NULL) = (a-, a+) */
void oracle_kt_interface(OracleCtx* o, const double* qcL, const double* qpL, const double* qcR,
                         const double* qpR, double gcf, int dir, double* H, double* speeds);
double oracle_ipow(double x, double y);
// element-wise over n values (OpenMP): x**y, and settling_velocity with gravity grav
void oracle_ipow_n(long long n, const double* x, const double* y, double* out);
void oracle_limit_n(long long n, const double* v1, const double* v2, const double* v3,
                    const double* z1, const double* z2, const double* z3, int limiter,
                    double theta, double* out);
void oracle_settling_velocity_n(long long n, const double* diam, const double* rhos,
                                const double* rhoc, const double* ikv, double grav,
                                double* out);
double oracle_limit(double v1, double v2, double v3, double z1, double z2,
                    double z3, int limiter, double theta);

#ifdef __cplusplus
}
#endif

#endif
