/*
 * imex_gpu.h -- C ABI of the B200 (sm_100a) IMEX_SfloW2D time step.
 *
 * The reference (demichie/IMEX_SfloW2D_v2, Fortran 90 + OpenMP) has no FFI:
 * its driver calls argument-less module routines that communicate through
 * module globals.  This header is the drop-in boundary for those calls.  Each
 * entry point names the reference routine it replaces:
 *
 *   imex_gpu_check_solve          <- check_solve(solve_all)      src/solver_2d.f90:666-857
 *   imex_gpu_timestep             <- timestep                    src/solver_2d.f90:872-1005
 *   imex_gpu_rk_step              <- imex_RK_solver              src/solver_2d.f90:1021-1632
 *   imex_gpu_erosion_deposition   <- update_erosion_deposition_cell(dt)
 *                                                                src/solver_2d.f90:2380-2595
 *   imex_gpu_set_state/get_state  <- the module arrays q, qp     src/solver_2d.f90:68,157
 *   imex_gpu_advance              <- one pass of the driver loop src/IMEX_SfloW2D.f90:337-389
 *   imex_gpu_advance_host         <- the same pass with q held on the host
 *                                    (check_solve, timestep, dt clipping, imex_RK_solver,
 *                                     update_erosion_deposition_cell, t = t + dt)
 *
 * All functions return an int status (IMEX_OK = 0).  Host arrays are owned by
 * the caller and are only read or written during the call (synchronous).
 * Layouts are the Fortran ones: q(n_vars,nx,ny) column-major, i.e. element
 * (i,j,k) (0-based) at i + n_vars*(j + nx*k); cell planes (nx,ny) at j + nx*k;
 * x-staggered planes (nx+1,ny) at j + (nx+1)*k; y-staggered (nx,ny+1) at j + nx*k.
 * Cell indices reported back (first bad cell) are 1-based (j,k) as in Fortran.
 *
 * No function traps, asserts or spins without a bound on the device.
 */
#ifndef IMEX_GPU_H
#define IMEX_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IMEX_MAX_SOLID 4
#define IMEX_MAX_VARS (4 + IMEX_MAX_SOLID)
#define IMEX_ABI_VERSION 1

/* Status codes.  1..6 mirror the reference's fatal prints (which print and
 * then block on READ(*,*) before continuing with the same values); the
 * step is completed exactly as the reference completes it after the read. */
enum {
  IMEX_OK = 0,
  IMEX_ENAN = 1,          /* NaN in q after the RK step     src/solver_2d.f90:1379 */
  IMEX_ENEGH = 2,         /* h < -1e-7 after the RK step    src/solver_2d.f90:1405 */
  IMEX_ENEGSOLID = 3,     /* solid <= -1e-7                 src/solver_2d.f90:1439 */
  IMEX_ELOWT = 4,         /* T < 273 K                      src/solver_2d.f90:1538 */
  IMEX_ESOLIDSUM = 5,     /* sum(solid) > q1 beyond 1e-10   src/solver_2d.f90:1569 */
  IMEX_EEROSION = 6,      /* erosion/deposition checks      src/solver_2d.f90:2497,2520,2549 */
  IMEX_ETIMEOUT = 7,      /* a bounded device wait gave up (never expected) */
  IMEX_ECUDA = 8,         /* CUDA runtime error; see imex_gpu_last_error() */
  IMEX_EINVAL = 9,        /* invalid argument / sizes */
  IMEX_EUNSUPPORTED = 10, /* a reference option outside the implemented path */
  IMEX_ENOMEM = 11,
  IMEX_ENODEVICE = 12
};

/* Bits of ImexStats.error_mask (one per reference check). */
#define IMEX_ERRBIT(code) (1u << (code))

typedef struct ImexBC {
  int32_t flag;   /* 0 Dirichlet, 1 Neumann (slope value), 2 one-sided slope */
  int32_t pad_;
  double value;
} ImexBC;         /* TYPE bc, src/parameters_2d.f90:341-344 */

/*
 * Run parameters.  Field names follow the reference namelists
 * (src/inpout_2d.f90:315-376) and module variables.  Derived constants
 * (rho_a_amb, inv_pres, 1/rho_s, dx/2, 1/dx, eps_sing**4, the complex-step
 * size n_vars*epsilon) are computed inside imex_gpu_create with the
 * reference's formulas.
 */
typedef struct ImexParams {
  int32_t abi_version;          /* must be IMEX_ABI_VERSION */
  /* grid: src/geometry_2d.f90:185-300 */
  int32_t nx, ny;               /* comp_cells_x, comp_cells_y */
  int32_t n_solid;              /* 1..IMEX_MAX_SOLID; n_vars = 4 + n_solid */
  double x0, y0, cell_size;
  double eps_sing;              /* MIN(MIN(dx**4,dy**4),1e-10), geometry_2d.f90:286-290 */
  /* numerics: NUMERIC_PARAMETERS */
  int32_t n_rk;                 /* 2 (the only tableau with a non-trivial implicit stage used here) */
  int32_t limiter[IMEX_MAX_VARS + 2]; /* limiter(1:n_vars+2); (n_vars+1,n_vars+2) = (2,3) */
  double cfl, max_dt, reconstr_coeff, theta;
  /* flags: NEWRUN_PARAMETERS etc. */
  int32_t energy_flag, alpha_flag, gas_flag, liquid_flag;
  int32_t rheology_flag, rheology_model;  /* models 0 (none), 1 Voellmy-Salm, 6 quadratic */
  int32_t slope_correction_flag, curvature_term_flag;
  int32_t radial_source_flag, lateral_source_flag, bottom_radial_source_flag;
  int32_t settling_flag, entrainment_flag, erodible_deposit_flag, topo_change_flag;
  int32_t pad_;
  /* boundary conditions bcW/E/S/N(n_vars) */
  ImexBC bcW[IMEX_MAX_VARS], bcE[IMEX_MAX_VARS], bcS[IMEX_MAX_VARS], bcN[IMEX_MAX_VARS];
  /* physical constants: constitutive_2d.f90:33-262 */
  double grav;
  double T_ambient, pres, sp_heat_a, sp_gas_const_a, kin_visc_c;
  double rho_s[IMEX_MAX_SOLID], diam_s[IMEX_MAX_SOLID], sp_heat_s[IMEX_MAX_SOLID];
  double mu, xi, friction_factor;
  double maximum_solid_packing;
  /* radial / lateral inlet: RADIAL_SOURCE_PARAMETERS (after read_param's
   * conversion of MFR/Ri into h_source, vel_source, alphas_source) */
  double h_source, vel_source, T_source;
  double alphas_source[IMEX_MAX_SOLID];
  double time_param[4];
  /* mass exchange: SOLID_TRANSPORT_PARAMETERS */
  double erosion_coeff, erodible_porosity, T_erodible, alphastot_min;
  double erodible_fract[IMEX_MAX_SOLID];
  double rho_c_sub;             /* pres/(R_a*T_erodible), inpout_2d.f90:1733 */
  double coeff_porosity;        /* erodible_porosity/(1-erodible_porosity), inpout_2d.f90:1683 */
} ImexParams;

/*
 * Static per-run planes (host pointers, Fortran layout, copied at create).
 * Required: B_prime_x_geom, B_prime_y_geom, solve_mask_time.
 * grav_coeff, d_grav_coeff_dx, grav_coeff_stag_x/y: required when
 *   slope_correction_flag; otherwise NULL (the reference sets them to 1 / 0).
 * B_second_*_geom: required when curvature_term_flag, else NULL.
 * source_cell/sourceE..N/source*_vect_*: required when radial_source_flag.
 * B_cent, B_nodata: optional (NULL = zero / false).
 * erodible, deposit, erosion: required when erosion_coeff>0 or settling_flag.
 */
typedef struct ImexStatic {
  const double* B_cent;            /* (nx,ny) */
  const double* B_prime_x_geom;    /* (nx,ny) */
  const double* B_prime_y_geom;
  const double* B_second_xx_geom;
  const double* B_second_xy_geom;
  const double* B_second_yy_geom;
  const double* grav_coeff;
  const double* d_grav_coeff_dx;
  const double* grav_coeff_stag_x; /* (nx+1,ny) */
  const double* grav_coeff_stag_y; /* (nx,ny+1) */
  const int32_t* source_cell;      /* (nx,ny) 0 solved, 1 inlet interior, 2 inlet ring */
  const int8_t* sourceE;
  const int8_t* sourceW;
  const int8_t* sourceS;
  const int8_t* sourceN;
  const double* sourceE_vect_x;
  const double* sourceE_vect_y;
  const double* sourceW_vect_x;
  const double* sourceW_vect_y;
  const double* sourceS_vect_x;
  const double* sourceS_vect_y;
  const double* sourceN_vect_x;
  const double* sourceN_vect_y;
  const int8_t* B_nodata;          /* (nx,ny) */
  const double* solve_mask_time;   /* (nx,ny) release time per cell */
  const double* erodible;          /* (n_solid,nx,ny) */
  const double* deposit;           /* (nx,ny,n_solid) */
  const double* erosion;           /* (nx,ny,n_solid) */
} ImexStatic;

typedef struct ImexStats {
  int64_t solve_cells;             /* cells in solve_mask at the last check_solve */
  int64_t newton_cells;            /* cells that entered solve_rk_step in the last step */
  int64_t newton_iters;            /* sum of nl_iter at exit over those cells */
  int64_t lnsrch_trials;           /* eval_f calls made by lnsrch */
  int64_t newton_maxit_cells;      /* cells that used all max_nl_iter iterations */
  int64_t newton_hist[16];         /* histogram of nl_iter (1..15, >=16 in the last bin) */
  uint32_t error_mask;             /* OR of IMEX_ERRBIT(code) since the last stats read */
  int32_t first_error_code;        /* code of the lowest-index offending cell (0 = none) */
  int32_t first_error_j, first_error_k; /* 1-based cell of that code */
  double dt;                       /* last dt used */
  double t;                        /* model time held by the context */
  int64_t steps;                   /* steps taken through imex_gpu_advance */
  int64_t kernel_launches;         /* kernels launched by the context since create */
  int64_t warm_fallback_cells;     /* warm starts redone from q_si in the last step */
} ImexStats;

typedef struct ImexCtx ImexCtx;

/* Context lifetime.  device < 0 selects the current CUDA device. */
int imex_gpu_create(const ImexParams* p, const ImexStatic* s, int device, ImexCtx** out);
int imex_gpu_destroy(ImexCtx* ctx);

/* State transfer (host q in Fortran layout q(n_vars,nx,ny)). */
int imex_gpu_set_state(ImexCtx* ctx, const double* q, double t);
int imex_gpu_get_state(ImexCtx* ctx, double* q, double* qp /* (n_vars+2,nx,ny) or NULL */);
/* Mass-exchange planes back to the host (any pointer may be NULL). */
int imex_gpu_get_exchange(ImexCtx* ctx, double* erodible, double* deposit,
                          double* erosion, double* B_cent);

/* The reference's per-step routines, one call each. */
int imex_gpu_check_solve(ImexCtx* ctx, double t, int solve_all, int64_t* n_solve_cells);
int imex_gpu_timestep(ImexCtx* ctx, double* dt);

/* The same CFL time step as imex_gpu_timestep, for callers that must not
 * allocate device memory at the time of the call: drivers living under a
 * fixed device-memory reservation (another framework's pool already owns the
 * GPU) or running in phases where allocation calls are not allowed.  It has
 * no counterpart in the reference.  Nothing is allocated: its only scratch
 * is a fixed array built into the library (8 MiB, held on every GPU that
 * loads it until exit), one slot per 32x8-cell tile, so grids above
 * 1,048,576 tiles (about 268 million cells) are rejected with IMEX_EINVAL
 * and a message in imex_gpu_last_error.  Inputs are the context's state and
 * mask (from imex_gpu_check_solve); the output is *dt on the host.  Unlike
 * imex_gpu_timestep it leaves the stage-1 fluxes uncomputed.  The call is
 * synchronous: it copies dt to the caller's host variable and waits for its
 * stream, so it must not be called while its stream (or, in global capture
 * mode, any stream) is being captured into a CUDA graph.  The first call on
 * a device also looks up the array's device address.  All calls share the
 * array: calls that overlap on one GPU race with each other. */
int imex_gpu_timestep_noalloc(ImexCtx* ctx, double* dt);
int imex_gpu_rk_step(ImexCtx* ctx, double t, double dt);
int imex_gpu_erosion_deposition(ImexCtx* ctx, double dt);
/* topography_reconstruction (src/geometry_2d.f90:535-860) on the device from
 * the context's B_cent: the *_geom slopes and curvatures the step reads and,
 * with slope correction, grav_coeff, d_grav_coeff_dx and the staggered
 * grav_coeff.  imex_gpu_advance runs it after every step when
 * topo_change_flag is set (as the driver does, src/IMEX_SfloW2D.f90:387);
 * with topo_change_flag the grid needs at least 5 cells per direction. */
int imex_gpu_topography_reconstruction(ImexCtx* ctx);

/* Masks back to the host: solve_mask (nx,ny), solve_mask_x (nx+1,ny),
 * solve_mask_y (nx,ny+1); 0/1 bytes.  Any pointer may be NULL. */
int imex_gpu_get_masks(ImexCtx* ctx, int8_t* solve_mask, int8_t* mask_x, int8_t* mask_y);

/*
 * n_steps passes of the driver loop body (src/IMEX_SfloW2D.f90:339-389) with
 * dt clipping on the device (no host round trip per step):
 *   dt = min(dt_cfl, t_end - t, t_output - t, 1.1*0.5*(dt_old + dt_old_old)).
 * dt_old/dt_old_old live in the context (initialised to dt0 by
 * imex_gpu_set_clock).  t_output < 0 disables that clip.
 * If use_graph != 0 the step sequence is captured once into a CUDA graph and
 * replayed.  t (on return) is the model time after the last step.
 */
int imex_gpu_set_clock(ImexCtx* ctx, double t, double dt0, double t_end, double t_output);
int imex_gpu_advance(ImexCtx* ctx, int n_steps, int use_graph, double* t);

/*
 * One pass of the driver loop (src/IMEX_SfloW2D.f90:339-389) for a driver
 * that keeps q on the host, as the reference's module arrays are: the result
 * of imex_gpu_set_state(ctx, q_in, t); imex_gpu_advance(ctx, 1, 0, t_out);
 * imex_gpu_get_state(ctx, q_out, NULL), bit for bit, with the transfers
 * overlapped with the step.  The grid goes up and comes back in row bands
 * on a second stream: the masks and fluxes of a band start as soon as the
 * band and its neighbour rows are on the device, and a band's rows return
 * once its assembly and erosion/deposition are done (stage 2's Newton
 * passes, which wait for the global dt, run on the whole grid in between).
 * q_in and q_out are q(n_vars, nx, ny) in Fortran order and may be the same
 * array; page-locked host memory lets the copies overlap.  Returns like
 * imex_gpu_advance (a reference check's code after the step completed).
 * With a warm start, harvest, moving bed, output sweep or profiling on, the
 * three calls run one after the other.  Synchronous.
 */
int imex_gpu_advance_host(ImexCtx* ctx, const double* q_in, double t, double* q_out,
                          double* t_out);

int imex_gpu_stats(ImexCtx* ctx, ImexStats* st, int reset_errors);
const char* imex_gpu_last_error(ImexCtx* ctx);

/* Synchronise the context stream (for host timing of asynchronous work). */
int imex_gpu_sync(ImexCtx* ctx);

/* Run the context's work on a caller's CUDA stream (a cudaStream_t; NULL
 * returns to the context's own stream), e.g. a framework's current stream so
 * that its events time the step. */
int imex_gpu_set_stream(ImexCtx* ctx, void* stream);

/* Device-resident buffers for callers that bring their own device arrays
 * (benchmarks): SoA planes q[v][k][pitch] of the context, and its pitch in
 * elements.  The pointer stays valid for the context's life. */
int imex_gpu_device_state(ImexCtx* ctx, double** q_dev, int64_t* pitch);

/* Measurement helpers (no counterpart in the reference).
 * imex_gpu_profile(ctx, 1) records CUDA events around the kernels that
 * imex_gpu_advance launches without a graph, on the context stream;
 * imex_gpu_kernel_times returns, per kernel id, the summed event time in ms
 * and the number of timed launches since the last call.  Ids: 0 mask,
 * 1 flux (stage 1 + CFL), 2 stage 2 up to Newton iteration 1, 3 Newton
 * iterations 2.. (three launches), 4 stage-2 assembly, 5 erosion/deposition;
 * n_kernels must be at least 6.  imex_gpu_measure_fp64_peak times an FP64 FMA-chain kernel
 * and returns the achieved GFLOP/s (2 flops per FMA). */
int imex_gpu_profile(ImexCtx* ctx, int enable);
int imex_gpu_kernel_times(ImexCtx* ctx, double* total_ms, int64_t* launches, int n_kernels);
int imex_gpu_measure_fp64_peak(int device, double* gflops);

/*
 * The driver's output sweep after each step on the device
 * (src/IMEX_SfloW2D.f90:391-485, first form :253-309): qp(1) for the
 * volume print, the running maxima hmax, pdynmax and mod_vel_max, the
 * vulnerability table, and the per-step mass / volume / area / solid-mass
 * print.  imex_gpu_post_init takes the VULNERABILITY_TABLE_PARAMETERS levels
 * (at most 10 of each kind, none negative; one kind given alone makes the
 * other a single level 0, as read_param does), zeroes the fields and runs the
 * first sweep over the current solve cells; call it right after
 * imex_gpu_set_state, as the driver runs its sweep right after the first
 * check_solve.  From then on imex_gpu_advance runs the sweep after every
 * step (also inside its CUDA graph); callers of the per-routine entry points
 * call imex_gpu_post_step after the step.  imex_gpu_post_diag returns the
 * driver's print values (dx*dy times the sums; area counts q(1) > 1e-7);
 * its sums are taken in a fixed order on the device, so they equal the
 * reference's sequential SUM to rounding, not bit for bit.
 * imex_gpu_get_post writes hmax, pdynmax, mod_vel_max (nx,ny) and
 * vuln_table (n_table,nx,ny) as 0/1 bytes; any pointer may be NULL.
 */
typedef struct ImexPostDiag {
  double mass, volume, area, solid_mass;
} ImexPostDiag;
int imex_gpu_post_init(ImexCtx* ctx, int n_thickness_levels, const double* thickness_levels,
                       int n_dyn_pres_levels, const double* dyn_pres_levels);
int imex_gpu_post_step(ImexCtx* ctx, ImexPostDiag* diag /* NULL: no print values */);
int imex_gpu_post_diag(ImexCtx* ctx, ImexPostDiag* diag);
int imex_gpu_get_post(ImexCtx* ctx, double* hmax, double* pdynmax, double* mod_vel_max,
                      int8_t* vuln_table, int* n_table);

/*
 * Learned Newton warm start (no counterpart in the reference).  A small
 * network (12 inputs -> 3 x 64 SiLU -> 2 outputs; BF16 weights on tensor
 * cores, FP32 accumulation) proposes the two momentum components that stage
 * 2's Newton solve (src/solver_2d.f90:1660-1994) starts from; the solve then
 * runs in FP64 to the reference's own exit tests, its scaling taken from the
 * proposed start.  A start that does not converge in 100 iterations or ends
 * non-finite is redone from q_si (the plain start); ImexStats counts those.
 * Results equal the plain method's to the solver's tolerance, not bit for
 * bit.  Training pairs come from the solver itself: imex_gpu_harvest_start
 * records, for every stride-th Newton cell of each following stage 2, the 12
 * inputs and the converged momentum change per unit q(1), up to `capacity`
 * pairs, into device buffers that imex_gpu_harvest_data exposes (valid until
 * the next harvest_start or destroy).  The network is trained on them with
 * imex_mlp_train (own forward/backward/Adam kernels) and attached with
 * imex_gpu_set_warmstart (NULL returns to the plain start; the network must
 * outlive its use).  Inputs and targets are normalised by imex_mlp_set_norm
 * (x mean[12], x std[12], y mean[2], y std[2]).
 */
typedef struct ImexMLP ImexMLP;
#define IMEX_MLP_NPARAM 9928
int imex_mlp_create(int device, uint64_t seed, ImexMLP** out);
int imex_mlp_destroy(ImexMLP* net);
int imex_mlp_get_params(ImexMLP* net, float* params /* IMEX_MLP_NPARAM */);
int imex_mlp_set_params(ImexMLP* net, const float* params);
int imex_mlp_set_norm(ImexMLP* net, const float* norm /* 28 floats */);
int imex_mlp_get_norm(ImexMLP* net, float* norm);
int imex_mlp_predict(ImexMLP* net, const float* x /* (n,12) */, int64_t n, float* y /* (n,2) */);
int imex_mlp_loss_grad(ImexMLP* net, const float* x, const float* y, int64_t n, float* loss,
                       float* grad /* IMEX_MLP_NPARAM */);
int imex_mlp_train(ImexMLP* net, const float* x_dev, const float* y_dev, int64_t n, int epochs,
                   int batch, float lr, uint64_t seed, float* loss_per_epoch);
const char* imex_mlp_last_error(ImexMLP* net);
int imex_gpu_set_warmstart(ImexCtx* ctx, ImexMLP* net);
int imex_gpu_harvest_start(ImexCtx* ctx, int64_t capacity, int stride);
int imex_gpu_harvest_stop(ImexCtx* ctx);
int imex_gpu_harvest_data(ImexCtx* ctx, const float** x_dev, const float** y_dev, int64_t* n);

/*
 * Ensembles: many independent runs (members), each with its own grid,
 * parameters and static planes, advanced together on one GPU.  This replaces
 * the reference's process-level ensemble (EXAMPLES/EXAMPLE_ENSEMBLE_ETNA:
 * create_ensemble.py samples the inputs, launch_jobs.py:13-30 runs one
 * single-threaded IMEX_SfloW2D process per member); the sampling of inputs
 * stays with the caller.
 *
 * imex_gpu_ensemble_create makes one context per member (params[m],
 * statics[m]).  imex_gpu_ensemble_member returns member m's context for the
 * single-context calls (set_state, set_clock, get_state, get_exchange, stats,
 * get_masks); do not call imex_gpu_advance or the per-routine calls on a
 * member while the ensemble advances.  imex_gpu_ensemble_advance runs n_steps
 * driver-loop passes (as imex_gpu_advance) of every member from one CUDA
 * graph that forks the members over K streams; its first calls time one real
 * step for K = 1, 2, 4, ... up to min(members, 32) and keep the fastest K
 * (results do not depend on K).  It returns the first status code found
 * (member order) and, in *first_bad_member, that member (-1: none).
 * imex_gpu_ensemble_tuning reports the chosen K and the timed candidates.
 *
 * When all members share one solid-class count and none uses the learned
 * start, the harvest, the output sweep or a moving bed, the ensemble runs
 * batched instead: every phase of the step is one persistent kernel for all
 * members (a fixed grid walking device-built work lists: all tiles for the
 * mask, the tiles holding a solve cell for the fluxes, stage 2 and erosion,
 * the members' Newton lists laid end to end for the iteration passes), 13
 * or 14 launches per step for the whole ensemble, captured once in a CUDA
 * graph and replayed.  Its first six steps are timed with the tile shapes
 * of the mask and flux passes (32x8, 16x16, 32x4 cells) in the order
 * 1 2 3 3 2 1, and the shape with the smallest total is kept;
 * imex_gpu_ensemble_tile_shape reports the chosen shape (0x0: not batched or
 * not tuned yet) and the timed steps.  Results equal each member's single
 * run bit for bit in both modes.
 */
typedef struct ImexEnsemble ImexEnsemble;
int imex_gpu_ensemble_create(int n_members, const ImexParams* const* params,
                             const ImexStatic* const* statics, int device, ImexEnsemble** out);
int imex_gpu_ensemble_destroy(ImexEnsemble* ens);
int imex_gpu_ensemble_member(ImexEnsemble* ens, int m, ImexCtx** ctx);
int imex_gpu_ensemble_advance(ImexEnsemble* ens, int n_steps, int* first_bad_member);
int imex_gpu_ensemble_tuning(ImexEnsemble* ens, int* k_streams, int* n_tried, int* tried_k,
                             float* tried_ms, int cap);
/* mode 0 (the default): batched when the members allow it; mode 2: always
 * per-member graphs over streams.  Takes effect at the next advance. */
int imex_gpu_ensemble_set_mode(ImexEnsemble* ens, int mode);
int imex_gpu_ensemble_tile_shape(ImexEnsemble* ens, int* tx, int* ty, int* n_tried,
                                 int* tried_tx, int* tried_ty, float* tried_ms, int cap);
const char* imex_gpu_ensemble_last_error(ImexEnsemble* ens);

/*
 * output_solution (src/inpout_2d.f90:5683-6180) from the device state.
 * imex_gpu_output enqueues, on the context's stream, the values the
 * reference prints and the copies of them into pinned host memory, then
 * returns; a host thread formats and writes the files while later steps
 * run (call imex_gpu_output_wait before reading them; a new
 * imex_gpu_output waits for the previous one).  Files, named as the
 * reference names them with idx = lettera(output_idx-1):
 *   cons:     RUN_idx.q_2d ('(2e20.12,100(e20.12))': x, y, q(1:n_vars)),
 *             RUN_erosion_idx.q_2d / RUN_erodible_idx.q_2d (erosion_coeff>0),
 *             RUN_deposit_idx.q_2d (settling_flag), RUN_B_idx.q_2d
 *             (topo_change_flag); like the reference it sets |q| < 1e-20
 *             to 0 in the state;
 *   phys:     RUN_idx.p_2d ('100ES15.7E2') with the columns of :6142-6148
 *             for this library's physics (no additional gas, liquid,
 *             stochastic or pore-pressure variables: alphal, shear_vel,
 *             Rouse_no and inertial_number print as 0, and mu_eff takes the
 *             excess pore pressure as 0 where the reference reads element 1
 *             of an empty array); hmax/pdynmax/mod_vel_max come from the
 *             post-step planes (0 without imex_gpu_post_init); like the
 *             reference it sets DEPOSIT/EROSION below 1e-20 to 0;
 *   esri:     RUN_idx.asc (h), RUN_T_idx.asc, RUN_dep_SSSS_idx.asc and
 *             RUN_depTot_idx.asc (settling_flag), RUN_ers_SSSS_idx.asc and
 *             RUN_ersTot_idx.asc (erosion_coeff>0), output_esri (:6306-6613);
 *   max_grid: RUN_max.asc from hmax (output_max, :6195-6235; needs
 *             imex_gpu_post_init).
 * The list-directed files of output_esri's first call (dem_esri*.asc) and
 * the NetCDF-4 output are not written.  threads: formatting threads (0 = all
 * cores).  A failed write is reported by the next imex_gpu_output_wait.
 */
typedef struct ImexOutputSpec {
  const char* run_name;   /* TRIM(run_name): path prefix of every file */
  int output_idx;         /* output_idx after the reference's increment */
  double time;            /* model time of the output (informational) */
  int cons, phys, esri, max_grid;
  int threads;
} ImexOutputSpec;
int imex_gpu_output(ImexCtx* ctx, const ImexOutputSpec* spec);
int imex_gpu_output_wait(ImexCtx* ctx);
/* One value through the writers' Fortran edit descriptors (kind 0 Ew.d,
 * 1 ESw.dEe, 2 Iw, 3 Fw.d) into buf, NUL-terminated; returns the length, or
 * -1 for bad arguments.  Host code: needs no GPU. */
int imex_format_edit(int kind, double value, int w, int d, int e, char* buf, int cap);

/*
 * Set-up on the device (no context needed).  Inputs and outputs are host
 * arrays in the reference's column-major layouts; each call copies its
 * inputs to `device` (< 0: the current one), runs one kernel and copies the
 * result back.  *kernel_ms (may be NULL) receives the kernel's device time.
 * Errors: IMEX_EINVAL with a message in imex_setup_last_error().
 *
 * imex_setup_dem replaces init_grid's DEM sampling (src/geometry_2d.f90:
 * 320-342): B_nodata = interp_2d_nodata (:1242-1296) on the heights as read,
 * B_cent = interp_2d_scalar (:1174-1226) on MAX(0, heights), at the cell
 * centres of the nx*ny grid with origin (x0, y0) and spacing cell_size (1
 * along an axis of one cell, :250-266).  z is topography_profile(3,:,:):
 * (ncols, nrows), row 1 the southernmost; node (j,k) sits at
 * (xllcorner+(j-0.5)*cellsize, yllcorner+(k-0.5)*cellsize)
 * (src/inpout_2d.f90:3572-3605).  A cell centre west or south of the first
 * node (where the reference would index outside the DEM) is an error.
 *
 * imex_setup_cell_fract replaces compute_cell_fract (src/geometry_2d.f90:
 * 1678-1773): the share of each cell's 200x200 subgrid points inside the
 * ellipse of centre (xs, ys), semi-axes rs, r2s, rotated by angle_deg, as
 * REAL(count)/40000 in single precision; 0 outside the bounding square.
 * cos/sin of the angle come from the host's libm.
 *
 * imex_setup_regrid replaces the restart regridding of read_solution
 * (src/inpout_2d.f90:5203-5246 with regrid_scalar, src/geometry_2d.f90:
 * 1491-1534): the area-weighted average of the raster fin (ncols, nrows,
 * row 1 southernmost, cell edges at xllcorner+(j-1)*cellsize) over each
 * cell [x0+(j-1)*cell_size, x0+j*cell_size] x [...]; values equal to
 * nodata count as 0.  The reference's loop bounds are kept (the raster's
 * last column is never read: ix2 <= ncols).
 */
int imex_setup_dem(int device, int ncols, int nrows, double xllcorner, double yllcorner,
                   double cellsize, double nodata, const double* z, int nx, int ny, double x0,
                   double y0, double cell_size, double* B_cent, int8_t* B_nodata,
                   float* kernel_ms);
int imex_setup_cell_fract(int device, int nx, int ny, double x0, double y0, double cell_size,
                          double xs, double ys, double rs, double r2s, double angle_deg,
                          double* cell_fract, float* kernel_ms);
int imex_setup_regrid(int device, int ncols, int nrows, double xllcorner, double yllcorner,
                      double cellsize, double nodata, const double* fin, int nx, int ny,
                      double x0, double y0, double cell_size, double* fout, float* kernel_ms);
const char* imex_setup_last_error(void);

/* Point functions of the step evaluated on the device, element by element,
 * for host arrays of n values (copied in, evaluated, copied out); a check of
 * the CUDA point functions against another implementation on any inputs.
 *   fn 0  x**y, the table-driven power of the mass-exchange closures:
 *         out = a**b (c, d unused)
 *   fn 1  settling_velocity(diam = a, rhos = b, rhoc = c, 1/kin_visc = d)
 *         with gravity g          src/constitutive_2d.f90:5148-5214
 *   fn 2  the limiter-1 (minmod) slope of values a, b, c at centres 0, d, 2d
 *         by the equal-spacing path of the flux kernel
 *   fn 3  limit(a, b, c at centres 0, d, 2d) with limiter g (0..7), theta 1
 *         src/geometry_2d.f90:1555-1676
 *   fn 4  the kernels' test of a rounded quotient against a threshold,
 *         taken without the division where certain: 1 if a/b < c, else 0
 * Returns IMEX_EINVAL for another fn or n < 0, IMEX_ENODEVICE without a GPU. */
int imex_gpu_point_eval(int fn, long long n, const double* a, const double* b, const double* c,
                        const double* d, double g, double* out);

/* Build information: "sm_100a fmad=0 ..." */
const char* imex_gpu_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* IMEX_GPU_H */
