! imex_gpu_iface.f90 -- Fortran 2003 ISO_C_BINDING declarations of the C ABI
! in imex_gpu.h, for the reference driver (src/IMEX_SfloW2D.f90).
!
! The derived types mirror ImexBC, ImexParams, ImexStatic, ImexStats,
! ImexPostDiag and ImexOutputSpec field for field, in the same order and with
! the same kinds (C_INT32_T, C_INT64_T, C_DOUBLE, C_INT, C_PTR); the
! interfaces bind the entry points a driver calls, with the C argument
! order.  Every function returns the int status of imex_gpu.h (IMEX_OK = 0).
! Host arrays are passed by reference in the reference's Fortran layouts
! (q(n_vars,nx,ny), cell planes (nx,ny), staggered planes (nx+1,ny) and
! (nx,ny+1)); static planes go into imex_static as C_LOC of the allocated
! module arrays (C_NULL_PTR where a plane is unused).
!
! The driver calls it replaces (src/IMEX_SfloW2D.f90):
!   CALL check_solve(.FALSE.)              :341-349  -> imex_gpu_check_solve
!   CALL timestep                          :357      -> imex_gpu_timestep
!   CALL imex_RK_solver                    :383      -> imex_gpu_rk_step
!   CALL update_erosion_deposition_cell(dt):385      -> imex_gpu_erosion_deposition
!   IF (topo_change_flag) CALL topography_reconstruction
!                                          :387      -> imex_gpu_topography_reconstruction
MODULE imex_gpu_iface

  USE, INTRINSIC :: ISO_C_BINDING

  IMPLICIT NONE

  INTEGER, PARAMETER :: IMEX_MAX_SOLID = 4
  INTEGER, PARAMETER :: IMEX_MAX_VARS = 4 + IMEX_MAX_SOLID
  INTEGER, PARAMETER :: IMEX_ABI_VERSION = 1

  INTEGER(C_INT), PARAMETER :: IMEX_OK = 0, IMEX_ENAN = 1, IMEX_ENEGH = 2,      &
       IMEX_ENEGSOLID = 3, IMEX_ELOWT = 4, IMEX_ESOLIDSUM = 5, IMEX_EEROSION = 6,&
       IMEX_ETIMEOUT = 7, IMEX_ECUDA = 8, IMEX_EINVAL = 9, IMEX_EUNSUPPORTED = 10,&
       IMEX_ENOMEM = 11, IMEX_ENODEVICE = 12

  TYPE, BIND(C) :: imex_bc
     INTEGER(C_INT32_T) :: flag
     INTEGER(C_INT32_T) :: pad_
     REAL(C_DOUBLE) :: value
  END TYPE imex_bc

  TYPE, BIND(C) :: imex_params
     INTEGER(C_INT32_T) :: abi_version
     INTEGER(C_INT32_T) :: nx, ny
     INTEGER(C_INT32_T) :: n_solid
     REAL(C_DOUBLE) :: x0, y0, cell_size
     REAL(C_DOUBLE) :: eps_sing
     INTEGER(C_INT32_T) :: n_rk
     INTEGER(C_INT32_T) :: limiter(IMEX_MAX_VARS + 2)
     REAL(C_DOUBLE) :: cfl, max_dt, reconstr_coeff, theta
     INTEGER(C_INT32_T) :: energy_flag, alpha_flag, gas_flag, liquid_flag
     INTEGER(C_INT32_T) :: rheology_flag, rheology_model
     INTEGER(C_INT32_T) :: slope_correction_flag, curvature_term_flag
     INTEGER(C_INT32_T) :: radial_source_flag, lateral_source_flag
     INTEGER(C_INT32_T) :: bottom_radial_source_flag
     INTEGER(C_INT32_T) :: settling_flag, entrainment_flag
     INTEGER(C_INT32_T) :: erodible_deposit_flag, topo_change_flag
     INTEGER(C_INT32_T) :: pad_
     TYPE(imex_bc) :: bcW(IMEX_MAX_VARS), bcE(IMEX_MAX_VARS)
     TYPE(imex_bc) :: bcS(IMEX_MAX_VARS), bcN(IMEX_MAX_VARS)
     REAL(C_DOUBLE) :: grav
     REAL(C_DOUBLE) :: T_ambient, pres, sp_heat_a, sp_gas_const_a, kin_visc_c
     REAL(C_DOUBLE) :: rho_s(IMEX_MAX_SOLID), diam_s(IMEX_MAX_SOLID)
     REAL(C_DOUBLE) :: sp_heat_s(IMEX_MAX_SOLID)
     REAL(C_DOUBLE) :: mu, xi, friction_factor
     REAL(C_DOUBLE) :: maximum_solid_packing
     REAL(C_DOUBLE) :: h_source, vel_source, T_source
     REAL(C_DOUBLE) :: alphas_source(IMEX_MAX_SOLID)
     REAL(C_DOUBLE) :: time_param(4)
     REAL(C_DOUBLE) :: erosion_coeff, erodible_porosity, T_erodible, alphastot_min
     REAL(C_DOUBLE) :: erodible_fract(IMEX_MAX_SOLID)
     REAL(C_DOUBLE) :: rho_c_sub
     REAL(C_DOUBLE) :: coeff_porosity
  END TYPE imex_params

  TYPE, BIND(C) :: imex_static
     TYPE(C_PTR) :: B_cent
     TYPE(C_PTR) :: B_prime_x_geom, B_prime_y_geom
     TYPE(C_PTR) :: B_second_xx_geom, B_second_xy_geom, B_second_yy_geom
     TYPE(C_PTR) :: grav_coeff, d_grav_coeff_dx
     TYPE(C_PTR) :: grav_coeff_stag_x, grav_coeff_stag_y
     TYPE(C_PTR) :: source_cell
     TYPE(C_PTR) :: sourceE, sourceW, sourceS, sourceN
     TYPE(C_PTR) :: sourceE_vect_x, sourceE_vect_y
     TYPE(C_PTR) :: sourceW_vect_x, sourceW_vect_y
     TYPE(C_PTR) :: sourceS_vect_x, sourceS_vect_y
     TYPE(C_PTR) :: sourceN_vect_x, sourceN_vect_y
     TYPE(C_PTR) :: B_nodata
     TYPE(C_PTR) :: solve_mask_time
     TYPE(C_PTR) :: erodible, deposit, erosion
  END TYPE imex_static

  TYPE, BIND(C) :: imex_stats
     INTEGER(C_INT64_T) :: solve_cells, newton_cells, newton_iters
     INTEGER(C_INT64_T) :: lnsrch_trials, newton_maxit_cells
     INTEGER(C_INT64_T) :: newton_hist(16)
     INTEGER(C_INT32_T) :: error_mask
     INTEGER(C_INT32_T) :: first_error_code
     INTEGER(C_INT32_T) :: first_error_j, first_error_k
     REAL(C_DOUBLE) :: dt
     REAL(C_DOUBLE) :: t
     INTEGER(C_INT64_T) :: steps
     INTEGER(C_INT64_T) :: kernel_launches
     INTEGER(C_INT64_T) :: warm_fallback_cells
  END TYPE imex_stats

  TYPE, BIND(C) :: imex_post_diag
     REAL(C_DOUBLE) :: mass, volume, area, solid_mass
  END TYPE imex_post_diag

  TYPE, BIND(C) :: imex_output_spec
     TYPE(C_PTR) :: run_name             ! TRIM(run_name)//C_NULL_CHAR
     INTEGER(C_INT) :: output_idx
     REAL(C_DOUBLE) :: time
     INTEGER(C_INT) :: cons, phys, esri, max_grid
     INTEGER(C_INT) :: threads
  END TYPE imex_output_spec

  INTERFACE

     ! ---- context
     INTEGER(C_INT) FUNCTION imex_gpu_create(p, s, device, ctx)                &
          BIND(C, name="imex_gpu_create")
       IMPORT :: C_INT, C_PTR, imex_params, imex_static
       TYPE(imex_params), INTENT(IN) :: p
       TYPE(imex_static), INTENT(IN) :: s
       INTEGER(C_INT), VALUE :: device
       TYPE(C_PTR), INTENT(OUT) :: ctx
     END FUNCTION imex_gpu_create

     INTEGER(C_INT) FUNCTION imex_gpu_destroy(ctx) BIND(C, name="imex_gpu_destroy")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION imex_gpu_destroy

     ! ---- state (module arrays q, qp)
     INTEGER(C_INT) FUNCTION imex_gpu_set_state(ctx, q, t)                     &
          BIND(C, name="imex_gpu_set_state")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(IN) :: q(*)
       REAL(C_DOUBLE), VALUE :: t
     END FUNCTION imex_gpu_set_state

     INTEGER(C_INT) FUNCTION imex_gpu_get_state(ctx, q, qp)                    &
          BIND(C, name="imex_gpu_get_state")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: q(*), qp(*)
     END FUNCTION imex_gpu_get_state

     INTEGER(C_INT) FUNCTION imex_gpu_get_exchange(ctx, erodible, deposit,     &
          erosion, B_cent) BIND(C, name="imex_gpu_get_exchange")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: erodible(*), deposit(*), erosion(*), B_cent(*)
     END FUNCTION imex_gpu_get_exchange

     ! ---- the per-step routines
     INTEGER(C_INT) FUNCTION imex_gpu_check_solve(ctx, t, solve_all, n_solve)  &
          BIND(C, name="imex_gpu_check_solve")
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT64_T
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), VALUE :: t
       INTEGER(C_INT), VALUE :: solve_all
       INTEGER(C_INT64_T), INTENT(OUT) :: n_solve
     END FUNCTION imex_gpu_check_solve

     INTEGER(C_INT) FUNCTION imex_gpu_timestep(ctx, dt) BIND(C, name="imex_gpu_timestep")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: dt
     END FUNCTION imex_gpu_timestep

     INTEGER(C_INT) FUNCTION imex_gpu_timestep_noalloc(ctx, dt)                &
          BIND(C, name="imex_gpu_timestep_noalloc")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: dt
     END FUNCTION imex_gpu_timestep_noalloc

     INTEGER(C_INT) FUNCTION imex_gpu_rk_step(ctx, t, dt) BIND(C, name="imex_gpu_rk_step")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), VALUE :: t, dt
     END FUNCTION imex_gpu_rk_step

     INTEGER(C_INT) FUNCTION imex_gpu_erosion_deposition(ctx, dt)              &
          BIND(C, name="imex_gpu_erosion_deposition")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), VALUE :: dt
     END FUNCTION imex_gpu_erosion_deposition

     INTEGER(C_INT) FUNCTION imex_gpu_topography_reconstruction(ctx)           &
          BIND(C, name="imex_gpu_topography_reconstruction")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION imex_gpu_topography_reconstruction

     INTEGER(C_INT) FUNCTION imex_gpu_get_masks(ctx, solve_mask, mask_x, mask_y)&
          BIND(C, name="imex_gpu_get_masks")
       IMPORT :: C_INT, C_PTR, C_INT8_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT8_T), INTENT(OUT) :: solve_mask(*), mask_x(*), mask_y(*)
     END FUNCTION imex_gpu_get_masks

     ! ---- whole driver-loop passes on the device
     INTEGER(C_INT) FUNCTION imex_gpu_set_clock(ctx, t, dt0, t_end, t_output)  &
          BIND(C, name="imex_gpu_set_clock")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), VALUE :: t, dt0, t_end, t_output
     END FUNCTION imex_gpu_set_clock

     INTEGER(C_INT) FUNCTION imex_gpu_advance(ctx, n_steps, use_graph, t)      &
          BIND(C, name="imex_gpu_advance")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: n_steps, use_graph
       REAL(C_DOUBLE), INTENT(OUT) :: t
     END FUNCTION imex_gpu_advance

     ! one driver-loop pass with q kept on the host: q_in at time t in, the
     ! state after the step out (may be the same array), transfers overlapped
     INTEGER(C_INT) FUNCTION imex_gpu_advance_host(ctx, q_in, t, q_out,      &
          t_out) BIND(C, name="imex_gpu_advance_host")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(IN) :: q_in(*)
       REAL(C_DOUBLE), VALUE :: t
       REAL(C_DOUBLE), INTENT(INOUT) :: q_out(*)
       REAL(C_DOUBLE), INTENT(OUT) :: t_out
     END FUNCTION imex_gpu_advance_host

     INTEGER(C_INT) FUNCTION imex_gpu_stats(ctx, st, reset_errors)             &
          BIND(C, name="imex_gpu_stats")
       IMPORT :: C_INT, C_PTR, imex_stats
       TYPE(C_PTR), VALUE :: ctx
       TYPE(imex_stats), INTENT(OUT) :: st
       INTEGER(C_INT), VALUE :: reset_errors
     END FUNCTION imex_gpu_stats

     TYPE(C_PTR) FUNCTION imex_gpu_last_error(ctx) BIND(C, name="imex_gpu_last_error")
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION imex_gpu_last_error

     INTEGER(C_INT) FUNCTION imex_gpu_sync(ctx) BIND(C, name="imex_gpu_sync")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION imex_gpu_sync

     ! ---- the driver's output sweep (src/IMEX_SfloW2D.f90:253-309, 391-485)
     INTEGER(C_INT) FUNCTION imex_gpu_post_init(ctx, n_thickness_levels,       &
          thickness_levels, n_dyn_pres_levels, dyn_pres_levels)                &
          BIND(C, name="imex_gpu_post_init")
       IMPORT :: C_INT, C_PTR, C_DOUBLE
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: n_thickness_levels
       REAL(C_DOUBLE), INTENT(IN) :: thickness_levels(*)
       INTEGER(C_INT), VALUE :: n_dyn_pres_levels
       REAL(C_DOUBLE), INTENT(IN) :: dyn_pres_levels(*)
     END FUNCTION imex_gpu_post_init

     INTEGER(C_INT) FUNCTION imex_gpu_post_step(ctx, diag)                     &
          BIND(C, name="imex_gpu_post_step")
       IMPORT :: C_INT, C_PTR, imex_post_diag
       TYPE(C_PTR), VALUE :: ctx
       TYPE(imex_post_diag), INTENT(OUT) :: diag
     END FUNCTION imex_gpu_post_step

     INTEGER(C_INT) FUNCTION imex_gpu_post_diag(ctx, diag)                     &
          BIND(C, name="imex_gpu_post_diag")
       IMPORT :: C_INT, C_PTR, imex_post_diag
       TYPE(C_PTR), VALUE :: ctx
       TYPE(imex_post_diag), INTENT(OUT) :: diag
     END FUNCTION imex_gpu_post_diag

     INTEGER(C_INT) FUNCTION imex_gpu_get_post(ctx, hmax, pdynmax, mod_vel_max, &
          vuln_table, n_table) BIND(C, name="imex_gpu_get_post")
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_INT8_T
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_DOUBLE), INTENT(OUT) :: hmax(*), pdynmax(*), mod_vel_max(*)
       INTEGER(C_INT8_T), INTENT(OUT) :: vuln_table(*)
       INTEGER(C_INT), INTENT(OUT) :: n_table
     END FUNCTION imex_gpu_get_post

     ! ---- output_solution (src/inpout_2d.f90:5683-6180) from the device
     INTEGER(C_INT) FUNCTION imex_gpu_output(ctx, spec) BIND(C, name="imex_gpu_output")
       IMPORT :: C_INT, C_PTR, imex_output_spec
       TYPE(C_PTR), VALUE :: ctx
       TYPE(imex_output_spec), INTENT(IN) :: spec
     END FUNCTION imex_gpu_output

     INTEGER(C_INT) FUNCTION imex_gpu_output_wait(ctx) BIND(C, name="imex_gpu_output_wait")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION imex_gpu_output_wait

     ! ---- set-up on the device (no context)
     INTEGER(C_INT) FUNCTION imex_setup_dem(device, ncols, nrows, xllcorner,   &
          yllcorner, cellsize, nodata, z, nx, ny, x0, y0, cell_size, B_cent,   &
          B_nodata, kernel_ms) BIND(C, name="imex_setup_dem")
       IMPORT :: C_INT, C_DOUBLE, C_INT8_T, C_FLOAT
       INTEGER(C_INT), VALUE :: device, ncols, nrows
       REAL(C_DOUBLE), VALUE :: xllcorner, yllcorner, cellsize, nodata
       REAL(C_DOUBLE), INTENT(IN) :: z(*)
       INTEGER(C_INT), VALUE :: nx, ny
       REAL(C_DOUBLE), VALUE :: x0, y0, cell_size
       REAL(C_DOUBLE), INTENT(OUT) :: B_cent(*)
       INTEGER(C_INT8_T), INTENT(OUT) :: B_nodata(*)
       REAL(C_FLOAT), INTENT(OUT) :: kernel_ms
     END FUNCTION imex_setup_dem

     INTEGER(C_INT) FUNCTION imex_setup_cell_fract(device, nx, ny, x0, y0,     &
          cell_size, xs, ys, rs, r2s, angle_deg, cell_fract, kernel_ms)        &
          BIND(C, name="imex_setup_cell_fract")
       IMPORT :: C_INT, C_DOUBLE, C_FLOAT
       INTEGER(C_INT), VALUE :: device, nx, ny
       REAL(C_DOUBLE), VALUE :: x0, y0, cell_size, xs, ys, rs, r2s, angle_deg
       REAL(C_DOUBLE), INTENT(OUT) :: cell_fract(*)
       REAL(C_FLOAT), INTENT(OUT) :: kernel_ms
     END FUNCTION imex_setup_cell_fract

     INTEGER(C_INT) FUNCTION imex_setup_regrid(device, ncols, nrows, xllcorner,&
          yllcorner, cellsize, nodata, fin, nx, ny, x0, y0, cell_size, fout,   &
          kernel_ms) BIND(C, name="imex_setup_regrid")
       IMPORT :: C_INT, C_DOUBLE, C_FLOAT
       INTEGER(C_INT), VALUE :: device, ncols, nrows
       REAL(C_DOUBLE), VALUE :: xllcorner, yllcorner, cellsize, nodata
       REAL(C_DOUBLE), INTENT(IN) :: fin(*)
       INTEGER(C_INT), VALUE :: nx, ny
       REAL(C_DOUBLE), VALUE :: x0, y0, cell_size
       REAL(C_DOUBLE), INTENT(OUT) :: fout(*)
       REAL(C_FLOAT), INTENT(OUT) :: kernel_ms
     END FUNCTION imex_setup_regrid

     TYPE(C_PTR) FUNCTION imex_setup_last_error() BIND(C, name="imex_setup_last_error")
       IMPORT :: C_PTR
     END FUNCTION imex_setup_last_error

     ! ---- ensembles (one process for all members)
     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_create(n_members, params,       &
          statics, device, ens) BIND(C, name="imex_gpu_ensemble_create")
       IMPORT :: C_INT, C_PTR
       INTEGER(C_INT), VALUE :: n_members
       TYPE(C_PTR), INTENT(IN) :: params(*)       ! C_LOC of imex_params(m)
       TYPE(C_PTR), INTENT(IN) :: statics(*)      ! C_LOC of imex_static(m)
       INTEGER(C_INT), VALUE :: device
       TYPE(C_PTR), INTENT(OUT) :: ens
     END FUNCTION imex_gpu_ensemble_create

     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_destroy(ens)                    &
          BIND(C, name="imex_gpu_ensemble_destroy")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ens
     END FUNCTION imex_gpu_ensemble_destroy

     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_member(ens, m, ctx)             &
          BIND(C, name="imex_gpu_ensemble_member")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ens
       INTEGER(C_INT), VALUE :: m
       TYPE(C_PTR), INTENT(OUT) :: ctx
     END FUNCTION imex_gpu_ensemble_member

     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_advance(ens, n_steps,           &
          first_bad_member) BIND(C, name="imex_gpu_ensemble_advance")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ens
       INTEGER(C_INT), VALUE :: n_steps
       INTEGER(C_INT), INTENT(OUT) :: first_bad_member
     END FUNCTION imex_gpu_ensemble_advance

     ! 0: batched when the members allow it, 2: per-member graphs on streams
     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_set_mode(ens, mode)          &
          BIND(C, name="imex_gpu_ensemble_set_mode")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ens
       INTEGER(C_INT), VALUE :: mode
     END FUNCTION imex_gpu_ensemble_set_mode

     ! the batched mode's tile shape and the timed trial steps (up to cap)
     INTEGER(C_INT) FUNCTION imex_gpu_ensemble_tile_shape(ens, tx, ty,       &
          n_tried, tried_tx, tried_ty, tried_ms, cap)                        &
          BIND(C, name="imex_gpu_ensemble_tile_shape")
       IMPORT :: C_INT, C_FLOAT, C_PTR
       TYPE(C_PTR), VALUE :: ens
       INTEGER(C_INT), INTENT(OUT) :: tx, ty, n_tried
       INTEGER(C_INT), INTENT(OUT) :: tried_tx(*), tried_ty(*)
       REAL(C_FLOAT), INTENT(OUT) :: tried_ms(*)
       INTEGER(C_INT), VALUE :: cap
     END FUNCTION imex_gpu_ensemble_tile_shape

  END INTERFACE

END MODULE imex_gpu_iface
