"""ctypes mirror of include/imex_gpu.h (the C ABI of the B200 time step).

The structures here must match the header field for field; tests check the
sizes against the values the shared library reports.
"""
import ctypes as C

IMEX_MAX_SOLID = 4
IMEX_MAX_VARS = 4 + IMEX_MAX_SOLID
IMEX_ABI_VERSION = 1

IMEX_OK = 0
IMEX_ENAN = 1
IMEX_ENEGH = 2
IMEX_ENEGSOLID = 3
IMEX_ELOWT = 4
IMEX_ESOLIDSUM = 5
IMEX_EEROSION = 6
IMEX_ETIMEOUT = 7
IMEX_ECUDA = 8
IMEX_EINVAL = 9
IMEX_EUNSUPPORTED = 10
IMEX_ENOMEM = 11
IMEX_ENODEVICE = 12

STATUS_NAMES = {
    0: "IMEX_OK", 1: "IMEX_ENAN", 2: "IMEX_ENEGH", 3: "IMEX_ENEGSOLID",
    4: "IMEX_ELOWT", 5: "IMEX_ESOLIDSUM", 6: "IMEX_EEROSION",
    7: "IMEX_ETIMEOUT", 8: "IMEX_ECUDA", 9: "IMEX_EINVAL",
    10: "IMEX_EUNSUPPORTED", 11: "IMEX_ENOMEM", 12: "IMEX_ENODEVICE",
}


def errbit(code):
    return 1 << code


class ImexBC(C.Structure):
    _fields_ = [("flag", C.c_int32), ("pad_", C.c_int32), ("value", C.c_double)]


_MV = IMEX_MAX_VARS
_MS = IMEX_MAX_SOLID


class ImexParams(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("n_solid", C.c_int32),
        ("x0", C.c_double), ("y0", C.c_double), ("cell_size", C.c_double),
        ("eps_sing", C.c_double),
        ("n_rk", C.c_int32),
        ("limiter", C.c_int32 * (_MV + 2)),
        ("cfl", C.c_double), ("max_dt", C.c_double),
        ("reconstr_coeff", C.c_double), ("theta", C.c_double),
        ("energy_flag", C.c_int32), ("alpha_flag", C.c_int32),
        ("gas_flag", C.c_int32), ("liquid_flag", C.c_int32),
        ("rheology_flag", C.c_int32), ("rheology_model", C.c_int32),
        ("slope_correction_flag", C.c_int32), ("curvature_term_flag", C.c_int32),
        ("radial_source_flag", C.c_int32), ("lateral_source_flag", C.c_int32),
        ("bottom_radial_source_flag", C.c_int32),
        ("settling_flag", C.c_int32), ("entrainment_flag", C.c_int32),
        ("erodible_deposit_flag", C.c_int32), ("topo_change_flag", C.c_int32),
        ("pad_", C.c_int32),
        ("bcW", ImexBC * _MV), ("bcE", ImexBC * _MV),
        ("bcS", ImexBC * _MV), ("bcN", ImexBC * _MV),
        ("grav", C.c_double),
        ("T_ambient", C.c_double), ("pres", C.c_double), ("sp_heat_a", C.c_double),
        ("sp_gas_const_a", C.c_double), ("kin_visc_c", C.c_double),
        ("rho_s", C.c_double * _MS), ("diam_s", C.c_double * _MS),
        ("sp_heat_s", C.c_double * _MS),
        ("mu", C.c_double), ("xi", C.c_double), ("friction_factor", C.c_double),
        ("maximum_solid_packing", C.c_double),
        ("h_source", C.c_double), ("vel_source", C.c_double), ("T_source", C.c_double),
        ("alphas_source", C.c_double * _MS),
        ("time_param", C.c_double * 4),
        ("erosion_coeff", C.c_double), ("erodible_porosity", C.c_double),
        ("T_erodible", C.c_double), ("alphastot_min", C.c_double),
        ("erodible_fract", C.c_double * _MS),
        ("rho_c_sub", C.c_double), ("coeff_porosity", C.c_double),
    ]


_dp = C.POINTER(C.c_double)
_i8p = C.POINTER(C.c_int8)
_i32p = C.POINTER(C.c_int32)


class ImexStatic(C.Structure):
    _fields_ = [
        ("B_cent", _dp), ("B_prime_x_geom", _dp), ("B_prime_y_geom", _dp),
        ("B_second_xx_geom", _dp), ("B_second_xy_geom", _dp), ("B_second_yy_geom", _dp),
        ("grav_coeff", _dp), ("d_grav_coeff_dx", _dp),
        ("grav_coeff_stag_x", _dp), ("grav_coeff_stag_y", _dp),
        ("source_cell", _i32p),
        ("sourceE", _i8p), ("sourceW", _i8p), ("sourceS", _i8p), ("sourceN", _i8p),
        ("sourceE_vect_x", _dp), ("sourceE_vect_y", _dp),
        ("sourceW_vect_x", _dp), ("sourceW_vect_y", _dp),
        ("sourceS_vect_x", _dp), ("sourceS_vect_y", _dp),
        ("sourceN_vect_x", _dp), ("sourceN_vect_y", _dp),
        ("B_nodata", _i8p), ("solve_mask_time", _dp),
        ("erodible", _dp), ("deposit", _dp), ("erosion", _dp),
    ]


class ImexStats(C.Structure):
    _fields_ = [
        ("solve_cells", C.c_int64), ("newton_cells", C.c_int64),
        ("newton_iters", C.c_int64), ("lnsrch_trials", C.c_int64),
        ("newton_maxit_cells", C.c_int64), ("newton_hist", C.c_int64 * 16),
        ("error_mask", C.c_uint32), ("first_error_code", C.c_int32),
        ("first_error_j", C.c_int32), ("first_error_k", C.c_int32),
        ("dt", C.c_double), ("t", C.c_double),
        ("steps", C.c_int64), ("kernel_launches", C.c_int64),
        ("warm_fallback_cells", C.c_int64),
    ]


class ImexOutputSpec(C.Structure):
    _fields_ = [("run_name", C.c_char_p), ("output_idx", C.c_int), ("time", C.c_double),
                ("cons", C.c_int), ("phys", C.c_int), ("esri", C.c_int), ("max_grid", C.c_int),
                ("threads", C.c_int)]


class ImexPostDiag(C.Structure):
    _fields_ = [("mass", C.c_double), ("volume", C.c_double), ("area", C.c_double),
                ("solid_mass", C.c_double)]


def vulnerability_levels(thickness_levels, dyn_pres_levels):
    """read_param's rule for VULNERABILITY_TABLE_PARAMETERS
    (src/inpout_2d.f90:3630-3682): one kind given alone makes the other a
    single level 0."""
    t, d = list(thickness_levels), list(dyn_pres_levels)
    if t and not d:
        d = [0.0]
    if d and not t:
        t = [0.0]
    return t, d


# static plane name -> (dtype, shape kind) ; shape kinds: "c" cell (nx,ny),
# "sx" (nx+1,ny), "sy" (nx,ny+1), "e" (n_solid,nx,ny), "d" (nx,ny,n_solid)
STATIC_FIELDS = {
    "B_cent": ("f8", "c"), "B_prime_x_geom": ("f8", "c"), "B_prime_y_geom": ("f8", "c"),
    "B_second_xx_geom": ("f8", "c"), "B_second_xy_geom": ("f8", "c"),
    "B_second_yy_geom": ("f8", "c"), "grav_coeff": ("f8", "c"),
    "d_grav_coeff_dx": ("f8", "c"), "grav_coeff_stag_x": ("f8", "sx"),
    "grav_coeff_stag_y": ("f8", "sy"), "source_cell": ("i4", "c"),
    "sourceE": ("i1", "c"), "sourceW": ("i1", "c"), "sourceS": ("i1", "c"),
    "sourceN": ("i1", "c"),
    "sourceE_vect_x": ("f8", "c"), "sourceE_vect_y": ("f8", "c"),
    "sourceW_vect_x": ("f8", "c"), "sourceW_vect_y": ("f8", "c"),
    "sourceS_vect_x": ("f8", "c"), "sourceS_vect_y": ("f8", "c"),
    "sourceN_vect_x": ("f8", "c"), "sourceN_vect_y": ("f8", "c"),
    "B_nodata": ("i1", "c"), "solve_mask_time": ("f8", "c"),
    "erodible": ("f8", "e"), "deposit": ("f8", "d"), "erosion": ("f8", "d"),
}


def make_static(arrays):
    """Build an ImexStatic from a dict of numpy arrays (Fortran-ordered or
    1-D in Fortran element order).  Returns (struct, keepalive list)."""
    import numpy as np

    st = ImexStatic()
    keep = []
    for name, (dt, _kind) in STATIC_FIELDS.items():
        a = arrays.get(name)
        if a is None:
            continue
        a = np.asarray(a, dtype=dt)
        flat = np.ascontiguousarray(a.ravel(order="F"))
        keep.append(flat)
        ctype = {"f8": C.c_double, "i1": C.c_int8, "i4": C.c_int32}[dt]
        setattr(st, name, flat.ctypes.data_as(C.POINTER(ctype)))
    return st, keep
