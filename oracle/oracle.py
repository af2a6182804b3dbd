"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (liboracle.so).

The oracle restates the reference Fortran time step on the CPU; tests and the
benchmark's CPU baseline compare the CUDA path against it.  The product
package never imports this module.  Parity is unpinned against the reference
binary (no Fortran compiler in this image); see imex_oracle.h.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from imex_sflow2d_v2_b200.abi import ImexParams, ImexStatic, ImexStats, make_static

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}
CHECKER = "liboracle.so"
TIMING = "liboracle_timing.so"


def build(force=False, target=CHECKER):
    so = os.path.join(_HERE, target)
    src = os.path.join(_HERE, "imex_oracle.cpp")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "CXX=g++", target])
    return so


def timing_build_usable():
    """The timing build targets x86-64-v3 (AVX2, FMA, BMI2): usable when the
    host CPU reports those flags."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
        return {"avx2", "fma", "bmi2", "movbe"} <= flags
    except OSError:
        return False


def lib(target=CHECKER):
    """ctypes handle of the checker build (default) or of the timing build
    (TIMING: contraction on, instrument off; for the CPU baseline only)."""
    L = _LIBS.get(target)
    if L is None:
        so = build(target=target)
        L = C.CDLL(so)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [C.POINTER(ImexParams), C.POINTER(ImexStatic)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_state.argtypes = [vp, dp, C.c_double]
        L.oracle_get_state.argtypes = [vp, dp, dp]
        L.oracle_get_exchange.argtypes = [vp, dp, dp, dp, dp]
        L.oracle_check_solve.restype = C.c_int64
        L.oracle_check_solve.argtypes = [vp, C.c_double, C.c_int]
        L.oracle_timestep.restype = C.c_double
        L.oracle_timestep.argtypes = [vp]
        L.oracle_rk_step.restype = C.c_uint32
        L.oracle_rk_step.argtypes = [vp, C.c_double, C.c_double]
        L.oracle_erosion_deposition.restype = C.c_uint32
        L.oracle_erosion_deposition.argtypes = [vp, C.c_double]
        L.oracle_post_step.argtypes = [vp]
        i8p = C.POINTER(C.c_int8)
        L.oracle_get_masks.argtypes = [vp, i8p, i8p, i8p]
        L.oracle_set_clock.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_advance.restype = C.c_uint32
        L.oracle_advance.argtypes = [vp, C.c_int, dp]
        L.oracle_stats.argtypes = [vp, C.POINTER(ImexStats)]
        L.oracle_stale_wet_reads.restype = C.c_int64
        L.oracle_stale_wet_reads.argtypes = [vp]
        L.oracle_mass_budget.argtypes = [vp, dp]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_qc_to_qp.argtypes = [vp, dp, dp]
        L.oracle_qp_to_qc.argtypes = [vp, dp, dp]
        L.oracle_implicit_terms.argtypes = [vp, dp, dp, dp, dp]
        L.oracle_mixt_var.argtypes = [vp, dp, dp]
        L.oracle_local_speeds.argtypes = [vp, dp, C.c_double, C.c_int, dp]
        L.oracle_eval_fluxes.argtypes = [vp, dp, dp, C.c_double, C.c_int, dp]
        L.oracle_kt_interface.argtypes = [vp, dp, dp, dp, dp, C.c_double, C.c_int, dp, dp]
        L.oracle_solve_rk_step.restype = C.c_int
        L.oracle_solve_rk_step.argtypes = [vp, dp, dp, dp, C.c_double, C.c_double,
                                           C.c_double, C.c_double]
        L.oracle_ipow.restype = C.c_double
        L.oracle_ipow.argtypes = [C.c_double, C.c_double]
        L.oracle_ipow_n.argtypes = [C.c_longlong, dp, dp, dp]
        L.oracle_settling_velocity_n.argtypes = [C.c_longlong, dp, dp, dp, dp, C.c_double, dp]
        L.oracle_limit_n.argtypes = [C.c_longlong] + [dp] * 6 + [C.c_int, C.c_double, dp]
        L.oracle_post_init.argtypes = [vp, C.c_int, dp, C.c_int, dp]
        L.oracle_post_diag.argtypes = [vp, dp]
        L.oracle_get_post.argtypes = [vp, dp, dp, dp, C.POINTER(C.c_int8)]
        L.oracle_topography_reconstruction.argtypes = [vp]
        L.oracle_get_topo.argtypes = [vp] + [dp] * 7
        i8p = C.POINTER(C.c_int8)
        L.oracle_setup_dem.restype = C.c_int
        L.oracle_setup_dem.argtypes = ([C.c_int, C.c_int] + [C.c_double] * 4 + [dp, C.c_int, C.c_int]
                                       + [C.c_double] * 3 + [dp, i8p])
        L.oracle_cell_fract.argtypes = [C.c_int, C.c_int] + [C.c_double] * 8 + [dp]
        L.oracle_regrid.restype = C.c_int
        L.oracle_regrid.argtypes = ([C.c_int, C.c_int] + [C.c_double] * 4 + [dp, C.c_int, C.c_int]
                                    + [C.c_double] * 3 + [dp])
        L.oracle_output_prep.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp, dp]
        L.oracle_limit.restype = C.c_double
        L.oracle_limit.argtypes = [C.c_double] * 6 + [C.c_int, C.c_double]
        _LIBS[target] = L
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One oracle context; arrays use the Fortran layouts of imex_gpu.h."""

    def __init__(self, params, static_arrays, threads=None, timing=False):
        L = lib(TIMING if timing else CHECKER)
        self._L = L
        if threads is not None:
            L.oracle_set_threads(int(threads))
        self.params = params
        self.nx, self.ny, self.ns = params.nx, params.ny, params.n_solid
        self.nv = 4 + self.ns
        st, self._keep = make_static(static_arrays)
        self._h = L.oracle_create(C.byref(params), C.byref(st))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.oracle_destroy(h)
            self._h = None

    def set_state(self, q, t=0.0):
        q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel(order="F"))
        self._L.oracle_set_state(self._h, _p(q), float(t))

    def get_state(self, with_qp=False):
        q = np.zeros(self.nv * self.nx * self.ny)
        qp = np.zeros((self.nv + 2) * self.nx * self.ny) if with_qp else None
        self._L.oracle_get_state(self._h, _p(q), _p(qp) if with_qp else None)
        q = q.reshape((self.nv, self.nx, self.ny), order="F")
        if with_qp:
            return q, qp.reshape((self.nv + 2, self.nx, self.ny), order="F")
        return q

    def get_exchange(self):
        n = self.nx * self.ny
        er = np.zeros(self.ns * n)
        de = np.zeros(self.ns * n)
        eo = np.zeros(self.ns * n)
        B = np.zeros(n)
        self._L.oracle_get_exchange(self._h, _p(er), _p(de), _p(eo), _p(B))
        return (er.reshape((self.ns, self.nx, self.ny), order="F"),
                de.reshape((self.nx, self.ny, self.ns), order="F"),
                eo.reshape((self.nx, self.ny, self.ns), order="F"),
                B.reshape((self.nx, self.ny), order="F"))

    def check_solve(self, t, solve_all=False):
        return self._L.oracle_check_solve(self._h, float(t), int(solve_all))

    def timestep(self):
        return self._L.oracle_timestep(self._h)

    def rk_step(self, t, dt):
        return self._L.oracle_rk_step(self._h, float(t), float(dt))

    def erosion_deposition(self, dt):
        return self._L.oracle_erosion_deposition(self._h, float(dt))

    def post_step(self):
        self._L.oracle_post_step(self._h)

    def get_masks(self):
        nx, ny = self.nx, self.ny
        m = np.zeros(nx * ny, np.int8)
        mx = np.zeros((nx + 1) * ny, np.int8)
        my = np.zeros(nx * (ny + 1), np.int8)
        i8 = C.POINTER(C.c_int8)
        self._L.oracle_get_masks(self._h, m.ctypes.data_as(i8), mx.ctypes.data_as(i8),
                               my.ctypes.data_as(i8))
        return (m.reshape((nx, ny), order="F"), mx.reshape((nx + 1, ny), order="F"),
                my.reshape((nx, ny + 1), order="F"))

    def set_clock(self, t, dt0, t_end=1e300, t_output=-1.0):
        self._L.oracle_set_clock(self._h, float(t), float(dt0), float(t_end), float(t_output))

    def advance(self, n_steps):
        t = C.c_double(0.0)
        err = self._L.oracle_advance(self._h, int(n_steps), C.byref(t))
        return err, t.value

    def stats(self):
        s = ImexStats()
        self._L.oracle_stats(self._h, C.byref(s))
        return s

    def stale_wet_reads(self):
        return self._L.oracle_stale_wet_reads(self._h)

    def mass_budget(self):
        """Changes of SUM(q1) since set_state by cause: (border and inlet face
        fluxes, assembly fixes, erosion/deposition, face fluxes of the last
        step); multiply by dx*dy for mass."""
        out = np.zeros(4)
        self._L.oracle_mass_budget(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return tuple(float(x) for x in out)

    # the driver's output sweep
    def post_init(self, thickness_levels=(), dyn_pres_levels=()):
        from imex_sflow2d_v2_b200.abi import vulnerability_levels
        t, d = vulnerability_levels(thickness_levels, dyn_pres_levels)
        self._nt = len(t) * len(d)
        t = np.ascontiguousarray(t, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        self._L.oracle_post_init(self._h, len(t), _p(t), len(d), _p(d))

    def output_prep(self, cons, phys, esri):
        """(p2d (17+4ns, nx, ny), esr (2, nx, ny)) of output_solution, with its
        in-place changes to q, DEPOSIT and EROSION."""
        nx, ny, ns = self.nx, self.ny, self.ns
        p2d = np.zeros((17 + 4 * ns) * nx * ny)
        esr = np.zeros(2 * nx * ny)
        self._L.oracle_output_prep(self._h, int(cons), int(phys), int(esri), _p(p2d), _p(esr))
        return (p2d.reshape(17 + 4 * ns, ny, nx).transpose(0, 2, 1),
                esr.reshape(2, ny, nx).transpose(0, 2, 1))

    def post_diag(self):
        out = np.zeros(4)
        self._L.oracle_post_diag(self._h, _p(out))
        return tuple(out)

    def get_post(self):
        n = self.nx * self.ny
        a = [np.zeros(n) for _ in range(3)]
        v = np.zeros(max(self._nt, 1) * n, np.int8)
        self._L.oracle_get_post(self._h, _p(a[0]), _p(a[1]), _p(a[2]),
                              v.ctypes.data_as(C.POINTER(C.c_int8)))
        f = [x.reshape((self.nx, self.ny), order="F") for x in a]
        return f[0], f[1], f[2], v[:self._nt * n].reshape((self._nt, self.nx, self.ny), order="F")

    def topography_reconstruction(self):
        self._L.oracle_topography_reconstruction(self._h)

    def get_topo(self):
        """B_prime_x/y_geom, B_second_xx/xy/yy_geom, grav_coeff, d_grav_coeff_dx."""
        n = self.nx * self.ny
        a = [np.zeros(n) for _ in range(7)]
        self._L.oracle_get_topo(self._h, *[_p(x) for x in a])
        return [x.reshape((self.nx, self.ny), order="F") for x in a]

    # point functions
    def qc_to_qp(self, qc):
        qc = np.ascontiguousarray(qc, dtype=np.float64)
        out = np.zeros(self.nv + 2)
        self._L.oracle_qc_to_qp(self._h, _p(qc), _p(out))
        return out

    def qp_to_qc(self, qp):
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.zeros(self.nv)
        self._L.oracle_qp_to_qc(self._h, _p(qp), _p(out))
        return out

    def mixt_var(self, qp):
        """(Ri, rho_m, rho_c, red_grav) of one physical state."""
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.zeros(4)
        self._L.oracle_mixt_var(self._h, _p(qp), _p(out))
        return out

    def local_speeds(self, qp, gcf, d):
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.zeros(2)
        self._L.oracle_local_speeds(self._h, _p(qp), float(gcf), int(d), _p(out))
        return out

    def eval_fluxes(self, qc, qp, gcf, d):
        qc = np.ascontiguousarray(qc, dtype=np.float64)
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.zeros(self.nv)
        self._L.oracle_eval_fluxes(self._h, _p(qc), _p(qp), float(gcf), int(d), _p(out))
        return out

    def kt_interface(self, qcL, qpL, qcR, qpR, gcf, d):
        """(H, (a-, a+)) of one interface from its two face states."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (qcL, qpL, qcR, qpR)]
        H = np.zeros(self.nv)
        sp = np.zeros(2)
        self._L.oracle_kt_interface(self._h, *[_p(x) for x in a], float(gcf), int(d), _p(H),
                                    _p(sp))
        return H, sp

    def implicit_terms(self, q_re, q_im=None):
        q_re = np.ascontiguousarray(q_re, dtype=np.float64)
        q_im = None if q_im is None else np.ascontiguousarray(q_im, dtype=np.float64)
        re = np.zeros(self.nv)
        im = np.zeros(self.nv)
        self._L.oracle_implicit_terms(self._h, _p(q_re), _p(q_im) if q_im is not None else None,
                                    _p(re), _p(im))
        return re, im

    def solve_rk_step(self, qj, qj_old, rj, bx, by, dt, a_diag=1.0):
        qj = np.array(qj, dtype=np.float64)
        qo = np.ascontiguousarray(qj_old, dtype=np.float64)
        rj = np.ascontiguousarray(rj, dtype=np.float64)
        it = self._L.oracle_solve_rk_step(self._h, _p(qj), _p(qo), _p(rj), float(bx), float(by),
                                        float(dt), float(a_diag))
        return qj, it


def ipow(x, y):
    return lib().oracle_ipow(float(x), float(y))


def ipow_n(x, y):
    """x**y element by element (arrays of one shape)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(np.broadcast_to(y, x.shape), dtype=np.float64)
    out = np.empty_like(x)
    lib().oracle_ipow_n(x.size, _p(x), _p(y), _p(out))
    return out


def limit_n(v1, v2, v3, z1, z2, z3, limiter, theta=1.0):
    """limit() element by element (arrays broadcast to one shape)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64)
            for a in np.broadcast_arrays(v1, v2, v3, z1, z2, z3)]
    out = np.empty(arrs[0].shape)
    lib().oracle_limit_n(out.size, *[_p(a) for a in arrs], int(limiter), float(theta), _p(out))
    return out


def settling_velocity_n(diam, rhos, rhoc, ikv, grav):
    """settling_velocity element by element (arrays broadcast to one shape)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64)
            for a in np.broadcast_arrays(diam, rhos, rhoc, ikv)]
    out = np.empty(arrs[0].shape)
    lib().oracle_settling_velocity_n(out.size, *[_p(a) for a in arrs], float(grav), _p(out))
    return out


def limit(v1, v2, v3, z1, z2, z3, limiter, theta=1.0):
    return lib().oracle_limit(v1, v2, v3, z1, z2, z3, int(limiter), float(theta))


def setup_dem(z, xll, yll, cellsize, nodata, nx, ny, x0, y0, cell_size):
    """(B_cent, B_nodata, status) of init_grid's DEM sampling; z is (ncols, nrows)."""
    z = np.asfortranarray(z, dtype=np.float64)
    ncols, nrows = z.shape
    B = np.zeros((nx, ny), dtype=np.float64, order="F")
    N = np.zeros((nx, ny), dtype=np.int8, order="F")
    st = lib().oracle_setup_dem(ncols, nrows, xll, yll, cellsize, nodata, _p(z), nx, ny, x0, y0,
                                cell_size, _p(B), N.ctypes.data_as(C.POINTER(C.c_int8)))
    return B, N, st


def cell_fract(nx, ny, x0, y0, cell_size, xs, ys, rs, r2s, angle):
    out = np.zeros((nx, ny), dtype=np.float64, order="F")
    lib().oracle_cell_fract(nx, ny, x0, y0, cell_size, xs, ys, rs, r2s, angle, _p(out))
    return out


def regrid(fin, xll, yll, cellsize, nodata, nx, ny, x0, y0, cell_size):
    fin = np.asfortranarray(fin, dtype=np.float64)
    ncols, nrows = fin.shape
    out = np.zeros((nx, ny), dtype=np.float64, order="F")
    st = lib().oracle_regrid(ncols, nrows, xll, yll, cellsize, nodata, _p(fin), nx, ny, x0, y0,
                             cell_size, _p(out))
    return out, st
