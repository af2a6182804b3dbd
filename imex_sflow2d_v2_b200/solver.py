"""Host side of the B200 IMEX step: a thin ctypes layer over libimexgpu.so.

The class mirrors the reference's per-step routines (src/solver_2d.f90):
``check_solve`` (:666), ``timestep`` (:872), ``imex_RK_solver`` (:1021) and
``update_erosion_deposition_cell`` (:2380), plus ``advance`` for whole driver
loop passes (src/IMEX_SfloW2D.f90:337-389) executed on the device.  Arrays use
the reference's Fortran layouts: q(n_vars, nx, ny), qp(n_vars+2, nx, ny).

There is no CPU fallback: if the CUDA library cannot be loaded or no device
is present, construction raises.
"""
import ctypes as C
import os

import numpy as np

from .abi import (IMEX_OK, STATUS_NAMES, ImexOutputSpec, ImexParams, ImexPostDiag,
                  ImexStatic, ImexStats, make_static)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libimexgpu.so")
# fast mode: the same sources built with contracted multiply-adds; results
# differ from the exact mode (and the oracle) by rounding only
LIB_FAST_PATH = os.path.join(_HERE, "libimexgpu_fast.so")
_LIBS = {}


class ImexError(RuntimeError):
    def __init__(self, code, where, detail=""):
        self.code = code
        name = STATUS_NAMES.get(code, str(code))
        super().__init__("%s failed: %s %s" % (where, name, detail))


def load_library(path=None, fast=False):
    """Load libimexgpu.so, or libimexgpu_fast.so with `fast` (built by
    ``python -m imex_sflow2d_v2_b200.build``)."""
    if path is None:
        path = LIB_FAST_PATH if fast else LIB_PATH
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise RuntimeError("%s not found: build it with "
                           "`python -m imex_sflow2d_v2_b200.build`" % path)
    L = C.CDLL(path)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    i8p = C.POINTER(C.c_int8)
    i64p = C.POINTER(C.c_int64)
    sig = {
        "imex_gpu_create": ([C.POINTER(ImexParams), C.POINTER(ImexStatic), C.c_int,
                             C.POINTER(vp)], C.c_int),
        "imex_gpu_destroy": ([vp], C.c_int),
        "imex_gpu_set_state": ([vp, dp, C.c_double], C.c_int),
        "imex_gpu_get_state": ([vp, dp, dp], C.c_int),
        "imex_gpu_get_exchange": ([vp, dp, dp, dp, dp], C.c_int),
        "imex_gpu_check_solve": ([vp, C.c_double, C.c_int, i64p], C.c_int),
        "imex_gpu_timestep": ([vp, dp], C.c_int),
        "imex_gpu_timestep_noalloc": ([vp, dp], C.c_int),
        "imex_gpu_rk_step": ([vp, C.c_double, C.c_double], C.c_int),
        "imex_gpu_erosion_deposition": ([vp, C.c_double], C.c_int),
        "imex_gpu_get_masks": ([vp, i8p, i8p, i8p], C.c_int),
        "imex_gpu_set_clock": ([vp, C.c_double, C.c_double, C.c_double, C.c_double], C.c_int),
        "imex_gpu_advance": ([vp, C.c_int, C.c_int, dp], C.c_int),
        "imex_gpu_advance_host": ([vp, dp, C.c_double, dp, dp], C.c_int),
        "imex_gpu_stats": ([vp, C.POINTER(ImexStats), C.c_int], C.c_int),
        "imex_gpu_last_error": ([vp], C.c_char_p),
        "imex_gpu_sync": ([vp], C.c_int),
        "imex_gpu_device_state": ([vp, C.POINTER(dp), i64p], C.c_int),
        "imex_gpu_set_stream": ([vp, vp], C.c_int),
        "imex_gpu_profile": ([vp, C.c_int], C.c_int),
        "imex_gpu_kernel_times": ([vp, dp, i64p, C.c_int], C.c_int),
        "imex_gpu_measure_fp64_peak": ([C.c_int, dp], C.c_int),
        "imex_gpu_build_info": ([], C.c_char_p),
        "imex_gpu_point_eval": ([C.c_int, C.c_longlong, dp, dp, dp, dp, C.c_double, dp],
                                C.c_int),
        "imex_setup_dem": ([C.c_int, C.c_int, C.c_int] + [C.c_double] * 4 + [dp, C.c_int, C.c_int]
                           + [C.c_double] * 3 + [dp, i8p, C.POINTER(C.c_float)], C.c_int),
        "imex_setup_cell_fract": ([C.c_int, C.c_int, C.c_int] + [C.c_double] * 8
                                  + [dp, C.POINTER(C.c_float)], C.c_int),
        "imex_setup_regrid": ([C.c_int, C.c_int, C.c_int] + [C.c_double] * 4
                              + [dp, C.c_int, C.c_int] + [C.c_double] * 3
                              + [dp, C.POINTER(C.c_float)], C.c_int),
        "imex_setup_last_error": ([], C.c_char_p),
        "imex_gpu_output": ([vp, C.POINTER(ImexOutputSpec)], C.c_int),
        "imex_gpu_output_wait": ([vp], C.c_int),
        "imex_format_edit": ([C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_char_p,
                              C.c_int], C.c_int),
        "imex_gpu_post_init": ([vp, C.c_int, dp, C.c_int, dp], C.c_int),
        "imex_gpu_post_step": ([vp, C.POINTER(ImexPostDiag)], C.c_int),
        "imex_gpu_post_diag": ([vp, C.POINTER(ImexPostDiag)], C.c_int),
        "imex_gpu_get_post": ([vp, dp, dp, dp, i8p, C.POINTER(C.c_int)], C.c_int),
        "imex_mlp_create": ([C.c_int, C.c_uint64, C.POINTER(vp)], C.c_int),
        "imex_mlp_destroy": ([vp], C.c_int),
        "imex_mlp_get_params": ([vp, C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_set_params": ([vp, C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_set_norm": ([vp, C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_get_norm": ([vp, C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_predict": ([vp, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_loss_grad": ([vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64,
                                C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_train": ([vp, vp, vp, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64,
                            C.POINTER(C.c_float)], C.c_int),
        "imex_mlp_last_error": ([vp], C.c_char_p),
        "imex_gpu_set_warmstart": ([vp, vp], C.c_int),
        "imex_gpu_harvest_start": ([vp, C.c_int64, C.c_int], C.c_int),
        "imex_gpu_harvest_stop": ([vp], C.c_int),
        "imex_gpu_harvest_data": ([vp, C.POINTER(vp), C.POINTER(vp), i64p], C.c_int),
        "imex_gpu_ensemble_create": ([C.c_int, C.POINTER(C.POINTER(ImexParams)),
                                      C.POINTER(C.POINTER(ImexStatic)), C.c_int,
                                      C.POINTER(vp)], C.c_int),
        "imex_gpu_ensemble_destroy": ([vp], C.c_int),
        "imex_gpu_ensemble_member": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
        "imex_gpu_ensemble_advance": ([vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "imex_gpu_ensemble_tuning": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int],
                                     C.c_int),
        "imex_gpu_ensemble_set_mode": ([vp, C.c_int], C.c_int),
        "imex_gpu_ensemble_tile_shape": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int],
                                         C.c_int),
        "imex_gpu_ensemble_last_error": ([vp], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIBS[path] = L
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def measure_fp64_peak(device=-1):
    """GFLOP/s of an FP64 FMA-chain kernel on the current device."""
    L = load_library()
    g = C.c_double(0.0)
    rc = L.imex_gpu_measure_fp64_peak(int(device), C.byref(g))
    if rc != IMEX_OK:
        raise ImexError(rc, "imex_gpu_measure_fp64_peak")
    return g.value


class ImexSolver:
    """One device context holding the state of one run.  `fast` selects the
    library built with contracted multiply-adds (results equal the exact
    mode's to rounding, not bit for bit)."""

    def __init__(self, params, static_arrays, device=-1, _handle=None, fast=False):
        self.lib = load_library(fast=fast)
        self.params = params
        self.nx, self.ny, self.ns = params.nx, params.ny, params.n_solid
        self.nv = 4 + self.ns
        self._owned = _handle is None
        if _handle is not None:        # a member context owned by an ImexEnsemble
            self._keep = []
            self._h = _handle
            return
        st, self._keep = make_static(static_arrays)
        h = C.c_void_p()
        rc = self.lib.imex_gpu_create(C.byref(params), C.byref(st), int(device), C.byref(h))
        if rc != IMEX_OK:
            raise ImexError(rc, "imex_gpu_create")
        self._h = h

    def _check(self, rc, where):
        if rc != IMEX_OK and rc > 6:
            raise ImexError(rc, where, self.lib.imex_gpu_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self.lib.imex_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state
    def set_state(self, q, t=0.0):
        """q: (n_vars,nx,ny) array, or a flat float64 array already in Fortran
        element order (used as is, e.g. a pinned host buffer)."""
        if not (isinstance(q, np.ndarray) and q.ndim == 1 and q.dtype == np.float64
                and q.flags.c_contiguous):
            q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel(order="F"))
        return self._check(self.lib.imex_gpu_set_state(self._h, _p(q), float(t)), "set_state")

    def get_state(self, with_qp=False, out=None):
        """Returns q (n_vars,nx,ny); with `out` (flat float64, n_vars*nx*ny
        elements) the state is written there and `out` is returned."""
        n = self.nx * self.ny
        if out is not None and not with_qp:
            self._check(self.lib.imex_gpu_get_state(self._h, _p(out), None), "get_state")
            return out
        q = np.zeros(self.nv * n)
        qp = np.zeros((self.nv + 2) * n) if with_qp else None
        self._check(self.lib.imex_gpu_get_state(self._h, _p(q), _p(qp) if with_qp else None),
                    "get_state")
        q = q.reshape((self.nv, self.nx, self.ny), order="F")
        if with_qp:
            return q, qp.reshape((self.nv + 2, self.nx, self.ny), order="F")
        return q

    def get_exchange(self):
        n = self.nx * self.ny
        er, de, eo, B = (np.zeros(self.ns * n), np.zeros(self.ns * n),
                         np.zeros(self.ns * n), np.zeros(n))
        self._check(self.lib.imex_gpu_get_exchange(self._h, _p(er), _p(de), _p(eo), _p(B)),
                    "get_exchange")
        return (er.reshape((self.ns, self.nx, self.ny), order="F"),
                de.reshape((self.nx, self.ny, self.ns), order="F"),
                eo.reshape((self.nx, self.ny, self.ns), order="F"),
                B.reshape((self.nx, self.ny), order="F"))

    # -- the reference's routines
    def check_solve(self, t, solve_all=False):
        n = C.c_int64(0)
        self._check(self.lib.imex_gpu_check_solve(self._h, float(t), int(solve_all), C.byref(n)),
                    "check_solve")
        return n.value

    def timestep(self):
        dt = C.c_double(0.0)
        self._check(self.lib.imex_gpu_timestep(self._h, C.byref(dt)), "timestep")
        return dt.value

    # -- the driver's output sweep (src/IMEX_SfloW2D.f90:253-309, 391-485)
    def post_init(self, thickness_levels=(), dyn_pres_levels=()):
        """First output sweep with the VULNERABILITY_TABLE_PARAMETERS levels;
        afterwards advance() sweeps after every step."""
        tl = np.ascontiguousarray(thickness_levels, dtype=np.float64)
        pl = np.ascontiguousarray(dyn_pres_levels, dtype=np.float64)
        return self._check(self.lib.imex_gpu_post_init(self._h, len(tl), _p(tl), len(pl), _p(pl)),
                           "post_init")

    def post_step(self, diag=True):
        """The sweep after one step taken with the per-routine calls; returns
        the print values (mass, volume, area, solid_mass) when `diag`."""
        d = ImexPostDiag()
        self._check(self.lib.imex_gpu_post_step(self._h, C.byref(d) if diag else None),
                    "post_step")
        return (d.mass, d.volume, d.area, d.solid_mass) if diag else None

    # -- output_solution (src/inpout_2d.f90:5683-6180) from the device state
    def output(self, run_name, output_idx, time=0.0, cons=True, phys=True, esri=False,
               max_grid=False, threads=0):
        """Write the reference's output files for output number `output_idx`
        (files carry lettera(output_idx-1)) asynchronously: the call returns
        once the values are queued on the device; output_wait() waits for the
        files.  Like the reference, cons sets |q| < 1e-20 to 0 in the state
        and phys sets DEPOSIT/EROSION below 1e-20 to 0."""
        spec = ImexOutputSpec(str(run_name).encode(), int(output_idx), float(time), int(cons),
                              int(phys), int(esri), int(max_grid), int(threads))
        self._check(self.lib.imex_gpu_output(self._h, C.byref(spec)), "output")

    def output_wait(self):
        self._check(self.lib.imex_gpu_output_wait(self._h), "output_wait")

    def post_diag(self):
        d = ImexPostDiag()
        self._check(self.lib.imex_gpu_post_diag(self._h, C.byref(d)), "post_diag")
        return d.mass, d.volume, d.area, d.solid_mass

    def get_post(self):
        """(hmax, pdynmax, mod_vel_max) as (nx,ny) arrays and vuln_table as
        (n_table,nx,ny) 0/1 bytes."""
        n = self.nx * self.ny
        a = [np.zeros(n) for _ in range(3)]
        nt = C.c_int(0)
        self._check(self.lib.imex_gpu_get_post(self._h, None, None, None, None, C.byref(nt)),
                    "get_post")
        v = np.zeros(max(nt.value, 1) * n, np.int8)
        self._check(self.lib.imex_gpu_get_post(self._h, _p(a[0]), _p(a[1]), _p(a[2]),
                                               v.ctypes.data_as(C.POINTER(C.c_int8)),
                                               C.byref(nt)), "get_post")
        f = [x.reshape((self.nx, self.ny), order="F") for x in a]
        return f[0], f[1], f[2], v[:nt.value * n].reshape((nt.value, self.nx, self.ny), order="F")

    # -- learned Newton warm start
    def set_warmstart(self, net):
        """Start stage 2's Newton solves from `net`'s guess (an ImexMLP), or
        from q_si again with None."""
        return self._check(self.lib.imex_gpu_set_warmstart(self._h, net._h if net else None),
                           "set_warmstart")

    def harvest_start(self, capacity, stride=1):
        return self._check(self.lib.imex_gpu_harvest_start(self._h, int(capacity), int(stride)),
                           "harvest_start")

    def harvest_stop(self):
        return self._check(self.lib.imex_gpu_harvest_stop(self._h), "harvest_stop")

    def harvest_data(self):
        """(x device pointer, y device pointer, pairs): float32 rows of 12 and 2."""
        x, y = C.c_void_p(), C.c_void_p()
        n = C.c_int64(0)
        self._check(self.lib.imex_gpu_harvest_data(self._h, C.byref(x), C.byref(y), C.byref(n)),
                    "harvest_data")
        return x.value, y.value, n.value

    def timestep_noalloc(self):
        """CFL dt like timestep(), through the entry point that allocates
        nothing (its scratch is a fixed array inside the library)."""
        dt = C.c_double(0.0)
        self._check(self.lib.imex_gpu_timestep_noalloc(self._h, C.byref(dt)), "timestep_noalloc")
        return dt.value

    def imex_RK_solver(self, t, dt):
        return self._check(self.lib.imex_gpu_rk_step(self._h, float(t), float(dt)), "rk_step")

    def update_erosion_deposition_cell(self, dt):
        return self._check(self.lib.imex_gpu_erosion_deposition(self._h, float(dt)),
                           "erosion_deposition")

    def get_masks(self):
        nx, ny = self.nx, self.ny
        m = np.zeros(nx * ny, np.int8)
        mx = np.zeros((nx + 1) * ny, np.int8)
        my = np.zeros(nx * (ny + 1), np.int8)
        i8 = C.POINTER(C.c_int8)
        self._check(self.lib.imex_gpu_get_masks(self._h, m.ctypes.data_as(i8),
                                                mx.ctypes.data_as(i8), my.ctypes.data_as(i8)),
                    "get_masks")
        return (m.reshape((nx, ny), order="F"), mx.reshape((nx + 1, ny), order="F"),
                my.reshape((nx, ny + 1), order="F"))

    # -- driver loop on the device
    def set_clock(self, t, dt0, t_end=1e300, t_output=-1.0):
        return self._check(self.lib.imex_gpu_set_clock(self._h, float(t), float(dt0),
                                                       float(t_end), float(t_output)),
                           "set_clock")

    def advance(self, n_steps, use_graph=False):
        t = C.c_double(0.0)
        rc = self._check(self.lib.imex_gpu_advance(self._h, int(n_steps), int(bool(use_graph)),
                                                   C.byref(t)), "advance")
        return rc, t.value

    def advance_host(self, q, t, out=None):
        """One driver-loop pass from the host state q at time t to the host
        state after it (imex_gpu_advance_host: the same result as set_state,
        advance(1) and get_state, with the transfers overlapped by the step).
        q and `out` as for set_state/get_state (flat float64 arrays in
        Fortran element order are used as they are; they may be the same
        array).  Returns (status, q after the step, t after the step)."""
        if not (isinstance(q, np.ndarray) and q.ndim == 1 and q.dtype == np.float64
                and q.flags.c_contiguous):
            q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel(order="F"))
        shaped = out is None
        if out is None:
            out = np.empty(self.nv * self.nx * self.ny)
        tt = C.c_double(0.0)
        rc = self._check(self.lib.imex_gpu_advance_host(self._h, _p(q), float(t), _p(out),
                                                        C.byref(tt)), "advance_host")
        if shaped:
            out = out.reshape((self.nv, self.nx, self.ny), order="F")
        return rc, out, tt.value

    def stats(self, reset_errors=False):
        s = ImexStats()
        self._check(self.lib.imex_gpu_stats(self._h, C.byref(s), int(reset_errors)), "stats")
        return s

    def sync(self):
        return self._check(self.lib.imex_gpu_sync(self._h), "sync")

    def set_stream(self, stream_handle):
        """Run on a caller's cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); 0/None = own stream."""
        return self._check(self.lib.imex_gpu_set_stream(self._h, C.c_void_p(stream_handle or None)),
                           "set_stream")

    KERNELS = ("mask", "flux", "stage2_first", "stage2_iter", "stage2_post", "erosion")

    def profile(self, enable=True):
        return self._check(self.lib.imex_gpu_profile(self._h, int(bool(enable))), "profile")

    def kernel_times(self):
        """{kernel: (total_ms, launches)} since the last call (profile on)."""
        nk = len(self.KERNELS)
        ms = (C.c_double * nk)()
        n = (C.c_int64 * nk)()
        self._check(self.lib.imex_gpu_kernel_times(self._h, ms, n, nk), "kernel_times")
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNELS)}

    def device_state(self):
        p = C.POINTER(C.c_double)()
        pitch = C.c_int64(0)
        self._check(self.lib.imex_gpu_device_state(self._h, C.byref(p), C.byref(pitch)),
                    "device_state")
        return C.cast(p, C.c_void_p).value, pitch.value


class ImexEnsemble:
    """Independent runs (members) advanced together on one GPU: batched (every
    phase one persistent kernel for all members, the step one CUDA graph),
    or through per-member graphs forked over streams when the members cannot
    share the batched kernels (the reference runs one process per member,
    EXAMPLES/EXAMPLE_ENSEMBLE_ETNA/launch_jobs.py).  `members` is a list of
    (params, static_arrays); member m's context is ``self.member(m)`` (an
    ImexSolver view for set_state, set_clock, get_state, stats ...)."""

    def __init__(self, members, device=-1):
        self.lib = load_library()
        n = len(members)
        self._keep = []
        P = (C.POINTER(ImexParams) * n)()
        S = (C.POINTER(ImexStatic) * n)()
        for m, (params, static_arrays) in enumerate(members):
            st, keep = make_static(static_arrays)
            self._keep.append((params, st, keep))
            P[m] = C.pointer(params)
            S[m] = C.pointer(st)
        h = C.c_void_p()
        rc = self.lib.imex_gpu_ensemble_create(n, P, S, int(device), C.byref(h))
        if rc != IMEX_OK:
            raise ImexError(rc, "imex_gpu_ensemble_create")
        self._h = h
        self._views = []
        for m, (params, _) in enumerate(members):
            ch = C.c_void_p()
            self.lib.imex_gpu_ensemble_member(self._h, m, C.byref(ch))
            self._views.append(ImexSolver(params, None, _handle=ch))

    def __len__(self):
        return len(self._views)

    def member(self, m):
        return self._views[m]

    def advance(self, n_steps):
        """n_steps driver-loop passes of every member; returns (status, first
        member with a non-zero status or -1)."""
        bad = C.c_int(-1)
        rc = self.lib.imex_gpu_ensemble_advance(self._h, int(n_steps), C.byref(bad))
        if rc > 6:
            raise ImexError(rc, "imex_gpu_ensemble_advance",
                            self.lib.imex_gpu_ensemble_last_error(self._h).decode())
        return rc, bad.value

    def tuning(self):
        """(chosen stream count, [(candidate, ms of its timed step), ...])."""
        k = C.c_int(0)
        n = C.c_int(0)
        tk = (C.c_int * 16)()
        tm = (C.c_float * 16)()
        self.lib.imex_gpu_ensemble_tuning(self._h, C.byref(k), C.byref(n), tk, tm, 16)
        return k.value, [(tk[i], tm[i]) for i in range(min(n.value, 16))]

    def set_mode(self, per_member_graphs=False):
        """Per-member graphs over streams even when the members could be
        batched (per_member_graphs=True), or batched when possible."""
        rc = self.lib.imex_gpu_ensemble_set_mode(self._h, 2 if per_member_graphs else 0)
        if rc != 0:
            raise ImexError(rc, "imex_gpu_ensemble_set_mode")

    def tile_shape(self):
        """Batched mode: ((tx, ty) chosen, [((tx, ty), ms of its timed step),
        ...]); ((0, 0), []) when the members advance through per-member
        graphs."""
        tx, ty, n = C.c_int(0), C.c_int(0), C.c_int(0)
        ax = (C.c_int * 8)()
        ay = (C.c_int * 8)()
        ms = (C.c_float * 8)()
        self.lib.imex_gpu_ensemble_tile_shape(self._h, C.byref(tx), C.byref(ty), C.byref(n), ax,
                                              ay, ms, 8)
        return (tx.value, ty.value), [((ax[i], ay[i]), ms[i]) for i in range(min(n.value, 8))]

    def close(self):
        if getattr(self, "_h", None):
            for v in self._views:
                v._h = None
            self.lib.imex_gpu_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class ImexMLP:
    """The warm-start network (12 -> 64 -> 64 -> 64 -> 2, SiLU; BF16 weights on
    tensor cores, FP32 accumulate) with its training kernels."""

    N_IN, N_OUT = 12, 2
    NPARAM = 16 * 64 + 64 + 2 * (64 * 64 + 64) + 64 * 8 + 8

    def __init__(self, seed=1, device=-1):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.imex_mlp_create(int(device), int(seed), C.byref(h))
        if rc != IMEX_OK:
            raise ImexError(rc, "imex_mlp_create")
        self._h = h

    def _check(self, rc, where):
        if rc != IMEX_OK:
            raise ImexError(rc, where, self.lib.imex_mlp_last_error(self._h).decode())

    def params(self):
        out = np.zeros(self.NPARAM, np.float32)
        self._check(self.lib.imex_mlp_get_params(self._h, _fp(out)), "get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.imex_mlp_set_params(self._h, _fp(p)), "set_params")

    def set_norm(self, x_mean, x_std, y_mean, y_std):
        n = np.ascontiguousarray(np.concatenate([x_mean, x_std, y_mean, y_std]), np.float32)
        self._check(self.lib.imex_mlp_set_norm(self._h, _fp(n)), "set_norm")

    def norm(self):
        n = np.zeros(2 * self.N_IN + 2 * self.N_OUT, np.float32)
        self._check(self.lib.imex_mlp_get_norm(self._h, _fp(n)), "get_norm")
        return n

    def predict(self, x):
        """Normalised inputs (n, 12) -> normalised outputs (n, 2)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.N_OUT), np.float32)
        self._check(self.lib.imex_mlp_predict(self._h, _fp(x), x.shape[0], _fp(y)), "predict")
        return y

    def loss_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(self.NPARAM, np.float32)
        loss = C.c_float(0.0)
        self._check(self.lib.imex_mlp_loss_grad(self._h, _fp(x), _fp(y), x.shape[0],
                                                C.byref(loss), _fp(g)), "loss_grad")
        return loss.value, g

    def train(self, x_dev, y_dev, n, epochs=4, batch=4096, lr=1e-3, seed=7):
        """Adam over a device-resident set (pointers to normalised float32
        rows); returns the per-epoch mean squared error."""
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(self.lib.imex_mlp_train(self._h, x_dev, y_dev, int(n), int(epochs),
                                            int(batch), float(lr), int(seed), _fp(losses)),
                    "train")
        return losses[:epochs]

    def close(self):
        if getattr(self, "_h", None):
            self.lib.imex_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def format_edit(kind, value, w, d=0, e=0):
    """One value through the output writers' Fortran edit descriptors:
    kind 0 = Ew.d, 1 = ESw.dEe, 2 = Iw, 3 = Fw.d (host code; no GPU)."""
    L = load_library()
    buf = C.create_string_buffer(128)
    n = L.imex_format_edit(int(kind), float(value), int(w), int(d), int(e), buf, 128)
    if n < 0:
        raise ValueError("imex_format_edit: bad arguments")
    return buf.value.decode()


def point_eval(fn, a, b, c=None, d=None, g=0.0, fast=False):
    """The device's point functions on host arrays (imex_gpu_point_eval):
    fn "ipow" gives a**b, fn "settling" settling_velocity(a, b, c, d) with
    gravity g, "minmod_uniform" the minmod slope of a, b, c at centres 0, d,
    2d by the flux kernel's equal-spacing path, "limit" limit() at those
    centres with limiter g, "quotient_below" 1.0 where a/b < c as the
    kernels evaluate it, else 0.0.  Arrays are broadcast to one shape."""
    code = {"ipow": 0, "settling": 1, "minmod_uniform": 2, "limit": 3, "quotient_below": 4}[fn]
    arrs = [np.ascontiguousarray(x, dtype=np.float64)
            for x in np.broadcast_arrays(a, b, *(() if code == 0 else (c, d)))]
    while len(arrs) < 4:
        arrs.append(arrs[0])
    out = np.empty(arrs[0].shape)
    L = load_library(fast=fast)
    p = [x.ctypes.data_as(C.POINTER(C.c_double)) for x in arrs]
    rc = L.imex_gpu_point_eval(code, out.size, *p, float(g),
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise ImexError(rc, "point_eval")
    return out
