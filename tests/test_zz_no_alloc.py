"""imex_gpu_timestep_noalloc against imex_gpu_timestep on the same states.

The allocation-free entry point must give the CFL dt of the ordinary one.
Both are folds of the same per-interface speeds with an exact minimum, so the
tolerance is zero: the two doubles are equal.  Each state is queried twice in
a row through the new entry point, and a second, smaller grid follows a
larger one so that tile minima left behind in the built-in scratch by the
first grid cannot leak into the second."""
import pytest

import cases
from imex_sflow2d_v2_b200.solver import ImexSolver

pytestmark = pytest.mark.gpu

DT_TOL = 0.0  # relative; exact minima of the same speeds


def _close(a, b):
    return abs(a - b) <= DT_TOL * max(abs(a), abs(b))


def _walk(p, st, q, nsteps):
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    t = 0.0
    seen = []
    for _ in range(nsteps):
        g.check_solve(t)
        d1 = g.timestep_noalloc()
        d2 = g.timestep_noalloc()
        d0 = g.timestep()
        assert _close(d1, d0), (d1, d0)
        assert _close(d2, d0), (d2, d0)
        seen.append(d0)
        g.imex_RK_solver(t, d0)
        t = t + d0
    return seen


def test_noalloc_dt_radial_then_dambreak():
    p, st, q = cases.radial(n=64)
    dts = _walk(p, st, q, 12)
    assert all(0.0 < d <= p.max_dt for d in dts)
    p, st, q = cases.dambreak(n=40)
    _walk(p, st, q, 12)


def test_noalloc_dt_fractal():
    p, st, q = cases.fractal_small()
    _walk(p, st, q, 6)


def test_noalloc_allocates_no_device_memory():
    """The entry point's defining property: once the first call on the
    device has resolved the scratch array's address (and the kernels are
    loaded), further calls leave the device's free memory unchanged."""
    import torch
    p, st, q = cases.radial(n=64)
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    g.check_solve(0.0)
    d0 = g.timestep()
    g.timestep_noalloc()
    g.sync()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        assert _close(g.timestep_noalloc(), d0)
    g.sync()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    g.close()


def test_noalloc_tile_limit_one_row_grids():
    """The built-in scratch holds one slot per 32x8 tile, 1,048,576 of them.
    A one-row grid of 32 * 1,048,576 cells needs exactly that many tiles: it
    is accepted and gives imex_gpu_timestep's dt (the fold then reduces the
    largest number of tile minima it takes).  One cell more needs one tile
    more and is rejected with IMEX_EINVAL, before any launch.  Each grid is
    a dam break along the row (33.5 M cells, about 9 GB on the device)."""
    import numpy as np
    from imex_sflow2d_v2_b200 import configs
    from imex_sflow2d_v2_b200.abi import IMEX_EINVAL
    from imex_sflow2d_v2_b200.solver import ImexError
    limit = 1 << 20
    for nx, fits in ((32 * limit, True), (32 * limit + 1, False)):
        p, st, q = configs.dambreak(nx=nx, ny=1, dx=0.05, x_split=nx * 0.05 * 0.5)
        g = ImexSolver(p, st)
        try:
            g.set_state(q, 0.0)
            del q, st
            g.check_solve(0.0)
            d0 = g.timestep()
            if fits:
                assert _close(g.timestep_noalloc(), d0)
                assert _close(g.timestep_noalloc(), d0)
            else:
                with pytest.raises(ImexError) as e:
                    g.timestep_noalloc()
                assert e.value.code == IMEX_EINVAL
                assert "1048577 tiles" in str(e.value), str(e.value)
            assert np.isfinite(d0) and d0 > 0.0
        finally:
            g.close()
