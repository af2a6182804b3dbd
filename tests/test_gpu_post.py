"""The driver's output sweep on the device (imex_gpu_post_*) against the
oracle's restatement of src/IMEX_SfloW2D.f90:253-309 and 391-485: running
maxima and the vulnerability table bit for bit after every step, the print
values (mass, volume, area, solid mass) within 1e-12 relative (the device
sums in a different order than Fortran's SUM; the area count is exact)."""
import numpy as np
import pytest

import cases
from imex_sflow2d_v2_b200.solver import ImexSolver
from oracle import Oracle

pytestmark = pytest.mark.gpu

THK = (0.05, 0.2, 0.5)
PDYN = (1.0, 50.0, 500.0, 5000.0)


def _close(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(abs(a), abs(b), 1e-300)


def _check(o, g):
    for a, b in zip(o.get_post(), g.get_post()):
        np.testing.assert_array_equal(a, b)
    do, dg = o.post_diag(), g.post_diag()
    assert do[2] == dg[2]
    for a, b in zip(do, dg):
        assert _close(a, b), (do, dg)


@pytest.mark.parametrize("case", ["radial", "dambreak"])
def test_post_sweep_stepwise(case):
    p, st, q = cases.radial(n=48) if case == "radial" else cases.dambreak(rheology=1)
    o = Oracle(p, st, threads=4)
    g = ImexSolver(p, st)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.post_init(THK, PDYN)
    _check(o, g)
    t = 0.0
    for step in range(15):
        o.check_solve(t)
        g.check_solve(t)
        dt = o.timestep()
        g.timestep()
        o.rk_step(t, dt)
        g.imex_RK_solver(t, dt)
        o.post_step()
        g.post_step(diag=False)
        t = t + dt
        _check(o, g)
    h, pd, mv, vuln = g.get_post()
    assert h.max() > 0 and vuln.shape[0] == len(THK) * len(PDYN) and vuln.any()


def test_post_sweep_in_advance_and_graph():
    p, st, q = cases.fractal_small()
    o = Oracle(p, st, threads=4)
    g = ImexSolver(p, st)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.set_clock(0.0, 1e-2)
    o.post_init((0.5,), ())         # pressure levels default to a single 0
    g.post_init((0.5,), ())
    for _ in range(5):
        o.advance(1)
    g.advance(5)
    _check(o, g)
    for _ in range(5):
        o.advance(1)
    rc, _ = g.advance(5, use_graph=True)   # the captured step holds the sweep too
    assert rc == 0
    _check(o, g)
