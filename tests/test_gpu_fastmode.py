"""Fast mode (the library built with contracted multiply-adds) against the
oracle on the three workloads at their stated sizes.

Fast mode is not bit-exact: each fused multiply-add rounds once where the
reference rounds twice.  Its acceptance bound is the north star's: solve
masks equal bit for bit at every compared step, conserved variables within
relative L1 1e-10 of the oracle, the model time within a relative 1e-12.
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


def _advance_fast(p, st, q, total, chunk):
    o = Oracle(p, st)
    g = ImexSolver(p, st, fast=True)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.set_clock(0.0, 1e-2)
    done = 0
    worst = 0.0
    while done < total:
        n = min(chunk, total - done)
        _, to = o.advance(n)
        _, tg = g.advance(n)
        done += n
        assert abs(tg - to) <= T_TOL * to, (done, to, tg)
        for a, b in zip(o.get_masks(), g.get_masks()):
            assert np.array_equal(a, b), done
        r = rel_l1(o.get_state(), g.get_state())
        worst = max(worst, r)
        assert r <= REL_L1_TOL, (done, r)
        assert g.stats().error_mask == o.stats().error_mask == 0
    return worst


def test_fast_radial_current_1024_2000_steps():
    p, st, q = configs.radial_current()
    print("fast radial worst rel_l1", _advance_fast(p, st, q, 2000, 250))


def test_fast_fractal_inlet_512_60_steps():
    p, st, q = configs.fractal_inlet(n=512, initial_layer=2.0)
    print("fast fractal worst rel_l1", _advance_fast(p, st, q, 60, 10))
