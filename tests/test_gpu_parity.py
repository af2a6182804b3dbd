"""Parity of the sm_100a path with the CPU oracle, through the C ABI.

Bit-exact where the arithmetic is +,-,*,/,sqrt (the dam-break, inlet and
slope cases): solve masks, CFL dt and every conserved variable equal bit for
bit after every step.  Cases that evaluate pow() (settling velocity, hindered
settling, entrainment) compare within relative L1 <= 1e-10, the tolerance the
rebuild is held to; their masks must still match exactly."""
import numpy as np
import pytest

import cases
from parity import lockstep, rel_l1

pytestmark = pytest.mark.gpu

VARIANTS = cases.dambreak_variants()


def assert_bitexact(recs, allow_errors=False):
    for r in recs:
        assert r["stale"] == 0, r
        assert r["cells"][0] == r["cells"][1], r
        assert r["mask_equal"], r
        assert r["dt"][0] == r["dt"][1], r
        assert r["q_equal"], r
        # the reference's checks fire identically on both sides
        assert r["err"][0] == r["err"][1], r
        if not allow_errors:
            assert r["err"][0][0] == 0, r


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_dambreak_variants_bitexact(name):
    p, st, q = VARIANTS[name]
    recs, o, g = lockstep(p, st, q, 25)
    assert_bitexact(recs)
    s_o, s_g = o.stats(), g.stats()
    assert (s_o.newton_cells, s_o.newton_iters, s_o.lnsrch_trials) == \
        (s_g.newton_cells, s_g.newton_iters, s_g.lnsrch_trials)


def test_radial_inlet_bitexact():
    p, st, q = cases.radial()
    recs, o, g = lockstep(p, st, q, 40)
    assert_bitexact(recs)


@pytest.mark.parametrize("rheology", [1, 6])
def test_slope_and_curvature_bitexact(rheology):
    p, st, q = cases.sloped(rheology=rheology)
    recs, o, g = lockstep(p, st, q, 30)
    # the raw CFL step on this steep-fronted slab drives a few cells below
    # h = -1e-7 (the reference's print-and-continue checks): both sides
    # report the same checks at the same first cell and carry on identically
    assert_bitexact(recs, allow_errors=True)


def test_reference_test2d_within_tolerance():
    p, st, q = cases.test2d()
    recs, o, g = lockstep(p, st, q, 60, erosion=True)
    for r in recs:
        assert r["mask_equal"], r
        assert r["rel_l1"] <= 1e-10, r
        assert r["dt"][1] == pytest.approx(r["dt"][0], rel=1e-10)
    er_o, de_o, eo_o, _ = o.get_exchange()
    er_g, de_g, eo_g, _ = g.get_exchange()
    assert rel_l1(de_o, de_g) <= 1e-10


def test_fractal_erosion_through_advance():
    p, st, q = cases.fractal_small()
    from imex_sflow2d_v2_b200.solver import ImexSolver
    from oracle import Oracle
    o = Oracle(p, st, threads=8)
    o.set_state(q, 0.0)
    o.set_clock(0.0, 1e-2)
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    g.set_clock(0.0, 1e-2)
    for step in range(40):
        eo, to = o.advance(1)
        eg, tg = g.advance(1)
        assert tg == pytest.approx(to, rel=1e-12)
        qo, qg = o.get_state(), g.get_state()
        assert rel_l1(qo, qg) <= 1e-10, step
    er_o, de_o, eo_o, _ = o.get_exchange()
    er_g, de_g, eo_g, _ = g.get_exchange()
    assert rel_l1(er_o, er_g) <= 1e-10
    assert rel_l1(de_o, de_g) <= 1e-10
    assert rel_l1(eo_o, eo_g) <= 1e-10


def test_advance_graph_equals_stepwise():
    from imex_sflow2d_v2_b200.solver import ImexSolver
    p, st, q = cases.radial()
    runs = []
    for use_graph in (False, True):
        g = ImexSolver(p, st)
        g.set_state(q, 0.0)
        g.set_clock(0.0, 1e-3)
        rc, t = g.advance(30, use_graph=use_graph)
        runs.append((g.get_state(), t, rc))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_error_codes_report_first_bad_cell():
    from imex_sflow2d_v2_b200 import abi
    from imex_sflow2d_v2_b200.solver import ImexSolver
    p, st, q = cases.dambreak(rheology=1)
    q = q.copy()
    q[:, 10, 12] = 0.0
    q[0, 10, 12] = -1.0e-3          # h below -1e-7: IMEX_ENEGH, state kept
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    t = 0.0
    g.check_solve(t)
    dt = g.timestep()
    rc = g.imex_RK_solver(t, dt)
    assert rc == abi.IMEX_ENEGH
    s = g.stats()
    assert s.error_mask & abi.errbit(abi.IMEX_ENEGH)
    assert (s.first_error_j, s.first_error_k) == (11, 13)


def test_repeat_runs_are_bit_identical():
    from imex_sflow2d_v2_b200.solver import ImexSolver
    p, st, q = cases.fractal_small()
    out = []
    for _ in range(2):
        g = ImexSolver(p, st)
        g.set_state(q, 0.0)
        g.set_clock(0.0, 1e-2)
        g.advance(20, use_graph=True)
        out.append(g.get_state())
    np.testing.assert_array_equal(out[0], out[1])
