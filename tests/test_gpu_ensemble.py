"""Ensemble advance against each member advanced alone through its own
context, and one member against the oracle, in both modes: batched (one
persistent kernel per phase for all members over device-built work lists,
the tile shape picked by the tuner) and per-member graphs forked over
streams (members that cannot share the batched kernels).  Members are
independent, so the results must be bit for bit those of the single runs
whatever tile shape or stream count the tuner picks."""
import numpy as np
import pytest

from imex_sflow2d_v2_b200 import configs
from imex_sflow2d_v2_b200.solver import ImexEnsemble, ImexSolver

pytestmark = pytest.mark.gpu

STEPS = 9   # more than the tuner's trial steps (3 tile shapes twice; 1, 2, 4 streams)
SHAPES = {(32, 8), (16, 16), (32, 4)}


def _members():
    return configs.ensemble_members(n_members=5, side_min=40, side_max=72, seed=7)


def _mixed_members():
    """Members with one and with two solid classes: no batched kernels."""
    mem = _members()[:3]
    for n in (36, 52):
        p, st, q = configs.radial_current(nx=n, ny=n + 7, dx=2.0, r_source=6.0, bump_sigma=20.0,
                                          mfr=4e5)
        mem.append((p, st, q, None))
    return mem


def _check_against_single_runs(mem, ens):
    for m, (p, st, q, s) in enumerate(mem):
        g = ImexSolver(p, st)
        g.set_state(q, 0.0)
        g.set_clock(0.0, 1e-2)
        g.advance(STEPS)
        np.testing.assert_array_equal(g.get_state(), ens.member(m).get_state())
        se, sg = ens.member(m).stats(), g.stats()
        assert se.t == sg.t and se.steps == sg.steps == STEPS
        assert se.solve_cells == sg.solve_cells
        assert (se.error_mask, se.first_error_code, se.first_error_j, se.first_error_k) == \
            (sg.error_mask, sg.first_error_code, sg.first_error_j, sg.first_error_k)
        assert (se.newton_cells, se.newton_iters, se.lnsrch_trials) == \
            (sg.newton_cells, sg.newton_iters, sg.lnsrch_trials)
        np.testing.assert_array_equal(g.get_masks()[0], ens.member(m).get_masks()[0])
        g.close()


def _run(mem):
    ens = ImexEnsemble([(p, st) for p, st, q, s in mem])
    for m, (p, st, q, s) in enumerate(mem):
        ens.member(m).set_state(q, 0.0)
        ens.member(m).set_clock(0.0, 1e-2)
    # the reference's assembly checks may fire (e.g. T < 273 K at a thin
    # front); they must fire identically in the single runs
    ens.advance(4)
    ens.advance(STEPS - 4)
    return ens


def test_batched_ensemble_equals_single_runs():
    mem = _members()
    ens = _run(mem)
    shape, tried = ens.tile_shape()
    assert shape in SHAPES and {s for s, ms in tried} == SHAPES and len(tried) == 6
    assert all(ms > 0.0 for s, ms in tried)
    _check_against_single_runs(mem, ens)
    ens.close()


def test_stream_ensemble_equals_single_runs():
    mem = _mixed_members()
    ens = _run(mem)
    assert ens.tile_shape()[0] == (0, 0)
    k, tried = ens.tuning()
    assert k in (1, 2, 4) and len(tried) == 3
    _check_against_single_runs(mem, ens)
    ens.close()


def test_ensemble_member_matches_oracle():
    from oracle import Oracle
    mem = _members()[:2]
    ens = ImexEnsemble([(p, st) for p, st, q, s in mem])
    for m, (p, st, q, s) in enumerate(mem):
        ens.member(m).set_state(q, 0.0)
        ens.member(m).set_clock(0.0, 1e-2)
    ens.advance(6)
    p, st, q, s = mem[1]
    o = Oracle(p, st, threads=4)
    o.set_state(q, 0.0)
    o.set_clock(0.0, 1e-2)
    for _ in range(6):
        o.advance(1)
    np.testing.assert_array_equal(o.get_state(), ens.member(1).get_state())
    ens.close()
