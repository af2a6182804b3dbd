"""Ensemble advance (one CUDA graph over all members, forked over streams)
against each member advanced alone through its own context, and one member
against the oracle.  Members are independent, so the results must be bit
for bit those of the single runs whatever stream count the tuner picks."""
import numpy as np
import pytest

from imex_sflow2d_v2_b200 import configs
from imex_sflow2d_v2_b200.solver import ImexEnsemble, ImexSolver

pytestmark = pytest.mark.gpu

STEPS = 9   # more than the tuner's trial steps (1, 2, 4 streams for 5 members)


def _members():
    return configs.ensemble_members(n_members=5, side_min=40, side_max=72, seed=7)


def test_ensemble_equals_single_runs():
    mem = _members()
    ens = ImexEnsemble([(p, st) for p, st, q, s in mem])
    for m, (p, st, q, s) in enumerate(mem):
        ens.member(m).set_state(q, 0.0)
        ens.member(m).set_clock(0.0, 1e-2)
    # the reference's assembly checks may fire (e.g. T < 273 K at a thin
    # front); they must fire identically in the single runs
    ens.advance(4)
    ens.advance(STEPS - 4)
    k, tried = ens.tuning()
    assert k in (1, 2, 4) and len(tried) == 3
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
        g.close()
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
