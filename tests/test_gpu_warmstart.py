"""Learned Newton warm start: pairs harvested from the solver, the network
trained by the library's kernels, stage 2 started from its guesses.  The
solves still end on the reference's own exit tests, so a warm-started step
equals the plain step to the solver's tolerance (relative L1 <= 1e-10 on q),
not bit for bit; a network that guesses badly costs iterations (and, if a
solve fails, a fallback to the plain start), not accuracy."""
import numpy as np
import pytest

import cases
from imex_sflow2d_v2_b200 import warmstart
from imex_sflow2d_v2_b200.solver import ImexMLP, ImexSolver
from parity import rel_l1

pytestmark = pytest.mark.gpu


def _developed(p, st, q, steps):
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    g.set_clock(0.0, 1e-2)
    g.advance(steps)
    return g


def _one_step(p, st, q, t, net):
    g = ImexSolver(p, st)
    g.set_state(q, t)
    g.set_clock(t, 1e-2)
    if net is not None:
        g.set_warmstart(net)
    g.advance(1)
    s = g.stats()
    out = g.get_state(), s.newton_iters / max(1, s.newton_cells), s.warm_fallback_cells
    g.close()
    return out


def test_harvest_train_and_warm_step_matches_plain():
    p, st, q = cases.fractal_small()
    g = _developed(p, st, q, 3)
    g.harvest_start(capacity=1 << 16, stride=1)
    g.advance(4)
    x, y = warmstart.harvested(g)
    assert x is not None and x.shape[0] > 1000 and x.shape[1] == 12
    net = ImexMLP(seed=2)
    n, losses = warmstart.train(net, g, epochs=8, batch=1024)
    assert losses[-1] < losses[0]
    g.harvest_stop()
    qs, t = g.get_state(), g.stats().t
    q_plain, it_plain, _ = _one_step(p, st, qs, t, None)
    q_warm, it_warm, fb = _one_step(p, st, qs, t, net)
    assert rel_l1(q_plain, q_warm) <= 1e-10
    assert np.isfinite(q_warm).all()
    print("iterations per Newton cell: plain %.3f learned %.3f fallback %d" % (it_plain, it_warm, fb))


def test_bad_network_costs_iterations_not_accuracy():
    p, st, q = cases.fractal_small()
    g = _developed(p, st, q, 3)
    qs, t = g.get_state(), g.stats().t
    net = ImexMLP(seed=3)
    net.set_params(net.params() * 50.0)          # wild guesses
    net.set_norm(np.zeros(12), np.ones(12), np.zeros(2), np.full(2, 10.0))
    q_plain, it_plain, _ = _one_step(p, st, qs, t, None)
    q_warm, it_warm, fb = _one_step(p, st, qs, t, net)
    assert np.isfinite(q_warm).all()
    assert rel_l1(q_plain, q_warm) <= 1e-8
    assert it_warm >= it_plain
