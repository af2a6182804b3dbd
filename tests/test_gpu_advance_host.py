"""imex_gpu_advance_host: one driver-loop pass from a host state to a host
state with the transfers overlapped by the step in row bands, against the
same pass taken as set_state, advance(1) and get_state.  Bit for bit: q,
the model time, the solve-cell and Newton counts, the reference checks and
the erosion/deposition planes, over consecutive steps (each step's input
is the previous output, as for a driver that keeps q on the host), on grids
of one to many bands, with the input and output in one array and in page-
locked memory."""
import numpy as np
import pytest
import torch

import cases
from imex_sflow2d_v2_b200 import configs
from imex_sflow2d_v2_b200.solver import ImexSolver

pytestmark = pytest.mark.gpu


def _stats(g):
    s = g.stats()
    return (s.solve_cells, s.newton_cells, s.newton_iters, s.lnsrch_trials, s.error_mask,
            s.first_error_code, s.first_error_j, s.first_error_k, s.dt, s.t)


def _compare(p, st, q, steps, pinned=False, same_array=False, exchange=False):
    a, b = ImexSolver(p, st), ImexSolver(p, st)
    for g in (a, b):
        g.set_clock(0.0, 1e-2)
    n = q.size
    qa = np.asarray(q, dtype=np.float64).ravel(order="F").copy()
    if pinned:
        buf = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        buf[:] = qa
        qb, out = buf, (buf if same_array else
                        torch.empty(n, dtype=torch.float64, pin_memory=True).numpy())
    else:
        qb = qa.copy()
        out = qb if same_array else np.empty(n)
    t = 0.0
    for step in range(steps):
        ra = a.set_state(qa, t)
        ra = a.advance(1)[0]
        ta = a.stats().t
        qa = a.get_state(out=np.empty(n))
        rb, qout, tb = b.advance_host(qb, t, out=out)
        assert tb == ta, step
        assert rb == ra, (step, ra, rb)
        assert np.array_equal(qout.view(np.uint64), qa.view(np.uint64)), step
        assert _stats(a) == _stats(b), step
        for ma, mb in zip(a.get_masks(), b.get_masks()):
            assert np.array_equal(ma, mb), step
        if exchange:
            for ea, eb in zip(a.get_exchange(), b.get_exchange()):
                assert np.array_equal(ea, eb), step
        qb = qout
        if not same_array:
            qb = qout.copy() if not pinned else qout
            if pinned:
                out = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        t = ta
    a.close()
    b.close()


def test_dambreak_many_bands():
    p, st, q = configs.dambreak()
    _compare(p, st, q, 20)


def test_fractal_inlet_erosion_pinned_same_array():
    p, st, q = configs.fractal_inlet(n=512, initial_layer=2.0)
    _compare(p, st, q, 8, pinned=True, same_array=True, exchange=True)


def test_radial_current_pinned():
    p, st, q = configs.radial_current(nx=256, ny=256)
    _compare(p, st, q, 30, pinned=True)


@pytest.mark.parametrize("case", ["one_row_60x1", "one_column_1x60", "single_cell_1x1",
                                  "tiny_3x5"])
def test_degenerate_grids(case):
    p, st, q = cases.edge_variants()[case]
    _compare(p, st, q, 5)


def test_ragged_band_rows():
    # 203 rows: 26 tile rows of 8 (the last one ragged) in bands of 1-2
    p, st, q = configs.dambreak(nx=97, ny=203)
    _compare(p, st, q, 10)
