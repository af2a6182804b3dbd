"""output_solution from the device (imex_gpu_output): the .q_2d family,
.p_2d, the ESRI grids and _max.asc written by the library's host thread
equal, byte for byte, the files the test restatement builds from the
oracle's values; the writer's in-place changes (q, DEPOSIT, EROSION) keep
the two runs in lockstep afterwards."""
import os

import numpy as np
import pytest

import cases
import fortran_format as FF
from imex_sflow2d_v2_b200.solver import ImexSolver
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _expected(o, p, run, idx, post):
    nx, ny, ns = p.nx, p.ny, p.n_solid
    dx = p.cell_size if nx > 1 else 1.0
    dy = p.cell_size if ny > 1 else 1.0
    xc, yc = FF.comp(p.x0, dx, nx), FF.comp(p.y0, dy, ny)
    s = FF.lettera(idx - 1)
    files = {}
    _, esr = o.output_prep(cons=1, phys=0, esri=1)        # driver qp, then the q zeroing
    q = o.get_state()
    er, de, eo, B = o.get_exchange()
    files["%s_%s.q_2d" % (run, s)] = FF.columns_file(xc, yc, [q[i] for i in range(4 + ns)], 0)
    files["%s_erosion_%s.q_2d" % (run, s)] = FF.columns_file(xc, yc, [eo[:, :, i] for i in range(ns)], 0)
    files["%s_erodible_%s.q_2d" % (run, s)] = FF.columns_file(xc, yc, [er[i] for i in range(ns)], 0)
    files["%s_deposit_%s.q_2d" % (run, s)] = FF.columns_file(xc, yc, [de[:, :, i] for i in range(ns)], 0)
    files["%s_B_%s.q_2d" % (run, s)] = FF.columns_file(xc, yc, [B], 0)
    p2d, _ = o.output_prep(cons=0, phys=1, esri=0)        # .p_2d, zeroing DEPOSIT/EROSION
    files["%s_%s.p_2d" % (run, s)] = FF.columns_file(xc, yc, list(p2d), 1)
    _, de, eo, _ = o.get_exchange()
    h, T = esr
    esri = lambda g: FF.esri_file(nx, ny, p.x0, p.y0, p.cell_size, g)
    files["%s_%s.asc" % (run, s)] = esri(np.where(h >= 1e-5, h, -9999.0))
    files["%s_T_%s.asc" % (run, s)] = esri(np.where(h >= 1e-5, T, -9999.0))
    for i in range(ns):
        files["%s_dep_%s_%s.asc" % (run, FF.lettera(i + 1), s)] = esri(np.where(de[:, :, i] > 0, de[:, :, i], -9999.0))
        files["%s_ers_%s_%s.asc" % (run, FF.lettera(i + 1), s)] = esri(np.where(eo[:, :, i] > 0, eo[:, :, i], -9999.0))

    def tot(a):
        t = np.zeros((nx, ny))
        for i in range(ns):
            t = t + a[:, :, i]
        return t / (1.0 - p.erodible_porosity)
    dt_, et_ = tot(de), tot(eo)
    files["%s_depTot_%s.asc" % (run, s)] = esri(np.where(dt_ > 0, dt_, -9999.0))
    files["%s_ersTot_%s.asc" % (run, s)] = esri(np.where(et_ > 0, et_, -9999.0))
    hmax = post[0]
    files["%s_max.asc" % run] = esri(np.where(hmax >= 1e-5, hmax, -9999.0))
    return files


def test_output_files_and_lockstep(tmp_path):
    p, st, q = cases.fractal_topo(n=40)
    o = Oracle(p, st, threads=4)
    g = ImexSolver(p, st)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.set_clock(0.0, 1e-2)
        x.post_init((0.5,), ())
    for _ in range(6):
        o.advance(1)
    g.advance(6)
    run_g = os.path.join(str(tmp_path), "gpu")
    g.output(run_g, 3, cons=True, phys=True, esri=True, max_grid=True, threads=3)
    g.advance(2)                       # steps queue behind the output's copies
    g.output_wait()
    want = _expected(o, p, "oracle", 3, o.get_post())
    assert len(want) == 5 + 1 + 2 + 2 * p.n_solid + 2 + 1
    for name, text in want.items():
        path = os.path.join(str(tmp_path), name.replace("oracle", "gpu", 1))
        with open(path) as f:
            got = f.read()
        assert got == text, name
    for _ in range(2):
        o.advance(1)
    for _ in range(3):
        o.advance(1)
    g.advance(3)
    qo, qg = o.get_state(), g.get_state()
    assert np.array_equal(qo.view(np.int64), qg.view(np.int64))
    for a, b in zip(o.get_exchange(), g.get_exchange()):
        assert np.array_equal(a.view(np.int64), b.view(np.int64))


def test_output_without_post_and_errors(tmp_path):
    p, st, q = cases.dambreak(rheology=1)
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    run = os.path.join(str(tmp_path), "d")
    with pytest.raises(Exception):      # the _max grid needs the post-step planes
        g.output(run, 1, cons=False, phys=False, esri=False, max_grid=True)
    g.output(run, 1, cons=True, phys=True)
    g.output_wait()
    assert os.path.exists(run + "_0000.q_2d") and os.path.exists(run + "_0000.p_2d")
    g.output(os.path.join(str(tmp_path), "missing-dir", "x"), 2, cons=True, phys=False)
    with pytest.raises(Exception):      # the failed write is reported by the wait
        g.output_wait()
