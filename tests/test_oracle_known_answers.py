"""Known-answer tests of the CPU oracle (the reference ships no golden
outputs; these pin the restatement with analytic properties)."""
import numpy as np
import pytest

import cases
from imex_sflow2d_v2_b200 import configs
from oracle import Oracle, ipow, limit


def run_oracle(p, st, q, n, dt0=1e-3):
    o = Oracle(p, st, threads=4)
    o.set_state(q, 0.0)
    o.set_clock(0.0, dt0)
    err = 0
    for _ in range(n):
        e, t = o.advance(1)
        err |= e
    return o, err


def test_limiter_table():
    # minmod, superbee, generalised minmod, MC, centred, one-sided
    z = (0.0, 1.0, 2.0)
    assert limit(0, 1, 3, *z, 1) == 1.0
    assert limit(0, 1, 0.5, *z, 1) == 0.0
    assert limit(0, 1, 3, *z, 0) == 0.0
    assert limit(0, 1, 3, *z, 2) == 2.0       # maxmod(minmod(2,2), minmod(4,1))
    assert limit(0, 1, 3, *z, 3, theta=1.3) == 1.3
    assert limit(0, 1, 3, *z, 4) == 1.5       # minmod(1.5, 2*1)
    assert limit(0, 1, 3, *z, 5) == 1.5
    assert limit(0, 1, 3, *z, 6) == 2.0
    assert limit(0, 1, 3, *z, 7) == 1.0
    assert limit(3, 1, 0, *z, 1) == -1.0


def test_flat_rest_state_is_steady():
    p, st, q = configs.dambreak(nx=24, ny=24, dx=0.25, h_left=0.5, h_right=0.5)
    o, err = run_oracle(p, st, q, 10)
    assert err == 0
    np.testing.assert_array_equal(o.get_state(), q)


def test_mass_conserved_before_waves_reach_boundary():
    p, st, q = configs.dambreak(nx=60, ny=30, dx=0.25, h_left=1.0, h_right=0.0, x_split=7.5)
    _, xc, _, _ = configs.grid(p)
    q[:, xc < 5.0, :] = 0.0          # a column of fluid away from the walls
    m0 = q[0].sum()
    o, err = run_oracle(p, st, q, 25)
    qq = o.get_state()
    assert qq[0, 0].max() == 0.0 and qq[0, -1].max() == 0.0
    assert abs(qq[0].sum() / m0 - 1.0) < 1e-13
    assert abs(qq[4].sum() / q[4].sum() - 1.0) < 1e-13


def test_dam_break_is_symmetric_in_y():
    p, st, q = cases.dambreak(rheology=1)
    o, err = run_oracle(p, st, q, 20)
    qq = o.get_state()
    np.testing.assert_array_equal(qq[0], qq[0][:, ::-1])
    np.testing.assert_array_equal(qq[1], qq[1][:, ::-1])
    np.testing.assert_array_equal(qq[2], -qq[2][:, ::-1])


def test_qp_qc_round_trip():
    p, st, q = cases.radial()
    o = Oracle(p, st)
    rng = np.random.default_rng(3)
    for _ in range(50):
        h = rng.uniform(0.01, 5.0)
        qp = np.array([h, h * rng.normal(), h * rng.normal(), rng.uniform(300, 1000),
                       0.003 * h, 0.002 * h, 0.0, 0.0])
        qp[6], qp[7] = qp[1] / h, qp[2] / h
        qc = o.qp_to_qc(qp)
        back = o.qc_to_qp(qc)
        np.testing.assert_allclose(back, qp, rtol=1e-12, atol=1e-14)


def test_complex_step_matches_central_difference():
    p, st, q = cases.dambreak(rheology=1)
    o = Oracle(p, st)
    qc = o.qp_to_qc(np.array([0.8, 0.8 * 2.0, 0.8 * -1.0, 400.0, 0.008, 2.0, -1.0]))
    hstep = 5 * np.finfo(float).eps
    for col in (1, 2):
        im = np.zeros(5)
        im[col] = hstep * abs(qc[col])
        re, imag = o.implicit_terms(qc, im)
        d_cs = imag / (hstep * abs(qc[col]))
        d = 1e-6 * abs(qc[col])
        qa, qb = qc.copy(), qc.copy()
        qa[col] += d
        qb[col] -= d
        d_fd = (o.implicit_terms(qa)[0] - o.implicit_terms(qb)[0]) / (2 * d)
        np.testing.assert_allclose(d_cs[1:3], d_fd[1:3], rtol=1e-5)


def test_newton_converges_to_the_implicit_balance():
    p, st, q = cases.dambreak(rheology=1)
    o = Oracle(p, st)
    dt = 0.01
    qold = o.qp_to_qc(np.array([0.8, 0.8 * 3.0, 0.8 * 1.5, 400.0, 0.008, 3.0, 1.5]))
    rj = np.zeros(5)
    qj, it = o.solve_rk_step(qold.copy(), qold, rj, 0.0, 0.0, dt)
    assert 1 <= it < 100
    nh, _ = o.implicit_terms(qj)
    F = qj - qold + dt * (rj - nh)
    assert np.abs(F[1:3]).max() < 1e-9 * np.abs(qold[1:3]).max()
    # friction only decelerates, keeping the direction
    assert abs(qj[1]) < abs(qold[1]) and np.sign(qj[1]) == np.sign(qold[1])
    assert qj[1] / qj[2] == pytest.approx(qold[1] / qold[2], rel=1e-12)


def dilate_reference(q1, border=True):
    wet = q1 > 0
    m = wet.copy()
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = True
    for _ in range(2):
        t = m.copy()
        inner = t[1:-1, 1:-1] | t[:-2, 1:-1] | t[2:, 1:-1] | t[1:-1, :-2] | t[1:-1, 2:]
        m[1:-1, 1:-1] = inner
    return m


def test_check_solve_mask_is_two_fold_dilation():
    p, st, q = configs.dambreak(nx=50, ny=40, dx=0.25, h_left=1.0, h_right=0.0, x_split=4.0)
    o = Oracle(p, st)
    o.set_state(q, 0.0)
    o.check_solve(0.0)
    m, mx, my = o.get_masks()
    np.testing.assert_array_equal(m.astype(bool), dilate_reference(q[0]))
    np.testing.assert_array_equal(mx[1:-1].astype(bool), m[:-1].astype(bool) | m[1:].astype(bool))


def test_test2d_fixture_runs_clean():
    p, st, q = cases.test2d()
    o, err = run_oracle(p, st, q, 20, dt0=1e-4)
    assert err == 0
    s = o.stats()
    assert s.newton_cells > 0
    assert o.stale_wet_reads() == 0


def test_ipow_accuracy_and_special_values():
    from decimal import Decimal, getcontext
    import math
    getcontext().prec = 50
    rng = np.random.default_rng(5)
    for y in (0.687, 4.65, 2.4, 1.5, 0.5):
        for x in np.concatenate([rng.uniform(0, 1, 300), rng.uniform(1, 1e3, 300),
                                 10 ** rng.uniform(-10, 6, 300)]):
            exact = float(Decimal(float(x)) ** Decimal(y))
            assert abs(ipow(x, y) - exact) <= 1 * math.ulp(exact), (x, y)
    assert ipow(1.0, 1.5) == 1.0 and ipow(0.0, 0.5) == 0.0 and ipow(2.0, 0.0) == 1.0
    assert math.isnan(ipow(-1.0, 0.5)) and ipow(-1.0, 0.0) == 1.0


def test_topography_reconstruction_matches_numpy_stencils():
    """The oracle's topography_reconstruction (reference summation order)
    against the independent numpy stencils of configs.topography_geom and
    configs.slope_correction_planes, on a rough seeded bed."""
    p, st, q = configs.dambreak(nx=23, ny=17, dx=0.7, rheology=1)
    rng = np.random.default_rng(9)
    B = np.asfortranarray(rng.standard_normal((23, 17)) * 3.0 + np.arange(23)[:, None] * 0.4)
    st = dict(st)
    st["B_cent"] = B
    p.slope_correction_flag = 1
    geo = configs.topography_geom(B, 0.7, 0.7)
    st.update(configs.slope_correction_planes(geo))
    o = Oracle(p, st, threads=1)
    o.topography_reconstruction()
    bx, by, bxx, bxy, byy, gc, dgc = o.get_topo()
    ref = [geo["B_prime_x_geom"], geo["B_prime_y_geom"], geo["B_second_xx_geom"],
           geo["B_second_xy_geom"], geo["B_second_yy_geom"]]
    for a, b in zip((bx, by, bxx, bxy, byy), ref):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    sc = configs.slope_correction_planes(geo)
    np.testing.assert_allclose(gc, sc["grav_coeff"], rtol=1e-12)
    np.testing.assert_allclose(dgc, sc["d_grav_coeff_dx"], rtol=1e-10, atol=1e-14)
