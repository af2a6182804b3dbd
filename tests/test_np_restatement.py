"""The oracle's point functions against a second, independent numpy
restatement of the Fortran (tests/np_restate.py) on seeded random states:
bit for bit.  This pins the oracle's reading of the reference independently
of the oracle's own code, for every state variable, every solid-class count
of the workloads and both alpha/energy formulations."""
import numpy as np
import pytest

import np_restate as R
from imex_sflow2d_v2_b200 import configs
from oracle import Oracle

N = 12000


def random_states(p, n, seed):
    """Physical states (n_vars+2, n): thickness log-uniform over 1e-16..1e3 m
    (dry, below machine epsilon, below eps_sing and thick), velocities with
    exact zeros, temperatures 250-1300 K, solid volume fractions summing to
    0..0.6 with some classes empty."""
    rng = np.random.default_rng(seed)
    ns = p.n_solid
    nv = 4 + ns
    h = 10.0 ** rng.uniform(-16.0, 3.0, n)
    h[rng.random(n) < 0.04] = 0.0
    u = rng.uniform(-30.0, 30.0, n)
    v = rng.uniform(-30.0, 30.0, n)
    u[rng.random(n) < 0.1] = 0.0
    v[rng.random(n) < 0.1] = 0.0
    T = rng.uniform(250.0, 1300.0, n)
    tot = rng.uniform(0.0, 0.6, n)
    w = rng.random((ns, n))
    w[rng.random((ns, n)) < 0.15] = 0.0
    w = w / np.maximum(w.sum(axis=0), 1e-300)
    al = w * tot
    qp = np.zeros((nv + 2, n))
    qp[0] = h
    qp[1] = h * u
    qp[2] = h * v
    qp[3] = T
    for i in range(ns):
        qp[4 + i] = al[i] if p.alpha_flag else al[i] * h
    qp[nv] = u
    qp[nv + 1] = v
    return qp


def setups():
    out = {}
    p, st, _ = configs.dambreak(nx=8, ny=8, rheology=1)
    out["one_class"] = (p, st)
    p, st, _ = configs.radial_current(nx=16, ny=16, r_source=4.0)
    out["two_classes_voellmy"] = (p, st)
    p, st, _ = configs.fractal_inlet(n=16, r_source=20.0)
    out["three_classes"] = (p, st)
    p, st, _ = configs.dambreak(nx=8, ny=8, rheology=1)
    p.alpha_flag = 1
    out["alpha_flag"] = (p, st)
    p, st, _ = configs.dambreak(nx=8, ny=8, rheology=1)
    p.energy_flag = 0
    out["no_energy"] = (p, st)
    return out


SETUPS = setups()


def columns(o, fn, arr, nout):
    out = np.empty((nout, arr.shape[1]))
    for c in range(arr.shape[1]):
        out[:, c] = fn(np.ascontiguousarray(arr[:, c]))
    return out


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return (a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))


@pytest.mark.parametrize("name", sorted(SETUPS))
def test_conversions_and_mixture(name):
    p, st = SETUPS[name]
    K = R.Consts(p)
    o = Oracle(p, st)
    qp = random_states(p, N, 11)
    nv = K.nv
    qc_o = columns(o, o.qp_to_qc, qp, nv)
    qc_n = R.qp_to_qc(K, qp)
    assert same_bits(qc_o, qc_n).all(), np.argwhere(~same_bits(qc_o, qc_n))[:5]
    qp_o = columns(o, o.qc_to_qp, qc_o, nv + 2)
    qp_n = R.qc_to_qp(K, qc_o)
    assert same_bits(qp_o, qp_n).all(), np.argwhere(~same_bits(qp_o, qp_n))[:5]
    mx_o = columns(o, o.mixt_var, qp, 4)
    mx_n = np.array(R.mixt_var(K, qp))
    assert same_bits(mx_o, mx_n).all(), np.argwhere(~same_bits(mx_o, mx_n))[:5]


@pytest.mark.parametrize("name", sorted(SETUPS))
@pytest.mark.parametrize("d", [1, 2])
def test_speeds_fluxes_and_kt_interface(name, d):
    p, st = SETUPS[name]
    K = R.Consts(p)
    o = Oracle(p, st)
    nv = K.nv
    rng = np.random.default_rng(20 + d)
    qpL = random_states(p, N, 31 + d)
    qpR = random_states(p, N, 41 + d)
    # a share of interfaces whose two faces are the same state, or have a zero
    # normal momentum on both sides (the zero-velocity rules)
    k = rng.random(N) < 0.05
    qpR[:, k] = qpL[:, k]
    z = rng.random(N) < 0.05
    for a in (qpL, qpR):
        a[d, z] = 0.0
        a[nv + d - 1, z] = 0.0
    gcf = np.where(rng.random(N) < 0.5, 1.0, rng.uniform(0.6, 1.0, N))
    qcL, qcR = R.qp_to_qc(K, qpL), R.qp_to_qc(K, qpR)
    sp_o = np.empty((2, N))
    fl_o = np.empty((nv, N))
    H_o = np.empty((nv, N))
    a_o = np.empty((2, N))
    for c in range(N):
        sp_o[:, c] = o.local_speeds(qpL[:, c], gcf[c], d)
        fl_o[:, c] = o.eval_fluxes(qcL[:, c], qpL[:, c], gcf[c], d)
        H_o[:, c], a_o[:, c] = o.kt_interface(qcL[:, c], qpL[:, c], qcR[:, c], qpR[:, c],
                                              gcf[c], d)
    sp_n = np.array(R.local_speeds(K, qpL, gcf, d))
    fl_n = R.eval_fluxes(K, qcL, qpL, gcf, d)
    H_n, aN, aP = R.kt_interface(K, qcL, qpL, qcR, qpR, gcf, d)
    assert same_bits(sp_o, sp_n).all(), np.argwhere(~same_bits(sp_o, sp_n))[:5]
    assert same_bits(fl_o, fl_n).all(), np.argwhere(~same_bits(fl_o, fl_n))[:5]
    assert same_bits(a_o, np.array([aN, aP])).all()
    assert same_bits(H_o, H_n).all(), np.argwhere(~same_bits(H_o, H_n))[:5]
    # the rules were exercised
    assert (aN == aP).any() and (~(aN == aP)).any()


@pytest.mark.parametrize("name", ["one_class", "two_classes_voellmy", "three_classes"])
def test_voellmy_implicit_terms(name):
    p, st = SETUPS[name]
    assert p.rheology_model == 1
    K = R.Consts(p)
    o = Oracle(p, st)
    qc = R.qp_to_qc(K, random_states(p, N, 51))
    nh_o = np.empty_like(qc)
    for c in range(N):
        nh_o[:, c] = o.implicit_terms(np.ascontiguousarray(qc[:, c]))[0]
    nh_n = R.voellmy_implicit(K, qc)
    ok = same_bits(nh_o, nh_n)
    assert ok.all(), (np.argwhere(~ok)[:5], nh_o[~ok][:5], nh_n[~ok][:5])
    assert (nh_n[1] != 0.0).sum() > N // 2
