"""The device's point functions against the oracle's on inputs far beyond
what a run produces (imex_gpu_point_eval): the table-driven x**y of the
mass-exchange closures, and the settling velocity's fixed-point iteration
(src/constitutive_2d.f90:5148-5214).  Both bit for bit.

The device evaluates x**y with bit operations in place of frexp and ldexp
on their common ranges and the settling loop's exit test without the
division where its answer is certain; the inputs below cover subnormal and
huge x, results near overflow and underflow, and settling states whose
relative change lands next to the 1e-6 threshold.  The limiters
(src/geometry_2d.f90:1555-1676) take the signs of finite operands without
dividing, and the flux kernel's minmod on equally spaced centres divides
once; both are compared with the oracle's limit() on values with zeros,
ties, both signs, infinities and NaN, and spacings down to where the
quotients overflow.
"""
import numpy as np
import pytest

from imex_sflow2d_v2_b200.solver import point_eval
from oracle import ipow_n, limit_n, settling_velocity_n

pytestmark = pytest.mark.gpu


def _same_bits(a, b):
    a = np.ascontiguousarray(a).view(np.uint64)
    b = np.ascontiguousarray(b).view(np.uint64)
    return a == b


@pytest.mark.parametrize("fast", [False, True])
def test_ipow_equals_oracle(fast):
    rng = np.random.default_rng(7)
    n = 1 << 21
    x = np.exp(rng.uniform(np.log(1e-320), np.log(1e308), n))
    x[:4096] = np.exp(rng.uniform(np.log(4e-324), np.log(2.3e-308), 4096))   # subnormal
    x[4096:8192] = 1.0 + rng.uniform(-1e-6, 1e-6, 4096)
    y = rng.choice([0.687, 2.4, 1.5, 0.5, 4.65, -0.5, 3.0], n)
    y[::3] = rng.uniform(-6.0, 6.0, (n + 2) // 3)
    specials = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 2.0, 0.5, 1e-300,
                         5e-324, 1.7e308])
    xs, ys = np.meshgrid(specials, np.array([0.0, 0.687, -0.687, 2.4, np.nan, 1.0, -1.0]))
    x = np.concatenate([x, xs.ravel()])
    y = np.concatenate([y, ys.ravel()])
    # results next to overflow and underflow: y*log(x) near 709.78 and -745.1
    edge = rng.uniform(700.0, 709.9, 4096)
    x = np.concatenate([x, np.full(4096, np.e ** 2), np.full(4096, np.e ** -2)])
    y = np.concatenate([y, edge / 2.0, rng.uniform(700.0, 745.5, 4096) / 2.0])
    g = point_eval("ipow", x, y, fast=fast)
    o = ipow_n(x, y)
    if fast:
        # the fast build contracts the log's sums into multiply-adds
        fin = np.isfinite(o) & (np.abs(o) > 1e-300)
        assert np.array_equal(np.isnan(g), np.isnan(o))
        assert np.array_equal(np.isinf(g), np.isinf(o))
        assert np.allclose(g[fin], o[fin], rtol=1e-14, atol=0.0)
        return
    same = _same_bits(g, o) | (np.isnan(g) & np.isnan(o))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, [(x[i], y[i], g[i], o[i]) for i in bad[:5]]


@pytest.mark.parametrize("fast", [False, True])
def test_settling_velocity_equals_oracle(fast):
    rng = np.random.default_rng(11)
    n = 1 << 20
    diam = np.exp(rng.uniform(np.log(1e-7), np.log(3e-2), n))
    rhos = rng.uniform(200.0, 8000.0, n)
    rhoc = np.exp(rng.uniform(np.log(1e-3), np.log(3000.0), n))
    ikv = np.exp(rng.uniform(np.log(1e2), np.log(1e7), n))
    # the workloads' carrier: air between 250 and 1300 K, kinematic
    # viscosity 1.48e-5, three particle sizes
    m = n // 4
    rhoc[:m] = 101300.0 / (287.051 * rng.uniform(250.0, 1300.0, m))
    ikv[:m] = 1.0 / 1.48e-5
    diam[:m] = rng.choice([1e-5, 1e-4, 1e-3], m)
    rhos[:m] = 2500.0
    g = point_eval("settling", diam, rhos, rhoc, ikv, g=9.81, fast=fast)
    o = settling_velocity_n(diam, rhos, rhoc, ikv, 9.81)
    if fast:
        # contracted multiply-adds round once where the reference rounds
        # twice; the iteration then ends within its own 1e-6 tolerance
        assert np.allclose(g, o, rtol=1e-5, atol=0.0)
        return
    bad = np.flatnonzero(~_same_bits(g, o))
    assert bad.size == 0, [(diam[i], rhos[i], rhoc[i], ikv[i], g[i], o[i]) for i in bad[:5]]
    assert (o[rhos <= rhoc] == 0.0).all()


def _limiter_inputs(rng, n):
    mag = np.exp(rng.uniform(np.log(1e-30), np.log(1e30), (3, n)))
    v = mag * rng.choice([-1.0, 1.0], (3, n))
    v[:, : n // 8] = rng.integers(-3, 4, (3, n // 8)).astype(np.float64)   # zeros, ties
    v[1, n // 8: n // 4] = v[0, n // 8: n // 4]                            # flat pairs
    k = n // 4
    v[0, k: k + 64] = np.inf
    v[1, k + 64: k + 128] = -np.inf
    v[2, k + 128: k + 192] = np.nan
    v[:, k + 192: k + 256] = 1e300 * rng.choice([-1.0, 1.0], (3, 64))
    dz = np.exp(rng.uniform(np.log(1e-12), np.log(1e4), n))
    dz[: 256] = 1e-300
    return v, dz


def test_minmod_uniform_equals_limit():
    rng = np.random.default_rng(5)
    n = 1 << 20
    v, dz = _limiter_inputs(rng, n)
    g = point_eval("minmod_uniform", v[0], v[1], v[2], dz)
    o = limit_n(v[0], v[1], v[2], 0.0, dz, 2.0 * dz, 1)
    same = _same_bits(g, o) | (np.isnan(g) & np.isnan(o))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, [(v[:, i], dz[i], g[i], o[i]) for i in bad[:5]]


@pytest.mark.parametrize("limiter", range(8))
def test_limit_equals_oracle(limiter):
    rng = np.random.default_rng(100 + limiter)
    n = 1 << 18
    v, dz = _limiter_inputs(rng, n)
    g = point_eval("limit", v[0], v[1], v[2], dz, g=float(limiter))
    o = limit_n(v[0], v[1], v[2], 0.0, dz, 2.0 * dz, limiter)
    same = _same_bits(g, o) | (np.isnan(g) & np.isnan(o))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, [(v[:, i], dz[i], g[i], o[i]) for i in bad[:5]]


def test_quotient_below_threshold_equals_ieee():
    """The kernels' test of a rounded quotient against a threshold (the
    settling loop's 1e-6, the Newton step's EPSILON), taken without the
    division where the answer is certain, against numpy's IEEE division:
    quotients next to the thresholds, both signs, zeros, infinities, NaN,
    extreme magnitudes."""
    rng = np.random.default_rng(21)
    n = 1 << 21
    b = np.exp(rng.uniform(np.log(1e-300), np.log(1e300), n)) * rng.choice([-1.0, 1.0], n)
    b[: n // 4] = rng.uniform(-2.0, 2.0, n // 4)
    c = np.where(rng.random(n) < 0.5, 1e-6, 2.220446049250313e-16)
    # a = |b|*c*(1 + k*2^-52): quotients next to the threshold on either side
    k = rng.integers(-6, 7, n).astype(np.float64)
    a = np.abs(b) * c * (1.0 + k * 2.0 ** -52)
    m = n // 2
    a[m:] = np.exp(rng.uniform(np.log(1e-300), np.log(1e300), n - m)) * rng.choice([-1.0, 1.0], n - m)
    specials = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 1e-310, 1e308])
    sa, sb = np.meshgrid(specials, specials)
    a = np.concatenate([a, sa.ravel()])
    b = np.concatenate([b, sb.ravel()])
    c = np.concatenate([c, np.full(sa.size, 1e-6)])
    g = point_eval("quotient_below", a, b, c, c)
    with np.errstate(all="ignore"):
        want = (a / b < c).astype(np.float64)
    bad = np.flatnonzero(g != want)
    assert bad.size == 0, [(a[i], b[i], c[i], g[i], want[i]) for i in bad[:5]]
