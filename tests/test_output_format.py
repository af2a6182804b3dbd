"""The output writers' Fortran edit descriptors (libimexgpu's host
formatter, no GPU needed) against known gfortran strings and against the
test restatement in fortran_format.py."""
import math

import numpy as np
import pytest

import fortran_format as FF
from imex_sflow2d_v2_b200.solver import format_edit

KNOWN = [
    # (kind, value, w, d, e, text)
    (0, 1234.5, 20, 12, 0, "  0.123450000000E+04"),
    (0, -0.000123456789, 20, 12, 0, " -0.123456789000E-03"),
    (0, 0.0, 20, 12, 0, "  0.000000000000E+00"),
    (0, 1e100, 20, 12, 0, "  0.100000000000+101"),
    (0, 9.9999999999995, 20, 12, 0, "  0.100000000000E+02"),
    (1, 1234.5, 15, 7, 2, "  1.2345000E+03"),
    (1, -0.000123456789, 15, 7, 2, " -1.2345679E-04"),
    (1, 1e-100, 15, 7, 2, "***************"),
    (1, -9999.0, 12, 3, 3, " -9.999E+003"),
    (1, 0.0, 12, 3, 3, "  0.000E+000"),
    (2, 4096, 5, 0, 0, " 4096"),
    (2, -9999, 5, 0, 0, "-9999"),
    (2, 123456, 5, 0, 0, "*****"),
    (3, 0.0, 15, 3, 0, "          0.000"),
    (3, -12.3456, 15, 3, 0, "        -12.346"),
]


@pytest.mark.parametrize("kind,v,w,d,e,text", KNOWN)
def test_known_strings(kind, v, w, d, e, text):
    assert format_edit(kind, v, w, d, e) == text
    py = {0: lambda: FF.fE(v, w, d), 1: lambda: FF.fES(v, w, d, e),
          2: lambda: FF.fI(int(v), w), 3: lambda: FF.fF(v, w, d)}[kind]()
    assert py == text


def test_random_values_match_restatement():
    rng = np.random.default_rng(5)
    vals = list(10.0 ** rng.uniform(-320, 300, 3000) * rng.choice([-1.0, 1.0], 3000))
    vals += [0.0, -0.0, math.nan, math.inf, -math.inf, 5e-324, 1.7976931348623157e308,
             0.5, 0.05, 0.15, 2.5, 1e-20, 9.99999995e-5, 99.99999995]
    for v in vals:
        assert format_edit(0, v, 20, 12) == FF.fE(v, 20, 12), v
        assert format_edit(1, v, 15, 7, 2) == FF.fES(v, 15, 7, 2), v
        assert format_edit(1, v, 12, 3, 3) == FF.fES(v, 12, 3, 3), v
        if abs(v) < 1e9 or math.isnan(v) or math.isinf(v):
            assert format_edit(3, v, 15, 3) == FF.fF(v, 15, 3), v


def test_lettera():
    assert FF.lettera(0) == "0000"
    assert FF.lettera(12) == "0012"
    assert FF.lettera(9999) == "9999"
    assert FF.lettera(10000) == ":000"   # CHAR(48+10), as the reference computes it
