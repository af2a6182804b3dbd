"""CPU-side checks of the C ABI: the shared library loads, exports every
function include/imex_gpu.h declares, and the ctypes mirror matches the C
struct layout (compiled here with gcc)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from imex_sflow2d_v2_b200 import abi, build
from imex_sflow2d_v2_b200.solver import load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "imex_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(imex_gpu_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return load_library()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_build_info(lib):
    info = lib.imex_gpu_build_info().decode()
    assert "sm_100a" in info and "fmad=false" in info


def _c_layout():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "imex_gpu.h"
#define OFF(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  printf("ImexParams %zu\nImexStatic %zu\nImexStats %zu\nImexBC %zu\nImexPostDiag %zu\n",
         sizeof(ImexParams), sizeof(ImexStatic), sizeof(ImexStats), sizeof(ImexBC),
         sizeof(ImexPostDiag));
  printf("ImexOutputSpec %zu\n", sizeof(ImexOutputSpec));
  OFF(ImexOutputSpec, time); OFF(ImexOutputSpec, cons); OFF(ImexOutputSpec, threads);
  OFF(ImexParams, limiter); OFF(ImexParams, cfl); OFF(ImexParams, bcW); OFF(ImexParams, bcN);
  OFF(ImexParams, grav); OFF(ImexParams, rho_s); OFF(ImexParams, time_param);
  OFF(ImexParams, erodible_fract); OFF(ImexParams, coeff_porosity);
  OFF(ImexStatic, erosion); OFF(ImexStats, error_mask); OFF(ImexStats, kernel_launches);
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(src, "w").write(prog)
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, src])
        out = subprocess.check_output([exe]).decode()
    vals = {}
    for line in out.splitlines():
        k, v = line.split()
        vals[k] = int(v)
    return vals


def test_ctypes_mirror_matches_c_layout():
    c = _c_layout()
    assert c["ImexParams"] == C.sizeof(abi.ImexParams)
    assert c["ImexStatic"] == C.sizeof(abi.ImexStatic)
    assert c["ImexStats"] == C.sizeof(abi.ImexStats)
    assert c["ImexBC"] == C.sizeof(abi.ImexBC)
    assert c["ImexPostDiag"] == C.sizeof(abi.ImexPostDiag)
    assert c["ImexOutputSpec"] == C.sizeof(abi.ImexOutputSpec)
    for key, v in c.items():
        if "." in key:
            t, f = key.split(".")
            assert getattr(getattr(abi, t), f).offset == v, key


def test_create_rejects_unsupported_options_without_a_device(lib):
    from imex_sflow2d_v2_b200 import configs
    p, st, q = configs.dambreak(nx=8, ny=8, dx=1.0)
    p.n_rk = 3
    s, keep = abi.make_static(st)
    h = C.c_void_p()
    rc = lib.imex_gpu_create(C.byref(p), C.byref(s), -1, C.byref(h))
    assert rc == abi.IMEX_EUNSUPPORTED
    p.n_rk = 2
    p.limiter[0] = 9
    rc = lib.imex_gpu_create(C.byref(p), C.byref(s), -1, C.byref(h))
    assert rc == abi.IMEX_EINVAL
