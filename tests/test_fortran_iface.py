"""The Fortran binding (include/imex_gpu_iface.f90) against the C ABI, without
a Fortran compiler: every TYPE, BIND(C) has the fields of its C struct in the
same order with the same kinds and array lengths (checked against the ctypes
mirror, which tests/test_abi_cpu.py checks against the header), and every
bound function exists in include/imex_gpu.h and in the library with the
same number of arguments."""
import os
import re

import ctypes as C
import pytest

from imex_sflow2d_v2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "imex_gpu_iface.f90")
HEADER = os.path.join(ROOT, "include", "imex_gpu.h")

KINDS = {"INTEGER(C_INT32_T)": "i32", "INTEGER(C_INT)": "i32", "INTEGER(C_INT64_T)": "i64",
         "REAL(C_DOUBLE)": "f64", "REAL(C_FLOAT)": "f32", "TYPE(C_PTR)": "ptr",
         "INTEGER(C_INT8_T)": "i8"}


def fortran_lines():
    """Statements of the file: comments stripped, continuations joined."""
    out, cur = [], ""
    for raw in open(F90):
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        if line.endswith("&"):
            cur += line[:-1] + " "
            continue
        out.append((cur + line).strip())
        cur = ""
    return out


def parameters(lines):
    env = {}
    for ln in lines:
        m = re.match(r"INTEGER, PARAMETER :: (.*)", ln)
        if m:
            for part in m.group(1).split(","):
                name, expr = part.split("=")
                env[name.strip()] = eval(expr, {}, dict(env))
    return env


def split_decls(text):
    """'a, b(3), c(N + 2)' -> [(name, dim expr or None)]."""
    out, depth, cur = [], 0, ""
    for ch in text + ",":
        if ch == "," and depth == 0:
            m = re.match(r"\s*(\w+)\s*(?:\((.*)\))?\s*$", cur)
            out.append((m.group(1), m.group(2)))
            cur = ""
            continue
        depth += ch == "("
        depth -= ch == ")"
        cur += ch
    return out


def fortran_types():
    lines = fortran_lines()
    env = parameters(lines)
    types, name = {}, None
    for ln in lines:
        m = re.match(r"TYPE, BIND\(C\) :: (\w+)$", ln)
        if m:
            name = m.group(1)
            types[name] = []
            continue
        if name and ln.startswith("END TYPE"):
            name = None
            continue
        if name:
            decl, rest = [x.strip() for x in ln.split("::")]
            kind = KINDS.get(decl) or ("type:" + re.match(r"TYPE\((\w+)\)", decl).group(1))
            for fld, dim in split_decls(rest):
                n = eval(dim, {}, dict(env)) if dim else 1
                types[name].append((fld.lower(), kind, n))
    return types


def ctypes_kind(t):
    if isinstance(t, type) and issubclass(t, C.Array):
        return ctypes_kind(t._type_)[0], t._length_
    if t in (C.c_int32, C.c_uint32):
        return "i32", 1
    if t is C.c_int64:
        return "i64", 1
    if t is C.c_double:
        return "f64", 1
    if t is C.c_char_p or t is C.c_void_p or (isinstance(t, type) and issubclass(t, C._Pointer)):
        return "ptr", 1
    return "type:" + t.__name__, 1


PAIRS = {"imex_bc": abi.ImexBC, "imex_params": abi.ImexParams, "imex_static": abi.ImexStatic,
         "imex_stats": abi.ImexStats, "imex_post_diag": abi.ImexPostDiag,
         "imex_output_spec": abi.ImexOutputSpec}
CTYPE_TO_F = {"type:ImexBC": "type:imex_bc"}


@pytest.mark.parametrize("fname", sorted(PAIRS))
def test_bind_c_type_matches_c_struct(fname):
    ft = fortran_types()[fname]
    cs = PAIRS[fname]
    cfields = []
    for name, t in cs._fields_:
        kind, n = ctypes_kind(t)
        cfields.append((name.lower(), CTYPE_TO_F.get(kind, kind), n))
    assert ft == cfields


def header_prototypes():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"(?:int|const char\*)\s+(imex_\w+)\s*\(([^)]*)\)\s*;", text):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return protos


def fortran_functions():
    funcs = {}
    for ln in fortran_lines():
        m = re.match(r".*FUNCTION (\w+)\(([^)]*)\)\s*BIND\(C, name=\"(\w+)\"\)", ln)
        if m:
            args = [a for a in m.group(2).split(",") if a.strip()]
            funcs[m.group(3)] = (m.group(1), len(args))
    return funcs


def test_bound_functions_exist_with_the_c_argument_counts():
    protos = header_prototypes()
    funcs = fortran_functions()
    assert len(funcs) >= 30
    from imex_sflow2d_v2_b200.solver import load_library
    lib = load_library()
    for cname, (fname, nargs) in funcs.items():
        assert fname == cname
        assert cname in protos, cname
        assert protos[cname] == nargs, (cname, protos[cname], nargs)
        assert hasattr(lib, cname), cname


def test_the_driver_calls_are_bound():
    """The calls of the reference's driver loop that the drop-in replaces
    (src/IMEX_SfloW2D.f90:341-389)."""
    funcs = fortran_functions()
    for name in ("imex_gpu_check_solve", "imex_gpu_timestep", "imex_gpu_rk_step",
                 "imex_gpu_erosion_deposition", "imex_gpu_topography_reconstruction",
                 "imex_gpu_set_state", "imex_gpu_get_state", "imex_gpu_advance"):
        assert name in funcs
