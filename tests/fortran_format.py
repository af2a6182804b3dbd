"""Test restatement of the reference's output files (src/inpout_2d.f90:
5683-6180, 6195-6235, 6306-6613): Fortran Ew.d / ESw.dEe / Iw / Fw.d as
gfortran writes them, and the .q_2d / .p_2d / ESRI file layouts, built from
oracle values.  The GPU writers' files must equal these byte for byte."""
import math


def _right(s, w):
    return "*" * w if len(s) > w else " " * (w - len(s)) + s


def _special(v, w):
    if math.isnan(v):
        return _right("NaN", w)
    if math.isinf(v):
        if v < 0:
            return _right("-Infinity" if w >= 9 else "-Inf", w)
        return _right("Infinity" if w >= 8 else "Inf", w)
    return None


def _digits(a, sig):
    s = "%.*e" % (sig - 1, a)
    mant, ex = s.split("e")
    return mant.replace(".", ""), int(ex)


def fE(v, w, d):
    sp = _special(v, w)
    if sp is not None:
        return sp
    a = abs(v)
    if a == 0.0:
        dig, ex = "0" * d, 0
    else:
        dig, x = _digits(a, d)
        ex = x + 1
    if abs(ex) <= 99:
        es = "E%s%02d" % ("-" if ex < 0 else "+", abs(ex))
    elif abs(ex) <= 999:
        es = "%s%03d" % ("-" if ex < 0 else "+", abs(ex))
    else:
        return "*" * w
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    return _right("%s0.%s%s" % (sign, dig, es), w)


def fES(v, w, d, e):
    sp = _special(v, w)
    if sp is not None:
        return sp
    a = abs(v)
    if a == 0.0:
        dig, x = "0" * (d + 1), 0
    else:
        dig, x = _digits(a, d + 1)
    if abs(x) >= 10 ** e:
        return "*" * w
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    return _right("%s%s.%sE%s%0*d" % (sign, dig[0], dig[1:], "-" if x < 0 else "+", e, abs(x)), w)


def fI(v, w):
    return _right("%d" % v, w)


def fF(v, w, d):
    sp = _special(v, w)
    if sp is not None:
        return sp
    return _right("%.*f" % (d, v), w)


def lettera(k):
    thou = k // 1000
    hund = (k - thou * 1000) // 100
    ten = (k - thou * 1000 - hund * 100) // 10
    one = k - thou * 1000 - hund * 100 - ten * 10
    return "".join(chr(c + 48) for c in (thou, hund, ten, one))


def comp(o, d, n):
    return [0.5 * ((o + (j - 1) * d) + (o + j * d)) for j in range(1, n + 1)]


def columns_file(xc, yc, cols, kind):
    """cols: list of (nx, ny) arrays.  kind 0: E20.12, 1: ES15.7E2."""
    nx, ny = len(xc), len(yc)
    f = (lambda v: fE(v, 20, 12)) if kind == 0 else (lambda v: fES(v, 15, 7, 2))
    out = []
    for k in range(ny):
        for j in range(nx):
            out.append(f(xc[j]) + f(yc[k]) + "".join(f(float(c[j, k])) for c in cols) + "\n")
        out.append("  \n")
    out.append("  \n  \n")
    return "".join(out)


def esri_file(nx, ny, x0, y0, cell_size, grid):
    """grid: (nx, ny) values as printed (NODATA already applied)."""
    out = ["ncols " + fI(nx, 5) + "\n", "nrows " + fI(ny, 5) + "\n",
           "xllcorner " + fF(x0, 15, 3) + "\n", "yllcorner " + fF(y0, 15, 3) + "\n",
           "cellsize " + fF(cell_size, 15, 3) + "\n", "NODATA_value " + fI(-9999, 5) + "\n"]
    for k in range(ny - 1, -1, -1):
        row = []
        for j in range(nx):
            row.append(fES(float(grid[j, k]), 12, 3, 3))
            if (j + 1) % 2000 == 0 or j + 1 == nx:
                row.append("\n")
        out.append("".join(row))
    return "".join(out)
