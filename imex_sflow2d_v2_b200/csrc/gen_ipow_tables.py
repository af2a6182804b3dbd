"""Writes ipow_tables.h: the tables of the table-driven x**y (ipow) shared
by the CUDA path and the CPU oracle.  Exact decimal arithmetic at 60 digits:

  INVC[i]   the double nearest 1/c_i, c_i = 1 + (i + 1/2)/128, i = 0..127
  LOGC[i]   -log(INVC[i]) as an unevaluated sum hi + lo of two doubles
  EXP2[j]   2**(j/64), j = 0..63, as hi + lo

Run: python gen_ipow_tables.py > ipow_tables.h
"""
from decimal import Decimal, getcontext

getcontext().prec = 60


def dd(x):
    hi = float(x)
    lo = float(x - Decimal(hi))
    return hi, lo


def hexf(v):
    return float(v).hex()


def main():
    invc, lhi, llo = [], [], []
    for i in range(128):
        c = Decimal(1) + (Decimal(i) + Decimal("0.5")) / Decimal(128)
        ic = float(Decimal(1) / c)
        h, l = dd(-Decimal(ic).ln())
        invc.append(ic)
        lhi.append(h)
        llo.append(l)
    ehi, elo = [], []
    ln2 = Decimal(2).ln()
    for j in range(64):
        h, l = dd((ln2 * Decimal(j) / Decimal(64)).exp())
        ehi.append(h)
        elo.append(l)
    out = ["// Generated by gen_ipow_tables.py (exact decimal arithmetic); do not edit.",
           "// Tables of the table-driven x**y shared by the CUDA path and the oracle.",
           "#pragma once", "#ifdef __CUDACC__", "#define IPOW_TABLE __device__ static const",
           "#else", "#define IPOW_TABLE static const", "#endif"]

    def emit(name, vals):
        out.append("IPOW_TABLE double %s[%d] = {" % (name, len(vals)))
        for k in range(0, len(vals), 3):
            out.append("    " + ", ".join(hexf(v) for v in vals[k:k + 3]) + ",")
        out.append("};")
    emit("IPOW_INVC", invc)
    emit("IPOW_LOGC_HI", lhi)
    emit("IPOW_LOGC_LO", llo)
    emit("IPOW_EXP2_HI", ehi)
    emit("IPOW_EXP2_LO", elo)
    print("\n".join(out))


if __name__ == "__main__":
    main()
