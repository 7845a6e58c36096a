"""Prints the log tables of gmath.h (gm_log, P. T. P. Tang's table-driven
logarithm, ACM TOMS 16(4), 1990): for j = 0..128, c_j = 1 + j/128,
  inv_j = 1/c_j rounded to 12 significant bits (inv_0 = 1),
  -log(inv_j) = th_j + tl_j, th_j rounded to a multiple of 2^-42 (so that
  k ln2_hi + th_j is exact for every exponent k), tl_j the rest rounded to
  double.
Computed with Python's decimal module at 70 digits.

    python galic_b200/csrc/gen_gmath_tables.py
"""
import math
from decimal import Decimal, getcontext

getcontext().prec = 70
N = 128


def round_sig(x, bits):
    e = math.frexp(float(x))[1]
    scale = Decimal(2) ** (bits - e)
    return float((x * scale).to_integral_value() / scale)


def round_grid(x, lsb_exp):
    scale = Decimal(2) ** (-lsb_exp)
    return float((x * scale).to_integral_value() / scale)


def tables():
    inv, th, tl = [], [], []
    for j in range(N + 1):
        c = Decimal(1) + Decimal(j) / Decimal(N)
        iv = round_sig(Decimal(1) / c, 12) if j else 1.0
        t = -(Decimal(iv).ln())
        h = round_grid(t, -42)
        inv.append(iv)
        th.append(h)
        tl.append(float(t - Decimal(h)))
    return inv, th, tl


def emit(name, arr):
    body = ", ".join(float(v).hex() for v in arr)
    return f"#define {name} {{{body}}}"


if __name__ == "__main__":
    inv, th, tl = tables()
    for name, arr in (("GM_LOG_INV", inv), ("GM_LOG_TH", th), ("GM_LOG_TL", tl)):
        print(emit(name, arr))
