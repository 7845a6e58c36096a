"""The project's elementary functions (galic_b200/csrc/gmath.h) against glibc.

gmath.h replaces log/atan2/sin/cos/acos/asin/exp on the orbit, sampling and set-up paths so that the CUDA
kernels and the CPU restatement agree bit for bit; these tests bound its
error against glibc over the argument ranges the path uses."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r'''
#include "gmath.h"
double t_log(double x) { return gm_log(x); }
double t_atan2(double y, double x) { return gm_atan2(y, x); }
double t_sin(double x) { return gm_sin(x); }
double t_cos(double x) { return gm_cos(x); }
double t_acos(double x) { return gm_acos(x); }
double t_exp(double x) { return gm_exp(x); }
double t_asin(double x) { return gm_asin(x); }
void t_sincos(double x, double *s, double *c) { gm_sincos(x, s, c); }
#include <math.h>
#include <stdint.h>
#include <string.h>
/* The orbit step's division by a per-model constant (div_by in model.cuh):
   q0 = a*y, q = q0 + (a - b*q0)*y with y = 1/b, both steps fused.  Counts the
   pairs of n random binary64 numbers (significands uniform, a over 60 binades,
   b over 40, plus a's with all-ones and nearly-zero significands) where q
   differs from a / b. */
static uint64_t xs(uint64_t *s) { *s ^= *s << 13; *s ^= *s >> 7; *s ^= *s << 17; return *s; }
static double mk(uint64_t *s, int e)
{
  uint64_t u = ((uint64_t) (1023 + e) << 52) | (xs(s) & ((1ULL << 52) - 1)); double d; memcpy(&d, &u, 8); return d;
}
long t_div_by_mismatches(long nb, long na, uint64_t seed)
{
  long bad = 0;
  for(long i = 0; i < nb; i++) {
    double b = mk(&seed, (int) (xs(&seed) % 40) - 20), y = 1.0 / b;
    for(long j = 0; j < na; j++) {
      double a = mk(&seed, (int) (xs(&seed) % 60) - 30);
      uint64_t u; memcpy(&u, &a, 8);
      if((j & 7) == 0) u |= ((1ULL << 52) - 1) ^ (xs(&seed) & 0xff);
      if((j & 7) == 1) u = (u & ~((1ULL << 52) - 1)) | (xs(&seed) & 0xff);
      memcpy(&a, &u, 8);
      double q0 = a * y, q = fma(fma(-q0, b, a), y, q0);
      bad += q != a / b;
    }
  }
  return bad;
}
'''


@pytest.fixture(scope="module")
def gm(tmp_path_factory):
    d = tmp_path_factory.mktemp("gm")
    src = d / "t.c"
    src.write_text(SRC)
    so = d / "libt.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I",
                    os.path.join(ROOT, "galic_b200", "csrc"), str(src), "-o", str(so), "-lm"], check=True)
    L = C.CDLL(str(so))
    for n, k in (("t_log", 1), ("t_atan2", 2), ("t_sin", 1), ("t_cos", 1), ("t_acos", 1), ("t_exp", 1), ("t_asin", 1)):
        f = getattr(L, n)
        f.restype = C.c_double
        f.argtypes = [C.c_double] * k
    L.t_sincos.restype = None
    L.t_sincos.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.t_div_by_mismatches.restype = C.c_long
    L.t_div_by_mismatches.argtypes = [C.c_long, C.c_long, C.c_uint64]
    return L


def ulps(a, b):
    if a == b:
        return 0.0
    return abs(a - b) / abs(math.nextafter(b, math.inf) - b)


def test_log_within_one_ulp(gm):
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-700, 700, 20000)), 1 + rng.random(20000) * 1e4,
                         [1.0, 2.0, 0.5, 1e-310, 5e-324, 1.7976931348623157e308]])
    assert max(ulps(gm.t_log(x), math.log(x)) for x in xs) <= 1.0
    assert gm.t_log(1.0) == 0.0
    assert math.isinf(gm.t_log(0.0)) and gm.t_log(0.0) < 0
    assert math.isnan(gm.t_log(-1.0))


def test_atan2_within_two_ulp_and_signed_zeros(gm):
    rng = np.random.default_rng(2)
    a = rng.uniform(-1, 1, 20000) * 10 ** rng.uniform(-5, 5, 20000)
    b = rng.uniform(-1, 1, 20000) * 10 ** rng.uniform(-5, 5, 20000)
    assert max(ulps(gm.t_atan2(y, x), math.atan2(y, x)) for y, x in zip(a, b)) <= 2.0
    for y, x in ((0.0, 0.0), (-0.0, 0.0), (0.0, -0.0), (-0.0, -0.0), (0.0, -1.0), (-0.0, -1.0), (1.0, 0.0),
                 (-1.0, 0.0), (math.inf, math.inf), (1.0, -math.inf)):
        assert gm.t_atan2(y, x) == math.atan2(y, x)
        assert math.copysign(1, gm.t_atan2(y, x)) == math.copysign(1, math.atan2(y, x))


def test_sin_cos_within_one_ulp(gm):
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-math.pi, math.pi, 20000), rng.uniform(-300, 300, 5000), [0.0, -0.0, 1e-30]])
    assert max(ulps(gm.t_sin(x), math.sin(x)) for x in xs) <= 1.0
    assert max(ulps(gm.t_cos(x), math.cos(x)) for x in xs) <= 1.0


def test_acos_within_two_ulp(gm):
    rng = np.random.default_rng(4)
    xs = np.concatenate([rng.uniform(-1, 1, 20000), [1.0, -1.0, 0.0, 1 - 2 ** -52, -1 + 2 ** -53]])
    assert max(ulps(gm.t_acos(x), math.acos(x)) for x in xs) <= 2.0
    assert math.isnan(gm.t_acos(1.5))


def test_exp_within_one_ulp(gm):
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-700, 700, 20000), rng.uniform(-40, 0, 20000), rng.uniform(-1, 1, 5000),
                         rng.uniform(-745, -708, 2000), [0.0, -0.0, 1.0, -1.0, 709.78, 1e-300, -1e-300]])
    assert max(ulps(gm.t_exp(x), math.exp(x)) for x in xs) <= 1.0
    assert gm.t_exp(0.0) == 1.0
    assert gm.t_exp(-800.0) == 0.0 and math.isinf(gm.t_exp(800.0)) and math.isinf(gm.t_exp(709.9))
    assert math.isnan(gm.t_exp(math.nan))


def test_asin_within_two_ulp(gm):
    rng = np.random.default_rng(6)
    xs = np.concatenate([rng.uniform(-1, 1, 20000), rng.uniform(-1e-3, 1e-3, 2000), [1.0, -1.0, 0.0, -0.0, 1 - 2 ** -52]])
    assert max(ulps(gm.t_asin(x), math.asin(x)) for x in xs) <= 2.0
    assert math.isnan(gm.t_asin(1.5))


def test_sincos_equals_sin_and_cos(gm):
    """gm_sincos (one reduction, both polynomials, selected by quadrant) gives
    gm_sin and gm_cos bit for bit, special and tiny arguments included."""
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.uniform(-math.pi, math.pi, 20000), rng.uniform(-1e4, 1e4, 2000),
                         [0.0, -0.0, 1e-300, -1e-9, 2.0 ** -28, math.pi / 4, math.pi / 2, -math.pi, math.pi,
                          float("inf"), float("nan")]])
    s, c = C.c_double(), C.c_double()
    for x in xs:
        gm.t_sincos(float(x), C.byref(s), C.byref(c))
        ws, wc = gm.t_sin(float(x)), gm.t_cos(float(x))
        assert (math.isnan(ws) and math.isnan(s.value)) or np.float64(s.value).tobytes() == np.float64(ws).tobytes()
        assert (math.isnan(wc) and math.isnan(c.value)) or np.float64(c.value).tobytes() == np.float64(wc).tobytes()


def _rn(x, p):
    """x rounded to nearest-even at p significant bits (x exact in binary64)."""
    m, e = np.frexp(x)
    return np.ldexp(np.rint(np.ldexp(m, p)), e - p)


@pytest.mark.parametrize("p", range(6, 13))
def test_div_by_reciprocal_exhaustive_at_small_precision(p):
    """The orbit step divides by per-model constants as q0 = RN(a*y),
    q = RN(q0 + RN(a - b*q0)*y) with y = RN(1/b) (div_by in model.cuh).  At
    precision p every pair of significands a, b in [1, 2) is checked against
    the correctly rounded a / b, formed from integers; other binades scale
    the same pairs.  Products here need at most 3p+1 bits, so binary64 holds
    them exactly and _rn gives the p-bit roundings."""
    lo, hi = 1 << (p - 1), 1 << p
    A = np.arange(lo, hi, dtype=np.int64)[None, :]
    B = np.arange(lo, hi, dtype=np.int64)[:, None]
    a = np.ldexp(A.astype(np.float64), -(p - 1))
    b = np.ldexp(B.astype(np.float64), -(p - 1))
    big = A >= B
    sh = np.where(big, p - 1, p)
    num = A << sh
    Q, R = num // B, num % B
    Q = Q + ((2 * R > B) | ((2 * R == B) & (Q & 1 == 1)))
    exact = np.ldexp(Q.astype(np.float64), -sh)
    y = _rn(1.0 / b, p)
    q0 = _rn(a * y, p)
    r = _rn(a - b * q0, p)
    q = _rn(q0 + r * y, p)
    assert np.array_equal(q, exact), int((q != exact).sum())


def test_div_by_reciprocal_random_binary64(gm):
    """The same sequence in binary64 against IEEE division on 1e8 pairs."""
    assert gm.t_div_by_mismatches(20000, 5000, 0x9E3779B97F4A7C15) == 0
