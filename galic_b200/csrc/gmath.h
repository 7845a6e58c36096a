/*
 * gmath.h - project-written double-precision elementary functions shared by
 * the CUDA kernels and the CPU restatement of GALIC's orbit-response path.
 *
 * Why this exists: GALIC's orbit loop (orbit_response.c:211-458 and the
 * lookups it calls in grid.c:15-197, grid.c:494-534, disp_fields.c:118-132)
 * calls log, atan2, sin and cos every step, and main.c:383-401 /
 * disp_fields.c:216-230 call acos.  CUDA's and glibc's implementations differ
 * in the last bit, which makes two otherwise identical FP64 trajectories drift
 * apart.  When the GPU kernel and the CPU restatement both evaluate these
 * functions with the code below, and both are built without floating-point
 * contraction (nvcc --fmad=false, gcc -ffp-contract=off), every operation in
 * the orbit is IEEE-754 basic arithmetic or sqrt (both correctly rounded on
 * both sides) or one of these functions, so the two produce bit-identical
 * orbits.
 *
 * Methods (all published; coefficients are exact Taylor coefficients, rounded
 * once to double, and the constants were computed to 60 digits with Python's
 * decimal module):
 * Polynomials are evaluated by Horner's rule with fused multiply-adds.
 *  - log:   Cody & Waite style reduction x = 2^k * m, m in [sqrt(1/2), sqrt(2)),
 *           log(m) = 2 atanh(s), s = (m-1)/(m+1), atanh by its Taylor series;
 *           the algebraic rewrite log(1+f) = f - (f^2/2 - s (f^2/2 + R)) keeps
 *           the leading term exact.  ln2 is split into a 32-fractional-bit head
 *           and a tail so that k*ln2_hi is exact.
 *  - atan2: reduction to t = min/max in [0,1], table-driven atan
 *           atan(t) = atan(c) + atan((t-c)/(1+t c)), c = k/8 (Gal's accurate
 *           table idea), Taylor series on |u| <= 1/16, quadrant fix-up with
 *           pi/2 and pi split into head + tail.
 *  - sin/cos: Cody & Waite three-part reduction by pi/2 (heads with 33
 *           significant bits), Taylor polynomials on |r| <= pi/4.  Accurate
 *           for |x| < 2^20; the orbit path only uses |x| <= pi.
 *  - acos:  acos(x) = atan2(sqrt((1-x)(1+x)), x); asin(x) = atan2(x, sqrt((1-x)(1+x))).
 *  - exp:   Cody & Waite reduction by ln2 (same split as log), Taylor series
 *           of degree 13, scaling by 2^k in two steps.
 * Measured against glibc over random arguments the error is within 1 ulp for
 * log, exp, sin and cos and within 2 ulp for atan2, acos and asin
 * (tests/test_gmath.py).
 */
#ifndef GALIC_GMATH_H
#define GALIC_GMATH_H

#include <stdint.h>

#ifdef __CUDACC__
#define GM_HD __host__ __device__ __forceinline__
#else
#define GM_HD static inline
#endif

typedef union { double d; uint64_t u; } gm_pun;

GM_HD uint64_t gm_bits(double x) { gm_pun p; p.d = x; return p.u; }
GM_HD double gm_from_bits(uint64_t u) { gm_pun p; p.u = u; return p.d; }
GM_HD int gm_isnan(double x) { return x != x; }
GM_HD double gm_fabs(double x) { return gm_from_bits(gm_bits(x) & 0x7fffffffffffffffULL); }
GM_HD double gm_copysign(double a, double s)
{
  return gm_from_bits((gm_bits(a) & 0x7fffffffffffffffULL) | (gm_bits(s) & 0x8000000000000000ULL));
}
GM_HD int gm_signbit(double x) { return (int) (gm_bits(x) >> 63); }

/* nearest integer, ties away from zero; |x| < 2^52 */
GM_HD double gm_round(double x)
{
  double a = gm_fabs(x);
  if(!(a < 4503599627370496.0)) return x;
  double t = (double) (int64_t) (a + 0.5);
  return gm_copysign(t, x);
}

/* fused multiply-add, correctly rounded on both sides (DFMA on the GPU,
 * the C library's fma on the host): Horner steps use it explicitly, so the
 * result does not depend on the compilers' contraction settings */
#ifdef __CUDA_ARCH__
#define gm_fma(a, b, c) __fma_rn((a), (b), (c))
#else
#define gm_fma(a, b, c) __builtin_fma((a), (b), (c))
#endif

#define GM_INF gm_from_bits(0x7ff0000000000000ULL)
#define GM_NAN gm_from_bits(0x7ff8000000000000ULL)

/* ---------------------------------------------------------------- log */
/* The special arguments (NaN, negative, zero, infinity) are selected at the
 * end instead of returned early, and the subnormal scaling is a selection:
 * the body is one basic block, so the several logs of an orbit step can be
 * interleaved by the compiler.  Values equal the early-return form's. */
GM_HD double gm_log(double x)
{
  const double ln2_hi = 0x1.62e42fee00000p-1;
  const double ln2_lo = 0x1.a39ef35793c76p-33;
  const double sqrt2 = 0x1.6a09e667f3bcdp+0;

  const int sub = (gm_bits(x) >> 52) == 0; /* +0 and positive subnormals: scale up by 2^54 */
  const double xs = sub ? x * 0x1.0p54 : x;
  const uint64_t u = gm_bits(xs);
  int k = (sub ? -54 : 0) + (int) ((u >> 52) & 0x7ff) - 1023;
  double m = gm_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
  const int up = m > sqrt2;
  m = up ? m * 0.5 : m;
  k += up;

  double f = m - 1.0;        /* exact (Sterbenz) */
  double s = f / (2.0 + f);  /* (m-1)/(m+1) */
  double z = s * s;
  /* R(z) = sum_{j>=1} 2 z^j / (2j+1) */
  double p = 0x1.8618618618618p-4;
  p = gm_fma(z, p, 0x1.af286bca1af28p-4);
  p = gm_fma(z, p, 0x1.e1e1e1e1e1e1ep-4);
  p = gm_fma(z, p, 0x1.1111111111111p-3);
  p = gm_fma(z, p, 0x1.3b13b13b13b14p-3);
  p = gm_fma(z, p, 0x1.745d1745d1746p-3);
  p = gm_fma(z, p, 0x1.c71c71c71c71cp-3);
  p = gm_fma(z, p, 0x1.2492492492492p-2);
  p = gm_fma(z, p, 0x1.999999999999ap-2);
  p = gm_fma(z, p, 0x1.5555555555555p-1);
  double R = z * p;
  double hfsq = 0.5 * f * f;
  double dk = (double) k;
  /* log(1+f) = f - (hfsq - s*(hfsq + R)) */
  const double r = dk * ln2_hi + ((f - (hfsq - (s * (hfsq + R) + dk * ln2_lo))));
  return gm_isnan(x) ? x : (x < 0 ? GM_NAN : (x == 0 ? -GM_INF : (x == GM_INF ? x : r)));
}

/* ---------------------------------------------------------------- atan */
/* atan(k/8) as head + tail, k = 0..8 (global read-only tables: a per-call
 * local array would be rebuilt in local memory on every call on the GPU) */
#define GM_ATAN_HI {0.0, 0x1.fd5ba9aac2f6ep-4, 0x1.f5b75f92c80ddp-3, 0x1.6f61941e4def1p-2, \
                    0x1.dac670561bb4fp-2, 0x1.1e00babdefeb4p-1, 0x1.4978fa3269ee1p-1, \
                    0x1.700a7c5784634p-1, 0x1.921fb54442d18p-1}
#define GM_ATAN_LO {0.0, -0x1.cd37686760c17p-59, 0x1.8ab6e3cf7afbdp-57, -0x1.c63aae6f6e918p-56, \
                    0x1.a2b7f222f65e2p-56, -0x1.928df287a668fp-58, 0x1.2419a87f2a458p-56, \
                    -0x1.8c34d25aadef6p-56, 0x1.1a62633145c07p-55}
#ifdef __CUDACC__
static __device__ const double gm_atan_hi_dev[9] = GM_ATAN_HI;
static __device__ const double gm_atan_lo_dev[9] = GM_ATAN_LO;
#endif
static const double gm_atan_hi_host[9] = GM_ATAN_HI;
static const double gm_atan_lo_host[9] = GM_ATAN_LO;

/* atan on [0,1] */
GM_HD double gm_atan_unit(double t)
{
#ifdef __CUDA_ARCH__
  const double *ah = gm_atan_hi_dev, *al = gm_atan_lo_dev;
#else
  const double *ah = gm_atan_hi_host, *al = gm_atan_lo_host;
#endif
  int k = (int) (t * 8.0 + 0.5);
  if(k > 8) k = 8;
  double c = (double) k * 0.125;
  double u = (t - c) / (1.0 + t * c);
  double z = u * u;
  double p = -0x1.1111111111111p-4;
  p = gm_fma(z, p, 0x1.3b13b13b13b14p-4);
  p = gm_fma(z, p, -0x1.745d1745d1746p-4);
  p = gm_fma(z, p, 0x1.c71c71c71c71cp-4);
  p = gm_fma(z, p, -0x1.2492492492492p-3);
  p = gm_fma(z, p, 0x1.999999999999ap-3);
  p = gm_fma(z, p, -0x1.5555555555555p-2);
  double atu = u + u * (z * p);
  return ah[k] + (al[k] + atu);
}

GM_HD double gm_atan2(double y, double x)
{
  const double pio2_hi = 0x1.921fb54442d18p+0, pio2_lo = 0x1.1a62633145c07p-54;
  const double pi_hi = 0x1.921fb54442d18p+1, pi_lo = 0x1.1a62633145c07p-53;
  const double pio4 = 0x1.921fb54442d18p-1;

  double ax = gm_fabs(x), ay = gm_fabs(y);
  int xneg = gm_signbit(x);

  /* t = min/max: ax/ay when ay > ax, else ay/ax (one division, one
   * atan_unit for every lane of a warp; the result does not depend on how
   * the choice is compiled).  Zero, infinite and NaN arguments take the
   * special values selected at the end (their t is not used). */
  const int swap = ay > ax;
  const int special = gm_isnan(x) || gm_isnan(y) || ay == 0.0 || ax == 0.0 || ax == GM_INF || ay == GM_INF;
  double t = (swap ? ax : ay) / (swap ? ay : ax);
  t = special ? 0.0 : t;
  double a = gm_atan_unit(t);
  double b = (pio2_hi - a) + pio2_lo;
  a = swap ? b : a;
  double c = (pi_hi - a) + pi_lo;
  a = xneg ? c : a;
  const double regular = gm_copysign(a, y);
  /* atan2(+-0, x), atan2(y, +-0), the infinite cases, NaN */
  const double sv = (gm_isnan(x) || gm_isnan(y)) ? x + y
                    : (ay == 0.0)                 ? gm_copysign(xneg ? pi_hi : 0.0, y)
                    : (ax == 0.0)                 ? gm_copysign(pio2_hi, y)
                    : (ax == GM_INF)              ? (ay == GM_INF ? gm_copysign(xneg ? 3.0 * pio4 : pio4, y)
                                                                  : gm_copysign(xneg ? pi_hi : 0.0, y))
                                                  : gm_copysign(pio2_hi, y);
  return special ? sv : regular;
}

/* ---------------------------------------------------------------- sin/cos */
GM_HD double gm_sin_poly(double r)
{
  double z = r * r;
  double p = 0x1.952c77030ad4ap-49;
  p = gm_fma(z, p, -0x1.ae7f3e733b81fp-41);
  p = gm_fma(z, p, 0x1.6124613a86d09p-33);
  p = gm_fma(z, p, -0x1.ae64567f544e4p-26);
  p = gm_fma(z, p, 0x1.71de3a556c734p-19);
  p = gm_fma(z, p, -0x1.a01a01a01a01ap-13);
  p = gm_fma(z, p, 0x1.1111111111111p-7);
  p = gm_fma(z, p, -0x1.5555555555555p-3);
  return r + r * (z * p);
}

GM_HD double gm_cos_poly(double r)
{
  double z = r * r;
  double p = -0x1.6827863b97d97p-53;
  p = gm_fma(z, p, 0x1.ae7f3e733b81fp-45);
  p = gm_fma(z, p, -0x1.93974a8c07c9dp-37);
  p = gm_fma(z, p, 0x1.1eed8eff8d898p-29);
  p = gm_fma(z, p, -0x1.27e4fb7789f5cp-22);
  p = gm_fma(z, p, 0x1.a01a01a01a01ap-16);
  p = gm_fma(z, p, -0x1.6c16c16c16c17p-10);
  p = gm_fma(z, p, 0x1.5555555555555p-5);
  double hz = 0.5 * z;
  double w = 1.0 - hz;
  return w + (((1.0 - w) - hz) + z * (z * p));
}

/* reduce x to r in [-pi/4, pi/4], returns quadrant n mod 4 */
GM_HD int gm_reduce_pio2(double x, double *r)
{
  const double two_over_pi = 0x1.45f306dc9c883p-1;
  const double P1 = 0x1.921fb54400000p+0, P2 = 0x1.0b4611a600000p-34, P3 = 0x1.3198a2e037073p-69;
  double n = gm_round(x * two_over_pi);
  *r = ((x - n * P1) - n * P2) - n * P3;
  return (int) (((int64_t) n) & 3);
}

GM_HD double gm_sin(double x)
{
  if(gm_isnan(x) || gm_fabs(x) == GM_INF) return GM_NAN;
  if(gm_fabs(x) < 0x1.0p-27) return x;
  double r;
  int q = gm_reduce_pio2(x, &r);
  switch(q) {
    case 0: return gm_sin_poly(r);
    case 1: return gm_cos_poly(r);
    case 2: return -gm_sin_poly(r);
    default: return -gm_cos_poly(r);
  }
}

GM_HD double gm_cos(double x)
{
  if(gm_isnan(x) || gm_fabs(x) == GM_INF) return GM_NAN;
  if(gm_fabs(x) < 0x1.0p-27) return 1.0;
  double r;
  int q = gm_reduce_pio2(x, &r);
  switch(q) {
    case 0: return gm_cos_poly(r);
    case 1: return -gm_sin_poly(r);
    case 2: return -gm_cos_poly(r);
    default: return gm_sin_poly(r);
  }
}

/* sin and cos of one argument: one reduction, both polynomials and the
 * quadrant's signs by selection, so a warp whose lanes sit in different
 * quadrants evaluates each polynomial once; *s and *c equal gm_sin(x) and
 * gm_cos(x) bit for bit */
GM_HD void gm_sincos(double x, double *s, double *c)
{
  const int bad = gm_isnan(x) || gm_fabs(x) == GM_INF;
  const int tiny = gm_fabs(x) < 0x1.0p-27;
  double r;
  const int q = gm_reduce_pio2(bad ? 0.0 : x, &r);
  const double ps = gm_sin_poly(r), pc = gm_cos_poly(r);
  const double sv = (q & 1) ? pc : ps, cv = (q & 1) ? ps : pc;
  const double sr = (q & 2) ? -sv : sv;       /* quadrants 2, 3: -sin, -cos poly */
  const double cr = ((q + 1) & 2) ? -cv : cv; /* quadrants 1, 2: -sin, -cos poly */
  *s = bad ? GM_NAN : (tiny ? x : sr);
  *c = bad ? GM_NAN : (tiny ? 1.0 : cr);
}

/* ---------------------------------------------------------------- exp */
/* Cody & Waite reduction x = k ln2 + r with k the integer nearest x/ln2
 * (|r| <= ln2/2; ln2 split as in gm_log, so k*ln2_hi is exact), e^r by its
 * Taylor series to degree 13 (truncation below 2^-57 relative), then the
 * scaling by 2^k in two exact-or-once-rounded steps, so that subnormal
 * results are rounded once. */
GM_HD double gm_exp(double x)
{
  const double ln2_hi = 0x1.62e42fee00000p-1;
  const double ln2_lo = 0x1.a39ef35793c76p-33;
  const double inv_ln2 = 0x1.71547652b82fep+0;

  if(gm_isnan(x)) return x;
  if(x > 710.0) return GM_INF;
  if(x < -746.0) return 0.0;
  double k = gm_round(x * inv_ln2);
  double r = (x - k * ln2_hi) - k * ln2_lo;
  double p = 0x1.6124613a86d09p-33; /* 1/13! */
  p = gm_fma(r, p, 0x1.1eed8eff8d898p-29);
  p = gm_fma(r, p, 0x1.ae64567f544e4p-26);
  p = gm_fma(r, p, 0x1.27e4fb7789f5cp-22);
  p = gm_fma(r, p, 0x1.71de3a556c734p-19);
  p = gm_fma(r, p, 0x1.a01a01a01a01ap-16);
  p = gm_fma(r, p, 0x1.a01a01a01a01ap-13);
  p = gm_fma(r, p, 0x1.6c16c16c16c17p-10);
  p = gm_fma(r, p, 0x1.1111111111111p-7);
  p = gm_fma(r, p, 0x1.5555555555555p-5);
  p = gm_fma(r, p, 0x1.5555555555555p-3);
  p = gm_fma(r, p, 0.5);
  p = gm_fma(r, p, 1.0);
  p = gm_fma(r, p, 1.0);
  int ki = (int) k;        /* |k| <= 1077 */
  int k1 = ki / 2, k2 = ki - k1;
  p *= gm_from_bits((uint64_t) (k1 + 1023) << 52); /* exact */
  return p * gm_from_bits((uint64_t) (k2 + 1023) << 52);
}

/* ---------------------------------------------------------------- acos */
GM_HD double gm_acos(double x)
{
  if(gm_isnan(x)) return x;
  if(x > 1.0 || x < -1.0) return GM_NAN;
  double s = (1.0 - x) * (1.0 + x);
#ifdef __CUDA_ARCH__
  double q = __dsqrt_rn(s);
#else
  double q = __builtin_sqrt(s);
#endif
  return gm_atan2(q, x);
}

/* ---------------------------------------------------------------- asin */
/* asin(x) = atan2(x, sqrt((1-x)(1+x))), the companion of gm_acos */
GM_HD double gm_asin(double x)
{
  if(gm_isnan(x)) return x;
  if(x > 1.0 || x < -1.0) return GM_NAN;
  double s = (1.0 - x) * (1.0 + x);
#ifdef __CUDA_ARCH__
  double q = __dsqrt_rn(s);
#else
  double q = __builtin_sqrt(s);
#endif
  return gm_atan2(x, q);
}

#endif
