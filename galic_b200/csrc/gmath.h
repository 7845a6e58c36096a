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
 *  - log:   Tang's table-driven method (ACM TOMS 16(4), 1990): x = 2^k m,
 *           r = m/c_j - 1 formed as one FMA with a 12-bit reciprocal of
 *           c_j = 1 + j/128, log(c_j) from a head/tail table, log1p(r) by its
 *           Taylor series; no division.  ln2 is split into a
 *           32-fractional-bit head and a tail so that k*ln2_hi is exact.
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
/* Tables of gm_log (galic_b200/csrc/gen_gmath_tables.py): inv_j = 1/(1 + j/128)
 * rounded to 12 significant bits, -log(inv_j) = th_j + tl_j with th_j on a
 * 2^-42 grid. */
#define GM_LOG_INV {0x1.0000000000000p+0, 0x1.fc00000000000p-1, 0x1.f820000000000p-1, 0x1.f440000000000p-1, 0x1.f080000000000p-1, 0x1.ecc0000000000p-1, 0x1.e920000000000p-1, 0x1.e580000000000p-1, 0x1.e1e0000000000p-1, 0x1.de60000000000p-1, 0x1.dae0000000000p-1, 0x1.d780000000000p-1, 0x1.d420000000000p-1, 0x1.d0c0000000000p-1, 0x1.cd80000000000p-1, 0x1.ca40000000000p-1, 0x1.c720000000000p-1, 0x1.c400000000000p-1, 0x1.c0e0000000000p-1, 0x1.bde0000000000p-1, 0x1.bac0000000000p-1, 0x1.b7e0000000000p-1, 0x1.b4e0000000000p-1, 0x1.b200000000000p-1, 0x1.af20000000000p-1, 0x1.ac60000000000p-1, 0x1.a980000000000p-1, 0x1.a6e0000000000p-1, 0x1.a420000000000p-1, 0x1.a160000000000p-1, 0x1.9ec0000000000p-1, 0x1.9c20000000000p-1, 0x1.99a0000000000p-1, 0x1.9700000000000p-1, 0x1.9480000000000p-1, 0x1.9200000000000p-1, 0x1.8fa0000000000p-1, 0x1.8d40000000000p-1, 0x1.8ac0000000000p-1, 0x1.8860000000000p-1, 0x1.8620000000000p-1, 0x1.83c0000000000p-1, 0x1.8180000000000p-1, 0x1.7f40000000000p-1, 0x1.7d00000000000p-1, 0x1.7ae0000000000p-1, 0x1.78a0000000000p-1, 0x1.7680000000000p-1, 0x1.7460000000000p-1, 0x1.7240000000000p-1, 0x1.7020000000000p-1, 0x1.6e20000000000p-1, 0x1.6c20000000000p-1, 0x1.6a20000000000p-1, 0x1.6820000000000p-1, 0x1.6620000000000p-1, 0x1.6420000000000p-1, 0x1.6240000000000p-1, 0x1.6060000000000p-1, 0x1.5e80000000000p-1, 0x1.5ca0000000000p-1, 0x1.5ac0000000000p-1, 0x1.58e0000000000p-1, 0x1.5720000000000p-1, 0x1.5560000000000p-1, 0x1.53a0000000000p-1, 0x1.51e0000000000p-1, 0x1.5020000000000p-1, 0x1.4e60000000000p-1, 0x1.4ca0000000000p-1, 0x1.4b00000000000p-1, 0x1.4960000000000p-1, 0x1.47a0000000000p-1, 0x1.4600000000000p-1, 0x1.4460000000000p-1, 0x1.42e0000000000p-1, 0x1.4140000000000p-1, 0x1.3fc0000000000p-1, 0x1.3e20000000000p-1, 0x1.3ca0000000000p-1, 0x1.3b20000000000p-1, 0x1.39a0000000000p-1, 0x1.3820000000000p-1, 0x1.36a0000000000p-1, 0x1.3520000000000p-1, 0x1.33a0000000000p-1, 0x1.3240000000000p-1, 0x1.30e0000000000p-1, 0x1.2f60000000000p-1, 0x1.2e00000000000p-1, 0x1.2ca0000000000p-1, 0x1.2b40000000000p-1, 0x1.29e0000000000p-1, 0x1.2880000000000p-1, 0x1.2740000000000p-1, 0x1.25e0000000000p-1, 0x1.24a0000000000p-1, 0x1.2340000000000p-1, 0x1.2200000000000p-1, 0x1.20c0000000000p-1, 0x1.1f80000000000p-1, 0x1.1e20000000000p-1, 0x1.1d00000000000p-1, 0x1.1bc0000000000p-1, 0x1.1a80000000000p-1, 0x1.1940000000000p-1, 0x1.1820000000000p-1, 0x1.16e0000000000p-1, 0x1.15c0000000000p-1, 0x1.1480000000000p-1, 0x1.1360000000000p-1, 0x1.1240000000000p-1, 0x1.1120000000000p-1, 0x1.0fe0000000000p-1, 0x1.0ec0000000000p-1, 0x1.0dc0000000000p-1, 0x1.0ca0000000000p-1, 0x1.0b80000000000p-1, 0x1.0a60000000000p-1, 0x1.0960000000000p-1, 0x1.0840000000000p-1, 0x1.0740000000000p-1, 0x1.0620000000000p-1, 0x1.0520000000000p-1, 0x1.0420000000000p-1, 0x1.0300000000000p-1, 0x1.0200000000000p-1, 0x1.0100000000000p-1, 0x1.0000000000000p-1}
#define GM_LOG_TH {0x0.0p+0, 0x1.0101575880000p-7, 0x1.fbea8b13c0000p-7, 0x1.7c61b1cf60000p-6, 0x1.f7a9b16780000p-6, 0x1.39f07ba0e8000p-5, 0x1.766d923c20000p-5, 0x1.b35dd9b588000p-5, 0x1.f0c30c1118000p-5, 0x1.163d6ef958000p-4, 0x1.345179b63c000p-4, 0x1.5188742260000p-4, 0x1.6ef528c058000p-4, 0x1.8c985e9ba0000p-4, 0x1.a956d3ecac000p-4, 0x1.c6494a2e40000p-4, 0x1.e2507702b0000p-4, 0x1.fe89139dbc000p-4, 0x1.0d79e7cd48000p-3, 0x1.1b35ae3b82000p-3, 0x1.299d30c606000p-3, 0x1.36f4c27578000p-3, 0x1.44f8b726f8000p-3, 0x1.527e5e4a1c000p-3, 0x1.601b076e7a000p-3, 0x1.6d35fee52c000p-3, 0x1.7b00916516000p-3, 0x1.87ad07c494000p-3, 0x1.9509aa0044000p-3, 0x1.a27cc30640000p-3, 0x1.af6895610e000p-3, 0x1.bc69684aee000p-3, 0x1.c8df7cb9a8000p-3, 0x1.d60a17f904000p-3, 0x1.e2a877a6b2000p-3, 0x1.ef5ade4dd0000p-3, 0x1.fb7d86eee4000p-3, 0x1.03d95a1d67000p-2, 0x1.0a504e97bb000p-2, 0x1.107e404ab1000p-2, 0x1.1661caecba000p-2, 0x1.1ca28c64bb000p-2, 0x1.22981fbef8000p-2, 0x1.2896a13e08000p-2, 0x1.2e9e2bce12000p-2, 0x1.34585a594c000p-2, 0x1.3a71c56bb5000p-2, 0x1.403d086cea000p-2, 0x1.4610bc29c6000p-2, 0x1.4becf95d98000p-2, 0x1.51d1d93104000p-2, 0x1.5765f1749e000p-2, 0x1.5d01dc49ff000p-2, 0x1.62a5afc061000p-2, 0x1.68518244d0000p-2, 0x1.6e056aa442000p-2, 0x1.73c1800dc1000p-2, 0x1.792955fdf4000p-2, 0x1.7e9883fa4a000p-2, 0x1.840f1e1266000p-2, 0x1.898d38a893000p-2, 0x1.8f12e87386000p-2, 0x1.94a0428036000p-2, 0x1.99d5d81306000p-2, 0x1.9f123f4bf7000p-2, 0x1.a4558a1c9c000p-2, 0x1.a99fcabdb8000p-2, 0x1.aef113b0bc000p-2, 0x1.b44977c149000p-2, 0x1.b9a90a06bd000p-2, 0x1.beacd9e272000p-2, 0x1.c3b6fb361e000p-2, 0x1.c92b7d6bb1000p-2, 0x1.ce42f18064000p-2, 0x1.d360e90c38000p-2, 0x1.d81ff2cce9000p-2, 0x1.dd4aa04e1c000p-2, 0x1.e21582ecdc000p-2, 0x1.e74d262789000p-2, 0x1.ec241d5e30000p-2, 0x1.f100f6c2eb000p-2, 0x1.f5e3c0b542000p-2, 0x1.facc89c9aa000p-2, 0x1.ffbb60ca86000p-2, 0x1.02582a5c9d000p-1, 0x1.04d5ba679b000p-1, 0x1.0720e5c40e000p-1, 0x1.096eb58872800p-1, 0x1.0bf52e7353800p-1, 0x1.0e4898611d000p-1, 0x1.109eb9e2e5000p-1, 0x1.12f799594f000p-1, 0x1.15533d3b8d800p-1, 0x1.17b1ac17cc000p-1, 0x1.19db6ba0ba800p-1, 0x1.1c3f41fa98000p-1, 0x1.1e6df676ff800p-1, 0x1.20d74d2fbb000p-1, 0x1.230b0d8bec000p-1, 0x1.25413d529c800p-1, 0x1.2779e1ec94000p-1, 0x1.29ee409f15800p-1, 0x1.2bf29f9842000p-1, 0x1.2e32c3d74d800p-1, 0x1.30757344f1000p-1, 0x1.32bab3a7b2000p-1, 0x1.34c80a8958000p-1, 0x1.37123b5498800p-1, 0x1.39240dde5d000p-1, 0x1.3b7344be40000p-1, 0x1.3d89a6b1a5800p-1, 0x1.3fa238ac24800p-1, 0x1.41bcff4860000p-1, 0x1.44163ef728000p-1, 0x1.4635bcf40e000p-1, 0x1.481abdce32800p-1, 0x1.4a3e862342800p-1, 0x1.4c649aff0f000p-1, 0x1.4e8d015787000p-1, 0x1.5079fd4736800p-1, 0x1.52a6d269bc800p-1, 0x1.5497c72923000p-1, 0x1.56c91d71cf800p-1, 0x1.58be1b857b000p-1, 0x1.5ab505b390800p-1, 0x1.5ced1e17c3800p-1, 0x1.5ee82aa241800p-1, 0x1.60e52f4578800p-1, 0x1.62e42fefa3800p-1}
#define GM_LOG_TL {0x0.0p+0, 0x1.bce251998b506p-44, 0x1.ec927b17e4e13p-50, -0x1.08fc8f849a447p-45, 0x1.42ad9271be7d7p-45, 0x1.eb129d642e577p-44, 0x1.ff0a82f1c24c1p-46, 0x1.d5674d6cf558ep-44, -0x1.caef3588b7d80p-45, -0x1.7f3b038d8e6ebp-46, 0x1.d4203d36150d0p-44, 0x1.30a1d96258b3ep-44, -0x1.5d462d767cadep-44, -0x1.37c377e430036p-44, 0x1.e63794c02c4afp-44, 0x1.8a5e8ab20c4e6p-44, -0x1.f897980522249p-45, 0x1.56594d82f7a82p-44, 0x1.cb422847849e4p-44, -0x1.20a2e76016a9dp-46, 0x1.d4d0079dc08d9p-44, -0x1.4d9e2683a54edp-44, 0x1.df6a4432b9bb4p-44, -0x1.4e60b8d4b411dp-44, 0x1.152d7d4dfc8e5p-44, -0x1.f127eb4f64e1fp-45, -0x1.ae75fcb067e57p-44, -0x1.70f53c386330ap-44, 0x1.f1e675b4d35c6p-44, 0x1.d954963274bb8p-44, -0x1.148288bf7a937p-45, 0x1.8f6d5d141f9bdp-45, 0x1.eee42f58e1e6ep-44, -0x1.5d6e06fc20d39p-44, 0x1.823817787081ap-44, -0x1.a211565bb8e11p-51, -0x1.1c061cdb8097bp-45, 0x1.a17880f236109p-44, 0x1.03094e6690c44p-44, -0x1.fb921823aafdap-48, -0x1.171fff9fc4abbp-44, -0x1.ac4f842f5566bp-46, -0x1.a1421609580dap-44, 0x1.a8ed027e16952p-44, 0x1.4300c128d1dc2p-45, -0x1.d4d9bf230f411p-44, -0x1.ce772094aef70p-44, 0x1.e6ef574487308p-44, -0x1.e82c9f310c8e6p-46, -0x1.bb33b20023a70p-44, 0x1.5b0faa20d9c8ep-44, -0x1.6532d93e0d82bp-44, 0x1.740ab8cfa5ed3p-45, 0x1.0f54a2beeff32p-45, -0x1.3c6e803ba0773p-44, 0x1.d5417249679bcp-46, -0x1.9be4811571280p-45, 0x1.e889b0253ca88p-44, -0x1.401a62f035dd6p-50, 0x1.fc03bddc7f361p-44, 0x1.1f666071e2f57p-44, 0x1.63e9b66795610p-45, 0x1.0e7bcb08c6b44p-44, 0x1.f2041f94ec30bp-48, -0x1.2edbfd41b7fc2p-45, -0x1.f70faf3f84ff8p-44, 0x1.1e89c5f87a311p-46, 0x1.de1e7f07adbd4p-44, -0x1.cae5e0256c925p-47, -0x1.308b53f5c09fdp-44, -0x1.4bac8923c3257p-44, 0x1.80ab596d9efcap-45, -0x1.bc058001e24cfp-44, 0x1.d0d0798270b2ap-44, 0x1.42cdb58440fd6p-44, -0x1.6c99c641aa0c0p-44, 0x1.2d8512df01afdp-44, -0x1.18dfb659ddea2p-47, -0x1.e146ba126ba84p-44, -0x1.83f91f5d1fb7bp-49, 0x1.cce779d37f3d8p-45, 0x1.717da2f1dc6a9p-44, -0x1.a707cbbfc4e25p-44, 0x1.d9555b2ef9e1dp-45, 0x1.22c6c4e98e18cp-45, -0x1.b298eb21bad44p-44, -0x1.c762ffd3f0109p-46, 0x1.6eab8ed791a8ap-44, 0x1.9b5899cd387d3p-46, -0x1.8f599fe1ffa30p-44, -0x1.b496635b07d06p-44, -0x1.0e0950a8ee2fbp-47, -0x1.33f1aba7961e6p-47, -0x1.52762a46c5b48p-44, -0x1.24c53bd2daeccp-44, -0x1.ca798412ff675p-44, 0x1.a58ba81b983aap-46, -0x1.b321c53d151e2p-49, -0x1.b40fe646de661p-44, 0x1.76dfca70af4b9p-44, -0x1.35b991994c90fp-45, -0x1.dfca5febcc6f0p-44, -0x1.e275c79e2c481p-44, -0x1.3a9e0d9bfad3ep-44, -0x1.ec82f533a1f99p-45, 0x1.e86c98c5d5b38p-45, 0x1.d4093fcac34bdp-46, -0x1.26a88b54debbfp-47, -0x1.6d8482a914e99p-45, 0x1.88bb6943a0521p-44, -0x1.39c19502bf0e1p-44, 0x1.49eb5a15b20a8p-46, 0x1.76fd6b90e2a84p-47, 0x1.ec58a3f8fb594p-44, -0x1.18b9515f69aa9p-44, -0x1.33ceb89775f8bp-50, -0x1.6d82b36043dcep-44, -0x1.ea4e6e935367dp-45, -0x1.d38fcbf3f2776p-46, -0x1.07e991980a7afp-45, -0x1.ffbbb2e12ec6dp-45, 0x1.d74b64ca8a320p-44, 0x1.07bafd1366e9ep-49, -0x1.422bd0cc58b53p-45, -0x1.faa7614266a70p-44, -0x1.1d52fdabeaa73p-44, 0x1.202380cda46bep-45, 0x1.c6ea5e681638dp-46, 0x1.ef35793c76730p-45}

#ifdef __CUDACC__
static __device__ const double gm_log_inv_dev[129] = GM_LOG_INV;
static __device__ const double gm_log_th_dev[129] = GM_LOG_TH;
static __device__ const double gm_log_tl_dev[129] = GM_LOG_TL;
#endif
static const double gm_log_inv_host[129] = GM_LOG_INV;
static const double gm_log_th_host[129] = GM_LOG_TH;
static const double gm_log_tl_host[129] = GM_LOG_TL;

/* Table-driven logarithm without a division (P. T. P. Tang, "Table-driven
 * implementation of the logarithm function in IEEE floating-point
 * arithmetic", ACM TOMS 16(4), 1990): x = 2^k m, m in [1,2);
 * j = round(128 (m - 1)); r = m inv_j - 1 with one rounding (FMA; |r| < 2^-7);
 * log x = (k ln2_hi + th_j) + (r + (r^2 P(r) + (k ln2_lo + tl_j))) with
 * P the Taylor coefficients of (log1p(r) - r) / r^2 to degree 8.  The head
 * k ln2_hi + th_j is exact (ln2_hi has 32 significant bits, th_j lies on a
 * 2^-42 grid).  Special arguments (NaN, negative, zero, infinity) are
 * selected at the end and the subnormal scaling is a selection: the body is
 * one basic block, so the several logs of an orbit step interleave. */
GM_HD double gm_log(double x)
{
  const double ln2_hi = 0x1.62e42fee00000p-1;
  const double ln2_lo = 0x1.a39ef35793c76p-33;
#ifdef __CUDA_ARCH__
  const double *T_inv = gm_log_inv_dev, *T_h = gm_log_th_dev, *T_l = gm_log_tl_dev;
#else
  const double *T_inv = gm_log_inv_host, *T_h = gm_log_th_host, *T_l = gm_log_tl_host;
#endif
  const int sub = (gm_bits(x) >> 52) == 0; /* +0 and positive subnormals: scale up by 2^54 */
  const double xs = sub ? x * 0x1.0p54 : x;
  const uint64_t u = gm_bits(xs);
  const int k = (sub ? -54 : 0) + (int) ((u >> 52) & 0x7ff) - 1023;
  const double m = gm_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
  const int j = (int) ((m - 1.0) * 128.0 + 0.5);                                      /* 0..128 */
  const double r = gm_fma(m, T_inv[j], -1.0);
  /* (log1p(r) - r) / r^2 = -1/2 + r/3 - r^2/4 + ... - r^6/8 */
  double p = -0x1.0000000000000p-3;
  p = gm_fma(r, p, 0x1.2492492492492p-3);
  p = gm_fma(r, p, -0x1.5555555555555p-3);
  p = gm_fma(r, p, 0x1.999999999999ap-3);
  p = gm_fma(r, p, -0x1.0000000000000p-2);
  p = gm_fma(r, p, 0x1.5555555555555p-2);
  p = gm_fma(r, p, -0.5);
  const double dk = (double) k;
  const double head = dk * ln2_hi + T_h[j]; /* exact */
  const double res = head + (r + ((r * r) * p + (dk * ln2_lo + T_l[j])));
  return gm_isnan(x) ? x : (x < 0 ? GM_NAN : (x == 0 ? -GM_INF : (x == GM_INF ? x : res)));
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
