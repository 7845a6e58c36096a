/*
 * grng.h - counter-based random numbers shared by the CUDA kernels and the
 * CPU oracle.
 *
 * GALIC draws every random number from one sequential GSL stream
 * (gsl_rng_ranlxd1 seeded 42+ThisTask, init.c:25-27).  The optimisation step
 * (optimize, main.c:365-435) consumes one uniform (the unused `dir_rnd`,
 * main.c:370) and then, per attempt of the escape-speed rejection loop
 * (main.c:415-435), three Gaussians via gsl_ran_gaussian.  A sequential stream
 * cannot be shared by thousands of GPU threads, so this project gives every
 * optimisation call its own stream of a counter-based generator,
 * Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11), keyed by (seed, particle, repetition serial).
 * The CPU oracle's GSL stand-in draws from the same streams, so the proposals
 * of both sides are identical.
 *
 * gaussian: Marsaglia & Bray's polar method (SIAM Review 6, 1964), the
 * method gsl_ran_gaussian uses: draw (x, y) uniform in the unit square until
 * 0 < x^2 + y^2 <= 1, return sigma * y * sqrt(-2 ln r2 / r2).  The logarithm
 * is gm_log so that both sides agree bit for bit.
 */
#ifndef GALIC_GRNG_H
#define GALIC_GRNG_H

#include <stdint.h>
#include "gmath.h"

typedef struct {
  uint32_t key[2];
  uint32_t ctr[4];   /* ctr[0..1]: block counter, ctr[2..3]: stream id */
  uint32_t buf[4];
  int have;          /* number of unused 32-bit words in buf (0, 2 or 4) */
} grng_t;

GM_HD void grng_mulhilo(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo)
{
  uint64_t p = (uint64_t) a * (uint64_t) b;
  *hi = (uint32_t) (p >> 32);
  *lo = (uint32_t) p;
}

/* Philox4x32 with 10 rounds */
GM_HD void grng_philox(const uint32_t in_ctr[4], const uint32_t in_key[2], uint32_t out[4])
{
  uint32_t c0 = in_ctr[0], c1 = in_ctr[1], c2 = in_ctr[2], c3 = in_ctr[3];
  uint32_t k0 = in_key[0], k1 = in_key[1];
  for(int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    grng_mulhilo(0xD2511F53u, c0, &hi0, &lo0);
    grng_mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

GM_HD void grng_init(grng_t *g, uint64_t seed, uint32_t stream_a, uint32_t stream_b)
{
  g->key[0] = (uint32_t) seed;
  g->key[1] = (uint32_t) (seed >> 32);
  g->ctr[0] = 0;
  g->ctr[1] = 0;
  g->ctr[2] = stream_a;
  g->ctr[3] = stream_b;
  g->have = 0;
}

/* uniform double in [0,1) with 53 random bits */
GM_HD double grng_uniform(grng_t *g)
{
  if(g->have == 0) {
    grng_philox(g->ctr, g->key, g->buf);
    if(++g->ctr[0] == 0) ++g->ctr[1];
    g->have = 4;
  }
  uint32_t a = g->buf[4 - g->have];
  uint32_t b = g->buf[5 - g->have];
  g->have -= 2;
  uint64_t bits = (((uint64_t) a << 32) | (uint64_t) b) >> 11;
  return (double) bits * 0x1.0p-53;
}

/* Uniform number k of a stream: words 2(k&1), 2(k&1)+1 of block k>>1 give
 * the k-th draw of grng_uniform, so any draw can be computed without the
 * ones before it. */
GM_HD double grng_uniform_at(uint64_t seed, uint32_t stream_a, uint32_t stream_b, uint64_t k)
{
  const uint32_t key[2] = {(uint32_t) seed, (uint32_t) (seed >> 32)};
  const uint32_t ctr[4] = {(uint32_t) (k >> 1), (uint32_t) (k >> 33), stream_a, stream_b};
  uint32_t out[4];
  grng_philox(ctr, key, out);
  const int w = (int) (k & 1) * 2;
  uint64_t bits = (((uint64_t) out[w] << 32) | (uint64_t) out[w + 1]) >> 11;
  return (double) bits * 0x1.0p-53;
}

/* index of the next uniform grng_uniform returns */
GM_HD uint64_t grng_position(const grng_t *g)
{
  uint64_t blocks = ((uint64_t) g->ctr[1] << 32) | g->ctr[0];
  return 2 * blocks - (uint64_t) (g->have / 2);
}

/* positions the stream so that the next grng_uniform returns draw k */
GM_HD void grng_seek(grng_t *g, uint64_t k)
{
  g->ctr[0] = (uint32_t) (k >> 1);
  g->ctr[1] = (uint32_t) (k >> 33);
  g->have = 0;
  if(k & 1) {
    grng_philox(g->ctr, g->key, g->buf);
    if(++g->ctr[0] == 0) ++g->ctr[1];
    g->have = 2;
  }
}

GM_HD double grng_gaussian(grng_t *g, double sigma)
{
  double x, y, r2;
  int guard = 0;
  do {
    x = -1.0 + 2.0 * grng_uniform(g);
    y = -1.0 + 2.0 * grng_uniform(g);
    r2 = x * x + y * y;
    if(++guard > 1000) return 0.0; /* probability ~ (1-pi/4)^1000: never */
  } while(r2 > 1.0 || r2 == 0);
#ifdef __CUDA_ARCH__
  return sigma * y * __dsqrt_rn(-2.0 * gm_log(r2) / r2);
#else
  return sigma * y * __builtin_sqrt(-2.0 * gm_log(r2) / r2);
#endif
}

#endif
