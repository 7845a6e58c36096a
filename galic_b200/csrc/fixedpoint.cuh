// Deterministic, order-independent accumulation of FP64 response values.
//
// GALIC sums every orbit's time-averaged response into per-type grids in
// particle order (main.c:214-223).  On the GPU thousands of orbits deposit
// concurrently; floating-point atomics would make every bin depend on the
// arrival order.  Instead each value v is rounded once to the integer
// X = round(v * 2^S) and split as X = H * 2^24 + L with 0 <= L < 2^24.  Two
// 64-bit integer atomics add H (signed) and L (unsigned) to a bin's word
// pair.  Integer addition is exact and associative, so the final pair is the
// same for any order; the bin value is H_sum * 2^(24-S) + L_sum * 2^-S.
//
// Range: S is chosen per field from a bound B on the field's total
// (S = 84 - ceil(log2 B)), so |H_sum| < 2^60 and the resolution is
// B * 2^-84 (~5e-26 B).  L_sum cannot overflow before 2^40 deposits per bin.
#ifndef GALIC_FIXEDPOINT_CUH
#define GALIC_FIXEDPOINT_CUH

#include <stdint.h>

struct FxWord {
  unsigned long long hi;  // two's-complement sum of H
  unsigned long long lo;  // sum of L
};

__device__ __forceinline__ void fx_split(double v, int S, long long *H, unsigned long long *L)
{
  double t = ldexp(v, S - 24);  // exact power-of-two scaling
  double fh = floor(t);         // exact
  double fr = t - fh;           // exact, in [0,1)
  long long h = (long long) fh;
  unsigned long long l = (unsigned long long) rint(fr * 16777216.0);  // fr * 2^24 exact, rounded once
  if(l == 16777216ULL) {
    l = 0;
    h += 1;
  }
  *H = h;
  *L = l;
}

// the word pair of t = v * 2^(S-24) (t given: a caller that scales many values
// by the same power of two and factor folds them into one multiplier; a
// power-of-two factor is exact, so the pair equals fx_split's)
__device__ __forceinline__ void fx_split_scaled(double t, long long *H, unsigned long long *L)
{
  double fh = floor(t);
  double fr = t - fh;
  long long h = (long long) fh;
  unsigned long long l = (unsigned long long) rint(fr * 16777216.0);
  if(l == 16777216ULL) {
    l = 0;
    h += 1;
  }
  *H = h;
  *L = l;
}

__device__ __forceinline__ void fx_add_scaled(FxWord *w, double t)
{
  if(t == 0.0) return;
  long long H;
  unsigned long long L;
  fx_split_scaled(t, &H, &L);
  if(H) atomicAdd(&w->hi, (unsigned long long) H);
  if(L) atomicAdd(&w->lo, L);
}

// adds v to the word pair w (no return value needed: red.global.add.u64)
__device__ __forceinline__ void fx_add(FxWord *w, double v, int S)
{
  if(v == 0.0) return;
  long long H;
  unsigned long long L;
  fx_split(v, S, &H, &L);
  if(H) atomicAdd(&w->hi, (unsigned long long) H);
  if(L) atomicAdd(&w->lo, L);
}

__host__ __device__ __forceinline__ double fx_value(FxWord w, int S)
{
  long long h = (long long) w.hi;
#ifdef __CUDA_ARCH__
  return ldexp((double) h, 24 - S) + ldexp((double) w.lo, -S);
#else
  return __builtin_ldexp((double) h, 24 - S) + __builtin_ldexp((double) w.lo, -S);
#endif
}

#endif
