// CTA-cooperative versions of GALIC's stack routines.
//
// A stack holds a quadtree pyramid of a 2^L x 2^L grid; level l starts at
// STACKOFFSET(l,0,0) = (4^l - 1)/3 (allvars.h:160).  One CTA keeps a whole
// stack in shared memory (L = 7: 21845 doubles, 171 KiB).
//
// stack_smooth_cta: smooth_stack (grid.c:1247-1265), level by level, same
//                   summation order.
// stack_diff_cta:   calc_stack_difference[_mod] (grid.c:1086-1151).  The
//                   reference recurses from the root and stops at a node when
//                   l == maxlevel or ref1[node] < thresh.  Evaluated bottom
//                   up instead: every node gets either its leaf term or the
//                   sum of its four children's values in the recursion's
//                   order ((c(2i,2j) + c(2i,2j+1)) + c(2i+1,2j)) + c(2i+1,2j+1),
//                   which gives the recursion's result bit for bit.  The
//                   values overwrite the stack in place (a node's own d1 is
//                   read before its value is written).
#ifndef GALIC_STACK_CUH
#define GALIC_STACK_CUH

__device__ __forceinline__ int stack_off(int l) { return ((1 << (2 * l)) - 1) / 3; }

__device__ __forceinline__ void stack_smooth_cta(double *s, int L)
{
  for(int l = L - 1; l >= 0; l--) {
    const int n = 1 << l, base = stack_off(l), cb = stack_off(l + 1), cn = n << 1;
    for(int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      int i = idx >> l, j = idx & (n - 1);
      s[base + idx] = s[cb + (2 * i) * cn + 2 * j] + s[cb + (2 * i + 1) * cn + 2 * j] +
                      s[cb + (2 * i) * cn + 2 * j + 1] + s[cb + (2 * i + 1) * cn + 2 * j + 1];
    }
    __syncthreads();
  }
}

// leaf term; mode 0 = calc_stack_difference, 1 = calc_stack_difference_mod
__device__ __forceinline__ double stack_leaf(double d1, double d2, double r1, double r2, double dist, int flag,
                                             int mod, double R200_20, double lowdisp)
{
  if(mod && flag == 2) {
    if(r2 > 0) return fabs(d1 - d2) * (r1 / r2) / (dist < R200_20 ? dist : R200_20);
    return 0;
  }
  if(flag) {
    if(r1 > 0 && r2 > 0) {
      double q2 = d2 / r2;
      return fabs(d1 / r1 - q2) / (q2 > lowdisp ? q2 : lowdisp);
    }
    return 0;
  }
  return fabs(d1 - d2) / (dist < R200_20 ? dist : R200_20);
}

// s: smoothed d1 stack in shared memory (overwritten); returns the result to
// every thread.  ref2/dist may be null where the reference passes NULL.
__device__ __forceinline__ double stack_diff_cta(double *s, const double *d2, const double *ref1, const double *ref2,
                                                 const double *dist, double thresh, int flag, int mod, int L,
                                                 double R200_20, double lowdisp)
{
  for(int l = L; l >= 0; l--) {
    const int n = 1 << l, base = stack_off(l);
    const int cb = stack_off(l + 1), cn = n << 1;
    for(int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const int node = base + idx;
      const double r1 = ref1[node];
      double v;
      if(l >= L || r1 < thresh) {
        v = stack_leaf(s[node], d2[node], r1, ref2 ? ref2[node] : 0.0, dist ? dist[node] : 0.0, flag, mod, R200_20,
                       lowdisp);
      } else {
        int i = idx >> l, j = idx & (n - 1);
        v = s[cb + (2 * i) * cn + 2 * j];
        v += s[cb + (2 * i) * cn + 2 * j + 1];
        v += s[cb + (2 * i + 1) * cn + 2 * j];
        v += s[cb + (2 * i + 1) * cn + 2 * j + 1];
      }
      s[node] = v;
    }
    __syncthreads();
  }
  double r = s[0];
  __syncthreads();
  return r;
}

// The same two routines for a pyramid whose finest level (level L) is not
// stored: fin(i) returns its value at grid index i = iz * 2^L + iR (a sum
// the caller forms on the fly from global memory), and s holds levels
// 0 .. L-1 only ((4^L - 1) / 3 doubles: 43 KiB at L = 7 instead of 171 KiB).
// Level L-1 is summed from fin() in smooth_stack's order; in the misfit a
// non-leaf node of level L-1 evaluates its four children's leaf terms from
// fin() and the reference arrays, in the recursion's order.  Same values,
// same operations: bit-identical to the stored-stack versions.
template <class F>
__device__ __forceinline__ void stack_smooth_cta_from(double *s, int L, const F &fin)
{
  {
    const int l = L - 1, n = 1 << l, base = stack_off(l), cn = n << 1;
    for(int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const int i = idx >> l, j = idx & (n - 1);
      s[base + idx] = fin((2 * i) * cn + 2 * j) + fin((2 * i + 1) * cn + 2 * j) + fin((2 * i) * cn + 2 * j + 1) +
                      fin((2 * i + 1) * cn + 2 * j + 1);
    }
    __syncthreads();
  }
  for(int l = L - 2; l >= 0; l--) {
    const int n = 1 << l, base = stack_off(l), cb = stack_off(l + 1), cn = n << 1;
    for(int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      int i = idx >> l, j = idx & (n - 1);
      s[base + idx] = s[cb + (2 * i) * cn + 2 * j] + s[cb + (2 * i + 1) * cn + 2 * j] +
                      s[cb + (2 * i) * cn + 2 * j + 1] + s[cb + (2 * i + 1) * cn + 2 * j + 1];
    }
    __syncthreads();
  }
}

template <class F>
__device__ __forceinline__ double stack_diff_cta_from(double *s, const F &fin, const double *d2, const double *ref1,
                                                      const double *ref2, const double *dist, double thresh,
                                                      int flag, int mod, int L, double R200_20, double lowdisp)
{
  const int cbL = stack_off(L);
  // leaf term of the finest-level node at grid index g
  auto fine_leaf = [&](int g) {
    const int node = cbL + g;
    return stack_leaf(fin(g), d2[node], ref1[node], ref2 ? ref2[node] : 0.0, dist ? dist[node] : 0.0, flag, mod,
                      R200_20, lowdisp);
  };
  for(int l = L - 1; l >= 0; l--) {
    const int n = 1 << l, base = stack_off(l);
    const int cb = stack_off(l + 1), cn = n << 1;
    for(int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
      const int node = base + idx;
      const double r1 = ref1[node];
      double v;
      if(r1 < thresh) {
        v = stack_leaf(s[node], d2[node], r1, ref2 ? ref2[node] : 0.0, dist ? dist[node] : 0.0, flag, mod, R200_20,
                       lowdisp);
      } else {
        const int i = idx >> l, j = idx & (n - 1);
        if(l == L - 1) {
          v = fine_leaf((2 * i) * cn + 2 * j);
          v += fine_leaf((2 * i) * cn + 2 * j + 1);
          v += fine_leaf((2 * i + 1) * cn + 2 * j);
          v += fine_leaf((2 * i + 1) * cn + 2 * j + 1);
        } else {
          v = s[cb + (2 * i) * cn + 2 * j];
          v += s[cb + (2 * i) * cn + 2 * j + 1];
          v += s[cb + (2 * i + 1) * cn + 2 * j];
          v += s[cb + (2 * i + 1) * cn + 2 * j + 1];
        }
      }
      s[node] = v;
    }
    __syncthreads();
  }
  double r = s[0];
  __syncthreads();
  return r;
}

#endif
