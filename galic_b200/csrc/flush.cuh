// Warp-cooperative flush of merged deposits into the fixed-point grids.
//
// Each lane of the batched orbit kernels merges the deposits of consecutive
// steps that fall into the same DG cell in registers (20 values: 4 corners x
// {m, m vr2, m vt2, m vq2, m vp2}).  When its cell changes, the lane only
// parks the 20 values (already scaled by mass/Tint) in its slot of a per-warp
// shared-memory queue.  At one fixed point of every loop iteration the whole
// warp drains all parked slots together: item k of slot s is handled by lane
// k mod 32, so the fixed-point conversion and the two integer atomics of every
// value run on full warps instead of on the one lane whose cell changed.
#ifndef GALIC_FLUSH_CUH
#define GALIC_FLUSH_CUH

#include "fixedpoint.cuh"
#include "kernels.cuh"

struct WarpQueue {
  double val[32][20];  // [slot][corner * 5 + field]
  int cell[32];        // base cell iz*Nb+iR of the slot
  int type[32];
  int list[32];        // compacted occupied slots of one drain
};

// all 32 lanes call this with the same `full` mask (slots to drain)
__device__ __forceinline__ void warp_drain(WarpQueue &q, unsigned full, FxWord *fx, const int *shift, int G, int Nb)
{
  const int lane = threadIdx.x & 31;
  if(full & (1u << lane)) q.list[__popc(full & ((1u << lane) - 1))] = lane;
  __syncwarp();
  const int items = __popc(full) * 20;
  for(int it = lane; it < items; it += 32) {
    const int s = q.list[it / 20];
    const int k = it - (it / 20) * 20;
    const int corner = k / 5, f = k - corner * 5;
    const int off = (corner & 1) + ((corner >> 1) ? Nb : 0);
    const int t = q.type[s];
    fx_add(&fx[((size_t) t * NG_COMMITTED + f) * G + q.cell[s] + off], q.val[s][k], shift[t * NG_COMMITTED + f]);
  }
  __syncwarp();
}

// FP32 variant.  A lane parks one record per grid node that leaves its
// accumulators: the node's word index and its five sums already scaled by
// value x 2^(shift-24) in FP32 (the orbit's mass/Tint and the field's
// fixed-point scale are folded into one FP32 factor per field class when the
// orbit starts).  The drain rounds each item to one
// signed 64-bit fixed-point word, X = round(scaled value), and adds it to the
// high word of the bin (the low word stays zero, so fx_value reads it
// unchanged).  shift - 24 is chosen so that no bin can overflow 2^62; the
// FP32 rounding of the scaled value (2^-24 relative) is far inside the FP32
// form's tolerance, and one atomic per value instead of two halves the L2
// atomic traffic.
struct WarpQueue32 {
  int base[32 * 4];      // word of the node's mass field; field f is base + f * Ngrid
  float val[32 * 4][5];  // the node's five sums, scaled to fixed point
  int n;                 // records parked since the last drain
  int gbase[32];         // per lane: first word of its orbit's grid set
  float2 scale[32];      // per lane: {mass field, energy fields} fixed-point factors
};

// a lane reserves room for `count` node records; returns the first index
__device__ __forceinline__ int queue32_reserve(WarpQueue32 &q, int count) { return atomicAdd(&q.n, count); }

// all 32 lanes call this at the same point of the loop; each lane adds the
// five words of one parked node record at a time
__device__ __forceinline__ void warp_drain32(WarpQueue32 &q, FxWord *fx, int G)
{
  __syncwarp();
  const int lane = threadIdx.x & 31;
  const int records = q.n;
  for(int r = lane; r < records; r += 32) {
    const int b = q.base[r];
#pragma unroll
    for(int f = 0; f < 5; f++) {
      const long long X = __float2ll_rn(q.val[r][f]);
      if(X) atomicAdd(&fx[b + f * G].hi, (unsigned long long) X);
    }
  }
  __syncwarp();
  if(lane == 0) q.n = 0;
  __syncwarp();
}

#endif
