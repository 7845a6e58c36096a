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

// Node-record variant (the FP32 form, and the FP64 form's batched kernel
// with FP64 sums).  A lane parks one record per grid node that leaves its
// accumulators: the node's index and its five sums.  The drain scales them
// by value x 2^(shift-24) in FP32 (the orbit's mass/Tint and the field's
// fixed-point scale folded into one FP32 factor per field class when the
// orbit starts, kept in the lane's queue header), rounds each item to one
// signed 64-bit fixed-point word, X = round(scaled value), and adds it to the
// high word of the bin (the low word stays zero, so fx_value reads it
// unchanged).  shift - 24 is chosen so that no bin can overflow 2^62; the
// FP32 rounding of the scaled value (2^-24 relative) is far inside the FP32
// form's tolerance, and one atomic per value instead of two halves the L2
// atomic traffic.
// Each lane parks its node records in its own column of the warp's queue
// (no reservation atomic); a lane parks at most 4 records per loop iteration
// (one cell's nodes), so the warp drains before any lane could pass PER.
// The drain compacts all lanes' records and every lane adds the five words of
// one record at a time, so the global atomics run on full warps.  PER is
// chosen per block size so that the queues fit the static shared memory.
template <int PER_, class T>
struct WarpQueueT {
  static constexpr int PER = PER_;
  int base[PER][32];  // the node's index in its grid (field f of the orbit's set: gbase + f * Ngrid + base)
  T val[PER][5][32];  // the node's five sums
  int off[32];        // drain: first compacted record of each lane
  int gbase[32];      // per lane: first word of its orbit's grid set
  T scale[2][32];     // per lane: {mass field, energy fields} fixed-point factors
};
template <int PER>
using WarpQueue32 = WarpQueueT<PER, float>;

// records per lane of a block of BLOCK threads (FP32 sums)
__host__ __device__ constexpr int queue32_per(int block) { return block <= 128 ? 8 : (block <= 192 ? 7 : 5); }

// true when some lane could not park another cell's nodes
template <int PER>
__device__ __forceinline__ bool queue32_due(int cnt)
{
  return __any_sync(0xffffffffu, cnt > PER - 4);
}

__device__ __forceinline__ long long to_fixed(float v) { return __float2ll_rn(v); }
__device__ __forceinline__ long long to_fixed(double v) { return __double2ll_rn(v); }

// all 32 lanes call this at the same point of the loop with their record
// counts; cnt is 0 on return
template <int PER, class T>
__device__ __forceinline__ void warp_drain_nodes(WarpQueueT<PER, T> &q, FxWord *fx, int G, int &cnt)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int incl = cnt;
#pragma unroll
  for(int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if(lane >= o) incl += y;
  }
  const int total = __shfl_sync(FULL, incl, 31);
  q.off[lane] = incl - cnt;
  __syncwarp();
  for(int r = lane; r < total; r += 32) {
    // the lane L whose records hold r: the last L with off[L] <= r
    int L = 0;
#pragma unroll
    for(int step = 16; step; step >>= 1)
      if(q.off[L + step] <= r) L += step;
    const int k = r - q.off[L];
    const int b = q.gbase[L] + q.base[k][L];
    const T sm = q.scale[0][L], se = q.scale[1][L];
#pragma unroll
    for(int f = 0; f < 5; f++) {
      const long long X = to_fixed(q.val[k][f][L] * (f == 0 ? sm : se));
      if(X) atomicAdd(&fx[b + f * G].hi, (unsigned long long) X);
    }
  }
  __syncwarp();
  cnt = 0;
}

// Exact variant (FP64 sums): every value v = sum x mass/Tint is added as the
// two-word fixed-point pair of fixedpoint.cuh:fx_add (resolution 2^-S, two
// integer atomics), so the bins carry the full FP64 resolution whatever the
// headroom of the field's range.  The lane header holds mass/Tint x
// 2^(S-24) per field class (scale), which gives the pair of fx_add(v, S)
// bit for bit: the power-of-two factor is exact.
template <int PER>
__device__ __forceinline__ void warp_drain_nodes_exact(WarpQueueT<PER, double> &q, FxWord *fx, int G, int &cnt)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int incl = cnt;
#pragma unroll
  for(int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if(lane >= o) incl += y;
  }
  const int total = __shfl_sync(FULL, incl, 31);
  q.off[lane] = incl - cnt;
  __syncwarp();
  for(int r = lane; r < total; r += 32) {
    int L = 0;
#pragma unroll
    for(int step = 16; step; step >>= 1)
      if(q.off[L + step] <= r) L += step;
    const int k = r - q.off[L];
    const int b = q.gbase[L] + q.base[k][L];
    const double sm = q.scale[0][L], se = q.scale[1][L];
#pragma unroll
    for(int f = 0; f < 5; f++) fx_add_scaled(&fx[b + f * G], q.val[k][f][L] * (f == 0 ? sm : se));
  }
  __syncwarp();
  cnt = 0;
}

template <int PER>
__device__ __forceinline__ void warp_drain32(WarpQueue32<PER> &q, FxWord *fx, int G, int &cnt)
{
  warp_drain_nodes(q, fx, G, cnt);
}

#endif
