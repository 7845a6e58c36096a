// GALIC's set-up sampling on the GPU:
//   galic_sample_density_targets  densitygrid_sample_targetresponse (grid.c:536-617)
//   galic_sample_energy_targets   calc_energy_grid_mass_maps (grid.c:941-1076)
//   galic_sample_positions        {halo,disk,bulge}_get_fresh_coordinate
//                                 (halo.c:17-40, disk.c:17-50, bulge.c:15-37)
//                                 as forcedensitygrid_calculate calls them
//                                 (grid.c:659-678)
//
// The reference draws from one sequential stream and stops after exactly
// ntarget kept samples, so which uniforms form which sample depends on every
// draw before it.  The GPU replays that loop in parallel:
//  * the stream stand-in (grng.h) gives uniform k directly;
//  * the draws are cut into chunks of CHUNK consecutive uniforms, one chunk
//    per thread, in windows of up to MAX_CHUNKS chunks;
//  * a sample is three draws (halo and bulge: radius, azimuth, polar angle;
//    disk: height, radius, azimuth) and is complete at its third draw.
//    Reading the stream is a three-state automaton: state 0 expects a
//    sample's first draw, 1 its second, 2 its third.  Halo and disk redraw
//    all three when the point falls outside Rmax, so state 0 always moves
//    to 1; the bulge redraws only its radius (bulge.c:19-28), so a radius
//    beyond Rmax keeps state 0.  A chunk maps a starting state to an ending
//    state; an exclusive scan of these maps (composition is associative)
//    gives every chunk its starting state.  A halo or disk chunk (96 = 3 x 32
//    draws) maps every state to itself, so those chunks start in state 0
//    without a scan;
//  * pass "count": every thread walks its chunk and counts the samples the
//    reference keeps (inside Rmax and, for the target maps, inside the test
//    sqrt(x^2 + z^2) < Rmax of grid.c:572 and grid.c:987); an exclusive sum
//    gives every chunk the rank of its first kept sample;
//  * pass "emit": the walk is repeated; kept samples of rank < remaining are
//    binned (or written out), and the one of rank remaining - 1 records the
//    stream position after its last draw.
// Bins are signed 64-bit fixed-point words, X = round(v 2^S) with S per
// field from a bound on the field's total, added with integer atomics: exact
// and independent of the order in which threads arrive.  The finished grid
// is scaled, smoothed (grid.c:1247-1265) and stored by one CTA per stack.
//
// Built with --fmad=false: every operation rounds like the CPU restatement's
// (gcc -ffp-contract=off) and the elementary functions are gmath.h's, so a
// sample's coordinates are bit-identical to the restatement's.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "context.cuh"
#include "galic_gpu.h"
#include "grng.h"
#include "model.cuh"
#include "setup.cuh"
#include "stack.cuh"

namespace {

constexpr int CHUNK = 96;           // draws per thread (3 x 32: a multiple of a sample)
constexpr int SAMPLES_PER_CHUNK = CHUNK / 3;
constexpr int MAX_CHUNKS = 1 << 21;  // chunks per window (2e8 draws)
constexpr int WALK_BLOCK = 256;

enum { PASS_MAP = 0, PASS_COUNT = 1, PASS_EMIT = 2 };

// STACKOFFSET(l, 0, 0) on the host (allvars.h:160)
int stack_off_host(int l) { return ((1 << (2 * l)) - 1) / 3; }
enum { MODE_DG = 0, MODE_EG = 1, MODE_POS = 2 };

// a (DG or EG) grid: cell of grid.c:494-534 / grid.c:896-939
struct Grid2 {
  double Rmin, lfac;  // lfac = log(Fac), the value the reference recomputes per call
  int nbin;
};

struct WalkArgs {
  uint64_t seed;
  uint32_t sa, sb;
  uint64_t first;  // absolute index of the window's first draw
  int nchunks;
  int mode;
  Shape S;
  // bulge: per-chunk composed maps (map pass) and their exclusive scan
  uint8_t *maps;
  const uint8_t *prefix;
  int state0;  // state at the window's first draw
  uint32_t *counts;          // count pass: kept samples per chunk
  uint8_t *end_state;        // count pass: state after the window's last draw
  const uint32_t *offsets;   // emit pass: rank of each chunk's first kept sample
  long long remaining;       // emit pass: samples still to keep
  unsigned long long *end;   // emit pass: position after the last kept sample
  Grid2 grid;
  long long *acc;  // [fields][nbin^2]
  int shift[5];
  DispTab D;
  double *pos_out;  // MODE_POS: 3 doubles per kept sample, from rank 0
  double disk_q_half;  // disk radius draws below it give R < 0.45 Rmax (quick_keep)
};

template <int TYPE>
__device__ __forceinline__ bool make_sample(const Shape &S, double d0, double d1, double d2, double *pos)
{
  if(TYPE == 1) return halo_draw(S, d0, d1, d2, pos);
  if(TYPE == 2) return disk_draw(S, d0, d1, d2, pos);
  bulge_place(S, bulge_radius(S, d0), d1, d2, pos);
  return true;
}

__device__ __forceinline__ int next_state(int s, bool radius_ok) { return s == 0 ? (radius_ok ? 1 : 0) : (s == 1 ? 2 : 0); }

// ---------------------------------------------------------------- binning

__device__ __forceinline__ void fx_add1(long long *w, double v, int S)
{
  const long long X = __double2ll_rn(ldexp(v, S));
  if(X) atomicAdd((unsigned long long *) w, (unsigned long long) X);
}

__device__ __forceinline__ void deposit(const WalkArgs &a, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = gm_fabs(pos[2]);
  double br = (gm_log(r / a.grid.Rmin + 1.0) / a.grid.lfac) - 0.5;
  double bz = (gm_log(z / a.grid.Rmin + 1.0) / a.grid.lfac) - 0.5;
  Cell c = cell_from_b(br, bz, a.grid.nbin);
  const int N = a.grid.nbin, G = N * N;
  const int i00 = c.iz * N + c.iR;
  const double w[4] = {(1 - c.fR) * (1 - c.fz), (c.fR) * (1 - c.fz), (1 - c.fR) * (c.fz), (c.fR) * (c.fz)};
  const int at[4] = {i00, i00 + 1, i00 + N, i00 + N + 1};
#pragma unroll
  for(int k = 0; k < 4; k++) fx_add1(&a.acc[at[k]], w[k], a.shift[0]);
  if(a.mode == MODE_EG) {
    double d[4];
    disp_rtp(a.D, pos, d);
#pragma unroll
    for(int f = 0; f < 4; f++)
#pragma unroll
      for(int k = 0; k < 4; k++) fx_add1(&a.acc[(size_t) (f + 1) * G + at[k]], w[k] * d[f], a.shift[f + 1]);
  }
}

// ---------------------------------------------------------------- the walk

// The count pass only needs each sample's keep decision.  Where a cheap
// bound settles it with a wide margin the coordinates are not evaluated:
// 1 = kept, 0 = not kept, -1 = evaluate exactly.  Halo and bulge:
// |pos|^2 = r^2 (sin^2 theta + cos^2 theta / stretch^2) with cos theta = 2u - 1,
// and the grid.c test sqrt(x^2 + z^2) < Rmax follows from |pos| < Rmax (the
// rounded sums are monotone).  Disk: below the radius draw q_half the Newton
// radius is under 0.45 Rmax, and with |z| < 0.85 Rmax the point is inside.
// The evaluated values differ from the bounds by a few ulp, far inside the
// 1e-7 margins; a sample near a boundary takes the exact path.
template <int TYPE>
__device__ __forceinline__ int quick_keep(const WalkArgs &a, double d0, double d1, double d2)
{
  const Shape &S = a.S;
  const double R2 = S.Rmax * S.Rmax;
  if(TYPE == 2) {
    if(!(d1 < a.disk_q_half)) return -1;
    const double z = S.Disk_Z0 / 2 * gm_log(d0 / (1 - d0));
    return gm_fabs(z) < 0.85 * S.Rmax ? 1 : -1;
  }
  const double s = (TYPE == 1) ? S.HaloStretch : S.BulgeStretch;
  if(!(s >= 0.01 && s <= 100.0)) return -1;
  if(TYPE == 3 && a.mode == MODE_POS) return 1;  // the radius was accepted when drawn
  const double r = (TYPE == 1) ? (d0 > 0 ? S.Halo_A * (d0 + sqrt(d0)) / (1 - d0) : 0.0) : bulge_radius(S, d0);
  const double c = d2 * 2 - 1;
  const double E = r * r * ((1 - c * c) + c * c / (s * s));
  if(E < R2 * (1 - 1e-7)) return 1;
  if(TYPE == 1 && E > R2 * (1 + 1e-7)) return 0;
  return -1;
}

template <int TYPE, int PASS>
__global__ void __launch_bounds__(WALK_BLOCK) k_sample_walk(const WalkArgs a)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= a.nchunks) return;
  const uint64_t k0 = a.first + (uint64_t) c * CHUNK;
  grng_t g;
  grng_init(&g, a.seed, a.sa, a.sb);
  grng_seek(&g, k0);

  if(PASS == PASS_MAP) {
    int m0 = 0, m1 = 1, m2 = 2;  // end state from starting states 0, 1, 2
    for(int i = 0; i < CHUNK; i++) {
      const double u = grng_uniform(&g);
      const bool ok = !(bulge_radius(a.S, u) > a.S.Rmax);
      m0 = next_state(m0, ok);
      m1 = next_state(m1, ok);
      m2 = next_state(m2, ok);
    }
    a.maps[c] = (uint8_t) (m0 | (m1 << 2) | (m2 << 4));
    return;
  }

  int st = (TYPE == 3) ? ((a.prefix[c] >> (2 * a.state0)) & 3) : 0;
  double u1 = 0, u2 = 0;  // draws k-1 and k-2
  if(st >= 1) u1 = grng_uniform_at(a.seed, a.sa, a.sb, k0 - 1);
  if(st == 2) u2 = grng_uniform_at(a.seed, a.sa, a.sb, k0 - 2);
  const long long base = (PASS == PASS_EMIT) ? (long long) a.offsets[c] : 0;
  if(PASS == PASS_EMIT && base >= a.remaining) return;
  uint32_t kept = 0;
  for(int i = 0; i < CHUNK; i++) {
    const double u = grng_uniform(&g);
    if(st == 0) {
      st = (TYPE == 3) ? (!(bulge_radius(a.S, u) > a.S.Rmax) ? 1 : 0) : 1;
    } else if(st == 1) {
      st = 2;
    } else {
      st = 0;
      double pos[3];
      int quick = -1;
      if(PASS == PASS_COUNT) quick = quick_keep<TYPE>(a, u2, u1, u);
      bool keep;
      if(quick >= 0) {
        keep = quick;
      } else {
        keep = make_sample<TYPE>(a.S, u2, u1, u, pos);
        if(keep && a.mode != MODE_POS) keep = sqrt(pos[0] * pos[0] + pos[2] * pos[2]) < a.S.Rmax;
      }
      if(keep) {
        if(PASS == PASS_EMIT) {
          const long long rank = base + kept;
          if(rank >= a.remaining) return;
          if(a.mode == MODE_POS) {
            a.pos_out[3 * rank] = pos[0];
            a.pos_out[3 * rank + 1] = pos[1];
            a.pos_out[3 * rank + 2] = pos[2];
          } else {
            deposit(a, pos);
          }
          if(rank == a.remaining - 1) *a.end = k0 + i + 1;
        }
        kept++;
      }
    }
    u2 = u1;
    u1 = u;
  }
  if(PASS == PASS_COUNT) {
    a.counts[c] = kept;
    if(c == a.nchunks - 1) *a.end_state = (uint8_t) st;
  }
}

// composition of chunk maps, earlier map first
struct ComposeMaps {
  __host__ __device__ __forceinline__ uint8_t operator()(uint8_t first, uint8_t then) const
  {
    int r = 0;
#pragma unroll
    for(int s = 0; s < 3; s++) r |= ((then >> (2 * ((first >> (2 * s)) & 3))) & 3) << (2 * s);
    return (uint8_t) r;
  }
};
constexpr uint8_t IDENTITY_MAP = 0 | (1 << 2) | (2 << 4);

// one CTA per stack: fixed point -> scaled finest level -> smoothed stack;
// renorm also applies grid.c:862-880 to the finest level
__global__ void __launch_bounds__(1024) k_sample_finish(const long long *acc, int shift, double scale, int L,
                                                        int renorm, double mtype, double *out)
{
  extern __shared__ double sm[];
  __shared__ double fac;
  __shared__ int apply;
  const int off = stack_off(L), G = 1 << (2 * L), Ns = stack_off(L + 1);
  for(int i = threadIdx.x; i < G; i += blockDim.x) sm[off + i] = ldexp((double) acc[i], -shift) * scale;
  __syncthreads();
  stack_smooth_cta(sm, L);
  if(renorm) {
    if(threadIdx.x == 0) {
      double msum = 0;  // in the reference's order
      for(int i = 0; i < G; i++) msum += sm[off + i];
      apply = msum > 0;
      fac = apply ? mtype / msum : 1.0;
    }
    __syncthreads();
    if(apply)
      for(int i = threadIdx.x; i < G; i += blockDim.x) sm[off + i] *= fac;
    __syncthreads();
  }
  for(int i = threadIdx.x; i < Ns; i += blockDim.x) out[i] = sm[i];
}

// ---------------------------------------------------------------- host side

struct Scratch {
  uint8_t *maps = nullptr, *prefix = nullptr, *end_state = nullptr;
  uint32_t *counts = nullptr, *offsets = nullptr;
  unsigned long long *end = nullptr;
  void *temp = nullptr;
  size_t temp_bytes = 0;
};

cudaError_t scratch_alloc(Scratch &s, cudaStream_t st)
{
  size_t b1 = 0, b2 = 0;
  cudaError_t e;
  if((e = cub::DeviceScan::ExclusiveScan(nullptr, b1, (uint8_t *) nullptr, (uint8_t *) nullptr, ComposeMaps(),
                                         IDENTITY_MAP, MAX_CHUNKS, st)))
    return e;
  if((e = cub::DeviceScan::ExclusiveSum(nullptr, b2, (uint32_t *) nullptr, (uint32_t *) nullptr, MAX_CHUNKS + 1, st)))
    return e;
  s.temp_bytes = std::max(b1, b2);
  if((e = cudaMallocAsync((void **) &s.maps, MAX_CHUNKS, st))) return e;
  if((e = cudaMallocAsync((void **) &s.prefix, MAX_CHUNKS, st))) return e;
  if((e = cudaMallocAsync((void **) &s.end_state, 16, st))) return e;
  if((e = cudaMallocAsync((void **) &s.counts, (MAX_CHUNKS + 1) * sizeof(uint32_t), st))) return e;
  if((e = cudaMallocAsync((void **) &s.offsets, (MAX_CHUNKS + 1) * sizeof(uint32_t), st))) return e;
  if((e = cudaMallocAsync((void **) &s.end, sizeof(unsigned long long), st))) return e;
  return cudaMallocAsync(&s.temp, std::max<size_t>(s.temp_bytes, 16), st);
}

void scratch_free(Scratch &s, cudaStream_t st)
{
  void *p[] = {s.maps, s.prefix, s.end_state, s.counts, s.offsets, s.end, s.temp};
  for(void *q : p)
    if(q) cudaFreeAsync(q, st);
  s = Scratch();
}

#define SCK(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if(e_ != cudaSuccess) {                                                                   \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                      \
      return GALIC_ERR_CUDA;                                                                  \
    }                                                                                         \
  } while(0)

template <int TYPE>
cudaError_t launch_walk(int pass, const WalkArgs &a, cudaStream_t st)
{
  const int grid = (a.nchunks + WALK_BLOCK - 1) / WALK_BLOCK;
  if(pass == PASS_MAP) k_sample_walk<TYPE, PASS_MAP><<<grid, WALK_BLOCK, 0, st>>>(a);
  else if(pass == PASS_COUNT) k_sample_walk<TYPE, PASS_COUNT><<<grid, WALK_BLOCK, 0, st>>>(a);
  else k_sample_walk<TYPE, PASS_EMIT><<<grid, WALK_BLOCK, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t walk(int type, int pass, const WalkArgs &a, cudaStream_t st)
{
  if(type == 1) return launch_walk<1>(pass, a, st);
  if(type == 2) return launch_walk<2>(pass, a, st);
  return launch_walk<3>(pass, a, st);
}

// The disk's radius draw q solves (1 + R) e^-R = 1 - q for R / Disk_H
// (disk.c:25-36), increasing in q: q(R) = 1 - (1 + R) e^-R at R = 0.45 Rmax /
// Disk_H bounds the draws whose radius is below 0.45 Rmax (0: no quick path).
double disk_q_half(const Shape &S)
{
  if(!(S.Disk_H > 0) || !(S.Rmax > 0) || !std::isfinite(S.Rmax / S.Disk_H)) return 0.0;
  const double R = 0.45 * S.Rmax / S.Disk_H;
  return 1.0 - (1.0 + R) * std::exp(-R);
}

// Draws `ntarget` kept samples of one type from the stream, window by
// window (see the top of this file).  a: mode, shape, deposit targets.
// Returns GALIC_OK, GALIC_ERR_CUDA or GALIC_ERR_REJECTION_CAP.
int run_type(int type, long long ntarget, galic_stream_t *stream, WalkArgs a, Scratch &s, cudaStream_t st,
             int *launches)
{
  uint64_t pos = stream->position;
  const uint64_t start = pos;
  // draws beyond which the reference loop is taken to accept nothing any more
  const uint64_t cap = 3 * (64 * (uint64_t) ntarget + (1ull << 26));
  long long remaining = ntarget;
  double rate = 0.9;  // kept samples per candidate, refined per window
  int state = 0;
  double *pos_base = a.pos_out;
  a.seed = stream->seed;
  a.sa = stream->a;
  a.sb = stream->b;
  a.maps = s.maps;
  a.prefix = s.prefix;
  a.counts = s.counts;
  a.offsets = s.offsets;
  a.end = s.end;
  a.end_state = s.end_state;
  a.disk_q_half = disk_q_half(a.S);
  while(remaining > 0) {
    double want = (double) remaining / rate * 1.02 + 64;
    long long nch = (long long) std::ceil(want / SAMPLES_PER_CHUNK);
    nch = std::min<long long>(std::max<long long>(nch, 1), MAX_CHUNKS);
    a.first = pos;
    a.nchunks = (int) nch;
    a.state0 = state;
    if(a.mode == MODE_POS) a.pos_out = pos_base + 3 * (ntarget - remaining);
    if(type == 3) {
      SCK(walk(type, PASS_MAP, a, st));
      size_t tb = s.temp_bytes;
      SCK(cub::DeviceScan::ExclusiveScan(s.temp, tb, s.maps, s.prefix, ComposeMaps(), IDENTITY_MAP, a.nchunks, st));
      *launches += 2;
    }
    SCK(cudaMemsetAsync(s.counts + a.nchunks, 0, sizeof(uint32_t), st));
    SCK(walk(type, PASS_COUNT, a, st));
    size_t tb = s.temp_bytes;
    SCK(cub::DeviceScan::ExclusiveSum(s.temp, tb, s.counts, s.offsets, a.nchunks + 1, st));
    uint32_t total = 0;
    uint8_t end_state = 0;
    SCK(cudaMemcpyAsync(&total, s.offsets + a.nchunks, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&end_state, s.end_state, 1, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    *launches += 2;
    if(total > 0) {
      a.remaining = remaining;
      SCK(walk(type, PASS_EMIT, a, st));
      *launches += 1;
    }
    if((long long) total >= remaining) {
      unsigned long long end = 0;
      SCK(cudaMemcpyAsync(&end, s.end, sizeof(end), cudaMemcpyDeviceToHost, st));
      SCK(cudaStreamSynchronize(st));
      pos = end;
      remaining = 0;
    } else {
      remaining -= total;
      pos += (uint64_t) a.nchunks * CHUNK;
      state = end_state;
      // a window that kept nothing makes the next one 8x larger
      rate = total ? std::max((double) total / ((double) a.nchunks * SAMPLES_PER_CHUNK), 1e-6)
                   : std::max(rate / 8, 1e-9);
      if(pos - start > cap) return GALIC_ERR_REJECTION_CAP;
    }
  }
  stream->position = pos;
  return GALIC_OK;
}

Shape make_shape(const galic_sample_params_t *sp)
{
  Shape S;
  S.Rmax = sp->Rmax;
  S.Halo_A = sp->Halo_A;
  S.HaloStretch = sp->HaloStretch;
  S.Disk_Z0 = sp->Disk_Z0;
  S.Disk_H = sp->Disk_H;
  S.Bulge_A = sp->Bulge_A;
  S.BulgeStretch = sp->BulgeStretch;
  return S;
}

// S of a signed 64-bit word whose total stays below 2^61 for totals up to `bound`
int shift_for(double bound)
{
  if(!(bound > 0) || !std::isfinite(bound)) bound = 1.0;
  return 61 - (int) std::ceil(std::log2(bound));
}

int set_fail(galic_ctx *ctx, int st)
{
  if(ctx) ctx->status = st;
  return st;
}

bool finish_attr_done[256];

cudaError_t prepare_finish()
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e) return e;
  if(dev >= 0 && dev < 256 && finish_attr_done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(k_sample_finish, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int) (stack_off_host(7 + 1) * sizeof(double)));
  if(!e && dev >= 0 && dev < 256) finish_attr_done[dev] = true;
  return e;
}

// the context's sampled targets of one type: DG (fields 1) or EG (fields 5)
int sample_targets(galic_ctx *ctx, const galic_sample_params_t *sp, long long ntarget, galic_stream_t *stream, int mode,
                   int renorm)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(!sp || !stream || ntarget < 1 || ntarget > (1ll << 40)) return set_fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  const galic_params_t &p = ctx->prm;
  const int L = ctx->L, N = 1 << L, G = N * N;
  if(mode == MODE_EG)
    for(int t = 1; t <= 3; t++)
      if(p.MType[t] > 0 && !ctx->have_disp[t]) return set_fail(ctx, GALIC_ERR_STATE);
  cudaStream_t st = ctx->stream;
  if(cudaSetDevice(ctx->device) || prepare_finish()) return set_fail(ctx, GALIC_ERR_CUDA);
  const int nf = (mode == MODE_EG) ? 5 : 1;
  Scratch s;
  long long *acc = nullptr;
  int rc = GALIC_OK;
  if(scratch_alloc(s, st) || cudaMallocAsync((void **) &acc, (size_t) nf * G * sizeof(long long), st)) {
    scratch_free(s, st);
    return set_fail(ctx, GALIC_ERR_CUDA);
  }
  int launches = 0;
  galic_stream_t cur = *stream;
  for(int t = 1; t <= 3 && rc == GALIC_OK; t++) {
    if(!(p.MType[t] > 0)) continue;
    WalkArgs a{};
    a.mode = mode;
    a.S = make_shape(sp);
    a.acc = acc;
    a.grid.Rmin = (mode == MODE_EG) ? p.EG_Rmin : p.DG_Rmin;
    a.grid.lfac = gm_log((mode == MODE_EG) ? p.EG_Fac : p.DG_Fac);
    a.grid.nbin = N;
    a.shift[0] = shift_for(2.0 * (double) ntarget);
    if(mode == MODE_EG) {
      DispTab &D = a.D;
      D.disp_r = ctx->d_disp[t][0];
      D.dispz = ctx->d_disp[t][1];
      D.dispphi = ctx->d_disp[t][2];
      D.tvr2 = ctx->d_disp[t][3];
      D.tvz2 = ctx->d_disp[t][4];
      D.vstream = ctx->d_vstream[t];
      D.tovs = p.TypeOfVelocityStructure[t];
      D.beta = (t == 1) ? sp->HaloBetaParameter : (t == 3 ? sp->BulgeBetaParameter : 0.0);
      D.beta_a = (t == 1) ? sp->Halo_A : sp->Bulge_A;
      D.FG_Rmin = p.FG_Rmin;
      D.lfg = gm_log(p.FG_Fac);
      D.FG_Nbin = p.FG_Nbin;
      // bounds of |value| per deposit (interpolations are convex combinations)
      const double *mx = ctx->disp_max[t];
      double vmax = 0;
      if(ctx->h_vstream[t].size())
        for(double v : ctx->h_vstream[t]) vmax = std::max(vmax, std::fabs(v));
      double b[4];
      const double bfac = (D.beta >= 1) ? 1.0 : std::max(1.0, std::fabs(1 - D.beta));
      if(D.tovs == 0) b[0] = b[1] = b[2] = b[3] = mx[0];
      else if(D.tovs == 1) {
        b[0] = mx[0];
        b[1] = b[2] = b[3] = mx[0] * bfac;
      } else if(D.tovs == 2) {
        b[0] = b[1] = mx[1];
        b[2] = mx[2];
        b[3] = mx[2] + vmax * vmax;
      } else {
        b[0] = mx[3];
        b[1] = mx[4];
        b[2] = mx[2];
        b[3] = mx[2] + vmax * vmax;
      }
      for(int f = 0; f < 4; f++) a.shift[f + 1] = shift_for(2.0 * (double) ntarget * b[f]);
    }
    if(cudaMemsetAsync(acc, 0, (size_t) nf * G * sizeof(long long), st)) {
      rc = GALIC_ERR_CUDA;
      break;
    }
    rc = run_type(t, ntarget, &cur, a, s, st, &launches);
    if(rc != GALIC_OK) break;
    const double scale = p.MType[t] / (double) ntarget;  // MType[type] / nsum (grid.c:604-611)
    const size_t smem = (size_t) stack_off_host(L + 1) * sizeof(double);
    for(int f = 0; f < nf; f++) {
      const int k = (mode == MODE_EG) ? T_EGM + f : T_DGM;
      double *out = ctx->d_targets + ((size_t) t * NT_TARGET + k) * ctx->Ns;
      k_sample_finish<<<1, 1024, smem, st>>>(acc + (size_t) f * G, a.shift[f], scale, L, renorm && mode == MODE_DG,
                                             p.MType[t], out);
      launches++;
    }
    if(cudaGetLastError()) rc = GALIC_ERR_CUDA;
    ctx->target_parts[t] |= (mode == MODE_EG) ? 2u : 1u;
    if(ctx->target_parts[t] == 3u) ctx->have_targets[t] = true;
  }
  if(cudaStreamSynchronize(st) && rc == GALIC_OK) rc = GALIC_ERR_CUDA;
  scratch_free(s, st);
  cudaFreeAsync(acc, st);
  if(rc == GALIC_OK) {
    *stream = cur;
    ctx->generation++;
  }
  ctx->last_launches = launches;
  return set_fail(ctx, rc);
}

}  // namespace

extern "C" int galic_set_dispersion(galic_ctx *ctx, int type, const double *disp_r, const double *dispz,
                                    const double *dispphi, const double *tilted_vr2, const double *tilted_vz2)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(type < 1 || type > 3) return set_fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  const int tovs = ctx->prm.TypeOfVelocityStructure[type];
  const double *src[5] = {disp_r, dispz, dispphi, tilted_vr2, tilted_vz2};
  const bool need[5] = {tovs == 0 || tovs == 1, tovs == 2, tovs == 2 || tovs == 3, tovs == 3, tovs == 3};
  for(int k = 0; k < 5; k++)
    if(need[k] && !src[k]) return set_fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(cudaSetDevice(ctx->device)) return set_fail(ctx, GALIC_ERR_CUDA);
  const size_t NF = (size_t) ctx->prm.FG_Nbin * ctx->prm.FG_Nbin;
  for(int k = 0; k < 5; k++) {
    ctx->disp_max[type][k] = 0;
    if(!src[k]) continue;
    if(!ctx->d_disp[type][k] && cudaMallocAsync((void **) &ctx->d_disp[type][k], NF * sizeof(double), ctx->stream))
      return set_fail(ctx, GALIC_ERR_CUDA);
    if(cudaMemcpyAsync(ctx->d_disp[type][k], src[k], NF * sizeof(double), cudaMemcpyHostToDevice, ctx->stream))
      return set_fail(ctx, GALIC_ERR_CUDA);
    const size_t n = (k == 0) ? (size_t) ctx->prm.FG_Nbin : NF;
    double m = 0;
    for(size_t i = 0; i < n; i++) m = std::max(m, std::fabs(src[k][i]));
    ctx->disp_max[type][k] = m;
  }
  ctx->have_disp[type] = true;
  ctx->generation++;
  if(cudaStreamSynchronize(ctx->stream)) return set_fail(ctx, GALIC_ERR_CUDA);  // the upload is complete on return
  return set_fail(ctx, GALIC_OK);
}

extern "C" int galic_sample_density_targets(galic_ctx *ctx, const galic_sample_params_t *sp, long long ntarget,
                                            galic_stream_t *stream, int renormalize)
{
  return sample_targets(ctx, sp, ntarget, stream, MODE_DG, renormalize);
}

extern "C" int galic_sample_energy_targets(galic_ctx *ctx, const galic_sample_params_t *sp, long long ntarget,
                                           galic_stream_t *stream)
{
  return sample_targets(ctx, sp, ntarget, stream, MODE_EG, 0);
}

extern "C" int galic_get_targets(galic_ctx *ctx, int type, double *dgs_mass, double *egs_mass, double *egs_r,
                                 double *egs_t, double *egs_p, double *egs_q)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(type < 1 || type > 3) return set_fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  double *dst[NT_TARGET] = {dgs_mass, egs_mass, egs_r, egs_t, egs_p, egs_q};
  if(cudaSetDevice(ctx->device)) return set_fail(ctx, GALIC_ERR_CUDA);
  for(int k = 0; k < NT_TARGET; k++)
    if(dst[k] && cudaMemcpyAsync(dst[k], ctx->d_targets + ((size_t) type * NT_TARGET + k) * ctx->Ns,
                                 ctx->Ns * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream))
      return set_fail(ctx, GALIC_ERR_CUDA);
  if(cudaStreamSynchronize(ctx->stream)) return set_fail(ctx, GALIC_ERR_CUDA);
  return set_fail(ctx, GALIC_OK);
}

extern "C" int galic_sample_positions(const galic_sample_params_t *sp, int type, long long n, galic_stream_t *stream,
                                      double *pos)
{
  if(!sp || !stream || type < 1 || type > 3 || n < 0 || n > (1ll << 34) || (n > 0 && !pos))
    return GALIC_ERR_INVALID_ARGUMENT;
  if(n == 0) return GALIC_OK;
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) || ndev < 1) return GALIC_ERR_NO_DEVICE;
  cudaStream_t st;
  if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) return GALIC_ERR_CUDA;
  Scratch s;
  double *d_pos = nullptr;
  int rc = GALIC_OK;
  if(scratch_alloc(s, st) || cudaMallocAsync((void **) &d_pos, (size_t) 3 * n * sizeof(double), st)) rc = GALIC_ERR_CUDA;
  galic_stream_t cur = *stream;
  if(rc == GALIC_OK) {
    WalkArgs a{};
    a.mode = MODE_POS;
    a.S = make_shape(sp);
    a.pos_out = d_pos;
    int launches = 0;
    rc = run_type(type, n, &cur, a, s, st, &launches);
  }
  if(rc == GALIC_OK && cudaMemcpyAsync(pos, d_pos, (size_t) 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st))
    rc = GALIC_ERR_CUDA;
  if(cudaStreamSynchronize(st) && rc == GALIC_OK) rc = GALIC_ERR_CUDA;
  scratch_free(s, st);
  if(d_pos) cudaFreeAsync(d_pos, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if(rc == GALIC_OK) *stream = cur;
  return rc;
}
