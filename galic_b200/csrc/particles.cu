// initialize_particles (set_particles.c:15-307) on the GPU.
//
// The reference draws every particle from one sequential stream: particle
// n starts where particle n-1 stopped, and how many draws a particle takes
// depends on its rejection loops (position inside Rmax, the Hernquist
// velocity by von Neumann rejection, the Gaussian velocity below the escape
// speed, Marsaglia's polar method).  The replay here finds every particle's
// first draw in parallel by speculative segment decoding:
//  * k_len on the first 65536 positions of a type's draws gives the mean
//    draws per particle, which sizes the segments (16 or 32 particles' worth
//    of positions each, a multiple of 32);
//  * k_seg_decode: one lane per segment initialises particles back to back
//    from the segment's first position, marking each start in a bitmap;
//  * k_seg_fix rounds: a segment whose entry (the largest exit before it) is
//    not where its chain began re-decodes from the entry until it lands on a
//    start it already has -- two chains that meet agree from there on, and
//    they mostly meet within a few particles -- or leaves the segment, and
//    then goes on into the next segments that no other lane walks this round;
//  * k_seg_count, a scan and k_seg_extract turn the bitmap into the start of
//    every particle;
//  * k_final: each particle is initialised once more from its start, this
//    time keeping its values; then one uniform per particle after the last
//    draw and a radix sort give the permutation.
// The halo's velocity rejection loop has a long tail near the centre; its
// draw pairs are tested 32 at a time by a whole warp (halo_velocity_warp).
// A chain whose rejection loop hits its cap of 10^6 tries ends there; if
// that happens before a type's last particle the call fails.  Built with
// --fmad=false and gmath.h's functions, so every particle is bit-identical
// to the CPU restatement.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "context.cuh"
#include "galic_gpu.h"
#include "grng.h"
#include "model.cuh"
#include "setup.cuh"

namespace {

constexpr int LOOP_CAP = 1000000;     // tries of every rejection loop
constexpr uint32_t LEN_CAPPED = 0xffffffffu;
constexpr int PROBE = 1 << 16;        // positions of the draws-per-particle estimate
constexpr int PBLOCK = 128;

struct PInit {
  DevModel M;
  Shape S;
  DispTab D[4];
  uint64_t seed;
  uint32_t sa, sb;
  double MaxVel, LowerDispLimit, TorbitFac;
};

struct POut {
  double *pos, *vel, *vel_theo, *vesc, *tint, *targets;
  int *counts;  // [4][4] raised to LowerDispLimit, then [16] non-positive Tint
};

// halo_get_potential_from_radius (halo.c:69-73)
__device__ __forceinline__ double halo_pot_r(const DevModel &M, double r) { return -M.G * M.Halo_Mass / (r + M.Halo_A); }

// halo_f_q (halo.c:136-147): pow(x, 1.5) = x sqrt(x), pow(x, 2.5) = x x sqrt(x)
__device__ double halo_f_q(const DevModel &M, double q)
{
  const double c = 2 * M.G * M.Halo_Mass / M.Halo_A;
  double pre = (M.Halo_Mass / (M.Halo_A * M.Halo_A * M.Halo_A)) / (4 * kPi * kPi * kPi * (c * sqrt(c)));
  const double u = 1 - q * q;
  return pre * (3 * gm_asin(q) + q * sqrt(1 - q * q) * (1 - 2 * q * q) * (8 * q * q * q * q - 8 * q * q - 3)) /
         (u * u * sqrt(u));
}

// halo_f (halo.c:151-157) with halo_E_to_q (halo.c:113-116)
__device__ __forceinline__ double halo_f(const DevModel &M, double rad, double vel)
{
  double E = 0.5 * vel * vel + halo_pot_r(M, rad);
  double q = sqrt(-E * M.Halo_A / (M.G * M.Halo_Mass));
  return halo_f_q(M, q);
}

// one call of the type's *_get_fresh_coordinate from the stream g
// (halo.c:17-40, disk.c:17-50, bulge.c:15-37); false when capped
template <int TYPE>
__device__ bool fresh_seq(const Shape &S, grng_t &g, double *pos)
{
  if constexpr(TYPE == 1 || TYPE == 2) {
    for(int it = 0; it < LOOP_CAP; it++) {
      const double d0 = grng_uniform(&g), d1 = grng_uniform(&g), d2 = grng_uniform(&g);
      if(TYPE == 1 ? halo_draw(S, d0, d1, d2, pos) : disk_draw(S, d0, d1, d2, pos)) return true;
    }
  } else {
    for(int it = 0; it < LOOP_CAP; it++) {
      const double r = bulge_radius(S, grng_uniform(&g));
      if(!(r > S.Rmax)) {
        const double d1 = grng_uniform(&g), d2 = grng_uniform(&g);
        bulge_place(S, r, d1, d2, pos);
        return true;
      }
    }
  }
  return false;
}

// The halo's velocity draw (halo.c:168-184 inside set_particles.c:92-99),
// warp-cooperative.  For the particle of lane L (radius r, stream position w)
// halo_generate_v tests draw pairs (w, w+1), (w+2, w+3), ... until the first
// accepted one, and set_particles.c repeats that while the speed is not below
// MaxVelInUnitsVesc Vesc.  Near the centre the acceptance is small and the
// number of pairs has a long tail; here the 32 lanes test 32 consecutive
// pairs of one particle at once and a ballot picks the first accepted pair,
// which is the sequential loop's result.  Every lane of the warp calls it;
// need: this lane has a draw to make.  Returns false when capped.
__device__ bool halo_velocity_warp(const PInit &P, bool need, double r, double vesc, uint64_t &w, double &vr_out)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const DevModel &M = P.M;
  bool ok = true;
  unsigned pending = __ballot_sync(FULL, need);
  while(pending) {
    const int L = __ffs(pending) - 1;
    const double rL = __shfl_sync(FULL, r, L), vescL = __shfl_sync(FULL, vesc, L);
    uint64_t wpos = __shfl_sync(FULL, (unsigned long long) w, L);
    double vr = 0;
    bool capped = false;
    long long tries = 0;  // pairs tested for this particle, over all of its draws
    do {
      const double pot = halo_pot_r(M, rL);
      const double v_max = sqrt(-2 * pot);
      const double f_max = v_max * v_max * halo_f(M, rL, 0);
      for(long long base = 0;; base += 32) {
        const uint64_t j = wpos + 2 * (uint64_t) (base + lane);
        const double v_guess = grng_uniform_at(P.seed, P.sa, P.sb, j) * v_max;
        const double x_aux = grng_uniform_at(P.seed, P.sa, P.sb, j + 1) * f_max;
        const bool accept = !(x_aux > v_guess * v_guess * halo_f(M, rL, v_guess));
        const unsigned mask = __ballot_sync(FULL, accept);
        if(mask) {
          const int first = __ffs(mask) - 1;
          vr = __shfl_sync(FULL, v_guess, first);
          wpos += 2 * (uint64_t) (base + first + 1);
          break;
        }
        tries += 32;
        if(tries >= LOOP_CAP) {
          capped = true;
          break;
        }
      }
    } while(!capped && vr >= P.MaxVel * vescL);
    if(lane == L) {
      w = wpos;
      vr_out = vr;
      ok = !capped;
    }
    pending &= pending - 1;
  }
  return ok;
}

// one iteration of initialize_particles' loop (set_particles.c:64-237) for a
// particle of type TYPE from stream position `start`, called by all 32 lanes
// of a warp together (active: the lane has a particle).  VS: the velocity
// structure's frame, 0 spherical (TypeOfVelocityStructure 0, 1, 3) or 1
// cylindrical (2); one launch has one type and one frame, so each kernel
// carries only its own branches.  Returns the draws it took (LEN_CAPPED when
// a rejection loop hit its cap).  With o != nullptr the particle's values are
// stored at index n.
template <int TYPE, int VS>
__device__ uint32_t init_one(const PInit &P, uint64_t start, bool active, const POut *o, int n)
{
  constexpr int type = TYPE;
  grng_t g;
  grng_init(&g, P.seed, P.sa, P.sb);
  grng_seek(&g, start);
  const DevModel &M = P.M;
  const LogConsts L = make_log_consts(M);
  double pos[3] = {0, 0, 0};
  bool ok = active && fresh_seq<TYPE>(P.S, g, pos);
  double vesc = 0, tint = 0, r = 0;
  FgCoord fc{};
  if(ok) {
    // forcegrid_get_escape_speed (grid.c:115-120), the acceleration, Tint
    vesc = sqrt(-2.0 * forcegrid_pot(M, L, pos));
    double acc[3];
    fc = fg_coord(M, L, pos);
    forcegrid_acc(M, fc, pos, acc);
    const double a = sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
    r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    tint = P.TorbitFac * 2 * kPi * r / sqrt(r * a);
  }
  double vt[3] = {0, 0, 0};
  if constexpr(TYPE == 1) {
    uint64_t w = grng_position(&g);
    double vr = 0;
    const bool vok = halo_velocity_warp(P, ok, r, vesc, w, vr);
    if(ok) {
      ok = vok;
      grng_seek(&g, w);
    }
    if(ok) {
      const double phi = grng_uniform(&g) * kPi * 2;
      const double theta = gm_acos(grng_uniform(&g) * 2 - 1);
      vt[0] = vr * gm_sin(theta) * gm_cos(phi);
      vt[1] = vr * gm_sin(theta) * gm_sin(phi);
      vt[2] = vr * gm_cos(theta);
    }
  }
  if(!ok) return LEN_CAPPED;
  const DispTab &D = P.D[type];
  double d[4];
  disp_rtp(D, pos, d);
  int low[4];
  for(int k = 0; k < 4; k++) {
    low[k] = d[k] <= P.LowerDispLimit;
    if(low[k]) d[k] = P.LowerDispLimit;
  }
  // get_vstream (disp_fields.c:118-132)
  const double vstr = vstream_at(M, fc, type);
  double V[3];
  const double sigmaR = sqrt(d[0]), sigmaT = sqrt(d[1]), sigmaP = sqrt(d[2]);
  if constexpr(VS == 0) {
    double v, vr, vphi, vtheta;
    int it = 0;
    do {
      if(++it > LOOP_CAP) return LEN_CAPPED;
      vr = grng_gaussian(&g, sigmaR);
      vtheta = grng_gaussian(&g, sigmaT);
      vphi = grng_gaussian(&g, sigmaP);
      vphi += vstr;
      v = sqrt(vr * vr + vphi * vphi + vtheta * vtheta);
    } while(P.MaxVel * vesc < v);
    if(o) {
      const double phi = gm_atan2(pos[1], pos[0]);
      const double theta = gm_acos(pos[2] / sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]));
      const double st = gm_sin(theta), ct = gm_cos(theta), sp = gm_sin(phi), cp = gm_cos(phi);
      const double er[3] = {st * cp, st * sp, ct};
      const double ePhi[3] = {-sp, cp, 0};
      const double eTheta[3] = {-ct * cp, -ct * sp, st};
      for(int k = 0; k < 3; k++) V[k] = vr * er[k] + vphi * ePhi[k] + vtheta * eTheta[k];
    }
  } else {
    double v, vR, vphi, vz;
    int it = 0;
    do {
      if(++it > LOOP_CAP) return LEN_CAPPED;
      vR = grng_gaussian(&g, sigmaR);
      vz = grng_gaussian(&g, sigmaT);
      vphi = grng_gaussian(&g, sigmaP);
      vphi += vstr;
      v = sqrt(vR * vR + vphi * vphi + vz * vz);
    } while(v >= P.MaxVel * vesc);
    if(o) {
      const double phi = gm_atan2(pos[1], pos[0]);
      const double sp = gm_sin(phi), cp = gm_cos(phi);
      const double eR[3] = {cp, sp, 0};
      const double ePhi[3] = {-sp, cp, 0};
      const double eZ[3] = {0, 0, 1};
      for(int k = 0; k < 3; k++) V[k] = vR * eR[k] + vphi * ePhi[k] + vz * eZ[k];
    }
  }
  const uint64_t len = grng_position(&g) - start;
  if(o) {
    for(int k = 0; k < 3; k++) {
      o->pos[3 * n + k] = pos[k];
      o->vel[3 * n + k] = V[k];
      o->vel_theo[3 * n + k] = vt[k];
    }
    o->vesc[n] = vesc;
    o->tint[n] = tint;
    if(!(tint > 0)) atomicAdd(&o->counts[16], 1);
    for(int k = 0; k < 4; k++) {
      o->targets[4 * n + k] = d[k];
      if(low[k]) atomicAdd(&o->counts[4 * type + k], 1);
    }
  }
  return len >= LEN_CAPPED ? LEN_CAPPED : (uint32_t) len;
}

// the successor of every position o in [0, R) from `base`: next[o] = o + the
// draws of a particle started at o, R when that is past R, R + 1 when a
// rejection loop capped (whole warps run init_one together: lanes past R only keep the others company)
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_len(const PInit P, uint64_t base, uint32_t R, uint32_t *next)
{
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = o < R;
  const uint32_t len = init_one<TYPE, VS>(P, base + (active ? o : 0), active, nullptr, 0);
  if(o >= R + 2) return;
  if(!active) {
    next[o] = o;
    return;
  }
  const uint64_t e = (uint64_t) o + len;
  next[o] = (len == LEN_CAPPED) ? R + 1 : (e < R ? (uint32_t) e : R);
}

// Segment decode.  The type's stream positions are cut into K segments of
// Lseg positions (Lseg a multiple of 32, a few particles' worth); bit q of
// the bitmap says that position q starts a particle of the chain recorded
// for q's segment.  Each segment's chain starts at its entry x[c] and leaves
// the segment at its exit cx[c] (the first start at or past the segment's
// end; POS_CAPPED when a rejection loop hit its cap).  One lane owns each
// segment and the segment's bitmap words.
constexpr uint64_t POS_CAPPED = ~0ull;

struct Segs {
  uint64_t Lseg;
  uint32_t K, W;   // segments; bitmap words per segment (Lseg / 32)
  uint32_t *bits;  // K * W
  uint64_t *x, *cx;
};

// clears positions [lo, hi) of the segment that starts at a (a multiple of 32)
__device__ void clear_bits(uint32_t *w, uint64_t a, uint64_t lo, uint64_t hi)
{
  for(uint64_t q = lo; q < hi;) {
    const uint32_t k = (uint32_t) ((q - a) >> 5), b = (uint32_t) (q & 31);
    const uint64_t wend = a + ((uint64_t) k + 1) * 32;
    const uint32_t nb = (uint32_t) ((hi < wend ? hi : wend) - q);  // 1 .. 32 - b
    w[k] &= ~(nb == 32 ? 0xffffffffu : ((1u << nb) - 1) << b);
    q += nb;
  }
}

__device__ __forceinline__ bool bit_at(const uint32_t *w, uint64_t a, uint64_t q)
{
  return (w[(q - a) >> 5] >> (q & 31)) & 1u;
}

// every segment decoded from its own first position (whole warps run
// init_one together: lanes past K only keep the others company)
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_seg_decode(const PInit P, uint64_t base, const Segs S, uint64_t *exit)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = c < S.K;
  const uint64_t a = (uint64_t) c * S.Lseg, end = a + S.Lseg;
  uint32_t *w = S.bits + (size_t) (valid ? c : 0) * S.W;
  uint64_t q = a;
  bool work = valid;
  while(__any_sync(0xffffffffu, work)) {
    const uint32_t len = init_one<TYPE, VS>(P, base + (work ? q : 0), work, nullptr, 0);
    if(work) {
      w[(q - a) >> 5] |= 1u << (q & 31);
      if(len == LEN_CAPPED || len == 0) {
        q = POS_CAPPED;
        work = false;
      } else {
        q += len;
        work = q < end;
      }
    }
  }
  if(valid) {
    S.x[c] = a;
    S.cx[c] = q;
    exit[c] = q;
  }
}

struct MaxU64 {
  __device__ __forceinline__ uint64_t operator()(uint64_t u, uint64_t v) const { return u > v ? u : v; }
};

// before a resynchronisation round: a segment's entry is the largest exit
// before it (exits never decrease along the true chain, and one long particle
// can span many segments); flag[c]: the entry differs from the one the
// segment's chain was decoded from, so the segment is walked this round
__global__ void k_seg_prep(const Segs S, const uint64_t *pmax, const uint64_t *exit_in, uint64_t *exit_out,
                           uint8_t *flag)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= S.K) return;
  const uint64_t e = c ? pmax[c - 1] : 0;
  flag[c] = e != POS_CAPPED && e != S.x[c];
  exit_out[c] = exit_in[c];
}

// one resynchronisation round: each flagged segment re-decodes from its
// entry until it lands on a start of its recorded chain (the chains agree
// from there on) or leaves the segment; positions it steps over lose their
// bits.  A walk that leaves with a new exit goes on into the next segment
// when that one is not flagged (so no two lanes touch one segment), as the
// next round would.  After round r segments 0 .. r are exact; the rounds end
// when no exit changes.
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_seg_fix(const PInit P, uint64_t base, const Segs S,
                                                    const uint64_t *pmax, const uint8_t *flag,
                                                    const uint64_t *exit_in, uint64_t *exit_out, int *changed)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  bool work = c < S.K && flag[c];
  uint32_t d = c;
  uint64_t a = (uint64_t) d * S.Lseg, end = a + S.Lseg;
  uint32_t *w = S.bits + (size_t) (work ? d : 0) * S.W;
  uint64_t q = work ? pmax[c - 1] : 0;  // flag[0] is never set
  if(work) {
    S.x[d] = q;
    clear_bits(w, a, a, q < end ? q : end);
  }
  while(__any_sync(0xffffffffu, work)) {
    bool step = false;
    if(work) {
      const bool left = q >= end;
      if(left || bit_at(w, a, q)) {  // left the segment, or joined the recorded chain
        const uint64_t out = left ? q : S.cx[d];
        S.cx[d] = out;
        exit_out[d] = out;
        work = false;
        if(out != exit_in[d]) {
          *changed = 1;
          if(d + 1 < S.K && !flag[d + 1]) {  // go on into the next segment
            d++;
            a = end;
            end = a + S.Lseg;
            w = S.bits + (size_t) d * S.W;
            S.x[d] = q;
            clear_bits(w, a, a, q < end ? q : end);
            work = true;
          }
        }
      } else {
        step = true;
      }
    }
    const uint32_t len = init_one<TYPE, VS>(P, base + (step ? q : 0), step, nullptr, 0);
    if(step) {
      w[(q - a) >> 5] |= 1u << (q & 31);
      if(len == LEN_CAPPED || len == 0) {
        clear_bits(w, a, q + 1, end);
        S.cx[d] = POS_CAPPED;
        exit_out[d] = POS_CAPPED;
        if(exit_in[d] != POS_CAPPED) *changed = 1;
        work = false;
      } else {
        const uint64_t n = q + len;
        clear_bits(w, a, q + 1, n < end ? n : end);
        q = n;
      }
    }
  }
}

// the first segment whose chain caps (every later one is cut off)
__global__ void k_seg_first_cap(const uint64_t *exit, uint32_t K, unsigned *first)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c < K && exit[c] == POS_CAPPED) atomicMin(first, c);
}

// starts per segment up to the first capped one; cnt[K] = 0 closes the scan
__global__ void k_seg_count(const Segs S, const unsigned *first, uint64_t *cnt)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c > S.K) return;
  uint64_t n = 0;
  if(c < S.K && c <= *first) {
    const uint32_t *w = S.bits + (size_t) c * S.W;
    for(uint32_t k = 0; k < S.W; k++) n += __popc(w[k]);
  }
  cnt[c] = n;
}

// start of particle i (i <= count; i = count is where the type's draws end)
__global__ void k_seg_extract(const Segs S, const unsigned *first, const uint64_t *off, int count,
                              uint64_t *starts)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= S.K || c > *first) return;
  uint64_t r = off[c];
  if(r > (uint64_t) count) return;
  const uint32_t *w = S.bits + (size_t) c * S.W;
  const uint64_t a = (uint64_t) c * S.Lseg;
  for(uint32_t k = 0; k < S.W && r <= (uint64_t) count; k++)
    for(uint32_t m = w[k]; m && r <= (uint64_t) count; m &= m - 1)
      starts[r++] = a + 32ull * k + (uint64_t) (__ffs(m) - 1);
}

// each particle once more from its start, keeping its values.  Thread j
// takes the particle of length rank (j mod 32) * warps + j / 32 (ord: the
// particles by length, longest first): the longest particles start first,
// one to a warp, and no warp holds two of them.
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_final(const PInit P, uint64_t base, const uint64_t *starts,
                                                  const int *ord, int count, int n0, POut o)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int warps = (count + 31) / 32;
  const long long rank = (long long) (j & 31) * warps + (j >> 5);
  const bool active = j < warps * 32 && rank < count;
  const int i = active ? ord[rank] : 0;
  init_one<TYPE, VS>(P, base + (active ? starts[i] : 0), active, &o, n0 + i);
}

// particle lengths as sort keys (clamped to 32 bits) and their indices
__global__ void k_len_keys(const uint64_t *starts, int count, uint32_t *key, int *idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= count) return;
  const uint64_t len = starts[i + 1] - starts[i];
  key[i] = len > 0xffffffffull ? 0xffffffffu : (uint32_t) len;
  idx[i] = i;
}

// permutation[].rnd (set_particles.c:298-301): the bits of a uniform in [0, 1)
// order like the value
__global__ void k_perm_keys(uint64_t seed, uint32_t sa, uint32_t sb, uint64_t first, int n, unsigned long long *keys,
                            int *vals)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  keys[i] = gm_bits(grng_uniform_at(seed, sa, sb, first + (uint64_t) i));
  vals[i] = i;
}

#define PCK(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if(e_ != cudaSuccess) {                                                                   \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                      \
      rc = GALIC_ERR_CUDA;                                                                    \
      goto done;                                                                              \
    }                                                                                         \
  } while(0)

int pfail(galic_ctx *ctx, int st)
{
  if(ctx) ctx->status = st;
  return st;
}

inline unsigned gblocks(long long n, int b) { return (unsigned) ((n + b - 1) / b); }

// f(TYPE, VS) with the particle type (1-3) and the velocity frame (0, 1) as
// compile-time constants
template <class F>
void with_kind(int type, int vs, F &&f)
{
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  using V0 = std::integral_constant<int, 0>;
  if(type == 1)
    vs ? f(I1{}, I1{}) : f(I1{}, V0{});
  else if(type == 2)
    vs ? f(I2{}, I1{}) : f(I2{}, V0{});
  else
    vs ? f(I3{}, I1{}) : f(I3{}, V0{});
}

}  // namespace

extern "C" int galic_initialize_particles(galic_ctx *ctx, const galic_sample_params_t *sp, double TorbitFac,
                                          galic_stream_t *stream, galic_particles_out_t *out)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(!sp || !stream) return pfail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  const galic_params_t &p = ctx->prm;
  const int nt[4] = {0, p.NType[1], p.NType[2], p.NType[3]};
  const double tmass[4] = {0, p.Halo_Mass, p.Disk_Mass, p.Bulge_Mass};
  const long long Nll = (long long) nt[1] + nt[2] + nt[3];
  if(nt[1] < 0 || nt[2] < 0 || nt[3] < 0 || Nll < 1 || Nll > (1ll << 28)) return pfail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  const int N = (int) Nll;
  if(!ctx->have_fg) return pfail(ctx, GALIC_ERR_STATE);
  for(int t = 1; t <= 3; t++)
    if(nt[t] > 0 && (!ctx->have_disp[t] || !ctx->d_vstream[t] || ctx->h_vstream[t].empty()))
      return pfail(ctx, GALIC_ERR_STATE);
  if(cudaSetDevice(ctx->device)) return pfail(ctx, GALIC_ERR_CUDA);
  cudaStream_t s = ctx->stream;
  int rc = GALIC_OK, launches = 0;
  double *d_f = nullptr;  // pos, vel, vel_theo (3N each), vesc, tint (N each), targets (4N)
  int *d_counts = nullptr, *d_vals = nullptr, *d_vals2 = nullptr;
  uint32_t *d_J = nullptr;
  uint64_t *d_starts = nullptr;  // inside d_seg
  char *d_seg = nullptr;
  unsigned long long *d_keys = nullptr, *d_keys2 = nullptr;
  void *d_tmp = nullptr;
  size_t J_cap = 0, seg_cap = 0;
  std::vector<int> h_counts(17);
  uint64_t pos = stream->position;
  PInit P{};
  POut O{};
  P.M = ctx->dm;
  P.S.Rmax = sp->Rmax;
  P.S.Halo_A = sp->Halo_A;
  P.S.HaloStretch = sp->HaloStretch;
  P.S.Disk_Z0 = sp->Disk_Z0;
  P.S.Disk_H = sp->Disk_H;
  P.S.Bulge_A = sp->Bulge_A;
  P.S.BulgeStretch = sp->BulgeStretch;
  P.seed = stream->seed;
  P.sa = stream->a;
  P.sb = stream->b;
  P.MaxVel = p.MaxVelInUnitsVesc;
  P.LowerDispLimit = p.LowerDispLimit;
  P.TorbitFac = TorbitFac;
  for(int t = 1; t <= 3; t++) {
    DispTab &D = P.D[t];
    D.disp_r = ctx->d_disp[t][0];
    D.dispz = ctx->d_disp[t][1];
    D.dispphi = ctx->d_disp[t][2];
    D.tvr2 = ctx->d_disp[t][3];
    D.tvz2 = ctx->d_disp[t][4];
    D.vstream = ctx->d_vstream[t];
    D.tovs = p.TypeOfVelocityStructure[t];
    D.beta = (t == 1) ? sp->HaloBetaParameter : (t == 3 ? sp->BulgeBetaParameter : 0.0);
    D.beta_a = (t == 1) ? p.Halo_A : p.Bulge_A;
    D.FG_Rmin = p.FG_Rmin;
    D.lfg = gm_log(p.FG_Fac);
    D.FG_Nbin = p.FG_Nbin;
  }
  PCK(cudaMallocAsync((void **) &d_f, (size_t) 15 * N * sizeof(double), s));
  PCK(cudaMallocAsync((void **) &d_counts, 17 * sizeof(int), s));
  PCK(cudaMemsetAsync(d_f, 0, (size_t) 15 * N * sizeof(double), s));
  PCK(cudaMemsetAsync(d_counts, 0, 17 * sizeof(int), s));
  O.pos = d_f;
  O.vel = d_f + 3 * (size_t) N;
  O.vel_theo = d_f + 6 * (size_t) N;
  O.vesc = d_f + 9 * (size_t) N;
  O.tint = d_f + 10 * (size_t) N;
  O.targets = d_f + 11 * (size_t) N;
  O.counts = d_counts;
  {
    int n0 = 0;
    for(int t = 1; t <= 3 && rc == GALIC_OK; n0 += nt[t], t++) {
      if(nt[t] == 0) continue;
      const int vs = p.TypeOfVelocityStructure[t] == 2 ? 1 : 0;
      // draws per particle, from the lengths at the segment's first positions
      uint32_t R = PROBE;
      std::vector<uint32_t> probe(PROBE + 2);
      if(J_cap < (size_t) R + 2) {
        if(d_J) cudaFreeAsync(d_J, s);
        J_cap = (size_t) R + 2;
        PCK(cudaMallocAsync((void **) &d_J, J_cap * sizeof(uint32_t), s));
      }
      with_kind(t, vs, [&](auto T, auto V) {
        k_len<decltype(T)::value, decltype(V)::value><<<gblocks(R + 2, PBLOCK), PBLOCK, 0, s>>>(P, pos, R, d_J);
      });
      launches++;
      PCK(cudaGetLastError());
      PCK(cudaMemcpyAsync(probe.data(), d_J, (R + 2) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      PCK(cudaStreamSynchronize(s));
      double sum = 0;
      long long valid = 0;
      for(uint32_t o = 0; o < R; o++)
        if(probe[o] < R && probe[o] > o) {
          sum += probe[o] - o;
          valid++;
        }
      if(valid < PROBE / 2) {  // most starts end in a capped loop
        rc = GALIC_ERR_REJECTION_CAP;
        break;
      }
      const double per = sum / valid;
      // particles per segment: enough segments to fill the GPU with lanes,
      // few enough rounds (two chains usually meet within a few particles,
      // but the spread of the halo's lengths gives a long tail)
      const int seg_particles = (t == 2) ? 32 : 16;
      const uint64_t Lseg = ((uint64_t) (per * seg_particles) + 31) / 32 * 32;
      for(int attempt = 0;; attempt++) {
        const double want = ((double) nt[t] + 1) * per * (1.05 + 0.25 * attempt);
        const double Kd = want / (double) Lseg + 2;
        if(Kd > 2.0e9 || Kd * (double) Lseg / 8 > (double) (8ull << 30)) {  // the bitmap's budget
          rc = GALIC_ERR_UNSUPPORTED;
          break;
        }
        Segs G{};
        G.Lseg = Lseg;
        G.K = (uint32_t) Kd;
        G.W = (uint32_t) (Lseg / 32);
        const size_t K = G.K;
        size_t tb = 0, tb2 = 0, tb3 = 0;
        PCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, (uint64_t *) nullptr, (uint64_t *) nullptr, K + 1, s));
        PCK(cub::DeviceScan::InclusiveScan(nullptr, tb2, (uint64_t *) nullptr, (uint64_t *) nullptr, MaxU64(), K, s));
        PCK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb3, (uint32_t *) nullptr, (uint32_t *) nullptr,
                                                      (int *) nullptr, (int *) nullptr, nt[t], 0, 32, s));
        tb = std::max(std::max(tb, tb2), tb3);
        const auto al = [](size_t n) { return (n + 255) / 256 * 256; };
        const size_t sz_bits = al(K * G.W * sizeof(uint32_t)), sz_k = al(K * sizeof(uint64_t)),
                     sz_k1 = al((K + 1) * sizeof(uint64_t)), sz_st = al(((size_t) nt[t] + 1) * sizeof(uint64_t)),
                     sz_n = al((size_t) nt[t] * sizeof(uint32_t));
        const size_t need = sz_bits + 5 * sz_k + al(K) + 2 * sz_k1 + 256 + al(tb) + sz_st + 4 * sz_n;
        if(seg_cap < need) {
          if(d_seg) cudaFreeAsync(d_seg, s);
          d_seg = nullptr;
          seg_cap = need;
          PCK(cudaMallocAsync((void **) &d_seg, seg_cap, s));
        }
        char *cur = d_seg;
        G.bits = (uint32_t *) cur, cur += sz_bits;
        G.x = (uint64_t *) cur, cur += sz_k;
        G.cx = (uint64_t *) cur, cur += sz_k;
        uint64_t *ex[2] = {(uint64_t *) cur, (uint64_t *) (cur + sz_k)};
        cur += 2 * sz_k;
        uint64_t *d_pmax = (uint64_t *) cur;
        cur += sz_k;
        uint8_t *d_flag = (uint8_t *) cur;
        cur += al(K);
        uint64_t *d_cnt = (uint64_t *) cur, *d_off = (uint64_t *) (cur + sz_k1);
        cur += 2 * sz_k1;
        unsigned *d_first = (unsigned *) cur;
        int *d_changed = (int *) (cur + 128);
        cur += 256;
        void *d_scan = cur;
        cur += al(tb);
        d_starts = (uint64_t *) cur;
        cur += sz_st;
        uint32_t *d_lkey = (uint32_t *) cur, *d_lkey2 = (uint32_t *) (cur + sz_n);
        int *d_lidx = (int *) (cur + 2 * sz_n), *d_ord = (int *) (cur + 3 * sz_n);
        PCK(cudaMemsetAsync(G.bits, 0, sz_bits, s));
        with_kind(t, vs, [&](auto T, auto V) {
          k_seg_decode<decltype(T)::value, decltype(V)::value>
              <<<gblocks((long long) K, PBLOCK), PBLOCK, 0, s>>>(P, pos, G, ex[0]);
        });
        launches++;
        PCK(cudaGetLastError());
        int fin = -1;
        for(size_t r = 1; r <= K + 1; r++) {  // segment r - 1 is exact after round r - 1
          int h_changed = 0;
          const uint64_t *in = ex[(r - 1) & 1];
          uint64_t *out_ = ex[r & 1];
          size_t tbr = tb;
          PCK(cub::DeviceScan::InclusiveScan(d_scan, tbr, in, d_pmax, MaxU64(), K, s));
          k_seg_prep<<<gblocks((long long) K, 256), 256, 0, s>>>(G, d_pmax, in, out_, d_flag);
          PCK(cudaMemsetAsync(d_changed, 0, sizeof(int), s));
          with_kind(t, vs, [&](auto T, auto V) {
            k_seg_fix<decltype(T)::value, decltype(V)::value>
                <<<gblocks((long long) K, PBLOCK), PBLOCK, 0, s>>>(P, pos, G, d_pmax, d_flag, in, out_, d_changed);
          });
          launches += 3;
          PCK(cudaGetLastError());
          PCK(cudaMemcpyAsync(&h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, s));
          PCK(cudaStreamSynchronize(s));
          if(!h_changed) {
            fin = (int) (r & 1);
            break;
          }
        }
        if(fin < 0) {  // cannot happen: round r fixes segment r for good
          rc = GALIC_ERR_CUDA;
          break;
        }
        PCK(cudaMemsetAsync(d_first, 0xff, sizeof(unsigned), s));
        k_seg_first_cap<<<gblocks((long long) K, 256), 256, 0, s>>>(ex[fin], G.K, d_first);
        k_seg_count<<<gblocks((long long) K + 1, 256), 256, 0, s>>>(G, d_first, d_cnt);
        size_t tbx = tb;
        PCK(cub::DeviceScan::ExclusiveSum(d_scan, tbx, d_cnt, d_off, K + 1, s));
        launches += 3;
        PCK(cudaGetLastError());
        uint64_t total = 0;
        unsigned first = 0;
        PCK(cudaMemcpyAsync(&total, d_off + K, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        PCK(cudaMemcpyAsync(&first, d_first, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        PCK(cudaStreamSynchronize(s));
        if(total < (uint64_t) nt[t] + 1) {
          if(first < G.K) {  // the chain caps before its last particle ends
            rc = GALIC_ERR_REJECTION_CAP;
            break;
          }
          continue;  // the segments were too few: enlarge them
        }
        k_seg_extract<<<gblocks((long long) K, 256), 256, 0, s>>>(G, d_first, d_off, nt[t], d_starts);
        launches++;
        PCK(cudaGetLastError());
        uint64_t end = 0;
        PCK(cudaMemcpyAsync(&end, d_starts + nt[t], sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        PCK(cudaStreamSynchronize(s));
        k_len_keys<<<gblocks(nt[t], 256), 256, 0, s>>>(d_starts, nt[t], d_lkey, d_lidx);
        tbx = tb;
        PCK(cub::DeviceRadixSort::SortPairsDescending(d_scan, tbx, d_lkey, d_lkey2, d_lidx, d_ord, nt[t], 0, 32, s));
        with_kind(t, vs, [&](auto T, auto V) {
          k_final<decltype(T)::value, decltype(V)::value>
              <<<gblocks(nt[t], PBLOCK), PBLOCK, 0, s>>>(P, pos, d_starts, d_ord, nt[t], n0, O);
        });
        launches += 3;
        PCK(cudaGetLastError());
        pos += end;
        break;
      }
    }
  }
  if(rc != GALIC_OK) goto done;
  PCK(cudaMemcpyAsync(h_counts.data(), d_counts, 17 * sizeof(int), cudaMemcpyDeviceToHost, s));
  PCK(cudaStreamSynchronize(s));
  for(int t = 1; t <= 3; t++)
    for(int k = 0; k < 4; k++)
      if(nt[t] > 0 && (double) h_counts[4 * t + k] / nt[t] > 0.05) rc = GALIC_ERR_UNSUPPORTED;
  if(rc == GALIC_OK && h_counts[16]) rc = GALIC_ERR_INVALID_ARGUMENT;  // galic_set_particles' tint check
  if(rc == GALIC_OK) {
    // the permutation (set_particles.c:298-303)
    size_t tb = 0;
    PCK(cudaMallocAsync((void **) &d_keys, (size_t) N * sizeof(unsigned long long), s));
    PCK(cudaMallocAsync((void **) &d_keys2, (size_t) N * sizeof(unsigned long long), s));
    PCK(cudaMallocAsync((void **) &d_vals, (size_t) N * sizeof(int), s));
    PCK(cudaMallocAsync((void **) &d_vals2, (size_t) N * sizeof(int), s));
    k_perm_keys<<<gblocks(N, 256), 256, 0, s>>>(P.seed, P.sa, P.sb, pos, N, d_keys, d_vals);
    PCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_keys, d_keys2, d_vals, d_vals2, N, 0, 64, s));
    PCK(cudaMallocAsync(&d_tmp, std::max<size_t>(tb, 16), s));
    PCK(cub::DeviceRadixSort::SortPairs(d_tmp, tb, d_keys, d_keys2, d_vals, d_vals2, N, 0, 64, s));
    launches += 2;
    if(out && out->permutation)
      PCK(cudaMemcpyAsync(out->permutation, d_vals2, (size_t) N * sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  if(out && (rc == GALIC_OK || rc == GALIC_ERR_UNSUPPORTED)) {
    // the particles straight into the caller's arrays; masses, types and IDs
    // by type (set_particles.c:38-62)
    double *dst[6] = {out->pos, out->vel, out->vel_theo, out->vesc, out->tint, out->targets};
    const size_t off[6] = {0, 3, 6, 9, 10, 11}, len[6] = {3, 3, 3, 1, 1, 4};
    for(int k = 0; k < 6; k++)
      if(dst[k])
        PCK(cudaMemcpyAsync(dst[k], d_f + off[k] * N, len[k] * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    for(int t = 1, n = 0; t <= 3; t++)
      for(int i = 0; i < nt[t]; i++, n++) {
        if(out->mass) out->mass[n] = tmass[t] / nt[t];
        if(out->type) out->type[n] = t;
        if(out->id) out->id[n] = n + 1;
      }
    for(int t = 0; t < 4; t++)
      for(int k = 0; k < 4; k++) out->low_disp[t][k] = h_counts[4 * t + k];
  }
  PCK(cudaStreamSynchronize(s));
  if(rc == GALIC_OK) {
    // the particles become the context's
    rc = galic_internal::set_particles_device(ctx, nt, tmass, d_f, d_f + 3 * (size_t) N, d_f + 10 * (size_t) N, d_f + 9 * (size_t) N,
                              d_f + 11 * (size_t) N);
    if(rc == GALIC_OK) pos += (uint64_t) N;
  }
done:
  for(void *q : {(void *) d_f, (void *) d_counts, (void *) d_vals, (void *) d_vals2, (void *) d_J, (void *) d_seg,
                 (void *) d_keys, (void *) d_keys2, d_tmp})
    if(q) cudaFreeAsync(q, s);
  cudaStreamSynchronize(s);
  ctx->last_launches = launches;
  if(rc != GALIC_OK) return pfail(ctx, rc);
  stream->position = pos;
  return pfail(ctx, GALIC_OK);
}
