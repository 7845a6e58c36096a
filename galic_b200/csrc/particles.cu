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
// draw pairs are tested 32 at a time by a whole warp (halo_velocity_warp),
// and a loop still open after 2048 pairs is deferred and searched by the
// whole GPU between launches (LongTab, k_long_search): the kernels resume
// their suspended lanes, which then find the loop's answer in a table.  A
// resynchronisation walk that has carried on through 4 segments stops too,
// and goes on through a window of particle lengths evaluated ahead by the
// whole GPU (k_win_len).  A chain whose rejection loop hits its cap of 10^6
// tries ends there; if that happens before a type's last particle the call
// fails.  Built with --fmad=false and gmath.h's functions, so every particle
// is bit-identical to the CPU restatement.
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
constexpr uint32_t LEN_DEFER = 0xfffffffeu;  // a halo velocity loop passed VEL_SHORT pairs unresolved
constexpr int VEL_SHORT = 2048;               // pairs a warp tests before it defers the loop
constexpr int MAX_TAKE = 4;                   // segments a walk takes over before it waits for a window
constexpr int WIN_SEGS = 32;                  // segments' worth of positions in a long walk's window
constexpr int WIN_SLOTS = 64;                 // windows evaluated together
constexpr int PROBE = 1 << 16;        // positions of the draws-per-particle estimate
constexpr int PBLOCK = 128;

// Long halo velocity loops.  A loop that has not accepted a pair after
// VEL_SHORT pairs is deferred: its start position and radius go to the
// request list and the lane's particle returns LEN_DEFER.  Between launches
// k_long_search tests the loop's further pairs with the whole GPU and
// k_long_insert records the first accepted pair in an open-addressing table
// keyed by the loop's start position; the deferring kernel then resumes its
// suspended lanes, which find the loop in the table.
constexpr unsigned long long LT_EMPTY = ~0ull;
constexpr long long LT_CAPPED = -1;  // no pair accepted within LOOP_CAP pairs

struct LongTab {
  unsigned long long *key;  // mask + 1 entries, LT_EMPTY when free
  long long *acc;           // accepted pair, counted from the loop's first draw pair
  unsigned long long mask;
  unsigned long long *rq_key;  // requests of the current launch
  double *rq_r;
  int *rq_n;  // [0] requests, [1] overflow
  int rq_cap;
};

__device__ __forceinline__ unsigned long long lt_slot(unsigned long long key, unsigned long long mask)
{
  return (key * 0x9E3779B97F4A7C15ull >> 17) & mask;
}

// accepted pair of the loop starting at `key`; -2 when it is not in the table
__device__ long long lt_find(const LongTab &T, unsigned long long key)
{
  unsigned long long i = lt_slot(key, T.mask);
  for(unsigned long long probe = 0; probe <= T.mask; probe++, i = (i + 1) & T.mask) {
    const unsigned long long k = T.key[i];
    if(k == key) return T.acc[i];
    if(k == LT_EMPTY) return -2;
  }
  return -2;
}

struct PInit {
  DevModel M;
  Shape S;
  DispTab D[4];
  uint64_t seed;
  uint32_t sa, sb;
  double MaxVel, LowerDispLimit, TorbitFac;
  LongTab T;
};

struct POut {
  double *pos, *vel, *vel_theo, *vesc, *tint, *targets;
  int *counts;  // [4][4] raised to LowerDispLimit, [16] non-positive Tint, [17] deferred in k_final
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
// number of pairs has a long tail (up to 10^5 pairs and more); here the 32
// lanes test 32 consecutive pairs of one particle at once and a ballot picks
// the first accepted pair, which is the sequential loop's result.  A loop
// still open after its first 32 pairs is looked up in the long-loop table;
// one still open after VEL_SHORT pairs is deferred (see LongTab).  Every lane
// of the warp calls it; need: this lane has a draw to make.  Returns 0, or
// LEN_CAPPED / LEN_DEFER for this lane.
__device__ __forceinline__ bool halo_pair(const PInit &P, double rL, double v_max, double f_max, uint64_t j,
                                          double &v_guess)
{
  v_guess = grng_uniform_at(P.seed, P.sa, P.sb, j) * v_max;
  const double x_aux = grng_uniform_at(P.seed, P.sa, P.sb, j + 1) * f_max;
  return !(x_aux > v_guess * v_guess * halo_f(P.M, rL, v_guess));
}

__device__ uint32_t halo_velocity_warp(const PInit &P, bool need, double r, double vesc, uint64_t &w,
                                       double &vr_out)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const DevModel &M = P.M;
  uint32_t res = 0;
  unsigned pending = __ballot_sync(FULL, need);
  while(pending) {
    const int L = __ffs(pending) - 1;
    const double rL = __shfl_sync(FULL, r, L), vescL = __shfl_sync(FULL, vesc, L);
    uint64_t wpos = __shfl_sync(FULL, (unsigned long long) w, L);
    double vr = 0;
    uint32_t st = 0;
    int redraws = 0;
    do {
      if(++redraws > LOOP_CAP) {  // speeds at or above MaxVelInUnitsVesc Vesc without end
        st = LEN_CAPPED;
        break;
      }
      const double pot = halo_pot_r(M, rL);
      const double v_max = sqrt(-2 * pot);
      const double f_max = v_max * v_max * halo_f(M, rL, 0);
      long long n = -2;
      for(long long base = 0; base < VEL_SHORT; base += 32) {
        double vg;
        const unsigned mask = __ballot_sync(FULL, halo_pair(P, rL, v_max, f_max, wpos + 2 * (uint64_t) (base + lane), vg));
        if(mask) {
          const int first = __ffs(mask) - 1;
          vr = __shfl_sync(FULL, vg, first);
          n = base + first;
          break;
        }
        if(base == 0) {  // a long loop: resolved already?
          const long long t = lt_find(P.T, wpos);
          if(t == LT_CAPPED) {
            st = LEN_CAPPED;
            break;
          }
          if(t >= 0) {
            n = t;
            vr = grng_uniform_at(P.seed, P.sa, P.sb, wpos + 2 * (uint64_t) t) * v_max;
            break;
          }
        }
      }
      if(st) break;
      if(n < 0) {  // still open after VEL_SHORT pairs
        if(lane == 0) {
          const int i = atomicAdd(&P.T.rq_n[0], 1);
          if(i < P.T.rq_cap) {
            P.T.rq_key[i] = wpos;
            P.T.rq_r[i] = rL;
          } else {
            P.T.rq_n[1] = 1;
          }
        }
        st = LEN_DEFER;
        break;
      }
      wpos += 2 * (uint64_t) (n + 1);
    } while(vr >= P.MaxVel * vescL);
    if(lane == L) {
      w = wpos;
      vr_out = vr;
      res = st;
    }
    pending &= pending - 1;
  }
  return res;
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
    const uint32_t vst = halo_velocity_warp(P, ok, r, vesc, w, vr);
    if(ok && vst) return vst;
    if(ok) grng_seek(&g, w);
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
  if(len == LEN_DEFER) {  // not counted in the estimate
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
  // a lane whose particle deferred a long loop: where it stopped (segment,
  // position of the particle), resumed by the next launch with resume = true
  uint8_t *susp;  // 1: a long loop deferred, 2: a long walk stopped
  uint32_t *rs_d;
  uint64_t *rs_q;
};

// Windows of particle lengths ahead of the stopped long walks: walk k (lane
// lane_of_slot) gets positions [lo[k], lo[k] + n) of the type's draws,
// evaluated by the whole GPU (k_win_len); LEN_DEFER where a long loop is
// still open, and then the walk evaluates the particle itself
struct Win {
  const uint32_t *len;  // [slots][n]
  const uint64_t *lo;   // [slots]
  const int *slot;      // [K]: the lane's window, -1 for none
  uint32_t n;
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
// init_one together: lanes past K only keep the others company); with
// resume, only the suspended segments, from where they stopped
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_seg_decode(const PInit P, uint64_t base, const Segs S, uint64_t *exit,
                                                       bool resume)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = c < S.K && (!resume || S.susp[c]);
  const uint64_t a = (uint64_t) c * S.Lseg, end = a + S.Lseg;
  uint32_t *w = S.bits + (size_t) (valid ? c : 0) * S.W;
  uint64_t q = a;
  if(valid && resume) {
    S.susp[c] = 0;
    q = S.rs_q[c];
  }
  bool work = valid, done = valid;
  while(__any_sync(0xffffffffu, work)) {
    const uint32_t len = init_one<TYPE, VS>(P, base + (work ? q : 0), work, nullptr, 0);
    if(work) {
      if(len == LEN_DEFER) {
        S.susp[c] = 1;
        S.rs_q[c] = q;
        work = done = false;
        continue;
      }
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
  if(done) {
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
// when no exit changes.  With resume, only the suspended walks go on, in the
// same round, from the segment and position where they stopped.
// resume: 0 a new round; 1 the walks that deferred a long loop; 2 the
// stopped long walks, each through its window in W.  A walk that has taken
// over max_take segments outside a window stops and waits for one.
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_seg_fix(const PInit P, uint64_t base, const Segs S,
                                                    const uint64_t *pmax, const uint8_t *flag,
                                                    const uint64_t *exit_in, uint64_t *exit_out, int *changed,
                                                    int resume, int max_take, Win W)
{
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const int sl = (resume == 2 && c < S.K) ? W.slot[c] : -1;
  bool work = c < S.K && (resume == 0 ? flag[c] != 0 : (resume == 1 ? S.susp[c] == 1 : sl >= 0));
  const uint64_t wlo = sl >= 0 ? W.lo[sl] : 0;
  uint32_t d = c;
  uint64_t q = 0;
  int taken = 0;
  if(work && resume) {
    S.susp[c] = 0;
    d = S.rs_d[c];
    q = S.rs_q[c];
  }
  uint64_t a = (uint64_t) d * S.Lseg, end = a + S.Lseg;
  uint32_t *w = S.bits + (size_t) (work ? d : 0) * S.W;
  if(work && !resume) {
    q = pmax[c - 1];  // flag[0] is never set
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
            if(resume != 2 && ++taken > max_take) {  // a long walk: on with a window
              S.susp[c] = 2;
              S.rs_d[c] = d;
              S.rs_q[c] = q;
              work = false;
            }
          }
        }
      } else {
        step = true;
      }
    }
    uint32_t len = LEN_DEFER;
    const bool in_win = step && sl >= 0 && q >= wlo && q - wlo < W.n;
    if(in_win) len = W.len[(size_t) sl * W.n + (q - wlo)];
    const bool eval = step && len == LEN_DEFER;
    const uint32_t len1 = init_one<TYPE, VS>(P, base + (eval ? q : 0), eval, nullptr, 0);
    if(eval) len = len1;
    if(step) {
      if(resume == 2 && !in_win) {  // past the window: another one
        S.susp[c] = 2;
        S.rs_d[c] = d;
        S.rs_q[c] = q;
        work = false;
        continue;
      }
      if(len == LEN_DEFER) {
        S.susp[c] = 1;
        S.rs_d[c] = d;
        S.rs_q[c] = q;
        work = false;
        continue;
      }
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

// lengths of the particles starting at the windows' positions
template <int TYPE, int VS>
__global__ void __launch_bounds__(PBLOCK) k_win_len(const PInit P, uint64_t base, const uint64_t *lo, uint32_t n,
                                                    uint32_t slots, uint32_t *len)
{
  const uint64_t o = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = o < (uint64_t) n * slots;
  const uint64_t at = active ? lo[o / n] + o % n : 0;
  const uint32_t l = init_one<TYPE, VS>(P, base + at, active, nullptr, 0);
  if(active) len[o] = l;
}

// Long-loop search: pairs [lo, lo + len) of request i (blockIdx.y), each
// thread a run of consecutive pairs; found[i] = the first accepted pair
__global__ void __launch_bounds__(256) k_long_search(const PInit P, const unsigned long long *key, const double *r,
                                                     long long lo, long long len, unsigned long long *found)
{
  const int i = blockIdx.y;
  if(found[i] != LT_EMPTY) return;
  constexpr int RUN = 8;
  const long long first = lo + ((long long) blockIdx.x * blockDim.x + threadIdx.x) * RUN;
  if(first >= lo + len) return;
  const double rL = r[i];
  const double v_max = sqrt(-2 * halo_pot_r(P.M, rL));
  const double f_max = v_max * v_max * halo_f(P.M, rL, 0);
  for(int k = 0; k < RUN; k++) {
    double vg;
    if(halo_pair(P, rL, v_max, f_max, key[i] + 2 * (uint64_t) (first + k), vg)) {
      atomicMin(&found[i], (unsigned long long) (first + k));
      return;
    }
  }
}

// requests still open after a search step
__global__ void k_long_open(const unsigned long long *found, int n, int *open)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n && found[i] == LT_EMPTY) atomicAdd(open, 1);
}

// results into the table (requests for one loop may repeat); open ones
// after LOOP_CAP pairs are capped
__global__ void k_long_insert(LongTab T, const unsigned long long *found, int n, int *full)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const unsigned long long key = T.rq_key[i];
  const long long v = found[i] == LT_EMPTY ? LT_CAPPED : (long long) found[i];
  unsigned long long s = lt_slot(key, T.mask);
  for(unsigned long long probe = 0; probe <= T.mask; probe++, s = (s + 1) & T.mask) {
    const unsigned long long prev = atomicCAS(&T.key[s], LT_EMPTY, key);
    if(prev == LT_EMPTY || prev == key) {
      T.acc[s] = v;  // the same value for every request of this key
      return;
    }
  }
  atomicAdd(full, 1);
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
  const uint32_t len = init_one<TYPE, VS>(P, base + (active ? starts[i] : 0), active, &o, n0 + i);
  if(active && len == LEN_DEFER) atomicAdd(&o.counts[17], 1);  // its values were not written
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

// Resolves the long loops requested since the last call: k_long_search over
// growing runs of pairs (4096, then x4) until every request has its first
// accepted pair or LOOP_CAP pairs were tested, then k_long_insert.  *n: the
// requests there were.  d_aux: 2 ints of scratch.  partial: the launch that
// made the requests (the probe, the windows) may lose some to a full list --
// its positions stay deferred and are evaluated again where they matter --
// so only the recorded ones are resolved; elsewhere a full list is an error.
int resolve_long(const PInit &P, cudaStream_t s, unsigned long long *d_found, int *d_aux, int *n, int &launches,
                 bool partial = false)
{
  int h[2] = {0, 0};
  if(cudaMemcpyAsync(h, P.T.rq_n, 2 * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
     cudaStreamSynchronize(s) != cudaSuccess)
    return GALIC_ERR_CUDA;
  if(h[1] && !partial) return GALIC_ERR_UNSUPPORTED;  // at most one request per lane: not reachable
  if(h[0] > P.T.rq_cap) h[0] = P.T.rq_cap;
  *n = h[0];
  if(h[0] == 0) return GALIC_OK;
  const int nreq = h[0];
  if(cudaMemsetAsync(d_found, 0xff, (size_t) nreq * sizeof(unsigned long long), s) != cudaSuccess)
    return GALIC_ERR_CUDA;
  for(long long lo = VEL_SHORT, len = 4096; lo < LOOP_CAP; lo += len, len *= 4) {
    if(lo + len > LOOP_CAP) len = LOOP_CAP - lo;
    const unsigned bx = (unsigned) ((len + 256 * 8 - 1) / (256 * 8));
    for(int r0 = 0; r0 < nreq; r0 += 65535) {
      const unsigned nr = (unsigned) std::min(65535, nreq - r0);
      k_long_search<<<dim3(bx, nr), 256, 0, s>>>(P, P.T.rq_key + r0, P.T.rq_r + r0, lo, len, d_found + r0);
      launches++;
    }
    int open = 0;
    if(cudaMemsetAsync(d_aux, 0, sizeof(int), s) != cudaSuccess) return GALIC_ERR_CUDA;
    k_long_open<<<gblocks(nreq, 256), 256, 0, s>>>(d_found, nreq, d_aux);
    launches++;
    if(cudaGetLastError() != cudaSuccess ||
       cudaMemcpyAsync(&open, d_aux, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess)
      return GALIC_ERR_CUDA;
    if(open == 0) break;
  }
  int full = 0;
  if(cudaMemsetAsync(d_aux + 1, 0, sizeof(int), s) != cudaSuccess) return GALIC_ERR_CUDA;
  k_long_insert<<<gblocks(nreq, 256), 256, 0, s>>>(P.T, d_found, nreq, d_aux + 1);
  launches++;
  if(cudaGetLastError() != cudaSuccess ||
     cudaMemcpyAsync(&full, d_aux + 1, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
     cudaMemsetAsync(P.T.rq_n, 0, 2 * sizeof(int), s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
    return GALIC_ERR_CUDA;
  return full ? GALIC_ERR_UNSUPPORTED : GALIC_OK;  // the table is sized far above the loops there can be
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
  void *d_tmp = nullptr, *d_long = nullptr;
  unsigned long long *d_found = nullptr;
  int *d_aux = nullptr;
  uint32_t *d_wlen = nullptr;
  uint64_t *d_wlo = nullptr;  // inside d_long
  int *d_wslot = nullptr;  // inside d_seg
  size_t win_cap = 0;
  std::vector<uint64_t> h_rsq;
  size_t J_cap = 0, seg_cap = 0;
  std::vector<int> h_counts(18);
  std::vector<uint8_t> h_susp;
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
  PCK(cudaMallocAsync((void **) &d_counts, 18 * sizeof(int), s));
  PCK(cudaMemsetAsync(d_f, 0, (size_t) 15 * N * sizeof(double), s));
  PCK(cudaMemsetAsync(d_counts, 0, 18 * sizeof(int), s));
  O.pos = d_f;
  O.vel = d_f + 3 * (size_t) N;
  O.vel_theo = d_f + 6 * (size_t) N;
  O.vesc = d_f + 9 * (size_t) N;
  O.tint = d_f + 10 * (size_t) N;
  O.targets = d_f + 11 * (size_t) N;
  O.counts = d_counts;
  {
    // long-loop table (about one loop in 2 000 passes VEL_SHORT pairs) and
    // the request list (at most one request per lane and launch)
    unsigned long long cap = 8192;
    while(cap < (unsigned long long) N / 16) cap <<= 1;
    const int rq_cap = std::max(N, PROBE) + 64;
    const size_t bytes = cap * 16 + (size_t) rq_cap * 24 + 64 + WIN_SLOTS * sizeof(uint64_t);
    PCK(cudaMallocAsync(&d_long, bytes, s));
    char *c = (char *) d_long;
    P.T.key = (unsigned long long *) c;
    P.T.acc = (long long *) (c + cap * 8);
    P.T.mask = cap - 1;
    P.T.rq_key = (unsigned long long *) (c + cap * 16);
    P.T.rq_r = (double *) (c + cap * 16 + (size_t) rq_cap * 8);
    d_found = (unsigned long long *) (c + cap * 16 + (size_t) rq_cap * 16);
    P.T.rq_n = (int *) (c + cap * 16 + (size_t) rq_cap * 24);
    d_aux = P.T.rq_n + 4;
    d_wlo = (uint64_t *) (c + cap * 16 + (size_t) rq_cap * 24 + 64);
    P.T.rq_cap = rq_cap;
    PCK(cudaMemsetAsync(P.T.key, 0xff, cap * 8, s));
    PCK(cudaMemsetAsync(P.T.rq_n, 0, 64, s));
  }
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
      // the long loops met are resolved and the probe repeated, so that the
      // estimate holds them (the few long ones weigh much in the mean)
      for(int rep = 0;; rep++) {
        with_kind(t, vs, [&](auto T, auto V) {
          k_len<decltype(T)::value, decltype(V)::value><<<gblocks(R + 2, PBLOCK), PBLOCK, 0, s>>>(P, pos, R, d_J);
        });
        launches++;
        PCK(cudaGetLastError());
        int nreq = 0;
        rc = resolve_long(P, s, d_found, d_aux, &nreq, launches, true);
        if(rc != GALIC_OK || nreq == 0 || rep >= 8) break;
      }
      if(rc != GALIC_OK) break;
      PCK(cudaMemsetAsync(P.T.rq_n, 0, 2 * sizeof(int), s));
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
        // bits, x, cx, exits x 2, pmax, flag, cnt, off, first/changed, scan scratch, starts,
        // length keys and order, resume positions, segments, suspended flags, window slots
        const size_t need = sz_bits + 5 * sz_k + al(K) + 2 * sz_k1 + 256 + al(tb) + sz_st + 4 * sz_n + sz_k +
                            al(K * sizeof(uint32_t)) + al(K) + al(K * sizeof(int));
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
        cur += 4 * sz_n;
        G.rs_q = (uint64_t *) cur;
        cur += sz_k;
        G.rs_d = (uint32_t *) cur;
        cur += al(K * sizeof(uint32_t));
        G.susp = (uint8_t *) cur;
        cur += al(K);
        d_wslot = (int *) cur;
        PCK(cudaMemsetAsync(G.bits, 0, sz_bits, s));
        PCK(cudaMemsetAsync(G.susp, 0, K, s));
        PCK(cudaMemsetAsync(d_wslot, 0xff, K * sizeof(int), s));
        for(int resume = 0;; resume++) {
          with_kind(t, vs, [&](auto T, auto V) {
            k_seg_decode<decltype(T)::value, decltype(V)::value>
                <<<gblocks((long long) K, PBLOCK), PBLOCK, 0, s>>>(P, pos, G, ex[0], resume > 0);
          });
          launches++;
          PCK(cudaGetLastError());
          int nreq = 0;
          rc = resolve_long(P, s, d_found, d_aux, &nreq, launches);
          if(rc != GALIC_OK || nreq == 0) break;
          if(resume > 100000) {  // each resume passes a resolved loop: cannot happen
            rc = GALIC_ERR_CUDA;
            break;
          }
        }
        if(rc != GALIC_OK) break;
        int fin = -1;
        for(size_t r = 1; r <= K + 1; r++) {  // segment r - 1 is exact after round r - 1
          int h_changed = 0;
          const uint64_t *in = ex[(r - 1) & 1];
          uint64_t *out_ = ex[r & 1];
          size_t tbr = tb;
          PCK(cub::DeviceScan::InclusiveScan(d_scan, tbr, in, d_pmax, MaxU64(), K, s));
          k_seg_prep<<<gblocks((long long) K, 256), 256, 0, s>>>(G, d_pmax, in, out_, d_flag);
          PCK(cudaMemsetAsync(d_changed, 0, sizeof(int), s));
          launches += 2;
          // the round, then the walks that deferred a long loop, then the long
          // walks, through windows of particle lengths evaluated ahead
          int mode = 0;
          Win win{};
          for(int it = 0;; it++) {
            if(it > 1000000) {  // every launch passes a resolved loop or a window: cannot happen
              rc = GALIC_ERR_CUDA;
              break;
            }
            with_kind(t, vs, [&](auto T, auto V) {
              k_seg_fix<decltype(T)::value, decltype(V)::value><<<gblocks((long long) K, PBLOCK), PBLOCK, 0, s>>>(
                  P, pos, G, d_pmax, d_flag, in, out_, d_changed, mode, MAX_TAKE, win);
            });
            launches++;
            PCK(cudaGetLastError());
            if(mode == 2) PCK(cudaMemsetAsync(d_wslot, 0xff, K * sizeof(int), s));
            int nreq = 0;
            rc = resolve_long(P, s, d_found, d_aux, &nreq, launches);
            if(rc != GALIC_OK) break;
            if(nreq) {
              mode = 1;
              win = Win{};
              continue;
            }
            // the stopped long walks, up to WIN_SLOTS at a time
            h_susp.resize(K);
            PCK(cudaMemcpyAsync(h_susp.data(), G.susp, K, cudaMemcpyDeviceToHost, s));
            PCK(cudaStreamSynchronize(s));
            std::vector<uint32_t> walks;
            for(uint32_t k = 0; k < (uint32_t) K && walks.size() < (size_t) WIN_SLOTS; k++)
              if(h_susp[k] == 2) walks.push_back(k);
            if(walks.empty()) break;
            const uint32_t wn = (uint32_t) (WIN_SEGS * Lseg), ns = (uint32_t) walks.size();
            h_rsq.resize(K);
            PCK(cudaMemcpyAsync(h_rsq.data(), G.rs_q, K * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
            PCK(cudaStreamSynchronize(s));
            std::vector<uint64_t> wlo(ns);
            std::vector<int> wslot(K, -1);
            for(uint32_t k = 0; k < ns; k++) {
              wlo[k] = h_rsq[walks[k]];
              wslot[walks[k]] = (int) k;
            }
            if(win_cap < (size_t) wn * ns) {
              if(d_wlen) cudaFreeAsync(d_wlen, s);
              d_wlen = nullptr;
              win_cap = (size_t) wn * WIN_SLOTS;
              PCK(cudaMallocAsync((void **) &d_wlen, win_cap * sizeof(uint32_t), s));
            }
            PCK(cudaMemcpyAsync(d_wlo, wlo.data(), ns * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
            PCK(cudaMemcpyAsync(d_wslot, wslot.data(), K * sizeof(int), cudaMemcpyHostToDevice, s));
            // the windows' lengths; the long loops met there are resolved into
            // the table, and the walks evaluate those particles themselves
            with_kind(t, vs, [&](auto T, auto V) {
              k_win_len<decltype(T)::value, decltype(V)::value>
                  <<<gblocks((long long) wn * ns, PBLOCK), PBLOCK, 0, s>>>(P, pos, d_wlo, wn, ns, d_wlen);
            });
            launches++;
            PCK(cudaGetLastError());
            int nw = 0;
            rc = resolve_long(P, s, d_found, d_aux, &nw, launches, true);
            if(rc != GALIC_OK) break;
            mode = 2;
            win = Win{d_wlen, d_wlo, d_wslot, wn};
          }
          if(rc != GALIC_OK) break;
          PCK(cudaMemcpyAsync(&h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, s));
          PCK(cudaStreamSynchronize(s));
          if(!h_changed) {
            fin = (int) (r & 1);
            break;
          }
        }
        if(rc != GALIC_OK) break;
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
  PCK(cudaMemcpyAsync(h_counts.data(), d_counts, 18 * sizeof(int), cudaMemcpyDeviceToHost, s));
  PCK(cudaStreamSynchronize(s));
  for(int t = 1; t <= 3; t++)
    for(int k = 0; k < 4; k++)
      if(nt[t] > 0 && (double) h_counts[4 * t + k] / nt[t] > 0.05) rc = GALIC_ERR_UNSUPPORTED;
  if(rc == GALIC_OK && h_counts[16]) rc = GALIC_ERR_INVALID_ARGUMENT;  // galic_set_particles' tint check
  // every particle of the chain had each of its long loops resolved while the
  // chain was decoded, so k_final finds them all in the table
  if(rc == GALIC_OK && h_counts[17]) rc = GALIC_ERR_CUDA;
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
  for(void *q : {(void *) d_f, (void *) d_counts, (void *) d_vals, (void *) d_vals2, (void *) d_J, (void *) d_seg, d_long, (void *) d_wlen,
                 (void *) d_keys, (void *) d_keys2, d_tmp})
    if(q) cudaFreeAsync(q, s);
  cudaStreamSynchronize(s);
  ctx->last_launches = launches;
  if(rc != GALIC_OK) return pfail(ctx, rc);
  stream->position = pos;
  return pfail(ctx, GALIC_OK);
}
