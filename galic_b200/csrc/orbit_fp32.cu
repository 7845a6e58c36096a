// FP32-integrate / FP64-accumulate form of calc_all_response_fields
// (main.c:151-231, orbit_response.c:155-491).
//
// Same algorithm as the FP64 form (orbit_fp64.cu) with these changes, all of
// which only move results within the stated tolerance of the FP64 oracle:
//  * positions, velocities, accelerations and the interpolation run in FP32;
//    position and velocity are carried as compensated sums (Kahan 1965: an
//    FP32 value plus an FP32 correction term), so the rounding of the many
//    small kicks and drifts does not build up over an orbit span;
//    the force grid is read from one "quad" table per particle type: for
//    every cell the four corners' DPotDR, DPotDz and Vstream[type] (three
//    float4, one 64-byte line), so a bilinear lookup is one cache line;
//  * log(x)/log(Fac) becomes log2(x) * (1/log2 Fac) (MUFU.LG2), divisions
//    become reciprocal multiplies, and accR (cos phi, sin phi) is evaluated as
//    accR (x/R, y/R), which is the same vector without atan2/sin/cos;
//  * the orbit time tall, the mass/timespan normalisation and every deposit
//    into the response grids stay FP64 (merged per cell in FP32 registers,
//    then rounded once into the exact fixed-point accumulators);
//  * the relative energy drift check uses FP64 potentials.
// Built with --fmad=true (this file keeps contraction on).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "flush.cuh"
#include "kernels.cuh"

namespace {

struct Model32 {
  float V200, f_orb, f_cc;
  float invFG, ilgFG;       // 1/FG_Rmin, 1/log2(FG_Fac)
  float invDG, ilgDG;       // 1/DG_Rmin, 1/log2(DG_Fac)
  float GMh, Ah, eps_h, haloscale;   // G*Halo_Mass, Halo_A, 1e-6 Halo_A, M200/Halo_Mass
  float GMb, Ab, eps_b;
  int tabulated, analytic_halo, analytic_bulge;
  int tovs[4];
  int vstream_zero[4];     // FG_Vstream[type] identically zero: its corners are not read
  int FG_Nbin, DG_Nbin;
  float fgmax;             // FG_Nbin - 1
  float dgmax;             // DG_Nbin - 1
  const float4 *quad[4];   // per type, per cell iz*N+iR: {DPotDR x4}, {DPotDz x4}, {Vstream x4}, pad
  const float *cellsize;
  long long step_cap;
};

__device__ __forceinline__ float frcp(float x) { return __frcp_rn(x); }

struct Cell32 {
  int iR, iz;
  float fR, fz;
};

__device__ __forceinline__ Cell32 cell32(float br, float bz, int nbin, float bmax)
{
  // (grid.c:20-55 / 494-534) inside the grid: bin = floor, fraction = rest;
  // beyond its last node: bin = nbin - 2, fraction 1 (branch-free)
  Cell32 c;
  br = fmaxf(br, 0.f);
  bz = fmaxf(bz, 0.f);
  const bool in_r = br < bmax, in_z = bz < bmax;
  const float fbr = floorf(br), fbz = floorf(bz);
  c.iR = in_r ? (int) fbr : nbin - 2;
  c.iz = in_z ? (int) fbz : nbin - 2;
  c.fR = in_r ? br - fbr : 1.f;
  c.fz = in_z ? bz - fbz : 1.f;
  return c;
}

// acceleration (grid.c:122-197) and streaming velocity (disp_fields.c:118-132)
// at x; both read the same float4 table corners
__device__ __forceinline__ void accel32(const Model32 &M, int type, const float *x, float *a, float *vstr)
{
  const float R2 = x[0] * x[0] + x[1] * x[1];
  const float R = sqrtf(R2);
  const float az_abs = fabsf(x[2]);
  const float jd = __log2f(fmaf(R, M.invFG, 1.f)) * M.ilgFG;
  const float id = __log2f(fmaf(az_abs, M.invFG, 1.f)) * M.ilgFG;
  const int N = M.FG_Nbin;
  Cell32 c = cell32(jd, id, N, M.fgmax);
  // corners in the quad: (iz,iR), (iz,iR+1), (iz+1,iR), (iz+1,iR+1)
  const float4 *Q = M.quad[type] + 4 * (c.iz * N + c.iR);
  const float4 qR = __ldg(&Q[0]), qZ = __ldg(&Q[1]);
  const float4 qV = M.vstream_zero[type] ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(&Q[2]);
  const float w00 = (1.f - c.fR) * (1.f - c.fz), w01 = c.fR * (1.f - c.fz);
  const float w10 = (1.f - c.fR) * c.fz, w11 = c.fR * c.fz;
  *vstr = qV.x * w00 + qV.z * w10 + qV.y * w01 + qV.w * w11;
  a[0] = a[1] = a[2] = 0.f;
  if(M.tabulated) {
    if(jd < M.fgmax && id < M.fgmax) {
      float accR = qR.x * w00 + qR.y * w01 + qR.z * w10 + qR.w * w11;
      float accz = qZ.x * w00 + qZ.y * w01 + qZ.z * w10 + qZ.w * w11;
      if(x[2] < 0) accz = -accz;
      const float inv = R > 0.f ? frcp(R) : 0.f;
      a[0] = accR * x[0] * inv;
      a[1] = accR * x[1] * inv;
      a[2] = accz;
    } else {
      const float r = sqrtf(R2 + x[2] * x[2]);
      const float rp = r + M.Ah;
      const float fac = M.haloscale * M.GMh * frcp((r + M.eps_h) * rp * rp);
      a[0] = -fac * x[0];
      a[1] = -fac * x[1];
      a[2] = -fac * x[2];
    }
  }
  if(M.analytic_halo | M.analytic_bulge) {
    const float r = sqrtf(R2 + x[2] * x[2]);
    float fac = 0.f;
    if(M.analytic_halo) {
      const float rp = r + M.Ah;
      fac += M.GMh * frcp((r + M.eps_h) * rp * rp);
    }
    if(M.analytic_bulge) {
      const float rp = r + M.Ab;
      fac += M.GMb * frcp((r + M.eps_b) * rp * rp);
    }
    a[0] -= fac * x[0];
    a[1] -= fac * x[1];
    a[2] -= fac * x[2];
  }
}

struct Proj32 {
  float vr2, vt2, vq2, vp2;
};

// orbit_response.c:222-273 in FP32; vstr is the streaming velocity at x
__device__ __forceinline__ Proj32 project32(int tovs, const float *x, const float *v, float vstr)
{
  Proj32 o;
  if(tovs == 2) {
    const float r2 = x[0] * x[0] + x[1] * x[1];
    const float vdx = v[0] * x[0] + v[1] * x[1];
    const float ir2 = frcp(r2);
    o.vr2 = vdx * vdx * ir2;
    const float vq = (v[1] * x[0] - v[0] * x[1]) * rsqrtf(r2);
    o.vq2 = vq * vq;
    o.vp2 = (vq - vstr) * (vq - vstr);
    o.vt2 = v[2] * v[2];
  } else {
    // Q = x cross (0,0,-1) = (-y, x, 0); T = x cross Q
    const float r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    const float vdx = v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
    o.vr2 = vdx * vdx * frcp(r2);
    const float q2 = x[0] * x[0] + x[1] * x[1];
    const float vq = (v[1] * x[0] - v[0] * x[1]) * rsqrtf(q2);
    o.vq2 = vq * vq;
    o.vp2 = (vq - vstr) * (vq - vstr);
    const float T0 = x[0] * x[2], T1 = x[1] * x[2], T2 = -q2;
    const float t2 = T0 * T0 + T1 * T1 + T2 * T2;
    const float vdT = v[0] * T0 + v[1] * T1 + v[2] * T2;
    o.vt2 = vdT * vdT * frcp(t2);
  }
  return o;
}

__device__ __forceinline__ Cell32 density_cell32(const Model32 &M, const float *x)
{
  const float r = sqrtf(x[0] * x[0] + x[1] * x[1]);
  const float br = __log2f(fmaf(r, M.invDG, 1.f)) * M.ilgDG - 0.5f;
  const float bz = __log2f(fmaf(fabsf(x[2]), M.invDG, 1.f)) * M.ilgDG - 0.5f;
  return cell32(br, bz, M.DG_Nbin, M.dgmax);
}

// Register-merged FP32 sums for the four grid nodes of the current DG cell.
// A node (z, r) always lives in accumulator slot ((z & 1) << 1) | (r & 1):
// the four nodes of any cell have the four parities, so when the orbit moves
// to a neighbouring cell the nodes both cells share stay in their slots
// untouched, and only the slots whose node changes are flushed and cleared.
// A deposit's corner c = 2 dz + dr of the cell lands in slot c ^ (2 (iz & 1) + (iR & 1)).
struct NodeAcc {
  int cur = -1, cur_iR = 0, cur_iz = 0;
  float a[4][5];
  // slot s of cell (iz, iR) holds node (iz + node_dz(s, iz), iR + node_dr(s, iR))
  __device__ __forceinline__ static int node_dz(int s, int iz) { return ((s >> 1) ^ iz) & 1; }
  __device__ __forceinline__ static int node_dr(int s, int iR) { return (s ^ iR) & 1; }
  // slots whose node is not a node of cell (iz, iR)
  __device__ __forceinline__ void leaving(int iR, int iz, bool out[4]) const
  {
    // along one axis a move by d leaves the node whose parity is that of the
    // boundary left behind (d = +1: the lower node, d = -1: the upper one),
    // both nodes when |d| > 1, none when d = 0
    const int dz = iz - cur_iz, dr = iR - cur_iR;
    const int bz = (dz > 0 ? cur_iz : cur_iz + 1) & 1, br = (dr > 0 ? cur_iR : cur_iR + 1) & 1;
    const bool zall = dz > 1 || dz < -1, rall = dr > 1 || dr < -1;
    bool lz[2], lr[2];
#pragma unroll
    for(int b = 0; b < 2; b++) {
      lz[b] = zall || (dz != 0 && b == bz);
      lr[b] = rall || (dr != 0 && b == br);
    }
#pragma unroll
    for(int s = 0; s < 4; s++) out[s] = lz[s >> 1] || lr[s & 1];
  }
  __device__ __forceinline__ void clear(const bool which[4])
  {
#pragma unroll
    for(int s = 0; s < 4; s++)
#pragma unroll
      for(int f = 0; f < 5; f++) a[s][f] = which[s] ? 0.f : a[s][f];
  }
  __device__ __forceinline__ void accumulate(int iR, int iz, float hdt, float fR, float fz, const Proj32 &p)
  {
    // weights in slot order: slot s holds corner (dz, dr) = ((s >> 1) ^ (iz & 1), (s & 1) ^ (iR & 1))
    const bool oz = iz & 1, orr = iR & 1;
    const float z0 = oz ? fz : 1.f - fz, z1 = oz ? 1.f - fz : fz;
    const float r0 = orr ? fR : 1.f - fR, r1 = orr ? 1.f - fR : fR;
    const float hz0 = hdt * z0, hz1 = hdt * z1;
    const float w[4] = {hz0 * r0, hz0 * r1, hz1 * r0, hz1 * r1};
#pragma unroll
    for(int k = 0; k < 4; k++) {
      a[k][0] += w[k];
      a[k][1] = fmaf(w[k], p.vr2, a[k][1]);
      a[k][2] = fmaf(w[k], p.vt2, a[k][2]);
      a[k][3] = fmaf(w[k], p.vq2, a[k][3]);
      a[k][4] = fmaf(w[k], p.vp2, a[k][4]);
    }
  }
};

// Sink of the batched kernels: on a cell change the nonzero sums of the
// leaving nodes are parked in the warp queue as (word index, scaled value)
// records, and the warp drains them together once enough wait (flush.cuh).
template <int PER>
struct Sink32 : NodeAcc {
  WarpQueue32<PER> *q;
  int lane, Nb;
  int cnt;  // records parked in this lane's queue column since the last drain
  // the orbit's first word (grid set x NG_COMMITTED x Ngrid) and the scale
  // factors mass/Tint x 2^(shift-24) of the mass and energy fields, kept in
  // the lane's queue header (read only when parking)
  __device__ __forceinline__ void set_orbit(int gbase, float scale_m, float scale_e)
  {
    q->gbase[lane] = gbase;
    q->scale[0][lane] = scale_m;
    q->scale[1][lane] = scale_e;
  }
  __device__ __forceinline__ void park_masked(const bool out[4])
  {
    // a node with no mass has no deposit at all (every field is weight x ...);
    // the records keep the raw sums and the node's index in the grid, the
    // drain adds the orbit's grid set and scale factors
    bool rec[4];
    int at[4], k = cnt;
#pragma unroll
    for(int s = 0; s < 4; s++) {
      rec[s] = out[s] && a[s][0] != 0.f;
      at[s] = k;
      k += rec[s] ? 1 : 0;
    }
#pragma unroll
    for(int s = 0; s < 4; s++) {
      if(rec[s]) {
        q->base[at[s]][lane] = (cur_iz + node_dz(s, cur_iz)) * Nb + cur_iR + node_dr(s, cur_iR);
#pragma unroll
        for(int f = 0; f < 5; f++) q->val[at[s]][f][lane] = a[s][f];
      }
    }
    cnt = k;
  }
  __device__ __forceinline__ void park()
  {
    if(cur < 0) return;
    const bool all[4] = {true, true, true, true};
    park_masked(all);
    cur = -1;
  }
  __device__ __forceinline__ void move_to(int iR, int iz)
  {
    if(cur >= 0) {
      bool out[4];
      leaving(iR, iz, out);
      park_masked(out);
      clear(out);
    } else {
      const bool all[4] = {true, true, true, true};
      clear(all);
    }
    cur = iz * Nb + iR;
    cur_iR = iR;
    cur_iz = iz;
  }
  // straight-line form of `if(cell changed) move_to(iR, iz)`: every lane runs
  // it (a warp nearly always has a lane whose cell changed), so the compiler
  // can interleave it with the rest of the step; on an unchanged cell no
  // slot leaves, on the orbit's first deposit every slot is cleared and
  // nothing is parked
  __device__ __forceinline__ void add(int iR, int iz, float hdt, float fR, float fz, const Proj32 &p)
  {
    const bool first = cur < 0;
    bool out[4];
    leaving(iR, iz, out);
#pragma unroll
    for(int s = 0; s < 4; s++) out[s] = first || out[s];
    if(!first) park_masked(out);
    clear(out);
    cur = iz * Nb + iR;
    cur_iR = iR;
    cur_iz = iz;
    accumulate(iR, iz, hdt, fR, fz, p);
  }
};

// Kahan compensated summation (W. Kahan, "Further remarks on reducing
// truncation errors", CACM 8(1), 1965): adds inc to the sum s whose exact
// value is s - c; c collects what each rounding of s lost.
__device__ __forceinline__ void comp_add(float &s, float &c, float inc)
{
  const float y = inc - c;
  const float t = s + y;
  c = __fsub_rn(__fsub_rn(t, s), y);  // explicit roundings: never contracted
  s = t;
}

struct State32 {
  float x[3], v[3], a[3];
  float xc[3], vc[3];  // compensation of x and v: the exact values are x - xc, v - vc
  double tall, timespan;
  int iR, iz;
  float fR, fz, radsign_prev;
  float pend;    // weight of the deferred end-of-step deposit
  float cs_val;
  Proj32 proj;
  int norbit, flag, type, tovs, steps, status;
};

enum { LANE_ACTIVE = 0, LANE_FINISH = 1, LANE_DONE = 2, LANE_LAST = 3, LANE_START = 4 };

// orbit_response.c:172-206 in FP32: initial state of one orbit
__device__ __forceinline__ void orbit32_init(const Model32 &M, State32 &s, const double *xd, const double *vd,
                                             int type, double timespan)
{
  for(int i = 0; i < 3; i++) {
    s.x[i] = (float) xd[i];
    s.v[i] = (float) vd[i];
    s.xc[i] = (float) ((double) s.x[i] - xd[i]);
    s.vc[i] = (float) ((double) s.v[i] - vd[i]);
  }
  s.type = type;
  s.tovs = M.tovs[type];
  s.tall = 0;
  s.timespan = timespan;
  s.radsign_prev = 0.f;
  s.norbit = 0;
  s.flag = 0;
  s.steps = 0;
  s.status = ORBIT_OK;
  float vstr;
  accel32(M, type, s.x, s.a, &vstr);
  Cell32 c = density_cell32(M, s.x);
  s.iR = c.iR;
  s.iz = c.iz;
  s.fR = c.fR;
  s.fz = c.fz;
  s.proj = project32(s.tovs, s.x, s.v, vstr);
  s.cs_val = __ldg(&M.cellsize[s.iz * M.DG_Nbin + s.iR]);
  s.pend = 0.f;
}

// one KDK step with its two deposits (orbit_response.c:211-458) in FP32;
// false once the orbit has ended (time span reached, step cap, non-finite).
// The end-of-step deposit and the next step's start deposit sit at the same
// position, cell and projections, so they are made as one deposit with the
// two half-step weights added (the last one when the orbit ends).
// DEFER_LAST: the last half-step's deposit is left to the caller
// (orbit32_last), so that one call parks at most one cell's nodes.
template <class Sink, bool DEFER_LAST = false>
__device__ __forceinline__ bool orbit32_step(const Model32 &M, State32 &s, Sink &sink)
{
  // get_timestep (orbit_response.c:16-26)
  const float vv = sqrtf(s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]);
  const float aa = sqrtf(s.a[0] * s.a[0] + s.a[1] * s.a[1] + s.a[2] * s.a[2]);
  const float t1 = M.f_orb * M.V200 * frcp(aa);
  const float t2 = M.f_cc * s.cs_val * frcp(vv);
  double dt = (double) fminf(t1, t2);
  if(s.timespan < dt + s.tall) {
    dt = s.timespan - s.tall;
    s.flag = 1;
  }
  const float hdt = 0.5f * (float) dt;
  const float fdt = (float) dt;
  sink.add(s.iR, s.iz, hdt + s.pend, s.fR, s.fz, s.proj);
#pragma unroll
  for(int i = 0; i < 3; i++) comp_add(s.v[i], s.vc[i], hdt * s.a[i]);
#pragma unroll
  for(int i = 0; i < 3; i++) comp_add(s.x[i], s.xc[i], fdt * (s.v[i] - s.vc[i]));
  float vstr;
  accel32(M, s.type, s.x, s.a, &vstr);
#pragma unroll
  for(int i = 0; i < 3; i++) comp_add(s.v[i], s.vc[i], hdt * s.a[i]);
  Cell32 c = density_cell32(M, s.x);
  s.iR = c.iR;
  s.iz = c.iz;
  s.fR = c.fR;
  s.fz = c.fz;
  // DG_CellSize of the new cell for the next step's time step, loaded now
  // (every step, no branch: an L1 hit) so that its latency overlaps the rest
  // of this step
  s.cs_val = __ldg(&M.cellsize[s.iz * M.DG_Nbin + s.iR]);
  s.proj = project32(s.tovs, s.x, s.v, vstr);
  s.pend = hdt;
  s.tall += dt;
  const float radsign = s.v[0] * s.x[0] + s.v[1] * s.x[1] + s.v[2] * s.x[2];
  if(radsign > 0.f && s.radsign_prev < 0.f) s.norbit++;
  s.radsign_prev = radsign;
  s.steps++;
  if(!(s.tall == s.tall)) {
    s.status = ORBIT_NONFINITE;
    return false;
  }
  if(s.steps > M.step_cap) {
    s.status = ORBIT_STEP_CAP;
    return false;
  }
  if(!DEFER_LAST && s.flag) sink.add(s.iR, s.iz, s.pend, s.fR, s.fz, s.proj);
  return !s.flag;
}

// the deposit orbit32_step<Sink, true> left when the orbit ended normally
template <class Sink>
__device__ __forceinline__ void orbit32_last(const State32 &s, Sink &sink)
{
  sink.add(s.iR, s.iz, s.pend, s.fR, s.fz, s.proj);
}

// Particle arrays of one model
struct Particles32 {
  const double *pos, *vel, *mass, *tint;
  const int *type;
  const int *order;  // processing order
  int *orbits;
};

// Work source of one model (the context path): the model's constants are
// kernel parameters, so every access is a constant-bank operand.
struct SingleSrc {
  DevModel M64;
  Model32 M;
  Particles32 P;
  int n, first, stride;  // orbits order[first + k * stride], k < n
  int *next;
  FxWord *fx;        // [4][NG_COMMITTED][Ngrid]
  const int *shift;  // [4][NG_COMMITTED]
  unsigned long long *steps_total;
  double *max_egy_err;
  int *status;
  __device__ __forceinline__ const Model32 &model(int) const { return M; }
  __device__ __forceinline__ const DevModel &model64(int) const { return M64; }
  __device__ __forceinline__ const Particles32 &particles(int) const { return P; }
  __device__ __forceinline__ int gridset(int, int type) const { return type; }
  __device__ __forceinline__ bool take(int &mi, int &p) const
  {
    const int k = atomicAdd(next, 1);
    if(k >= n) return false;
    mi = 0;
    const int kk = first + k * stride;
    p = P.order ? P.order[kk] : kk;
    return true;
  }
  __device__ __forceinline__ void flush_stats(int, unsigned long long st, double err, int stat) const
  {
    if(st) atomicAdd(steps_total, st);
    if(err > 0) atomicMax((unsigned long long *) max_egy_err, (unsigned long long) __double_as_longlong(err));
    if(stat) atomicMax(status, stat);
  }
};

// Work source of an ensemble: orbits of all member models form one index
// space (model-major, each model in its own processing order); per-step
// constants of every model sit in the parameter space and are indexed by the
// lane's model (uniform across a warp except where two models meet).
struct EnsembleMember {
  DevModel dm;
  Particles32 part;
};

struct EnsembleSrc {
  int nmodels, total;
  int offset[GALIC_ENSEMBLE_MAX + 1];  // first orbit index of each model
  Model32 m[GALIC_ENSEMBLE_MAX];
  const EnsembleMember *mem;
  int *next;
  FxWord *fx;        // [models * 4][NG_COMMITTED][Ngrid]
  const int *shift;  // [models * 4][NG_COMMITTED]
  unsigned long long *steps;  // [models]
  double *maxerr;             // [models]
  int *status;                // [models]
  __device__ __forceinline__ const Model32 &model(int mi) const { return m[mi]; }
  __device__ __forceinline__ const DevModel &model64(int mi) const { return mem[mi].dm; }
  __device__ __forceinline__ const Particles32 &particles(int mi) const { return mem[mi].part; }
  __device__ __forceinline__ int gridset(int mi, int type) const { return 4 * mi + type; }
  __device__ __forceinline__ bool take(int &mi, int &p) const
  {
    const int k = atomicAdd(next, 1);
    if(k >= total) return false;
    int lo = 0, hi = nmodels;
    while(hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if(offset[mid] <= k)
        lo = mid;
      else
        hi = mid;
    }
    mi = lo;
    p = mem[lo].part.order[k - offset[lo]];
    return true;
  }
  __device__ __forceinline__ void flush_stats(int mi, unsigned long long st, double err, int stat) const
  {
    if(st) atomicAdd(&steps[mi], st);
    if(err > 0) atomicMax((unsigned long long *) &maxerr[mi], (unsigned long long) __double_as_longlong(err));
    if(stat) atomicMax(&status[mi], stat);
  }
};

// per-lane values used only when an orbit starts or ends (shared memory)
struct LaneAux {
  double E0;                // energy at the orbit start (orbit_response.c:203)
  double err;               // largest relative energy error of the lane's orbits of model stat_mi
  unsigned long long steps; // their orbit-steps
  int status, stat_mi, p;
};

// log(FG_Fac) for the FP64 potential of the energy check (grid.c:68-74)
__device__ __forceinline__ LogConsts pot_logs(const DevModel &M)
{
  LogConsts c;
  c.lfg = gm_log(M.FG_Fac);
  c.ldg = c.leg = 0.0;
  return c;
}

template <int BLOCK, class Src>
__device__ __forceinline__ void calc_all_fp32_body(const Src &S)
{
  constexpr int PER = queue32_per(BLOCK);
  __shared__ WarpQueue32<PER> queues[BLOCK / 32];
  // values a lane needs only when an orbit starts or ends, out of registers
  __shared__ LaneAux aux_all[BLOCK];
  LaneAux &aux = aux_all[threadIdx.x];
  aux.p = -1;
  aux.stat_mi = 0;
  aux.steps = 0;
  aux.err = 0;
  aux.status = 0;
  __syncwarp();
  const int G = S.model64(0).DG_Ngrid;
  State32 s;
  Sink32<PER> sink;
  sink.q = &queues[threadIdx.x >> 5];
  sink.lane = threadIdx.x & 31;
  sink.cur = -1;
  sink.cnt = 0;
  int mi = 0;

  auto begin = [&]() -> bool {
    int nmi, p;
    if(!S.take(nmi, p)) {
      aux.p = -1;
      return false;
    }
    aux.p = p;
    if(nmi != aux.stat_mi) {  // statistics are kept per model
      S.flush_stats(aux.stat_mi, aux.steps, aux.err, aux.status);
      aux.steps = 0;
      aux.err = 0;
      aux.status = 0;
      aux.stat_mi = nmi;
    }
    mi = nmi;
    const Model32 &M = S.model(mi);
    const Particles32 &P = S.particles(mi);
    const int type = P.type[p];
    sink.Nb = M.DG_Nbin;
    {
      const int gs = S.gridset(mi, type);
      const double fac = P.mass[p] / P.tint[p];
      sink.set_orbit(gs * NG_COMMITTED * G, (float) ldexp(fac, S.shift[gs * NG_COMMITTED + GALIC_GRID_MASS_S] - 24),
                     (float) ldexp(fac, S.shift[gs * NG_COMMITTED + GALIC_GRID_R_S] - 24));
    }
    sink.cur = -1;
    double xd[3], vd[3];
    for(int i = 0; i < 3; i++) {
      xd[i] = P.pos[3 * p + i];
      vd[i] = P.vel[3 * p + i];
    }
    orbit32_init(M, s, xd, vd, type, P.tint[p]);
    const DevModel &M64 = S.model64(mi);
    aux.E0 = 0.5 * (vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]) + forcegrid_pot(M64, pot_logs(M64), xd);
    return true;
  };

  int state = begin() ? LANE_ACTIVE : LANE_DONE;
  for(;;) {
    const bool all_done = !__any_sync(0xffffffffu, state != LANE_DONE);
    // records carry the orbit's grid set and scale only through the lane's
    // queue header, so a lane drains them before it starts the next orbit
    if(queue32_due<PER>(sink.cnt) || __any_sync(0xffffffffu, (all_done || state == LANE_START) && sink.cnt > 0))
      warp_drain32(*sink.q, S.fx, G, sink.cnt);
    if(all_done) break;
    if(state == LANE_ACTIVE) {
      if(!orbit32_step<Sink32<PER>, true>(S.model(mi), s, sink)) state = s.status == ORBIT_OK ? LANE_LAST : LANE_FINISH;
    } else if(state == LANE_LAST) {
      orbit32_last(s, sink);
      state = LANE_FINISH;
    } else if(state == LANE_FINISH) {
      sink.park();
      S.particles(mi).orbits[aux.p] = s.norbit;
      aux.steps += (unsigned long long) s.steps;
      if(s.status != ORBIT_OK)
        aux.status = max(aux.status, s.status);
      else {
        const DevModel &M64 = S.model64(mi);
        double xd[3] = {s.x[0], s.x[1], s.x[2]};
        double vd0 = s.v[0], vd1 = s.v[1], vd2 = s.v[2];
        double E1 = 0.5 * (vd0 * vd0 + vd1 * vd1 + vd2 * vd2) + forcegrid_pot(M64, pot_logs(M64), xd);
        double e = fabs((E1 - aux.E0) / aux.E0);
        if(e > aux.err) aux.err = e;
      }
      state = LANE_START;
    } else if(state == LANE_START) {
      state = begin() ? LANE_ACTIVE : LANE_DONE;
    }
  }
  S.flush_stats(aux.stat_mi, aux.steps, aux.err, aux.status);
}

__global__ void __launch_bounds__(CALC_ALL_BLOCK_FP32, GALIC_FP32_MIN_BLOCKS)
    k_calc_all_fp32(const __grid_constant__ SingleSrc S)
{
  calc_all_fp32_body<CALC_ALL_BLOCK_FP32>(S);
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_ensemble_fp32(const __grid_constant__ EnsembleSrc S)
{
  calc_all_fp32_body<BLOCK>(S);
}

// Dense sink of one orbit: the node sums of NodeAcc, added into the orbit's
// own FP64 grids [5][Ngrid] when their node leaves the current cell, as
// reductions that return nothing (the thread does not wait for the grid's
// lines; one thread's reductions to one address apply in program order, so
// the bins are those of a load-add-store).
struct DenseSink32 : NodeAcc {
  double *grid;
  int G, Nb;
  __device__ __forceinline__ void flush_nodes(const bool out[4])
  {
#pragma unroll
    for(int s = 0; s < 4; s++) {
      if(!out[s]) continue;
      const int node = (cur_iz + node_dz(s, cur_iz)) * Nb + cur_iR + node_dr(s, cur_iR);
#pragma unroll
      for(int f = 0; f < 5; f++)
        if(a[s][f] != 0.f) atomicAdd(&grid[(size_t) f * G + node], (double) a[s][f]);
    }
  }
  __device__ __forceinline__ void flush()
  {
    if(cur < 0) return;
    const bool all[4] = {true, true, true, true};
    flush_nodes(all);
    cur = -1;
  }
  __device__ __forceinline__ void add(int iR, int iz, float hdt, float fR, float fz, const Proj32 &p)
  {
    if(iz * Nb + iR != cur) {
      if(cur >= 0) {
        bool out[4];
        leaving(iR, iz, out);
        flush_nodes(out);
        clear(out);
      } else {
        const bool all[4] = {true, true, true, true};
        clear(all);
      }
      cur = iz * Nb + iR;
      cur_iR = iR;
      cur_iz = iz;
    }
    accumulate(iR, iz, hdt, fR, fz, p);
  }
};

// produce_orbit_response_field_mod (orbit_response.c:155-491) in the FP32
// form, one thread per orbit, into dense per-orbit FP64 grids (unscaled; the
// mass/tall normalisation follows in k_scale_dense)
__global__ void __launch_bounds__(128) k_orbits_dense_fp32(const __grid_constant__ Model32 M,
                                                          const __grid_constant__ DevModel M64, OrbitBatch b)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= b.count) return;
  const int G = M64.DG_Ngrid;
  DenseSink32 sink;
  sink.grid = b.grids + (size_t) k * NF_ORBIT * G;
  sink.G = G;
  sink.Nb = M.DG_Nbin;
  State32 s;
  const double *xd = &b.pos[3 * k], *vd = &b.vel[3 * k];
  orbit32_init(M, s, xd, vd, b.type[k], b.timespan[k]);
  const LogConsts L = pot_logs(M64);
  double x0[3] = {xd[0], xd[1], xd[2]};
  const double E0 = 0.5 * (vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]) + forcegrid_pot(M64, L, x0);
  while(orbit32_step(M, s, sink)) {
  }
  sink.flush();
  b.tall[k] = s.tall;
  b.norbit[k] = s.norbit;
  b.steps[k] = s.steps;
  b.status[k] = s.status;
  double err = -1.0;
  if(s.status == ORBIT_OK) {
    double x1[3] = {s.x[0], s.x[1], s.x[2]};
    const double v0 = s.v[0], v1 = s.v[1], v2 = s.v[2];
    const double E1 = 0.5 * (v0 * v0 + v1 * v1 + v2 * v2) + forcegrid_pot(M64, L, x1);
    err = fabs((E1 - E0) / E0);
  }
  b.egy_err[k] = err;
}

Model32 make_model32(const DevModel &M64, const float4 *const quad[4], const float *cellsize32)
{
  Model32 M;
  M.V200 = (float) M64.V200;
  M.f_orb = (float) M64.f_orb;
  M.f_cc = (float) M64.f_cc;
  M.invFG = (float) (1.0 / M64.FG_Rmin);
  M.ilgFG = (float) (1.0 / std::log2(M64.FG_Fac));
  M.invDG = (float) (1.0 / M64.DG_Rmin);
  M.ilgDG = (float) (1.0 / std::log2(M64.DG_Fac));
  M.GMh = (float) (M64.G * M64.Halo_Mass);
  M.Ah = (float) M64.Halo_A;
  M.eps_h = (float) (1.0e-6 * M64.Halo_A);
  M.haloscale = (float) (M64.M200 / M64.Halo_Mass);
  M.GMb = (float) (M64.G * M64.Bulge_Mass);
  M.Ab = (float) M64.Bulge_A;
  M.eps_b = (float) (1.0e-6 * M64.Bulge_A);
  M.tabulated = M64.tabulated;
  M.analytic_halo = M64.analytic_halo;
  M.analytic_bulge = M64.analytic_bulge;
  for(int t = 0; t < 4; t++) {
    M.tovs[t] = M64.tovs[t];
    M.vstream_zero[t] = M64.vstream_zero[t];
    M.quad[t] = quad[t];
  }
  M.FG_Nbin = M64.FG_Nbin;
  M.DG_Nbin = M64.DG_Nbin;
  M.fgmax = (float) (M64.FG_Nbin - 1);
  M.dgmax = (float) (M64.DG_Nbin - 1);
  M.cellsize = cellsize32;
  M.step_cap = M64.step_cap;
  return M;
}

// tile variants of the ensemble kernel: threads per CTA, CTAs per SM asked of
// the register allocator
struct Variant {
  int block, min_blocks;
};
constexpr Variant kVariants[] = {{128, 4}, {256, 2}, {128, 5}, {192, 3}, {256, 3}, {128, 3}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <int V>
void *variant_kernel()
{
  return (void *) k_ensemble_fp32<kVariants[V].block, kVariants[V].min_blocks>;
}

void *ensemble_kernel(int v)
{
  switch(v) {
    case 0: return variant_kernel<0>();
    case 1: return variant_kernel<1>();
    case 2: return variant_kernel<2>();
    case 3: return variant_kernel<3>();
    case 4: return variant_kernel<4>();
    default: return variant_kernel<5>();
  }
}

}  // namespace

int calc_all_fp32_occupancy(int block)
{
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_calc_all_fp32, block, 0);
  return blocks;
}

int launch_calc_all_fp32(const DevModel &M64, const float4 *const quad[4], const float *cellsize32,
                         const CalcAllArgs &a, int grid, int block, cudaStream_t s)
{
  SingleSrc S;
  S.M64 = M64;
  S.M = make_model32(M64, quad, cellsize32);
  S.P.pos = a.pos;
  S.P.vel = a.vel;
  S.P.mass = a.mass;
  S.P.tint = a.tint;
  S.P.type = a.type;
  S.P.order = a.order;
  S.P.orbits = a.orbits;
  S.n = a.n;
  S.first = a.first;
  S.stride = a.stride;
  S.next = a.next;
  S.fx = a.fx;
  S.shift = a.shift;
  S.steps_total = a.steps_total;
  S.max_egy_err = a.max_egy_err;
  S.status = a.status;
  k_calc_all_fp32<<<grid, block, 0, s>>>(S);
  return 1;
}

void launch_orbits_dense_fp32(const DevModel &M64, const float4 *const quad[4], const float *cellsize32,
                              const OrbitBatch &b, cudaStream_t s)
{
  if(b.count <= 0) return;
  const Model32 M = make_model32(M64, quad, cellsize32);
  k_orbits_dense_fp32<<<(b.count + 127) / 128, 128, 0, s>>>(M, M64, b);
}

int ensemble_variant_count() { return kNumVariants; }

int ensemble_variant(int v, int *block, int *min_blocks)
{
  if(v < 0 || v >= kNumVariants) return 0;
  *block = kVariants[v].block;
  *min_blocks = kVariants[v].min_blocks;
  return 1;
}

int ensemble_occupancy(int v)
{
  int blocks = 0;
  if(v < 0 || v >= kNumVariants) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, ensemble_kernel(v), kVariants[v].block, 0);
  return blocks;
}

size_t ensemble_member_bytes() { return sizeof(EnsembleMember); }

void ensemble_fill_member(void *dst, const DevModel &dm, const double *pos, const double *vel, const double *mass,
                          const double *tint, const int *type, const int *order, int *orbits)
{
  EnsembleMember m;
  m.dm = dm;
  m.part.pos = pos;
  m.part.vel = vel;
  m.part.mass = mass;
  m.part.tint = tint;
  m.part.type = type;
  m.part.order = order;
  m.part.orbits = orbits;
  std::memcpy(dst, &m, sizeof(m));
}

cudaError_t launch_ensemble_fp32(const EnsembleLaunch &L, int v, int grid, cudaStream_t s)
{
  if(L.nmodels < 1 || L.nmodels > GALIC_ENSEMBLE_MAX || v < 0 || v >= kNumVariants) return cudaErrorInvalidValue;
  EnsembleSrc S;
  S.nmodels = L.nmodels;
  S.total = L.offset[L.nmodels];
  for(int k = 0; k <= L.nmodels; k++) S.offset[k] = L.offset[k];
  for(int k = L.nmodels + 1; k <= GALIC_ENSEMBLE_MAX; k++) S.offset[k] = S.total;
  for(int k = 0; k < L.nmodels; k++) S.m[k] = make_model32(L.dm[k], L.quad[k], L.cellsize32[k]);
  S.mem = (const EnsembleMember *) L.members;
  S.next = L.next;
  S.fx = L.fx;
  S.shift = L.shift;
  S.steps = L.steps;
  S.maxerr = L.maxerr;
  S.status = L.status;
  void *args[] = {&S};
  return cudaLaunchKernel(ensemble_kernel(v), dim3(grid), dim3(kVariants[v].block), args, 0, s);
}
