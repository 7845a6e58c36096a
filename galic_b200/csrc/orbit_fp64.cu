// FP64 orbit-response kernels (built with --fmad=false).
//
//  k_orbits_dense   produce_orbit_response_field[_mod] (orbit_response.c:33-491)
//                   with reference semantics: one thread per orbit, dense
//                   per-orbit grids accumulated in the reference's order.
//  k_scale_dense    the mass/tall normalisation (orbit_response.c:475-486).
//  k_calc_all_fp64  calc_all_response_fields (main.c:151-231): persistent
//                   threads pull orbits from a work counter; deposits of
//                   consecutive steps are summed per grid node in registers
//                   and flushed as exact fixed-point atomics into the
//                   per-type grids when their node leaves the orbit's cell.
//  k_instantaneous  calc_disp_components_for_particle + add_to_energy_grid
//                   (main.c:226-229).
//  k_fx_finalize    fixed-point words -> FP64 committed grids.
#include <cuda_runtime.h>

#include "flush.cuh"
#include "kernels.cuh"

namespace {

struct DenseSink {
  double *m, *r, *t, *q, *p;
  int Nb;
  int with_egy;
  // The bins of the cell the orbit is in, held in registers: c[f][corner]
  // for corners 00, 10, 01, 11.  A deposit adds to them in the reference's
  // order per bin (bin += value); when a deposit falls in another cell the
  // held bins are stored and the new cell's bins loaded (a bin two cells
  // share is stored before it is loaded again), and finish() stores the
  // last cell's.  Each orbit's grids are its own, so every bin receives the
  // reference's sequence of roundings, and the thread waits for the grid
  // only when the orbit changes cell instead of at every deposit.
  int cur = -1;  // grid index of the held cell's corner 00; -1: none
  double c[5][4];
  __device__ __forceinline__ double *field(int f) const
  {
    return f == 0 ? m : f == 1 ? r : f == 2 ? t : f == 3 ? q : p;
  }
  __device__ __forceinline__ void store_cell()
  {
    const int idx[4] = {cur, cur + 1, cur + Nb, cur + Nb + 1};
    const int nf = with_egy ? 5 : 1;
#pragma unroll
    for(int f = 0; f < 5; f++)
      if(f < nf) {
        double *g = field(f);
#pragma unroll
        for(int k = 0; k < 4; k++) g[idx[k]] = c[f][k];
      }
  }
  __device__ __forceinline__ void load_cell(int i00)
  {
    const int idx[4] = {i00, i00 + 1, i00 + Nb, i00 + Nb + 1};
    const int nf = with_egy ? 5 : 1;
#pragma unroll
    for(int f = 0; f < 5; f++)
      if(f < nf) {
        const double *g = field(f);
#pragma unroll
        for(int k = 0; k < 4; k++) c[f][k] = g[idx[k]];
      }
    cur = i00;
  }
  __device__ __forceinline__ void operator()(const Deposit &d)
  {
    const int i00 = d.iz * Nb + d.iR;
    if(i00 != cur) {
      if(cur >= 0) store_cell();
      load_cell(i00);
    }
    const double w[4] = {d.m00, d.m10, d.m01, d.m11};
#pragma unroll
    for(int k = 0; k < 4; k++) c[0][k] = c[0][k] + w[k];
    if(with_egy) {
#pragma unroll
      for(int k = 0; k < 4; k++) {
        c[1][k] = c[1][k] + w[k] * d.p.vr2;
        c[2][k] = c[2][k] + w[k] * d.p.vt2;
        c[3][k] = c[3][k] + w[k] * d.p.vq2;
        c[4][k] = c[4][k] + w[k] * d.p.vp2;
      }
    }
  }
  __device__ __forceinline__ void finish()
  {
    if(cur >= 0) store_cell();
    cur = -1;
  }
};

__global__ void k_orbits_dense(DevModel M, OrbitBatch b)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= b.count) return;
  LogConsts L = step_log_consts(M);
  const size_t G = (size_t) M.DG_Ngrid;
  double *base = b.grids + (size_t) k * NF_ORBIT * G;
  DenseSink sink{base + F_M * G, base + F_R * G, base + F_T * G, base + F_Q * G, base + F_P * G, M.DG_Nbin,
                 b.with_egy};
  OrbitState s;
  orbit_begin(M, L, s, &b.pos[3 * k], &b.vel[3 * k], b.timespan[k], b.type[k], b.with_egy != 0);
  while(orbit_step(M, L, s, b.with_egy != 0, sink)) {
  }
  sink.finish();
  b.tall[k] = s.tall;
  b.norbit[k] = s.norbit;
  b.steps[k] = s.steps;
  b.status[k] = s.status;
  b.egy_err[k] = s.status == ORBIT_OK ? orbit_energy_error(M, L, s) : -1.0;
}

// grids[k][f][i] *= mass[k] / tall[k]
__global__ void k_scale_dense(OrbitBatch b, int G)
{
  const size_t per = (size_t) NF_ORBIT * G;
  const size_t total = per * b.count;
  for(size_t idx = blockIdx.x * (size_t) blockDim.x + threadIdx.x; idx < total; idx += (size_t) gridDim.x * blockDim.x) {
    int k = (int) (idx / per);
    int f = (int) ((idx - k * per) / G);
    if(!b.with_egy && f != F_M) continue;
    double fac = b.mass[k] / b.tall[k];
    b.grids[idx] *= fac;
  }
}

// Node sink of the batched path.  The deposits of consecutive steps are
// summed per grid NODE in FP64 registers: node (z, r) lives in accumulator
// slot ((z & 1) << 1) | (r & 1), so the four nodes of any cell have the four
// parities, and when the orbit moves to a neighbouring cell the nodes the two
// cells share stay in place.  Only the slots whose node leaves are parked, as
// records {node index, 5 sums}, in the lane's column of the warp's queue; the
// warp drains all lanes' records together (flush.cuh:warp_drain_nodes_exact),
// each value scaled by mass/Tint and added as an exact two-word fixed-point
// pair (order independent).
template <int PER>
struct NodeSink64 {
  WarpQueueT<PER, double> *q;
  int lane, Nb;
  int cnt;  // records parked in this lane's column since the last drain
  int cur_iR, cur_iz;  // the current cell; cur_iz < 0: none
  double a[4][5];
  // fac x 2^(shift - 24) of the mass and the energy fields (exact scalings)
  __device__ __forceinline__ void set_orbit(int gbase, double scale_m, double scale_e)
  {
    q->gbase[lane] = gbase;
    q->scale[0][lane] = scale_m;
    q->scale[1][lane] = scale_e;
    cur_iz = -1;
  }
  // slot s of cell (iz, iR) holds node (iz + node_dz(s, iz), iR + node_dr(s, iR))
  __device__ __forceinline__ static int node_dz(int s, int iz) { return ((s >> 1) ^ iz) & 1; }
  __device__ __forceinline__ static int node_dr(int s, int iR) { return (s ^ iR) & 1; }
  __device__ __forceinline__ void park_masked(const bool out[4])
  {
    // record positions first, then predicated stores: straight-line code
    // for every lane of the warp
    bool rec[4];
    int at[4], k = cnt;
#pragma unroll
    for(int s = 0; s < 4; s++) {
      rec[s] = out[s] && a[s][0] != 0.0;  // a node without mass has no deposit at all
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
    if(cur_iz < 0) return;
    const bool all[4] = {true, true, true, true};
    park_masked(all);
    cur_iz = -1;
  }
  __device__ __forceinline__ void move_to(int iR, int iz)
  {
    bool out[4];
    if(cur_iz >= 0) {
      // along one axis a move by d leaves the node whose parity is that of
      // the boundary left behind, both nodes when |d| > 1, none when d = 0
      const int dz = iz - cur_iz, dr = iR - cur_iR;
      const int bz = (dz > 0 ? cur_iz : cur_iz + 1) & 1, br = (dr > 0 ? cur_iR : cur_iR + 1) & 1;
      const bool zall = dz > 1 || dz < -1, rall = dr > 1 || dr < -1;
#pragma unroll
      for(int s = 0; s < 4; s++)
        out[s] = (zall || (dz != 0 && (s >> 1) == bz)) || (rall || (dr != 0 && (s & 1) == br));
      park_masked(out);
    } else {
#pragma unroll
      for(int s = 0; s < 4; s++) out[s] = true;
    }
#pragma unroll
    for(int s = 0; s < 4; s++)
#pragma unroll
      for(int f = 0; f < 5; f++) a[s][f] = out[s] ? 0.0 : a[s][f];
    cur_iR = iR;
    cur_iz = iz;
  }
  __device__ __forceinline__ void operator()(const Deposit &d)
  {
    if(d.iz != cur_iz || d.iR != cur_iR) move_to(d.iR, d.iz);
    // slot s holds corner (dz, dr) = ((s >> 1) ^ (iz & 1), (s & 1) ^ (iR & 1));
    // corner weights: (0,0) m00, (0,1) m10, (1,0) m01, (1,1) m11
    const bool oz = d.iz & 1, orr = d.iR & 1;
    const double z0r0 = oz ? d.m01 : d.m00, z0r1 = oz ? d.m11 : d.m10;  // slot z-parity 0: dz = oz
    const double z1r0 = oz ? d.m00 : d.m01, z1r1 = oz ? d.m10 : d.m11;
    const double w[4] = {orr ? z0r1 : z0r0, orr ? z0r0 : z0r1, orr ? z1r1 : z1r0, orr ? z1r0 : z1r1};
    // the node sums are this form's own partial sums (the reference adds
    // every product to the grid bin in turn): fused, one rounding per term
#pragma unroll
    for(int k = 0; k < 4; k++) {
      a[k][0] += w[k];
      a[k][1] = fma(w[k], d.p.vr2, a[k][1]);
      a[k][2] = fma(w[k], d.p.vt2, a[k][2]);
      a[k][3] = fma(w[k], d.p.vq2, a[k][3]);
      a[k][4] = fma(w[k], d.p.vp2, a[k][4]);
    }
  }
};

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
  // non-negative doubles order like their bit patterns
  if(!(v >= 0)) return;
  atomicMax((unsigned long long *) addr, (unsigned long long) __double_as_longlong(v));
}

enum LaneState { LANE_ACTIVE = 0, LANE_FINISH = 1, LANE_DONE = 2, LANE_START = 3 };

// records per lane of the FP64 queue (FP64 sums: 40 B per record and lane)
constexpr int kPer64 = 8;

template <int MINB>
__global__ void __launch_bounds__(CALC_ALL_BLOCK_FP64, MINB) k_calc_all_fp64(DevModel M, CalcAllArgs A)
{
  __shared__ WarpQueueT<kPer64, double> queues[CALC_ALL_BLOCK_FP64 / 32];
  // the CTA's step count, largest energy error (as bits: non-negative
  // doubles order like them) and worst status, added to at each orbit's end
  // instead of being held in every thread's registers
  __shared__ unsigned long long cta_steps, cta_err_bits;
  __shared__ int cta_status;
  if(threadIdx.x == 0) {
    cta_steps = 0;
    cta_err_bits = 0;
    cta_status = 0;
  }
  __syncthreads();
  LogConsts L = step_log_consts(M);
  const int G = M.DG_Ngrid;
  OrbitState s;
  NodeSink64<kPer64> sink;
  sink.q = &queues[threadIdx.x >> 5];
  sink.lane = threadIdx.x & 31;
  sink.Nb = M.DG_Nbin;
  sink.cur_iz = -1;
  sink.cnt = 0;
  int p = -1;

  // fetch the next orbit for this lane; returns false when none is left
  auto fetch = [&]() -> bool {
    int k = atomicAdd(A.next, 1);
    if(k >= A.n) {
      p = -1;
      return false;
    }
    k = A.first + k * A.stride;
    p = A.order ? A.order[k] : k;
    const int type = A.type[p];
    const double fac = A.mass[p] / A.tint[p];
    sink.set_orbit(type * NG_COMMITTED * G, ldexp(fac, A.shift[type * NG_COMMITTED + GALIC_GRID_MASS_S] - 24),
                   ldexp(fac, A.shift[type * NG_COMMITTED + GALIC_GRID_R_S] - 24));
    orbit_begin(M, L, s, &A.pos[3 * p], &A.vel[3 * p], A.tint[p], type, true);
    return true;
  };

  int state = fetch() ? LANE_ACTIVE : LANE_DONE;
  for(;;) {
    const bool all_done = !__any_sync(0xffffffffu, state != LANE_DONE);
    // records take the orbit's grid set and scale from the lane's queue
    // header: a lane's records are drained before it starts the next orbit
    if(queue32_due<kPer64>(sink.cnt) ||
       __any_sync(0xffffffffu, (all_done || state == LANE_START) && sink.cnt > 0))
      warp_drain_nodes_exact(*sink.q, A.fx, G, sink.cnt);
    if(all_done) break;
    if(state == LANE_ACTIVE) {
      if(!orbit_step(M, L, s, true, sink)) state = LANE_FINISH;
    } else if(state == LANE_FINISH) {
      sink.park();
      A.orbits[p] = s.norbit;
      atomicAdd(&cta_steps, (unsigned long long) s.steps);
      if(s.status != ORBIT_OK)
        atomicMax(&cta_status, s.status);
      else {
        const double e = orbit_energy_error_from(M, L, s, &A.pos[3 * p], &A.vel[3 * p]);
        if(e >= 0) atomicMax(&cta_err_bits, (unsigned long long) __double_as_longlong(e));
      }
      state = LANE_START;
    } else if(state == LANE_START) {
      state = fetch() ? LANE_ACTIVE : LANE_DONE;
    }
  }
  __syncthreads();
  if(threadIdx.x == 0) {
    if(cta_steps) atomicAdd(A.steps_total, cta_steps);
    atomic_max_nonneg(A.max_egy_err, __longlong_as_double((long long) cta_err_bits));
    if(cta_status) atomicMax(A.status, cta_status);
  }
}

// main.c:226-229 for every particle: vdisp = projections of the current
// velocity; the instantaneous energy grids get mass and mass * v^2
__global__ void k_instantaneous(DevModel M, int n, int first, int stride, const double *pos, const double *vel,
                                const double *mass, const int *type, double *vdisp, FxWord *fx, const int *shift,
                                int Ngrid)
{
  int k = first + (blockIdx.x * blockDim.x + threadIdx.x) * stride;
  if(k >= n) return;
  LogConsts L = step_log_consts(M);
  int t = type[k];
  double d[4];
  disp_components(M, L, t, &pos[3 * k], &vel[3 * k], d);
  for(int j = 0; j < 4; j++) vdisp[4 * k + j] = d[j];
  // add_to_energy_grid (main.c:877-917)
  Cell c = energy_cell(M, L, &pos[3 * k]);
  const int Nb = 1 << M.EG_L;
  double m = mass[k];
  double vr2 = d[0] * m, vt2 = d[1] * m, vp2 = d[2] * m, vq2 = d[3] * m;
  const int cells[4] = {c.iz * Nb + c.iR, c.iz * Nb + c.iR + 1, (c.iz + 1) * Nb + c.iR, (c.iz + 1) * Nb + c.iR + 1};
  const double w[4] = {(1 - c.fR) * (1 - c.fz), (c.fR) * (1 - c.fz), (1 - c.fR) * (c.fz), (c.fR) * (c.fz)};
  FxWord *g = fx + (size_t) t * NG_COMMITTED * Ngrid;
  const int *sh = shift + t * NG_COMMITTED;
  for(int j = 0; j < 4; j++) {
    fx_add(&g[(size_t) GALIC_GRID_MASS_I * Ngrid + cells[j]], w[j] * m, sh[GALIC_GRID_MASS_I]);
    fx_add(&g[(size_t) GALIC_GRID_R_I * Ngrid + cells[j]], w[j] * vr2, sh[GALIC_GRID_R_I]);
    fx_add(&g[(size_t) GALIC_GRID_T_I * Ngrid + cells[j]], w[j] * vt2, sh[GALIC_GRID_T_I]);
    fx_add(&g[(size_t) GALIC_GRID_P_I * Ngrid + cells[j]], w[j] * vp2, sh[GALIC_GRID_P_I]);
    fx_add(&g[(size_t) GALIC_GRID_Q_I * Ngrid + cells[j]], w[j] * vq2, sh[GALIC_GRID_Q_I]);
  }
}

__global__ void k_fx_finalize(const FxWord *fx, const int *shift, double *out, int count, int Ngrid)
{
  size_t total = (size_t) count * Ngrid;
  for(size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < total; i += (size_t) gridDim.x * blockDim.x) {
    int g = (int) (i / Ngrid);
    out[i] = fx_value(fx[i], shift[g]);
  }
}

}  // namespace

void launch_orbits_dense(const DevModel &M, const OrbitBatch &b, cudaStream_t s)
{
  int block = 64;
  int grid = (b.count + block - 1) / block;
  if(grid > 0) k_orbits_dense<<<grid, block, 0, s>>>(M, b);
}

void launch_scale_dense(const DevModel &M, const OrbitBatch &b, cudaStream_t s)
{
  size_t total = (size_t) NF_ORBIT * M.DG_Ngrid * b.count;
  int grid = (int) ((total + 255) / 256);
  if(grid > 148 * 16) grid = 148 * 16;
  if(grid > 0) k_scale_dense<<<grid, 256, 0, s>>>(b, M.DG_Ngrid);
}

int calc_all_occupancy(int block)
{
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_calc_all_fp64<GALIC_FP64_MIN_BLOCKS>, block, 0);
  return blocks;
}

int launch_calc_all_fp64(const DevModel &M, const CalcAllArgs &a, int grid, int block, cudaStream_t s)
{
  k_calc_all_fp64<GALIC_FP64_MIN_BLOCKS><<<grid, block, 0, s>>>(M, a);
  return 1;
}

void launch_instantaneous(const DevModel &M, int n, const double *pos, const double *vel, const double *mass,
                          const int *type, double *vdisp, FxWord *fx, const int *shift, int Ngrid, cudaStream_t s,
                          int first, int stride)
{
  if(n <= first || stride < 1) return;
  const int count = (n - first + stride - 1) / stride;
  k_instantaneous<<<(count + 127) / 128, 128, 0, s>>>(M, n, first, stride, pos, vel, mass, type, vdisp, fx, shift,
                                                      Ngrid);
}

void launch_fx_finalize(const FxWord *fx, const int *shift, double *committed, int count, int Ngrid, cudaStream_t s)
{
  size_t total = (size_t) count * Ngrid;
  int grid = (int) ((total + 255) / 256);
  if(grid > 148 * 8) grid = 148 * 8;
  k_fx_finalize<<<grid, 256, 0, s>>>(fx, shift, committed, count, Ngrid);
}
