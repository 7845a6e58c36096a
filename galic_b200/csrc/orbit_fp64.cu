// FP64 orbit-response kernels (built with --fmad=false).
//
//  k_orbits_dense   produce_orbit_response_field[_mod] (orbit_response.c:33-491)
//                   with reference semantics: one thread per orbit, dense
//                   per-orbit grids accumulated in the reference's order.
//  k_scale_dense    the mass/tall normalisation (orbit_response.c:475-486).
//  k_calc_all_fp64  calc_all_response_fields (main.c:151-231): persistent
//                   threads pull orbits from a work counter; deposits of
//                   consecutive steps in the same cell are merged in
//                   registers and flushed as exact fixed-point atomics into
//                   the per-type grids.
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
  __device__ __forceinline__ void operator()(const Deposit &d)
  {
    int i00 = d.iz * Nb + d.iR, i10 = d.iz * Nb + (d.iR + 1);
    int i01 = (d.iz + 1) * Nb + d.iR, i11 = (d.iz + 1) * Nb + (d.iR + 1);
    m[i00] += d.m00;
    m[i10] += d.m10;
    m[i01] += d.m01;
    m[i11] += d.m11;
    if(with_egy) {
      r[i00] += d.m00 * d.p.vr2;
      r[i10] += d.m10 * d.p.vr2;
      r[i01] += d.m01 * d.p.vr2;
      r[i11] += d.m11 * d.p.vr2;
      t[i00] += d.m00 * d.p.vt2;
      t[i10] += d.m10 * d.p.vt2;
      t[i01] += d.m01 * d.p.vt2;
      t[i11] += d.m11 * d.p.vt2;
      q[i00] += d.m00 * d.p.vq2;
      q[i10] += d.m10 * d.p.vq2;
      q[i01] += d.m01 * d.p.vq2;
      q[i11] += d.m11 * d.p.vq2;
      p[i00] += d.m00 * d.p.vp2;
      p[i10] += d.m10 * d.p.vp2;
      p[i01] += d.m01 * d.p.vp2;
      p[i11] += d.m11 * d.p.vp2;
    }
  }
};

__global__ void k_orbits_dense(DevModel M, OrbitBatch b)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= b.count) return;
  LogConsts L = make_log_consts(M);
  const size_t G = (size_t) M.DG_Ngrid;
  double *base = b.grids + (size_t) k * NF_ORBIT * G;
  DenseSink sink{base + F_M * G, base + F_R * G, base + F_T * G, base + F_Q * G, base + F_P * G, M.DG_Nbin,
                 b.with_egy};
  OrbitState s;
  orbit_begin(M, L, s, &b.pos[3 * k], &b.vel[3 * k], b.timespan[k], b.type[k], b.with_egy != 0);
  while(orbit_step(M, L, s, b.with_egy != 0, sink)) {
  }
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

// Register-merged sink of the batched path: deposits of consecutive steps in
// the same cell are summed in registers; on a cell change the 20 sums are
// scaled by mass/Tint and parked in the lane's slot of the warp queue, which
// the whole warp drains into the fixed-point grids (flush.cuh).
struct QueueSink {
  WarpQueue *q;
  int lane, type, Nb;
  double fac;  // mass / timespan
  int cur;     // merged cell iz*Nb+iR, -1 if none
  bool parked;
  double a[4][5];
  __device__ __forceinline__ void park()
  {
    if(cur < 0) return;
#pragma unroll
    for(int c = 0; c < 4; c++)
#pragma unroll
      for(int f = 0; f < 5; f++) q->val[lane][c * 5 + f] = a[c][f] * fac;
    q->cell[lane] = cur;
    q->type[lane] = type;
    parked = true;
    cur = -1;
  }
  __device__ __forceinline__ void operator()(const Deposit &d)
  {
    int c = d.iz * Nb + d.iR;
    if(c != cur) {
      park();
#pragma unroll
      for(int k = 0; k < 4; k++)
#pragma unroll
        for(int f = 0; f < 5; f++) a[k][f] = 0;
      cur = c;
    }
    const double w[4] = {d.m00, d.m10, d.m01, d.m11};
#pragma unroll
    for(int k = 0; k < 4; k++) {
      a[k][0] += w[k];
      a[k][1] += w[k] * d.p.vr2;
      a[k][2] += w[k] * d.p.vt2;
      a[k][3] += w[k] * d.p.vq2;
      a[k][4] += w[k] * d.p.vp2;
    }
  }
};

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
  // non-negative doubles order like their bit patterns
  if(!(v >= 0)) return;
  atomicMax((unsigned long long *) addr, (unsigned long long) __double_as_longlong(v));
}

enum LaneState { LANE_ACTIVE = 0, LANE_FINISH = 1, LANE_DONE = 2 };

__global__ void __launch_bounds__(CALC_ALL_BLOCK_FP64, 3) k_calc_all_fp64(DevModel M, CalcAllArgs A)
{
  __shared__ WarpQueue queues[CALC_ALL_BLOCK_FP64 / 32];
  LogConsts L = make_log_consts(M);
  const int G = M.DG_Ngrid;
  OrbitState s;
  QueueSink sink;
  sink.q = &queues[threadIdx.x >> 5];
  sink.lane = threadIdx.x & 31;
  sink.Nb = M.DG_Nbin;
  sink.cur = -1;
  sink.parked = false;
  int p = -1;
  unsigned long long my_steps = 0;
  double my_err = 0;
  int my_status = 0;

  // fetch the next orbit for this lane; returns false when none is left
  auto fetch = [&]() -> bool {
    int k = atomicAdd(A.next, 1);
    if(k >= A.n) {
      p = -1;
      return false;
    }
    k = A.first + k * A.stride;
    p = A.order ? A.order[k] : k;
    int type = A.type[p];
    sink.type = type;
    sink.fac = A.mass[p] / A.tint[p];
    sink.cur = -1;
    orbit_begin(M, L, s, &A.pos[3 * p], &A.vel[3 * p], A.tint[p], type, true);
    return true;
  };

  int state = fetch() ? LANE_ACTIVE : LANE_DONE;
  for(;;) {
    const unsigned full = __ballot_sync(0xffffffffu, sink.parked);
    if(full) {
      warp_drain(*sink.q, full, A.fx, A.shift, G, M.DG_Nbin);
      sink.parked = false;
    }
    if(!__any_sync(0xffffffffu, state != LANE_DONE)) break;
    if(state == LANE_ACTIVE) {
      if(!orbit_step(M, L, s, true, sink)) state = LANE_FINISH;
    } else if(state == LANE_FINISH) {
      sink.park();
      A.orbits[p] = s.norbit;
      my_steps += (unsigned long long) s.steps;
      if(s.status != ORBIT_OK)
        my_status = max(my_status, s.status);
      else {
        double e = orbit_energy_error(M, L, s);
        if(e > my_err) my_err = e;
      }
      state = fetch() ? LANE_ACTIVE : LANE_DONE;
    }
  }
  if(my_steps) atomicAdd(A.steps_total, my_steps);
  atomic_max_nonneg(A.max_egy_err, my_err);
  if(my_status) atomicMax(A.status, my_status);
}

// main.c:226-229 for every particle: vdisp = projections of the current
// velocity; the instantaneous energy grids get mass and mass * v^2
__global__ void k_instantaneous(DevModel M, int n, int first, int stride, const double *pos, const double *vel,
                                const double *mass, const int *type, double *vdisp, FxWord *fx, const int *shift,
                                int Ngrid)
{
  int k = first + (blockIdx.x * blockDim.x + threadIdx.x) * stride;
  if(k >= n) return;
  LogConsts L = make_log_consts(M);
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
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_calc_all_fp64, block, 0);
  return blocks;
}

int launch_calc_all_fp64(const DevModel &M, const CalcAllArgs &a, int grid, int block, cudaStream_t s)
{
  k_calc_all_fp64<<<grid, block, 0, s>>>(M, a);
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
