// galic_orbit_responses_noalloc: the batched FP64 orbit-response binning of
// galic_calc_all_response_fields (main.c:151-223) for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside a host framework
// that owns every device allocation through its own pool, or a host process
// whose device-memory budget is fixed before the solver starts.  This entry
// point takes only caller-owned device buffers for its inputs and outputs and
// allocates nothing.  Its working memory (the exact fixed-point bin
// accumulators and two counters) is the file-scope array g_noalloc_scratch
// below: a fixed 3.75 MiB + 256 B per device, resident on every GPU that
// loads the library until the process exits.  The sizes it accepts are
// limited by that array: at most three particle types and DG_MaxLevel <= 7
// (16384 bins per grid); larger requests are rejected with GALIC_ERR_BUDGET.
//
// The array's name is only a host-side stand-in in host code.  Its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call made on the device; make that first call
// before any stream capture.  The cached address belongs to the device's
// context: after cudaDeviceReset it is stale, and the library must be
// reloaded.  All calls share the one array and leave the last call's
// contents in it; each call clears the accumulators and counters it uses
// before its kernel runs.  Calls whose work overlaps on the GPU (other
// streams, other host threads) race on the array and must be serialised by
// the caller.
//
// Particles are checked on the device before their orbit starts (a type
// outside 1..3, a non-positive or non-finite Tint or a non-finite mass):
// such a particle is skipped, deposits nothing, and the call returns
// GALIC_ERR_INVALID_ARGUMENT.  Step counts and energy errors are not
// returned; the context path reports them.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "kernels.cuh"

namespace {

constexpr int kTypes = 3;        // particle types 1..3
constexpr int kFields = NF_ORBIT;  // m, r, t, q, p
constexpr int kMaxGrid = 16384;  // DG_MaxLevel <= 7

// status words beyond OrbitStatus (the worst code seen wins)
enum { NOALLOC_OVERFLOW = 3, NOALLOC_INVALID = 4 };

struct NoAllocScratch {
  FxWord fx[kTypes * kFields * kMaxGrid];
  int next;
  int status;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

struct Shifts {
  int s[kTypes * kFields];
};

struct NoAllocArgs {
  int n;
  const double *pos, *vel, *mass, *tint;
  const int *type;
  int *orbits;
  NoAllocScratch *scratch;
  Shifts shift;
};

struct Slots {
  double val[32][20];
  int cell[32];
  int type[32];
  int list[32];
};

struct ParkSink {
  Slots *q;
  int lane, type, Nb;
  double fac;
  int cur;
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

__device__ __forceinline__ void drain(Slots &q, unsigned full, const NoAllocArgs &A, int G, int Nb)
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
    const int t = q.type[s] - 1;
    fx_add(&A.scratch->fx[((size_t) t * kFields + f) * G + q.cell[s] + off], q.val[s][k],
           A.shift.s[t * kFields + f]);
  }
  __syncwarp();
}

enum { ST_ACTIVE = 0, ST_FINISH = 1, ST_DONE = 2 };

__global__ void __launch_bounds__(128, 3) k_noalloc_orbits(DevModel M, NoAllocArgs A)
{
  __shared__ Slots queues[4];
  LogConsts L = step_log_consts(M);
  const int G = M.DG_Ngrid;
  OrbitState s;
  ParkSink sink;
  sink.q = &queues[threadIdx.x >> 5];
  sink.lane = threadIdx.x & 31;
  sink.Nb = M.DG_Nbin;
  sink.cur = -1;
  sink.parked = false;
  int p = -1;
  int my_status = 0;
  auto fetch = [&]() -> bool {
    for(;;) {
      const int k = atomicAdd(&A.scratch->next, 1);
      if(k >= A.n) return false;
      // an invalid particle would index outside the grids (type) or never
      // reach its time span (Tint): skip it and report it
      const int t = A.type[k];
      const double tint = A.tint[k], mass = A.mass[k];
      if(t >= 1 && t <= kTypes && tint > 0 && tint <= 1.0e300 && mass == mass && fabs(mass) <= 1.0e300) {
        p = k;
        break;
      }
      if(A.orbits) A.orbits[k] = 0;
      my_status = NOALLOC_INVALID;
    }
    sink.type = A.type[p];
    sink.fac = A.mass[p] / A.tint[p];
    sink.cur = -1;
    orbit_begin(M, L, s, &A.pos[3 * p], &A.vel[3 * p], A.tint[p], sink.type, true);
    return true;
  };
  int state = fetch() ? ST_ACTIVE : ST_DONE;
  for(;;) {
    const unsigned full = __ballot_sync(0xffffffffu, sink.parked);
    if(full) {
      drain(*sink.q, full, A, G, M.DG_Nbin);
      sink.parked = false;
    }
    if(!__any_sync(0xffffffffu, state != ST_DONE)) break;
    if(state == ST_ACTIVE) {
      if(!orbit_step(M, L, s, true, sink)) state = ST_FINISH;
    } else if(state == ST_FINISH) {
      sink.park();
      if(A.orbits) A.orbits[p] = s.norbit;
      if(s.status != ORBIT_OK) my_status = max(my_status, s.status);
      state = fetch() ? ST_ACTIVE : ST_DONE;
    }
  }
  if(my_status) atomicMax(&A.scratch->status, my_status);
}

// fixed-point words -> FP64 grids; a high word beyond 2^62 means the bins
// came close to the word's range (a phi_bound below max|FG_Pot|)
__global__ void k_noalloc_finalize(NoAllocScratch *sc, Shifts sh, double *out, int G)
{
  const size_t total = (size_t) kTypes * kFields * G;
  bool over = false;
  for(size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < total; i += (size_t) gridDim.x * blockDim.x) {
    const FxWord w = sc->fx[i];
    const long long h = (long long) w.hi;
    over |= h > (1LL << 62) || h < -(1LL << 62);
    out[i] = fx_value(w, sh.s[i / G]);
  }
  if(over) atomicMax(&sc->status, (int) NOALLOC_OVERFLOW);
}

std::mutex g_setup_mutex;
NoAllocScratch *g_scratch_ptr[64] = {nullptr};

int shift_for(double bound)
{
  if(!(bound > 0) || !std::isfinite(bound)) bound = 1.0;
  return 84 - (int) std::ceil(std::log2(bound));
}

}  // namespace

extern "C" int galic_orbit_responses_noalloc(const galic_params_t *prm, const double *d_fg_acc2,
                                             const double *d_fg_pot, const double *d_vstream,
                                             const double *d_cellsize, double phi_bound, int n,
                                             const double *d_pos, const double *d_vel, const double *d_mass,
                                             const double *d_tint, const int *d_type, double *d_out, int *d_orbits,
                                             void *stream)
{
  if(!prm || !d_fg_acc2 || !d_fg_pot || !d_vstream || !d_cellsize || !d_out || n < 0 ||
     (n > 0 && (!d_pos || !d_vel || !d_mass || !d_tint || !d_type)) || !(std::fabs(phi_bound) <= 1.0e300))
    return GALIC_ERR_INVALID_ARGUMENT;
  if(prm->DG_MaxLevel != prm->EG_MaxLevel || prm->DG_MaxLevel < 1 || prm->FG_Nbin < 2 || !(prm->Halo_Mass > 0))
    return GALIC_ERR_INVALID_ARGUMENT;
  if(!(prm->FG_Rmin > 0) || !(prm->FG_Fac > 1) || !(prm->DG_Rmin > 0) || !(prm->DG_Fac > 1) || !(prm->EG_Rmin > 0) ||
     !(prm->EG_Fac > 1))
    return GALIC_ERR_INVALID_ARGUMENT;
  const int L = prm->DG_MaxLevel;
  if(L > 7) return GALIC_ERR_BUDGET;  // 4^L bins per grid must fit the fixed scratch array
  const int G = 1 << (2 * L);
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GALIC_ERR_NO_DEVICE;
  NoAllocScratch *sc;
  {
    // once per device, with that device current: device address of the array
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if(!g_scratch_ptr[dev]) {
      void *p = nullptr;
      if(cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GALIC_ERR_CUDA;
      g_scratch_ptr[dev] = (NoAllocScratch *) p;
    }
    sc = g_scratch_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t) stream;
  DevModel M{};
  M.V200 = prm->V200;
  M.M200 = prm->M200;
  M.R200 = prm->R200;
  M.G = prm->G;
  M.Halo_Mass = prm->Halo_Mass;
  M.Halo_A = prm->Halo_A;
  M.Bulge_Mass = prm->Bulge_Mass;
  M.Bulge_A = prm->Bulge_A;
  M.f_orb = prm->TimeStepFactorOrbit;
  M.f_cc = prm->TimeStepFactorCellCross;
  M.LowerDispLimit = prm->LowerDispLimit;
  M.MaxVelInUnitsVesc = prm->MaxVelInUnitsVesc;
  M.tabulated = (prm->Disk_Mass > 0 || (prm->Halo_Mass > 0 && prm->SampleForceNhalo > 0) ||
                 (prm->Bulge_Mass > 0 && prm->SampleForceNbulge > 0))
                    ? 1
                    : 0;
  M.analytic_halo = (prm->Halo_Mass > 0 && prm->SampleForceNhalo == 0) ? 1 : 0;
  M.analytic_bulge = (prm->Bulge_Mass > 0 && prm->SampleForceNbulge == 0) ? 1 : 0;
  const size_t NF = (size_t) prm->FG_Nbin * prm->FG_Nbin;
  for(int t = 0; t < 4; t++) {
    M.tovs[t] = prm->TypeOfVelocityStructure[t];
    M.vstream_zero[t] = 0;
    M.vstream[t] = t >= 1 ? d_vstream + (t - 1) * NF : d_vstream;
  }
  M.FG_Nbin = prm->FG_Nbin;
  M.DG_Nbin = 1 << L;
  M.DG_L = L;
  M.EG_L = prm->EG_MaxLevel;
  M.DG_Ngrid = G;
  M.DG_Nstack = ((1 << (2 + 2 * L)) - 1) / 3;
  M.FG_Rmin = prm->FG_Rmin;
  M.FG_Fac = prm->FG_Fac;
  M.DG_Rmin = prm->DG_Rmin;
  M.DG_Fac = prm->DG_Fac;
  M.EG_Rmin = prm->EG_Rmin;
  M.EG_Fac = prm->EG_Fac;
  set_step_constants(M);
  M.fg_acc = (const double2 *) d_fg_acc2;
  M.fg_pot = d_fg_pot;
  M.cellsize = d_cellsize;
  M.step_cap = GALIC_STEP_CAP;

  NoAllocArgs A;
  A.n = n;
  A.pos = d_pos;
  A.vel = d_vel;
  A.mass = d_mass;
  A.tint = d_tint;
  A.type = d_type;
  A.orbits = d_orbits;
  A.scratch = sc;
  // same bounds as the context path: |phi| <= phi_bound + G M200 / a (+ bulge)
  double phi = std::fabs(phi_bound) + prm->G * prm->M200 / prm->Halo_A;
  if(prm->Bulge_Mass > 0 && prm->Bulge_A > 0) phi += prm->G * prm->Bulge_Mass / prm->Bulge_A;
  for(int t = 0; t < kTypes; t++) {
    double bm = prm->MType[t + 1] > 1e-300 ? prm->MType[t + 1] : 1e-300;
    for(int f = 0; f < kFields; f++) A.shift.s[t * kFields + f] = shift_for(f == 0 ? 2.0 * bm : bm * 2.0 * phi * 16.0);
  }
  // clear what must start at zero: the accumulators of this size and the counters
  if(cudaMemsetAsync(sc->fx, 0, (size_t) kTypes * kFields * G * sizeof(FxWord), s) != cudaSuccess ||
     cudaMemsetAsync(&sc->next, 0, sizeof(int) + sizeof(int), s) != cudaSuccess)
    return GALIC_ERR_CUDA;
  int sms = 0;
  if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  if(n > 0) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_noalloc_orbits, 128, 0);
    int grid = (per_sm > 0 ? per_sm : 1) * sms;
    int need = (n + 127) / 128;
    if(grid > need) grid = need;
    k_noalloc_orbits<<<grid, 128, 0, s>>>(M, A);
  }
  k_noalloc_finalize<<<sms * 4, 256, 0, s>>>(sc, A.shift, d_out, G);
  int status = 0;
  if(cudaGetLastError() != cudaSuccess) return GALIC_ERR_CUDA;
  if(cudaMemcpyAsync(&status, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
     cudaStreamSynchronize(s) != cudaSuccess)
    return GALIC_ERR_CUDA;
  if(status == NOALLOC_INVALID || status == ORBIT_NONFINITE) return GALIC_ERR_INVALID_ARGUMENT;
  if(status == NOALLOC_OVERFLOW) return GALIC_ERR_OVERFLOW;
  if(status == ORBIT_STEP_CAP) return GALIC_ERR_STEP_CAP;
  return GALIC_OK;
}
