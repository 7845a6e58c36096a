// C ABI of libgalic_cuda.so (include/galic_gpu.h): the context that replaces
// GALIC's globals, uploads, and the entry points that replace the reference
// functions.  Host code only; the kernels live in orbit_fp64.cu and
// fit_fp64.cu.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "context.cuh"
#include "galic_gpu.h"
#include "kernels.cuh"
#include "rep.cuh"


namespace {

const char *kStatusText[] = {"ok",
                             "invalid argument",
                             "an orbit exceeded the step cap",
                             "CUDA runtime error",
                             "no CUDA device",
                             "request exceeds the HBM budget",
                             "configuration not supported",
                             "rejection loop exceeded its cap (velocity proposal: 100000 tries; sampling: nothing lands inside Rmax)",
                             "fixed-point response bin out of range",
                             "call out of order"};

int fail(galic_ctx *c, int st)
{
  if(c) c->status = st;
  return st;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if(e_ != cudaSuccess) {                                                                       \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                          \
      return fail(ctx, GALIC_ERR_CUDA);                                                           \
    }                                                                                             \
  } while(0)

// Device memory of a context comes from the device's stream-ordered pool
// and is allocated and released in the context's stream: a context that
// starts or ends does not synchronise the device, so contexts driven from
// different host threads (the serving loop) do not stall one another.
template <class T>
cudaError_t dalloc(galic_ctx *ctx, T **p, size_t count)
{
  return cudaMallocAsync((void **) p, std::max<size_t>(count, 1) * sizeof(T), ctx->stream);
}

template <class T>
void dfree(galic_ctx *ctx, T *&p)
{
  if(p) cudaFreeAsync((void *) p, ctx->stream);
  p = nullptr;
}

// keep freed pool memory mapped (the default pool would return it to the
// driver at every synchronisation); process-local, once per device
cudaError_t keep_pool_memory(int device)
{
  static std::mutex mu;
  static bool done[256] = {false};
  std::lock_guard<std::mutex> lk(mu);
  if(device < 0 || device >= 256 || done[device]) return cudaSuccess;
  cudaMemPool_t pool;
  cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, device);
  if(e != cudaSuccess) return e;
  uint64_t threshold = UINT64_MAX;
  e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  if(e == cudaSuccess) done[device] = true;
  return e;
}

int stack_size(int L) { return ((1 << (2 + 2 * L)) - 1) / 3; }

// pinned staging area of at least `bytes` (null on failure)
char *stage(galic_ctx *ctx, size_t bytes)
{
  if(bytes <= ctx->stage_cap) return ctx->h_stage;
  if(ctx->h_stage) {
    cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(ctx->h_stage);
  }
  ctx->h_stage = nullptr;
  ctx->stage_cap = 0;
  const size_t cap = std::max<size_t>(bytes, 4096);
  if(cudaMallocHost((void **) &ctx->h_stage, cap) != cudaSuccess) return nullptr;
  ctx->stage_cap = cap;
  return ctx->h_stage;
}

int check_params(const galic_params_t *p)
{
  if(!p) return GALIC_ERR_INVALID_ARGUMENT;
  if(p->FG_Nbin < 2 || p->DG_MaxLevel < 1 || p->EG_MaxLevel < 1) return GALIC_ERR_INVALID_ARGUMENT;
  // eval_fit_mod indexes energy stacks with DG_MaxLevel (main.c:1056) and the
  // stacks are kept in one CTA's shared memory
  if(p->DG_MaxLevel != p->EG_MaxLevel || p->DG_MaxLevel > 7) return GALIC_ERR_UNSUPPORTED;
  if(!(p->FG_Rmin > 0) || !(p->FG_Fac > 1) || !(p->DG_Rmin > 0) || !(p->DG_Fac > 1) || !(p->EG_Rmin > 0) ||
     !(p->EG_Fac > 1))
    return GALIC_ERR_INVALID_ARGUMENT;
  for(int t = 1; t <= 3; t++)
    if(p->TypeOfVelocityStructure[t] < 0 || p->TypeOfVelocityStructure[t] > 3) return GALIC_ERR_INVALID_ARGUMENT;
  // grid.c:96-97 and 174-175: analytic components must be spherical
  if(p->Halo_Mass > 0 && p->SampleForceNhalo == 0 && p->HaloStretch != 1.0) return GALIC_ERR_UNSUPPORTED;
  if(p->Bulge_Mass > 0 && p->SampleForceNbulge == 0 && p->BulgeStretch != 1.0) return GALIC_ERR_UNSUPPORTED;
  if(!(p->Halo_Mass > 0)) return GALIC_ERR_UNSUPPORTED;  // off-grid fallback divides by Halo_Mass
  return GALIC_OK;
}

int ensure_orbit_scratch(galic_ctx *ctx, int count)
{
  if(count <= ctx->scratch_orbits) return GALIC_OK;
  dfree(ctx, ctx->d_b_pos); dfree(ctx, ctx->d_b_vel); dfree(ctx, ctx->d_b_mass); dfree(ctx, ctx->d_b_time); dfree(ctx, ctx->d_grids);
  dfree(ctx, ctx->d_b_tall); dfree(ctx, ctx->d_b_err); dfree(ctx, ctx->d_b_type); dfree(ctx, ctx->d_b_norbit); dfree(ctx, ctx->d_b_status);
  dfree(ctx, ctx->d_b_steps);
  CK(dalloc(ctx, &ctx->d_b_pos, 3 * (size_t) count));
  CK(dalloc(ctx, &ctx->d_b_vel, 3 * (size_t) count));
  CK(dalloc(ctx, &ctx->d_b_mass, count));
  CK(dalloc(ctx, &ctx->d_b_time, count));
  CK(dalloc(ctx, &ctx->d_grids, (size_t) count * NF_ORBIT * ctx->G));
  CK(dalloc(ctx, &ctx->d_b_tall, count));
  CK(dalloc(ctx, &ctx->d_b_err, count));
  CK(dalloc(ctx, &ctx->d_b_type, count));
  CK(dalloc(ctx, &ctx->d_b_norbit, count));
  CK(dalloc(ctx, &ctx->d_b_status, count));
  CK(dalloc(ctx, &ctx->d_b_steps, count));
  ctx->scratch_orbits = count;
  return GALIC_OK;
}

int ensure_rep_scratch(galic_ctx *ctx, int count)
{
  int st = ensure_orbit_scratch(ctx, 2 * count);
  if(st) return st;
  if(count <= ctx->scratch_rep) return GALIC_OK;
  dfree(ctx, ctx->d_idx); dfree(ctx, ctx->d_accepted); dfree(ctx, ctx->d_vel_try); dfree(ctx, ctx->d_F); dfree(ctx, ctx->d_inst_v);
  dfree(ctx, ctx->d_inst_cell); dfree(ctx, ctx->d_acc_list); dfree(ctx, ctx->d_acc_n); dfree(ctx, ctx->d_fac);
  CK(dalloc(ctx, &ctx->d_idx, count));
  CK(dalloc(ctx, &ctx->d_acc_list, count));
  CK(dalloc(ctx, &ctx->d_acc_n, count));  // one per repetition: at most count repetitions per window
  if(!ctx->d_inst0) CK(dalloc(ctx, &ctx->d_inst0, 16));
  CK(dalloc(ctx, &ctx->d_accepted, count));
  CK(dalloc(ctx, &ctx->d_vel_try, 3 * (size_t) count));
  CK(dalloc(ctx, &ctx->d_F, 2 * 9 * (size_t) count));  // 9 merit terms per evaluation
  CK(dalloc(ctx, &ctx->d_fac, 2 * (size_t) count));
  CK(dalloc(ctx, &ctx->d_inst_v, 4 * (size_t) count));
  CK(dalloc(ctx, &ctx->d_inst_cell, count));
  ctx->scratch_rep = count;
  return GALIC_OK;
}

}  // namespace

namespace galic_internal {

FitArgs make_fit_args(galic_ctx *ctx)
{
  FitArgs f;
  const galic_params_t &p = ctx->prm;
  f.L = ctx->L;
  f.Ngrid = ctx->G;
  f.Nstack = ctx->Ns;
  f.committed = ctx->d_committed;
  f.stacks = ctx->d_stacks;
  f.targets = ctx->d_targets;
  f.dgs_distance = ctx->d_dist;
  f.fit = ctx->d_fit;
  f.firstrun = ctx->d_firstrun;
  for(int t = 0; t < 4; t++) {
    // main.c:296 / 313: MinParticles * MType / NType, left to right
    f.thr_d[t] = p.NType[t] ? p.MinParticlesPerBinForDensityMeasurement * p.MType[t] / p.NType[t] : 0;
    f.thr_e[t] = p.NType[t] ? p.MinParticlesPerBinForDispersionMeasurement * p.MType[t] / p.NType[t] : 0;
    f.MType[t] = p.MType[t];
    f.present[t] = (t >= 1 && p.NType[t] > 0) ? 1 : 0;
    f.tovs[t] = p.TypeOfVelocityStructure[t];
  }
  f.R200_20 = p.R200 / 20.0;
  f.LowerDispLimit = p.LowerDispLimit;
  return f;
}

int fixed_point_shift(double bound)
{
  if(!(bound > 0) || !std::isfinite(bound)) bound = 1.0;
  int e = (int) std::ceil(std::log2(bound));
  return 84 - e;
}

// form: two-word exact words (FP64 form) or one signed word (FP32 form,
// flush.cuh:warp_drain_nodes); both keep every bin total inside the word's range
void set_shifts(galic_ctx *ctx, int *shift, int form)
{
  const galic_params_t &p = ctx->prm;
  // |potential| bound: tabulated part plus the analytic halo and bulge
  double phi = std::fabs(ctx->pot_min) + p.G * p.M200 / p.Halo_A;
  if(p.Bulge_Mass > 0 && p.Bulge_A > 0) phi += p.G * p.Bulge_Mass / p.Bulge_A;
  for(int t = 0; t < 4; t++) {
    double bm = std::max(p.MType[t], 1e-300);
    double be = bm * 2.0 * phi * 16.0;  // v^2 <= 2|phi| with a factor 16 headroom
    for(int g = 0; g < NG_COMMITTED; g++) {
      bool mass = (g == GALIC_GRID_MASS_S || g == GALIC_GRID_MASS_I);
      shift[t * NG_COMMITTED + g] = fixed_point_shift(mass ? 2.0 * bm : be) + (form == GALIC_FORM_FP32 ? 2 : 0);
    }
  }
}

// float4 tables of the FP32 form, rebuilt after any table upload
int ensure_tab32(galic_ctx *ctx)
{
  if(!ctx->tab32_dirty) return GALIC_OK;
  const int NF = ctx->prm.FG_Nbin * ctx->prm.FG_Nbin;
  if(ctx->h_dpotdr.size() != (size_t) NF) {
    ctx->h_dpotdr.assign(NF, 0.0);
    ctx->h_dpotdz.assign(NF, 0.0);
  }
  const int N = ctx->prm.FG_Nbin;
  std::vector<float4> tab(4 * (size_t) NF, make_float4(0.f, 0.f, 0.f, 0.f));
  for(int t = 1; t <= 3; t++) {
    if(!ctx->d_tab32[t]) CK(dalloc(ctx, &ctx->d_tab32[t], 4 * (size_t) NF));
    const bool hv = ctx->h_vstream[t].size() == (size_t) NF;
    for(int iz = 0; iz + 1 < N; iz++)
      for(int iR = 0; iR + 1 < N; iR++) {
        const int c[4] = {iz * N + iR, iz * N + iR + 1, (iz + 1) * N + iR, (iz + 1) * N + iR + 1};
        float r[4], z[4], v[4];
        for(int k = 0; k < 4; k++) {
          r[k] = (float) ctx->h_dpotdr[c[k]];
          z[k] = (float) ctx->h_dpotdz[c[k]];
          v[k] = hv ? (float) ctx->h_vstream[t][c[k]] : 0.f;
        }
        float4 *e = &tab[4 * (size_t) (iz * N + iR)];
        e[0] = make_float4(r[0], r[1], r[2], r[3]);
        e[1] = make_float4(z[0], z[1], z[2], z[3]);
        e[2] = make_float4(v[0], v[1], v[2], v[3]);
      }
    CK(cudaMemcpyAsync(ctx->d_tab32[t], tab.data(), 4 * (size_t) NF * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
  }
  if(!ctx->d_cellsize32) CK(dalloc(ctx, &ctx->d_cellsize32, ctx->G));
  std::vector<float> cs(ctx->G);
  for(int i = 0; i < ctx->G; i++) cs[i] = (float) ctx->h_cellsize[i];
  CK(cudaMemcpyAsync(ctx->d_cellsize32, cs.data(), ctx->G * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  ctx->tab32_dirty = false;
  return GALIC_OK;
}

}  // namespace galic_internal

using namespace galic_internal;

extern "C" const char *galic_status_string(int status)
{
  if(status < 0 || status >= (int) (sizeof(kStatusText) / sizeof(kStatusText[0]))) return "unknown status";
  return kStatusText[status];
}

extern "C" int galic_get_params(const galic_ctx *ctx, galic_params_t *out)
{
  if(!ctx || !out) return GALIC_ERR_INVALID_ARGUMENT;
  *out = ctx->prm;
  return GALIC_OK;
}

extern "C" int galic_last_status(const galic_ctx *ctx) { return ctx ? ctx->status : GALIC_ERR_INVALID_ARGUMENT; }

namespace galic_internal {
int ctx_create(const galic_params_t *prm, int priority, galic_ctx **out);
}

extern "C" int galic_ctx_create(const galic_params_t *prm, galic_ctx **out)
{
  return galic_internal::ctx_create(prm, 0, out);
}

// priority: of the context's streams (cudaStreamCreateWithPriority; 0 is the
// default, lower numbers run first): the serving loop gives jobs admitted
// while few others run precedence over later ones
int galic_internal::ctx_create(const galic_params_t *prm, int priority, galic_ctx **out)
{
  galic_ctx *ctx = nullptr;
  if(!out) return GALIC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int st = check_params(prm);
  if(st) return st;
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GALIC_ERR_NO_DEVICE;
  }
  ctx = new galic_ctx();
  ctx->prm = *prm;
  cudaGetDevice(&ctx->device);
  CK(keep_pool_memory(ctx->device));
  ctx->priority = priority;
  CK(cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, priority));
  for(int k = 0; k < 3; k++) CK(cudaEventCreate(&ctx->ev[k]));
  CK(prepare_fit_kernels());
  ctx->L = prm->DG_MaxLevel;
  ctx->G = 1 << (2 * ctx->L);
  ctx->Ns = stack_size(ctx->L);
  const int NF = prm->FG_Nbin * prm->FG_Nbin;
  CK(dalloc(ctx, &ctx->d_fg_acc, NF));
  CK(dalloc(ctx, &ctx->d_fg_pot, NF));
  for(int t = 1; t <= 3; t++) {
    CK(dalloc(ctx, &ctx->d_vstream[t], NF));
    CK(cudaMemsetAsync(ctx->d_vstream[t], 0, NF * sizeof(double), ctx->stream));
  }
  CK(cudaMemsetAsync(ctx->d_fg_acc, 0, NF * sizeof(double2), ctx->stream));
  CK(cudaMemsetAsync(ctx->d_fg_pot, 0, NF * sizeof(double), ctx->stream));
  CK(dalloc(ctx, &ctx->d_cellsize, ctx->G));
  CK(dalloc(ctx, &ctx->d_dist, ctx->Ns));
  CK(dalloc(ctx, &ctx->d_targets, (size_t) 4 * NT_TARGET * ctx->Ns));
  CK(cudaMemsetAsync(ctx->d_targets, 0, (size_t) 4 * NT_TARGET * ctx->Ns * sizeof(double), ctx->stream));
  CK(dalloc(ctx, &ctx->d_committed, (size_t) 4 * NG_COMMITTED * ctx->G));
  CK(cudaMemsetAsync(ctx->d_committed, 0, (size_t) 4 * NG_COMMITTED * ctx->G * sizeof(double), ctx->stream));
  CK(dalloc(ctx, &ctx->d_stacks, (size_t) 4 * NG_COMMITTED * ctx->Ns));
  CK(dalloc(ctx, &ctx->d_fx, (size_t) 4 * NG_COMMITTED * ctx->G));
  CK(dalloc(ctx, &ctx->d_shift, 4 * NG_COMMITTED));
  CK(dalloc(ctx, &ctx->d_fit, 4 * 7 + 4 * 5));
  CK(cudaMemsetAsync(ctx->d_fit, 0, (4 * 7 + 4 * 5) * sizeof(double), ctx->stream));
  CK(dalloc(ctx, &ctx->d_firstrun, 4));
  CK(cudaMemsetAsync(ctx->d_firstrun, 0, 4 * sizeof(int), ctx->stream));
  CK(dalloc(ctx, &ctx->d_counters, 9));
  CK(cudaMemsetAsync(ctx->d_counters, 0, 9 * sizeof(unsigned long long), ctx->stream));
  CK(dalloc(ctx, &ctx->d_status, 1));
  CK(dalloc(ctx, &ctx->d_next, 1));
  CK(dalloc(ctx, &ctx->d_maxerr, 1));
  CK(dalloc(ctx, &ctx->d_rep_stats, 2));

  DevModel &M = ctx->dm;
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
  for(int t = 0; t < 4; t++) {
    M.tovs[t] = prm->TypeOfVelocityStructure[t];
    M.vstream_zero[t] = 1;
  }
  M.FG_Nbin = prm->FG_Nbin;
  M.DG_Nbin = 1 << ctx->L;
  M.DG_L = ctx->L;
  M.EG_L = prm->EG_MaxLevel;
  M.DG_Ngrid = ctx->G;
  M.DG_Nstack = ctx->Ns;
  M.FG_Rmin = prm->FG_Rmin;
  M.FG_Fac = prm->FG_Fac;
  M.DG_Rmin = prm->DG_Rmin;
  M.DG_Fac = prm->DG_Fac;
  M.EG_Rmin = prm->EG_Rmin;
  M.EG_Fac = prm->EG_Fac;
  set_step_constants(M);
  M.fg_acc = ctx->d_fg_acc;
  M.fg_pot = ctx->d_fg_pot;
  for(int t = 0; t < 4; t++) M.vstream[t] = ctx->d_vstream[t];
  M.cellsize = ctx->d_cellsize;
  M.step_cap = GALIC_STEP_CAP;
  *out = ctx;
  return GALIC_OK;
}

extern "C" void galic_ctx_destroy(galic_ctx *ctx)
{
  if(!ctx) return;
  cudaStreamSynchronize(ctx->stream);
  dfree(ctx, ctx->d_fg_acc); dfree(ctx, ctx->d_fg_pot);
  for(int t = 0; t < 4; t++) dfree(ctx, ctx->d_vstream[t]);
  for(int t = 0; t < 4; t++)
    for(int k = 0; k < 5; k++) dfree(ctx, ctx->d_disp[t][k]);
  dfree(ctx, ctx->d_cellsize); dfree(ctx, ctx->d_dist); dfree(ctx, ctx->d_targets); dfree(ctx, ctx->d_committed); dfree(ctx, ctx->d_stacks);
  dfree(ctx, ctx->d_fx); dfree(ctx, ctx->d_shift); dfree(ctx, ctx->d_fit); dfree(ctx, ctx->d_firstrun); dfree(ctx, ctx->d_counters);
  dfree(ctx, ctx->d_status); dfree(ctx, ctx->d_next); dfree(ctx, ctx->d_maxerr);
  dfree(ctx, ctx->d_pos); dfree(ctx, ctx->d_vel); dfree(ctx, ctx->d_mass); dfree(ctx, ctx->d_tint); dfree(ctx, ctx->d_vesc);
  dfree(ctx, ctx->d_ptargets); dfree(ctx, ctx->d_vdisp); dfree(ctx, ctx->d_type); dfree(ctx, ctx->d_orbits); dfree(ctx, ctx->d_order);
  dfree(ctx, ctx->d_b_pos); dfree(ctx, ctx->d_b_vel); dfree(ctx, ctx->d_b_mass); dfree(ctx, ctx->d_b_time); dfree(ctx, ctx->d_grids);
  dfree(ctx, ctx->d_b_tall); dfree(ctx, ctx->d_b_err); dfree(ctx, ctx->d_b_type); dfree(ctx, ctx->d_b_norbit); dfree(ctx, ctx->d_b_status);
  dfree(ctx, ctx->d_b_steps);
  dfree(ctx, ctx->d_idx); dfree(ctx, ctx->d_accepted); dfree(ctx, ctx->d_vel_try); dfree(ctx, ctx->d_F); dfree(ctx, ctx->d_inst_v);
  dfree(ctx, ctx->d_inst_cell); dfree(ctx, ctx->d_acc_list); dfree(ctx, ctx->d_acc_n); dfree(ctx, ctx->d_inst0);
  dfree(ctx, ctx->d_fac); dfree(ctx, ctx->d_idx_all); dfree(ctx, ctx->d_fit_hist); dfree(ctx, ctx->d_rep_stats);
  for(int t = 0; t < 4; t++) dfree(ctx, ctx->d_tab32[t]);
  dfree(ctx, ctx->d_cellsize32);
  for(int k = 0; k < 3; k++)
    if(ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
  if(ctx->stream2) {
    cudaStreamSynchronize(ctx->stream2);
    cudaStreamDestroy(ctx->stream2);
  }
  for(int k = 0; k < 5; k++)
    if(ctx->ev2[k]) cudaEventDestroy(ctx->ev2[k]);
  if(ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  if(ctx->h_stage) cudaFreeHost(ctx->h_stage);
  delete ctx;
}

extern "C" int galic_set_force_grid(galic_ctx *ctx, const double *pot, const double *dpotdr, const double *dpotdz)
{
  if(!ctx || !pot || !dpotdr || !dpotdz) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  const int NF = ctx->prm.FG_Nbin * ctx->prm.FG_Nbin;
  std::vector<double2> acc(NF);
  double pmin = 0;
  for(int i = 0; i < NF; i++) {
    acc[i] = make_double2(dpotdr[i], dpotdz[i]);
    if(pot[i] < pmin) pmin = pot[i];
  }
  ctx->pot_min = pmin;
  ctx->h_dpotdr.assign(dpotdr, dpotdr + NF);
  ctx->h_dpotdz.assign(dpotdz, dpotdz + NF);
  ctx->tab32_dirty = true;
  CK(cudaMemcpyAsync(ctx->d_fg_acc, acc.data(), NF * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_fg_pot, pot, NF * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->have_fg = true;
  CK(cudaStreamSynchronize(ctx->stream));  // the upload is complete on return
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_set_vstream(galic_ctx *ctx, int type, const double *v)
{
  if(!ctx || !v || type < 1 || type > 3) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  const int NF = ctx->prm.FG_Nbin * ctx->prm.FG_Nbin;
  int zero = 1;
  for(int i = 0; i < NF && zero; i++) {
    uint64_t b;
    memcpy(&b, &v[i], 8);
    if(b != 0) zero = 0;  // only +0.0 everywhere allows skipping the lookup
  }
  ctx->dm.vstream_zero[type] = zero;
  ctx->h_vstream[type].assign(v, v + NF);
  ctx->tab32_dirty = true;
  CK(cudaMemcpyAsync(ctx->d_vstream[type], v, NF * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // the upload is complete on return
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_set_density_geometry(galic_ctx *ctx, const double *cellsize, const double *dist)
{
  if(!ctx || !cellsize || !dist) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  CK(cudaMemcpyAsync(ctx->d_cellsize, cellsize, ctx->G * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->h_cellsize.assign(cellsize, cellsize + ctx->G);
  ctx->tab32_dirty = true;
  CK(cudaMemcpyAsync(ctx->d_dist, dist, ctx->Ns * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->have_geom = true;
  CK(cudaStreamSynchronize(ctx->stream));  // the upload is complete on return
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_set_targets(galic_ctx *ctx, int type, const double *dgs_mass, const double *egs_mass,
                                 const double *egs_r, const double *egs_t, const double *egs_p, const double *egs_q)
{
  if(!ctx || type < 1 || type > 3 || !dgs_mass || !egs_mass || !egs_r || !egs_t || !egs_p || !egs_q)
    return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  const double *src[NT_TARGET] = {dgs_mass, egs_mass, egs_r, egs_t, egs_p, egs_q};
  for(int k = 0; k < NT_TARGET; k++)
    CK(cudaMemcpyAsync(ctx->d_targets + ((size_t) type * NT_TARGET + k) * ctx->Ns, src[k], ctx->Ns * sizeof(double),
                  cudaMemcpyHostToDevice, ctx->stream));
  ctx->have_targets[type] = true;
  CK(cudaStreamSynchronize(ctx->stream));  // the upload is complete on return
  return fail(ctx, GALIC_OK);
}

namespace {
cudaError_t order_by_type_radius(galic_ctx *ctx);
}

extern "C" int galic_set_particles(galic_ctx *ctx, int n, const double *pos, const double *vel, const double *mass,
                                   const double *tint, const double *vesc, const int *type, const double *targets)
{
  if(!ctx || n <= 0 || !pos || !vel || !mass || !tint || !vesc || !type || !targets)
    return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  for(int i = 0; i < n; i++)
    if(type[i] < 1 || type[i] > 3 || !(tint[i] > 0)) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  if(n != ctx->n) {
    dfree(ctx, ctx->d_pos); dfree(ctx, ctx->d_vel); dfree(ctx, ctx->d_mass); dfree(ctx, ctx->d_tint); dfree(ctx, ctx->d_vesc);
    dfree(ctx, ctx->d_ptargets); dfree(ctx, ctx->d_vdisp); dfree(ctx, ctx->d_type); dfree(ctx, ctx->d_orbits); dfree(ctx, ctx->d_order);
    CK(dalloc(ctx, &ctx->d_order, n));
    CK(dalloc(ctx, &ctx->d_pos, 3 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_vel, 3 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_mass, n));
    CK(dalloc(ctx, &ctx->d_tint, n));
    CK(dalloc(ctx, &ctx->d_vesc, n));
    CK(dalloc(ctx, &ctx->d_ptargets, 4 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_vdisp, 4 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_type, n));
    CK(dalloc(ctx, &ctx->d_orbits, n));
    ctx->n = n;
  }
  CK(cudaMemcpyAsync(ctx->d_pos, pos, 3 * (size_t) n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_vel, vel, 3 * (size_t) n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_mass, mass, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_tint, tint, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_vesc, vesc, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_ptargets, targets, 4 * (size_t) n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_type, type, n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_vdisp, 0, 4 * (size_t) n * sizeof(double), ctx->stream));
  // by type, then by radius: neighbouring lanes then integrate orbits of one
  // type (one velocity structure, no divergent projections) that start at
  // similar radii and read nearby force-grid cells; results do not depend on
  // the order.  Sorted on the GPU from the uploaded positions and types.
  CK(order_by_type_radius(ctx));
  CK(cudaMemsetAsync(ctx->d_orbits, 0, n * sizeof(int), ctx->stream));
  ctx->have_response = false;
  CK(cudaStreamSynchronize(ctx->stream));  // the upload is complete on return
  return fail(ctx, GALIC_OK);
}

namespace {

// masses and types of particles stored type by type
__global__ void k_particle_meta(int n, int n1, int n12, double m1, double m2, double m3, double *mass, int *type)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const int t = i < n1 ? 1 : (i < n12 ? 2 : 3);
  type[i] = t;
  mass[i] = t == 1 ? m1 : (t == 2 ? m2 : m3);
}

// r^2 as it orders (non-negative doubles order like their bits)
__global__ void k_radius_keys(int n, const double *pos, unsigned long long *key, int *idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const double *p = pos + 3 * (size_t) i;
  const double r2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  key[i] = (unsigned long long) __double_as_longlong(r2);
  idx[i] = i;
}

__global__ void k_type_keys(int n, const int *type, const int *idx, int *key)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  key[i] = type[idx[i]];
}

// the orbit order (by type, then by radius, ties in index order) of the
// context's particles into d_order: a stable radix sort by r^2, then a
// stable one by type (1-3: two bits)
cudaError_t order_by_type_radius(galic_ctx *ctx)
{
  const int n = ctx->n;
  cudaStream_t s = ctx->stream;
  const unsigned g = (unsigned) ((n + 255) / 256);
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  int *i0 = nullptr, *i1 = nullptr, *t0 = nullptr, *t1 = nullptr;
  void *tmp = nullptr;
  size_t tb = 0, tb2 = 0, tbx;
  cudaError_t e = cudaMallocAsync((void **) &k0, 2 * (size_t) n * sizeof(unsigned long long), s);
  if(e == cudaSuccess) e = cudaMallocAsync((void **) &i0, 4 * (size_t) n * sizeof(int), s);
  if(e == cudaSuccess) {
    k1 = k0 + n;
    i1 = i0 + n;
    t0 = i1 + n;
    t1 = t0 + n;
    e = cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, i0, i1, n, 0, 64, s);
  }
  if(e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb2, t0, t1, i1, ctx->d_order, n, 0, 2, s);
  if(e == cudaSuccess) e = cudaMallocAsync(&tmp, std::max<size_t>(std::max(tb, tb2), 16), s);
  if(e == cudaSuccess) {
    k_radius_keys<<<g, 256, 0, s>>>(n, ctx->d_pos, k0, i0);
    tbx = std::max(tb, tb2);
    e = cub::DeviceRadixSort::SortPairs(tmp, tbx, k0, k1, i0, i1, n, 0, 64, s);
  }
  if(e == cudaSuccess) {
    k_type_keys<<<g, 256, 0, s>>>(n, ctx->d_type, i1, t0);
    tbx = std::max(tb, tb2);
    e = cub::DeviceRadixSort::SortPairs(tmp, tbx, t0, t1, i1, ctx->d_order, n, 0, 2, s);
  }
  if(e == cudaSuccess) e = cudaGetLastError();
  for(void *q : {(void *) k0, (void *) i0, tmp})
    if(q) cudaFreeAsync(q, s);
  return e;
}

}  // namespace

namespace galic_internal {

cudaError_t keep_device_pool(int device) { return keep_pool_memory(device); }

// installs particles whose arrays are on the device, stored type by type
// (nt[t] particles of type t, masses tmass[t] / nt[t]), as galic_set_particles
// does from the host
int set_particles_device(galic_ctx *ctx, const int nt[4], const double tmass[4], const double *pos,
                         const double *vel, const double *tint, const double *vesc, const double *targets)
{
  const int n = nt[1] + nt[2] + nt[3];
  if(n <= 0) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  cudaStream_t s = ctx->stream;
  ctx->generation++;
  if(n != ctx->n) {
    dfree(ctx, ctx->d_pos); dfree(ctx, ctx->d_vel); dfree(ctx, ctx->d_mass); dfree(ctx, ctx->d_tint); dfree(ctx, ctx->d_vesc);
    dfree(ctx, ctx->d_ptargets); dfree(ctx, ctx->d_vdisp); dfree(ctx, ctx->d_type); dfree(ctx, ctx->d_orbits); dfree(ctx, ctx->d_order);
    ctx->n = 0;
    CK(dalloc(ctx, &ctx->d_order, n));
    CK(dalloc(ctx, &ctx->d_pos, 3 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_vel, 3 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_mass, n));
    CK(dalloc(ctx, &ctx->d_tint, n));
    CK(dalloc(ctx, &ctx->d_vesc, n));
    CK(dalloc(ctx, &ctx->d_ptargets, 4 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_vdisp, 4 * (size_t) n));
    CK(dalloc(ctx, &ctx->d_type, n));
    CK(dalloc(ctx, &ctx->d_orbits, n));
    ctx->n = n;
  }
  const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(ctx->d_pos, pos, 3 * (size_t) n * sizeof(double), dd, s));
  CK(cudaMemcpyAsync(ctx->d_vel, vel, 3 * (size_t) n * sizeof(double), dd, s));
  CK(cudaMemcpyAsync(ctx->d_tint, tint, n * sizeof(double), dd, s));
  CK(cudaMemcpyAsync(ctx->d_vesc, vesc, n * sizeof(double), dd, s));
  CK(cudaMemcpyAsync(ctx->d_ptargets, targets, 4 * (size_t) n * sizeof(double), dd, s));
  CK(cudaMemsetAsync(ctx->d_vdisp, 0, 4 * (size_t) n * sizeof(double), s));
  CK(cudaMemsetAsync(ctx->d_orbits, 0, n * sizeof(int), s));
  k_particle_meta<<<(unsigned) ((n + 255) / 256), 256, 0, s>>>(n, nt[1], nt[1] + nt[2], nt[1] ? tmass[1] / nt[1] : 0.0,
                                                                nt[2] ? tmass[2] / nt[2] : 0.0,
                                                                nt[3] ? tmass[3] / nt[3] : 0.0, ctx->d_mass, ctx->d_type);
  CK(cudaGetLastError());
  CK(order_by_type_radius(ctx));
  ctx->have_response = false;
  CK(cudaStreamSynchronize(s));
  return fail(ctx, GALIC_OK);
}

}  // namespace galic_internal

extern "C" int galic_get_particles(galic_ctx *ctx, double *vel, int *orbits, double *vdisp)
{
  if(!ctx || ctx->n == 0) return fail(ctx, GALIC_ERR_STATE);
  CK(cudaStreamSynchronize(ctx->stream));
  if(vel) CK(cudaMemcpyAsync(vel, ctx->d_vel, 3 * (size_t) ctx->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if(orbits) CK(cudaMemcpyAsync(orbits, ctx->d_orbits, ctx->n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  if(vdisp) CK(cudaMemcpyAsync(vdisp, ctx->d_vdisp, 4 * (size_t) ctx->n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return fail(ctx, GALIC_OK);
}

namespace {

double one_orbit(galic_ctx *ctx, double *pos, double *vel, double *grids[5], double mass, double timespan,
                 int *orbitstaken, int type, int with_egy)
{
  if(!ctx) return -1.0;
  if(!pos || !vel || !grids[0] || !orbitstaken || (with_egy && (!grids[1] || !grids[2] || !grids[3] || !grids[4])) ||
     type < 1 || type > 3 || !ctx->have_geom) {
    fail(ctx, !ctx->have_geom ? GALIC_ERR_STATE : GALIC_ERR_INVALID_ARGUMENT);
    return -1.0;
  }
  if(ensure_orbit_scratch(ctx, 1)) return -1.0;
  const int G = ctx->G;
  OrbitBatch b;
  b.count = 1;
  b.pos = ctx->d_b_pos;
  b.vel = ctx->d_b_vel;
  b.mass = ctx->d_b_mass;
  b.timespan = ctx->d_b_time;
  b.type = ctx->d_b_type;
  b.grids = ctx->d_grids;
  b.tall = ctx->d_b_tall;
  b.norbit = ctx->d_b_norbit;
  b.steps = ctx->d_b_steps;
  b.egy_err = ctx->d_b_err;
  b.status = ctx->d_b_status;
  b.with_egy = with_egy;
  cudaStream_t s = ctx->stream;
  auto ck = [&](cudaError_t e) {
    if(e != cudaSuccess) {
      fprintf(stderr, "galic_cuda: %s\n", cudaGetErrorString(e));
      fail(ctx, GALIC_ERR_CUDA);
      return false;
    }
    return true;
  };
  if(!ck(cudaMemcpyAsync(ctx->d_b_pos, pos, 3 * sizeof(double), cudaMemcpyHostToDevice, s)) ||
     !ck(cudaMemcpyAsync(ctx->d_b_vel, vel, 3 * sizeof(double), cudaMemcpyHostToDevice, s)) ||
     !ck(cudaMemcpyAsync(ctx->d_b_mass, &mass, sizeof(double), cudaMemcpyHostToDevice, s)) ||
     !ck(cudaMemcpyAsync(ctx->d_b_time, &timespan, sizeof(double), cudaMemcpyHostToDevice, s)) ||
     !ck(cudaMemcpyAsync(ctx->d_b_type, &type, sizeof(int), cudaMemcpyHostToDevice, s)) ||
     !ck(cudaMemsetAsync(ctx->d_grids, 0, (size_t) NF_ORBIT * G * sizeof(double), s)))
    return -1.0;
  launch_orbits_dense(ctx->dm, b, s);
  launch_scale_dense(ctx->dm, b, s);
  double tall = 0;
  int norbit = 0, status = 0;
  if(!ck(cudaMemcpyAsync(&tall, ctx->d_b_tall, sizeof(double), cudaMemcpyDeviceToHost, s)) ||
     !ck(cudaMemcpyAsync(&norbit, ctx->d_b_norbit, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
     !ck(cudaMemcpyAsync(&status, ctx->d_b_status, sizeof(int), cudaMemcpyDeviceToHost, s)))
    return -1.0;
  for(int f = 0; f < (with_egy ? NF_ORBIT : 1); f++)
    if(!ck(cudaMemcpyAsync(grids[f], ctx->d_grids + (size_t) f * G, G * sizeof(double), cudaMemcpyDeviceToHost, s)))
      return -1.0;
  if(!ck(cudaStreamSynchronize(s)) || !ck(cudaGetLastError())) return -1.0;
  ctx->last_launches = 2;
  if(status == ORBIT_STEP_CAP) {
    fail(ctx, GALIC_ERR_STEP_CAP);
    return -1.0;
  }
  if(status == ORBIT_NONFINITE) {
    fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
    return -1.0;
  }
  *orbitstaken = norbit;
  fail(ctx, GALIC_OK);
  return tall;
}

}  // namespace

extern "C" double galic_produce_orbit_response_field_mod(galic_ctx *ctx, double *pos, double *vel, int id,
                                                         double *mfield, double *egyfield_r, double *egyfield_t,
                                                         double *egyfield_q, double *egyfield_p, double mass,
                                                         double timespan, int *orbitstaken, int type)
{
  (void) id;
  double *g[5] = {mfield, egyfield_r, egyfield_t, egyfield_q, egyfield_p};
  return one_orbit(ctx, pos, vel, g, mass, timespan, orbitstaken, type, 1);
}

extern "C" double galic_produce_orbit_response_field(galic_ctx *ctx, double *pos, double *vel, int id,
                                                     double *mfield, double mass, double timespan, int *orbitstaken)
{
  (void) id;
  double *g[5] = {mfield, nullptr, nullptr, nullptr, nullptr};
  return one_orbit(ctx, pos, vel, g, mass, timespan, orbitstaken, 1, 0);
}

namespace {

int check_calc_all(galic_ctx *ctx, int form)
{
  if(form != GALIC_FORM_FP64 && form != GALIC_FORM_FP32) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(ctx->n == 0 || !ctx->have_geom) return fail(ctx, GALIC_ERR_STATE);
  if(form == GALIC_FORM_FP32) {
    int st = ensure_tab32(ctx);
    if(st) return st;
  }
  for(int t = 1; t <= 3; t++)
    if(ctx->prm.NType[t] > 0 && !ctx->have_targets[t]) return fail(ctx, GALIC_ERR_STATE);
  return GALIC_OK;
}

// main.c:151-231 for the orbits order[first + k * stride] and the particles
// first, first + stride, ...: zeroes the accumulators and leaves every
// deposit in fixed point (no synchronisation)
int enqueue_orbits(galic_ctx *ctx, int form, int first, int stride, int *launches)
{
  cudaStream_t s = ctx->stream;
  const int G = ctx->G;
  int shift[4 * NG_COMMITTED];
  set_shifts(ctx, shift, form);
  CK(cudaMemcpyAsync(ctx->d_shift, shift, sizeof(shift), cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev[0], s));
  CK(cudaMemsetAsync(ctx->d_fx, 0, (size_t) 4 * NG_COMMITTED * G * sizeof(FxWord), s));
  CK(cudaMemsetAsync(ctx->d_next, 0, sizeof(int), s));
  CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s));
  CK(cudaMemsetAsync(ctx->d_maxerr, 0, sizeof(double), s));
  CK(cudaMemsetAsync(ctx->d_counters + 8, 0, sizeof(unsigned long long), s));
  CalcAllArgs a;
  a.n = first < ctx->n ? (ctx->n - first + stride - 1) / stride : 0;
  a.first = first;
  a.stride = stride;
  a.pos = ctx->d_pos;
  a.vel = ctx->d_vel;
  a.mass = ctx->d_mass;
  a.tint = ctx->d_tint;
  a.type = ctx->d_type;
  a.order = ctx->d_order;
  a.next = ctx->d_next;
  a.fx = ctx->d_fx;
  a.shift = ctx->d_shift;
  a.orbits = ctx->d_orbits;
  a.steps_total = ctx->d_counters + 8;
  a.max_egy_err = ctx->d_maxerr;
  a.status = ctx->d_status;
  const int block = form == GALIC_FORM_FP32 ? CALC_ALL_BLOCK_FP32 : CALC_ALL_BLOCK_FP64;
  int per_sm = form == GALIC_FORM_FP32 ? calc_all_fp32_occupancy(block) : calc_all_occupancy(block);
  if(per_sm < 1) per_sm = 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  int grid = per_sm * sms;
  const int need = (a.n + block - 1) / block;
  if(grid > need) grid = need;
  CK(cudaEventRecord(ctx->ev[1], s));
  if(grid > 0) {
    if(form == GALIC_FORM_FP32)
      *launches += launch_calc_all_fp32(ctx->dm, ctx->d_tab32, ctx->d_cellsize32, a, grid, block, s);
    else
      *launches += launch_calc_all_fp64(ctx->dm, a, grid, block, s);
  }
  CK(cudaEventRecord(ctx->ev[2], s));
  launch_instantaneous(ctx->dm, ctx->n, ctx->d_pos, ctx->d_vel, ctx->d_mass, ctx->d_type, ctx->d_vdisp, ctx->d_fx,
                       ctx->d_shift, G, s, first, stride);
  *launches += 1;
  CK(cudaGetLastError());
  return GALIC_OK;
}

// fixed point -> committed grids, then calc_global_fit (main.c:251-362)
int enqueue_finish(galic_ctx *ctx, int *launches)
{
  launch_fx_finalize(ctx->d_fx, ctx->d_shift, ctx->d_committed, 4 * NG_COMMITTED, ctx->G, ctx->stream);
  *launches += 1;
  *launches += launch_global_fit(make_fit_args(ctx), ctx->stream);
  CK(cudaGetLastError());
  return GALIC_OK;
}

// waits for the stream; records timing, steps and the worst orbit status
int collect(galic_ctx *ctx, int launches, bool with_timing)
{
  cudaStream_t s = ctx->stream;
  char *h = stage(ctx, 32);
  if(!h) return fail(ctx, GALIC_ERR_CUDA);
  CK(cudaMemcpyAsync(h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h + 8, ctx->d_counters + 8, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h + 16, ctx->d_maxerr, sizeof(double), cudaMemcpyDeviceToHost, s));
  cudaEvent_t ev_end;
  CK(cudaEventCreate(&ev_end));
  CK(cudaEventRecord(ev_end, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  int status;
  unsigned long long steps;
  std::memcpy(&status, h, sizeof(int));
  std::memcpy(&steps, h + 8, sizeof(steps));
  std::memcpy(&ctx->last_max_egy_err, h + 16, sizeof(double));
  if(with_timing) {
    float ms_total = 0, ms_orbit = 0;
    CK(cudaEventElapsedTime(&ms_total, ctx->ev[0], ev_end));
    CK(cudaEventElapsedTime(&ms_orbit, ctx->ev[1], ctx->ev[2]));
    ctx->last_ms_total = ms_total;
    ctx->last_ms_orbit = ms_orbit;
  }
  cudaEventDestroy(ev_end);
  ctx->last_steps = (long long) steps;
  ctx->last_launches = launches;
  if(status == ORBIT_STEP_CAP) return fail(ctx, GALIC_ERR_STEP_CAP);
  if(status == ORBIT_NONFINITE) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  return GALIC_OK;
}

}  // namespace

extern "C" int galic_calc_all_response_fields(galic_ctx *ctx, int form)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  int st = check_calc_all(ctx, form);
  if(st) return st;
  int launches = 0;
  if((st = enqueue_orbits(ctx, form, 0, 1, &launches))) return st;
  if((st = enqueue_finish(ctx, &launches))) return st;
  if((st = collect(ctx, launches, true))) return st;
  ctx->have_response = true;
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_calc_all_shard(galic_ctx *ctx, int form, int rank, int world)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(world < 1 || rank < 0 || rank >= world) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  int st = check_calc_all(ctx, form);
  if(st) return st;
  int launches = 0;
  ctx->have_response = false;
  ctx->shard_form = form;
  if((st = enqueue_orbits(ctx, form, rank, world, &launches))) return st;
  return fail(ctx, collect(ctx, launches, true));
}

extern "C" int galic_accumulators(galic_ctx *ctx, void **device_ptr, size_t *words)
{
  if(!ctx || !device_ptr || !words) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  *device_ptr = (void *) ctx->d_fx;
  *words = (size_t) 4 * NG_COMMITTED * ctx->G * 2;
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_calc_all_finish(galic_ctx *ctx)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(ctx->shard_form < 0) return fail(ctx, GALIC_ERR_STATE);
  int launches = 0;
  int st = enqueue_finish(ctx, &launches);
  if(st) return st;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->last_launches = launches;
  ctx->shard_form = -1;
  ctx->have_response = true;
  return fail(ctx, GALIC_OK);
}

namespace {

// device arguments of `count` optimised particles starting at the context's
// scratch (one repetition, or a window of repetitions of per_rep each)
RepArgs make_rep_args(galic_ctx *ctx, int count, uint64_t seed, uint32_t rep_serial, int per_rep)
{
  RepArgs R;
  R.count = count;
  R.idx = ctx->d_idx;
  R.seed = seed;
  R.rep_serial = rep_serial;
  R.per_rep = per_rep;
  R.p_pos = ctx->d_pos;
  R.p_vel = ctx->d_vel;
  R.p_mass = ctx->d_mass;
  R.p_tint = ctx->d_tint;
  R.p_vesc = ctx->d_vesc;
  R.p_targets = ctx->d_ptargets;
  R.p_vdisp = ctx->d_vdisp;
  R.p_type = ctx->d_type;
  R.p_orbits = ctx->d_orbits;
  R.b_pos = ctx->d_b_pos;
  R.b_vel = ctx->d_b_vel;
  R.b_mass = ctx->d_b_mass;
  R.b_time = ctx->d_b_time;
  R.b_type = ctx->d_b_type;
  R.b_norbit = ctx->d_b_norbit;
  R.grids = ctx->d_grids;
  R.b_tall = ctx->d_b_tall;
  R.fac = ctx->d_fac;
  R.vel_try = ctx->d_vel_try;
  R.F = ctx->d_F;
  R.accepted = ctx->d_accepted;
  R.acc_list = ctx->d_acc_list;
  R.acc_n = ctx->d_acc_n;
  R.inst0 = ctx->d_inst0;
  R.inst_v = ctx->d_inst_v;
  R.inst_cell = ctx->d_inst_cell;
  R.tries = ctx->d_counters;
  R.changes = ctx->d_counters + 4;
  for(int t = 0; t < 4; t++) {
    R.fac_rs[t] = ctx->prm.fac_value_rs[t];
    R.fac_ts[t] = ctx->prm.fac_value_ts[t];
    R.fac_qs[t] = ctx->prm.fac_value_qs[t];
    R.fac_ps[t] = ctx->prm.fac_value_ps[t];
  }
  R.status = ctx->d_status;
  return R;
}

// the 2 * count old / trial orbits of make_rep_args' particles
OrbitBatch make_rep_batch(galic_ctx *ctx, int count)
{
  OrbitBatch b;
  b.count = 2 * count;
  b.pos = ctx->d_b_pos;
  b.vel = ctx->d_b_vel;
  b.mass = ctx->d_b_mass;
  b.timespan = ctx->d_b_time;
  b.type = ctx->d_b_type;
  b.grids = ctx->d_grids;
  b.tall = ctx->d_b_tall;
  b.norbit = ctx->d_b_norbit;
  b.steps = ctx->d_b_steps;
  b.egy_err = ctx->d_b_err;
  b.status = ctx->d_b_status;
  b.with_egy = 1;
  return b;
}

// uploads `count` particle indices and clears the status words; returns the
// pinned staging block (status, per-orbit status and steps are read back
// into it by finish_rep_window), or null
char *begin_rep_window(galic_ctx *ctx, const int *idx, int count, size_t *off_st, size_t *off_ost, size_t *off_steps)
{
  cudaStream_t s = ctx->stream;
  *off_st = ((size_t) count * sizeof(int) + 15) & ~(size_t) 15;
  *off_ost = *off_st + 16;
  *off_steps = (*off_ost + 2 * (size_t) count * sizeof(int) + 15) & ~(size_t) 15;
  char *h = stage(ctx, *off_steps + 2 * (size_t) count * sizeof(long long));
  if(!h) return nullptr;
  std::memcpy(h, idx, count * sizeof(int));
  if(cudaMemcpyAsync(ctx->d_idx, h, count * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
     cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s) != cudaSuccess ||
     cudaMemsetAsync(ctx->d_b_status, 0, 2 * (size_t) count * sizeof(int), s) != cudaSuccess)
    return nullptr;
  return h;
}

// waits for the window's work; adds its orbit-steps to *steps; returns the
// worst status of the window
int finish_rep_window(galic_ctx *ctx, char *h, int count, size_t off_st, size_t off_ost, size_t off_steps,
                      long long *steps)
{
  cudaStream_t s = ctx->stream;
  if(cudaMemcpyAsync(h + off_st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
     cudaMemcpyAsync(h + off_ost, ctx->d_b_status, 2 * (size_t) count * sizeof(int), cudaMemcpyDeviceToHost, s) !=
         cudaSuccess ||
     cudaMemcpyAsync(h + off_steps, ctx->d_b_steps, 2 * (size_t) count * sizeof(long long), cudaMemcpyDeviceToHost,
                     s) != cudaSuccess ||
     cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return GALIC_ERR_CUDA;
  int status;
  std::memcpy(&status, h + off_st, sizeof(int));
  const int *ost = (const int *) (h + off_ost);
  const long long *st = (const long long *) (h + off_steps);
  for(int k = 0; k < 2 * count; k++) {
    *steps += st[k];
    if(ost[k] == ORBIT_STEP_CAP) status = std::max(status, (int) GALIC_ERR_STEP_CAP);
  }
  return status;
}

}  // namespace

extern "C" int galic_optimize_rep(galic_ctx *ctx, const int *idx, int count, uint64_t seed, uint32_t rep_serial,
                                  int form)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(form != GALIC_FORM_FP64 && form != GALIC_FORM_FP32) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(!ctx->have_response) return fail(ctx, GALIC_ERR_STATE);
  if(form == GALIC_FORM_FP32) {
    int st = ensure_tab32(ctx);
    if(st) return st;
  }
  if(count < 0 || (count > 0 && !idx)) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  // every particle at most once per repetition: the reference evaluates a
  // repetition against committed state and P[n] only changes for n itself
  std::vector<char> seen(ctx->n, 0);
  for(int k = 0; k < count; k++) {
    if(idx[k] < 0 || idx[k] >= ctx->n || seen[idx[k]]) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
    seen[idx[k]] = 1;
  }
  cudaStream_t s = ctx->stream;
  FitArgs f = make_fit_args(ctx);
  if(count == 0) {  // init_updates + commit_updates with no particle: only the fit
    ctx->last_launches = launch_global_fit(f, s);
    CK(cudaStreamSynchronize(s));
    return fail(ctx, GALIC_OK);
  }
  int st = ensure_rep_scratch(ctx, count);
  if(st) return st;
  size_t off_st, off_ost, off_steps;
  char *h = begin_rep_window(ctx, idx, count, &off_st, &off_ost, &off_steps);
  if(!h) return fail(ctx, GALIC_ERR_CUDA);
  RepArgs R = make_rep_args(ctx, count, seed, rep_serial, 0);
  OrbitBatch b = make_rep_batch(ctx, count);
  ctx->last_launches = form == GALIC_FORM_FP32 ? launch_rep(ctx->dm, R, f, b, s, ctx->d_tab32, ctx->d_cellsize32)
                                               : launch_rep(ctx->dm, R, f, b, s);
  long long tot = 0;
  int status = finish_rep_window(ctx, h, count, off_st, off_ost, off_steps, &tot);
  ctx->last_steps = tot;
  if(status) return fail(ctx, status);
  return fail(ctx, GALIC_OK);
}

namespace {

// one window of repetitions: reps [r0, r1); dep: some particle of the
// window was optimised in the window before it
struct RepWindow {
  int r0, r1;
  bool dep;
};

// the orbit batch of `count` orbit pairs starting at pair `first` of the
// context's scratch
OrbitBatch batch_slice(const OrbitBatch &b, int first, int count, int G)
{
  OrbitBatch o = b;
  const size_t k = 2 * (size_t) first;
  o.count = 2 * count;
  o.pos = b.pos + 3 * k;
  o.vel = b.vel + 3 * k;
  o.mass = b.mass + k;
  o.timespan = b.timespan + k;
  o.type = b.type + k;
  o.grids = b.grids + k * NF_ORBIT * G;
  o.tall = b.tall + k;
  o.norbit = b.norbit + k;
  o.steps = b.steps + k;
  o.egy_err = b.egy_err + k;
  o.status = b.status + k;
  return o;
}

__global__ void k_window_stats(const long long *steps, const int *status, int n, unsigned long long *total,
                               int *worst)
{
  long long my = 0;
  int w = 0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    my += steps[i];
    w = max(w, status[i]);
  }
  if(my) atomicAdd(total, (unsigned long long) my);
  if(w) atomicMax(worst, w);
}

}  // namespace

extern "C" int galic_optimize_reps(galic_ctx *ctx, const int *idx, int count, int reps, uint64_t seed,
                                   uint32_t rep_serial, int form, size_t window_bytes, double *fits)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(form != GALIC_FORM_FP64 && form != GALIC_FORM_FP32) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(!ctx->have_response) return fail(ctx, GALIC_ERR_STATE);
  if(count < 0 || reps < 0 || (count > 0 && reps > 0 && !idx)) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(form == GALIC_FORM_FP32) {
    int st = ensure_tab32(ctx);
    if(st) return st;
  }
  // each repetition's particles distinct and in range (as galic_optimize_rep)
  std::vector<int> last_rep(ctx->n, -1);
  for(int r = 0; r < reps; r++)
    for(int k = 0; k < count; k++) {
      const int n = idx[(size_t) r * count + k];
      if(n < 0 || n >= ctx->n || last_rep[n] == r) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
      last_rep[n] = r;
    }
  cudaStream_t s = ctx->stream;
  FitArgs f = make_fit_args(ctx);
  int launches = 0;
  if(reps > 0 && fits) {
    if(ctx->fit_hist_cap < (size_t) reps) {
      dfree(ctx, ctx->d_fit_hist);
      CK(dalloc(ctx, &ctx->d_fit_hist, (size_t) reps * 28));
      ctx->fit_hist_cap = reps;
    }
  }
  auto record_fit = [&](int r) -> cudaError_t {
    if(!fits) return cudaSuccess;
    return cudaMemcpyAsync(ctx->d_fit_hist + (size_t) r * 28, ctx->d_fit, 28 * sizeof(double),
                           cudaMemcpyDeviceToDevice, s);
  };
  auto copy_fits = [&]() -> int {
    if(!fits || reps == 0) return GALIC_OK;
    CK(cudaMemcpyAsync(fits, ctx->d_fit_hist, (size_t) reps * 28 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GALIC_OK;
  };
  if(count == 0) {
    for(int r = 0; r < reps; r++) {
      launches += launch_global_fit(f, s);
      CK(record_fit(r));
    }
    int st = copy_fits();
    if(st) return st;
    CK(cudaStreamSynchronize(s));
    ctx->last_launches = launches;
    ctx->last_steps = 0;
    return fail(ctx, GALIC_OK);
  }
  // per optimised particle: two orbits' dense grids plus their small arrays
  const size_t per_particle = 2 * ((size_t) NF_ORBIT * ctx->G * sizeof(double) + 128);
  if(window_bytes == 0) window_bytes = (size_t) 4 << 30;
  // the windows: each one's particles all distinct (the old orbit of a
  // particle optimised twice would depend on the first outcome) and its
  // grids within window_bytes (at least one repetition)
  std::fill(last_rep.begin(), last_rep.end(), -1);
  std::vector<RepWindow> wins;
  int maxM = 0;
  for(int r0 = 0; r0 < reps;) {
    int r1 = r0;
    bool dep = false;
    while(r1 < reps) {
      if(r1 > r0 && (size_t) (r1 - r0 + 1) * count * per_particle > window_bytes) break;
      bool repeat = false, before = false;
      for(int k = 0; k < count; k++) {
        const int q = last_rep[idx[(size_t) r1 * count + k]];
        repeat |= q >= r0;
        before |= q >= 0 && q < r0 && !wins.empty() && q >= wins.back().r0;
      }
      if(repeat && r1 > r0) break;
      dep |= before;
      for(int k = 0; k < count; k++) last_rep[idx[(size_t) r1 * count + k]] = r1;
      r1++;
    }
    wins.push_back({r0, r1, dep});
    maxM = std::max(maxM, (r1 - r0) * count);
    r0 = r1;
  }
  // two halves of the scratch: the orbits of window w + 1 run on the second
  // stream while window w commits on the context's stream
  const int nbuf = wins.size() > 1 ? 2 : 1;
  int st = ensure_rep_scratch(ctx, nbuf * maxM);
  if(st) return st;
  if(ctx->idx_cap < (size_t) reps * count) {
    dfree(ctx, ctx->d_idx_all);
    CK(dalloc(ctx, &ctx->d_idx_all, (size_t) reps * count));
    ctx->idx_cap = (size_t) reps * count;
  }
  if(!ctx->stream2) {
    CK(cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking, ctx->priority));
    for(int k = 0; k < 5; k++) CK(cudaEventCreateWithFlags(&ctx->ev2[k], cudaEventDisableTiming));
  }
  cudaStream_t so = ctx->stream2;
  // every index of the call in one copy; staged through pinned memory
  {
    char *h = stage(ctx, (size_t) reps * count * sizeof(int));
    if(!h) return fail(ctx, GALIC_ERR_CUDA);
    std::memcpy(h, idx, (size_t) reps * count * sizeof(int));
    CK(cudaMemcpyAsync(ctx->d_idx_all, h, (size_t) reps * count * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s));
  CK(cudaMemsetAsync(ctx->d_rep_stats, 0, sizeof(unsigned long long) + sizeof(int) * 2, s));
  // ev2[2]: the context's stream reached this point (scratch allocated, indices uploaded)
  CK(cudaEventRecord(ctx->ev2[2], s));
  CK(cudaStreamWaitEvent(so, ctx->ev2[2], 0));
  const RepArgs Rall = make_rep_args(ctx, nbuf * maxM, seed, rep_serial, count);
  const OrbitBatch ball = make_rep_batch(ctx, nbuf * maxM);
  unsigned long long *d_total = (unsigned long long *) ctx->d_rep_stats;
  int *d_worst = (int *) (ctx->d_rep_stats + 1);
  for(size_t w = 0; w < wins.size(); w++) {
    const int half = (int) (w % nbuf), W = wins[w].r1 - wins[w].r0, M = W * count;
    RepArgs R = rep_slice(Rall, half * maxM, M, ctx->G);
    R.idx = ctx->d_idx_all + (size_t) wins[w].r0 * count;
    R.per_rep = count;
    R.rep_serial = rep_serial + (uint32_t) wins[w].r0;
    const OrbitBatch b = batch_slice(ball, half * maxM, M, ctx->G);
    // the half is free once the window before the previous one has
    // committed; a window whose particles were optimised in the previous
    // window waits for that window's commit as well
    if(w >= 2) CK(cudaStreamWaitEvent(so, ctx->ev2[half], 0));
    if(wins[w].dep && w >= 1) CK(cudaStreamWaitEvent(so, ctx->ev2[1 - half], 0));
    CK(cudaMemsetAsync(b.status, 0, (size_t) b.count * sizeof(int), so));
    launches += form == GALIC_FORM_FP32 ? launch_rep_orbits(ctx->dm, R, b, so, ctx->d_tab32, ctx->d_cellsize32)
                                        : launch_rep_orbits(ctx->dm, R, b, so);
    // ev2[3 + half]: this window's orbits are done (a wait takes the event's
    // state at the time of the wait, so the event can be recorded again for
    // the window after next)
    CK(cudaEventRecord(ctx->ev2[3 + half], so));
    CK(cudaStreamWaitEvent(s, ctx->ev2[3 + half], 0));
    // each repetition's evaluation against the state its predecessors
    // committed, acceptance and commit, in order
    for(int j = 0; j < W; j++) {
      launches += launch_rep_commit(ctx->dm, rep_slice(R, j * count, count, ctx->G), f, s);
      CK(record_fit(wins[w].r0 + j));
    }
    k_window_stats<<<(b.count + 255) / 256 < 148 ? (b.count + 255) / 256 : 148, 256, 0, s>>>(b.steps, b.status,
                                                                                             b.count, d_total, d_worst);
    launches++;
    CK(cudaEventRecord(ctx->ev2[half], s));
  }
  // totals of the call
  char *h = stage(ctx, 32);
  if(!h) return fail(ctx, GALIC_ERR_CUDA);
  CK(cudaMemcpyAsync(h, ctx->d_rep_stats, 16, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h + 16, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  unsigned long long tot;
  int worst, status;
  std::memcpy(&tot, h, 8);
  std::memcpy(&worst, h + 8, 4);
  std::memcpy(&status, h + 16, 4);
  ctx->last_steps = (long long) tot;
  ctx->last_launches = launches;
  if(worst == ORBIT_STEP_CAP) status = std::max(status, (int) GALIC_ERR_STEP_CAP);
  if(status) return fail(ctx, status);
  st = copy_fits();
  if(st) return st;
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_get_fit(galic_ctx *ctx, double *out)
{
  if(!ctx || !out) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  char *h = stage(ctx, 4 * 7 * sizeof(double));
  if(!h) return fail(ctx, GALIC_ERR_CUDA);
  CK(cudaMemcpyAsync(h, ctx->d_fit, 4 * 7 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, h, 4 * 7 * sizeof(double));
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_get_counters(galic_ctx *ctx, long long *tries, long long *changes)
{
  if(!ctx || !tries || !changes) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  unsigned long long c[8];
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpyAsync(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  for(int t = 0; t < 4; t++) {
    tries[t] = (long long) c[t];
    changes[t] = (long long) c[4 + t];
  }
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_get_response(galic_ctx *ctx, int type, int which, double *out)
{
  if(!ctx || !out || type < 1 || type > 3 || which < 0 || which >= GALIC_GRID_COUNT)
    return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpyAsync(out, ctx->d_committed + ((size_t) type * NG_COMMITTED + which) * ctx->G, ctx->G * sizeof(double),
                cudaMemcpyDeviceToHost, ctx->stream));
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_set_step_cap(galic_ctx *ctx, long long cap)
{
  if(!ctx || cap < 1) return fail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  ctx->generation++;
  ctx->dm.step_cap = cap;
  return fail(ctx, GALIC_OK);
}

extern "C" int galic_last_timing(const galic_ctx *ctx, double *ms_total, double *ms_orbit_kernel)
{
  if(!ctx || !ms_total || !ms_orbit_kernel) return GALIC_ERR_INVALID_ARGUMENT;
  *ms_total = ctx->last_ms_total;
  *ms_orbit_kernel = ctx->last_ms_orbit;
  return GALIC_OK;
}

extern "C" double galic_last_max_energy_error(const galic_ctx *ctx) { return ctx ? ctx->last_max_egy_err : 0; }

extern "C" long long galic_last_orbit_steps(const galic_ctx *ctx) { return ctx ? ctx->last_steps : 0; }
extern "C" int galic_last_kernel_launches(const galic_ctx *ctx) { return ctx ? ctx->last_launches : 0; }
