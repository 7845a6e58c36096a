// Ensembles: many galaxy models advanced by one persistent FP32 launch per
// iteration, the whole iteration replayed from a CUDA graph.
//
// One iteration of a member is calc_all_response_fields (main.c:151-246) with
// its calc_global_fit (main.c:251-362), as galic_calc_all_response_fields
// does for one context in the FP32 form.  The ensemble keeps the members'
// own device state (particles, tables, targets, committed grids, stacks,
// fit) and adds one fixed-point accumulator block for all members, so that a
// single orbit kernel can serve every member: the orbits of all members form
// one work index space, each lane takes the next orbit of whichever member it
// belongs to, and deposits go to that member's grids.  The fixed-point sums
// are exact and order-independent, so a member's results do not depend on the
// other members, on the tile variant or on scheduling.
//
// The graph holds: accumulator and counter resets, the orbit kernel, and per
// member the instantaneous-energy kernel, the fixed-point read-out and the
// three merit kernels.  It captures the members' device pointers; any upload
// to a member (which may reallocate) invalidates the ensemble
// (GALIC_ERR_STATE), and the caller builds a new one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "context.cuh"
#include "galic_gpu.h"
#include "kernels.cuh"

using namespace galic_internal;

struct galic_ensemble {
  int device = 0;
  int nmodels = 0;
  int G = 0;
  std::vector<galic_ctx *> members;
  std::vector<unsigned> generation;
  cudaStream_t stream = nullptr;
  EnsembleLaunch L{};
  void *d_members = nullptr;
  int *d_next = nullptr;
  FxWord *d_fx = nullptr;
  int *d_shift = nullptr;
  unsigned long long *d_steps = nullptr;
  double *d_maxerr = nullptr;
  int *d_status = nullptr;
  unsigned long long *h_steps = nullptr;  // pinned
  double *h_maxerr = nullptr;             // pinned
  int *h_status = nullptr;                // pinned
  int variant = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_variant = -1;
  size_t graph_nodes = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double last_ms_total = 0, last_ms_orbit = 0;
  long long last_steps = 0;
  int status = 0;
};

namespace {

int efail(galic_ensemble *e, int st)
{
  if(e) e->status = st;
  return st;
}

#define ECK(call)                                                                                      \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if(e_ != cudaSuccess) {                                                                            \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                               \
      return efail(e, GALIC_ERR_CUDA);                                                                 \
    }                                                                                                  \
  } while(0)

void release_graph(galic_ensemble *e)
{
  if(e->exec) cudaGraphExecDestroy(e->exec);
  if(e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr;
  e->graph = nullptr;
  e->graph_variant = -1;
}

int persistent_grid(int variant, int total, int device)
{
  int block = 0, minb = 0;
  ensemble_variant(variant, &block, &minb);
  int per_sm = ensemble_occupancy(variant);
  if(per_sm < 1) per_sm = 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int grid = per_sm * sms;
  const int need = (total + block - 1) / block;
  return std::max(1, std::min(grid, need));
}

bool members_unchanged(const galic_ensemble *e)
{
  for(int m = 0; m < e->nmodels; m++)
    if(e->members[m]->generation != e->generation[m]) return false;
  return true;
}

// one iteration of every member, enqueued on e->stream (no host
// synchronisation: this is what the graph captures); the events become
// event-record nodes of the graph (cudaEventRecordExternal)
int enqueue_iteration(galic_ensemble *e, int variant, int grid)
{
  cudaStream_t s = e->stream;
  const size_t fx_words = (size_t) e->nmodels * 4 * NG_COMMITTED * e->G;
  ECK(cudaEventRecordWithFlags(e->ev[0], s, cudaEventRecordExternal));
  ECK(cudaMemsetAsync(e->d_fx, 0, fx_words * sizeof(FxWord), s));
  ECK(cudaMemsetAsync(e->d_next, 0, sizeof(int), s));
  ECK(cudaMemsetAsync(e->d_steps, 0, e->nmodels * sizeof(unsigned long long), s));
  ECK(cudaMemsetAsync(e->d_maxerr, 0, e->nmodels * sizeof(double), s));
  ECK(cudaMemsetAsync(e->d_status, 0, e->nmodels * sizeof(int), s));
  ECK(cudaEventRecordWithFlags(e->ev[1], s, cudaEventRecordExternal));
  ECK(launch_ensemble_fp32(e->L, variant, grid, s));
  ECK(cudaEventRecordWithFlags(e->ev[2], s, cudaEventRecordExternal));
  for(int m = 0; m < e->nmodels; m++) {
    galic_ctx *c = e->members[m];
    FxWord *fx = e->d_fx + (size_t) m * 4 * NG_COMMITTED * e->G;
    const int *shift = e->d_shift + m * 4 * NG_COMMITTED;
    launch_instantaneous(c->dm, c->n, c->d_pos, c->d_vel, c->d_mass, c->d_type, c->d_vdisp, fx, shift, e->G, s);
    launch_fx_finalize(fx, shift, c->d_committed, 4 * NG_COMMITTED, e->G, s);
    launch_global_fit(make_fit_args(c), s);
  }
  ECK(cudaGetLastError());
  ECK(cudaEventRecordWithFlags(e->ev[3], s, cudaEventRecordExternal));
  return GALIC_OK;
}

int build_graph(galic_ensemble *e)
{
  release_graph(e);
  const int grid = persistent_grid(e->variant, e->L.offset[e->nmodels], e->device);
  ECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_iteration(e, e->variant, grid);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
  if(st) {
    if(g) cudaGraphDestroy(g);
    return st;
  }
  ECK(ce);
  e->graph = g;
  ECK(cudaGraphInstantiate(&e->exec, g, 0));
  ECK(cudaGraphGetNodes(g, nullptr, &e->graph_nodes));
  e->graph_variant = e->variant;
  return GALIC_OK;
}

int ensemble_setup(galic_ensemble *e, galic_ctx *const *members, int count, int dev, int G);

}  // namespace

extern "C" int galic_ensemble_create(galic_ctx *const *members, int count, galic_ensemble **out)
{
  galic_ensemble *e = nullptr;
  if(!members || !out || count < 1 || count > GALIC_ENSEMBLE_MAX) return GALIC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess) return GALIC_ERR_NO_DEVICE;
  const int G = members[0] ? members[0]->G : 0;
  for(int m = 0; m < count; m++) {
    galic_ctx *c = members[m];
    if(!c) return GALIC_ERR_INVALID_ARGUMENT;
    for(int k = 0; k < m; k++)
      if(members[k] == c) return GALIC_ERR_INVALID_ARGUMENT;
    if(c->device != dev || c->G != G) return GALIC_ERR_UNSUPPORTED;  // one device, one response-grid level
    if(c->n == 0 || !c->have_geom) return GALIC_ERR_STATE;
    for(int t = 1; t <= 3; t++)
      if(c->prm.NType[t] > 0 && !c->have_targets[t]) return GALIC_ERR_STATE;
  }
  e = new galic_ensemble();
  const int st = ensemble_setup(e, members, count, dev, G);
  if(st) {
    galic_ensemble_destroy(e);
    return st;
  }
  *out = e;
  return GALIC_OK;
}

namespace {

int ensemble_setup(galic_ensemble *e, galic_ctx *const *members, int count, int dev, int G)
{
  e->device = dev;
  e->nmodels = count;
  e->G = G;
  e->members.assign(members, members + count);
  ECK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  for(int k = 0; k < 4; k++) ECK(cudaEventCreate(&e->ev[k]));
  const size_t mb = ensemble_member_bytes();
  std::vector<char> host_members(mb * count);
  std::vector<int> shift(count * 4 * NG_COMMITTED);
  EnsembleLaunch &L = e->L;
  L.nmodels = count;
  L.offset[0] = 0;
  long long total = 0;
  for(int m = 0; m < count; m++) {
    galic_ctx *c = members[m];
    const int st = ensure_tab32(c);
    if(st) return st;
    total += c->n;
    if(total > (1LL << 30)) return GALIC_ERR_BUDGET;
    L.offset[m + 1] = (int) total;
    L.dm[m] = c->dm;
    for(int t = 0; t < 4; t++) L.quad[m][t] = c->d_tab32[t];
    L.cellsize32[m] = c->d_cellsize32;
    ensemble_fill_member(host_members.data() + mb * m, c->dm, c->d_pos, c->d_vel, c->d_mass, c->d_tint, c->d_type,
                         c->d_order, c->d_orbits);
    set_shifts(c, &shift[m * 4 * NG_COMMITTED], GALIC_FORM_FP32);
    e->generation.push_back(c->generation);
  }
  ECK(cudaMalloc(&e->d_members, mb * count));
  ECK(cudaMemcpy(e->d_members, host_members.data(), mb * count, cudaMemcpyHostToDevice));
  ECK(cudaMalloc(&e->d_next, sizeof(int)));
  ECK(cudaMalloc(&e->d_fx, (size_t) count * 4 * NG_COMMITTED * G * sizeof(FxWord)));
  ECK(cudaMalloc(&e->d_shift, shift.size() * sizeof(int)));
  ECK(cudaMemcpy(e->d_shift, shift.data(), shift.size() * sizeof(int), cudaMemcpyHostToDevice));
  ECK(cudaMalloc(&e->d_steps, count * sizeof(unsigned long long)));
  ECK(cudaMalloc(&e->d_maxerr, count * sizeof(double)));
  ECK(cudaMalloc(&e->d_status, count * sizeof(int)));
  ECK(cudaMallocHost(&e->h_steps, count * sizeof(unsigned long long)));
  ECK(cudaMallocHost(&e->h_maxerr, count * sizeof(double)));
  ECK(cudaMallocHost(&e->h_status, count * sizeof(int)));
  L.members = e->d_members;
  L.next = e->d_next;
  L.fx = e->d_fx;
  L.shift = e->d_shift;
  L.steps = e->d_steps;
  L.maxerr = e->d_maxerr;
  L.status = e->d_status;
  ECK(prepare_fit_kernels());
  return GALIC_OK;
}

}  // namespace

extern "C" void galic_ensemble_destroy(galic_ensemble *e)
{
  if(!e) return;
  if(e->stream) cudaStreamSynchronize(e->stream);
  release_graph(e);
  cudaFree(e->d_members);
  cudaFree(e->d_next);
  cudaFree(e->d_fx);
  cudaFree(e->d_shift);
  cudaFree(e->d_steps);
  cudaFree(e->d_maxerr);
  cudaFree(e->d_status);
  cudaFreeHost(e->h_steps);
  cudaFreeHost(e->h_maxerr);
  cudaFreeHost(e->h_status);
  for(int k = 0; k < 4; k++)
    if(e->ev[k]) cudaEventDestroy(e->ev[k]);
  if(e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

extern "C" int galic_ensemble_last_status(const galic_ensemble *e) { return e ? e->status : GALIC_ERR_INVALID_ARGUMENT; }

extern "C" int galic_ensemble_variants(int *block, int *min_blocks, int max)
{
  const int n = ensemble_variant_count();
  for(int v = 0; v < n && v < max; v++) ensemble_variant(v, &block[v], &min_blocks[v]);
  return n;
}

extern "C" int galic_ensemble_set_variant(galic_ensemble *e, int variant)
{
  if(!e || variant < 0 || variant >= ensemble_variant_count()) return efail(e, GALIC_ERR_INVALID_ARGUMENT);
  e->variant = variant;
  return efail(e, GALIC_OK);
}

extern "C" int galic_ensemble_calc_all(galic_ensemble *e)
{
  if(!e) return GALIC_ERR_INVALID_ARGUMENT;
  if(!members_unchanged(e)) return efail(e, GALIC_ERR_STATE);
  if(!e->exec || e->graph_variant != e->variant) {
    int st = build_graph(e);
    if(st) return st;
  }
  cudaStream_t s = e->stream;
  for(galic_ctx *c : e->members) ECK(cudaStreamSynchronize(c->stream));  // members' own work first
  ECK(cudaGraphLaunch(e->exec, s));
  ECK(cudaMemcpyAsync(e->h_steps, e->d_steps, e->nmodels * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  ECK(cudaMemcpyAsync(e->h_maxerr, e->d_maxerr, e->nmodels * sizeof(double), cudaMemcpyDeviceToHost, s));
  ECK(cudaMemcpyAsync(e->h_status, e->d_status, e->nmodels * sizeof(int), cudaMemcpyDeviceToHost, s));
  ECK(cudaStreamSynchronize(s));
  float ms_total = -1, ms_orbit = -1;
  if(cudaEventElapsedTime(&ms_total, e->ev[0], e->ev[3]) != cudaSuccess) ms_total = -1;
  if(cudaEventElapsedTime(&ms_orbit, e->ev[1], e->ev[2]) != cudaSuccess) ms_orbit = -1;
  e->last_ms_total = ms_total;
  e->last_ms_orbit = ms_orbit;
  e->last_steps = 0;
  int worst = 0;
  for(int m = 0; m < e->nmodels; m++) {
    galic_ctx *c = e->members[m];
    c->last_steps = (long long) e->h_steps[m];
    c->last_max_egy_err = e->h_maxerr[m];
    c->last_ms_total = ms_total;
    c->last_ms_orbit = ms_orbit;
    e->last_steps += (long long) e->h_steps[m];
    const int st = e->h_status[m] == ORBIT_STEP_CAP ? GALIC_ERR_STEP_CAP
                   : e->h_status[m] == ORBIT_NONFINITE ? GALIC_ERR_INVALID_ARGUMENT
                                                        : GALIC_OK;
    c->status = st;
    c->have_response = (st == GALIC_OK);
    worst = std::max(worst, st);
  }
  return efail(e, worst);
}

extern "C" int galic_ensemble_autotune(galic_ensemble *e, double sample_fraction, int *best, double *ms_per_variant)
{
  if(!e || !(sample_fraction > 0) || sample_fraction > 1) return efail(e, GALIC_ERR_INVALID_ARGUMENT);
  if(!members_unchanged(e)) return efail(e, GALIC_ERR_STATE);
  // the same kernel on the first part of every member's processing order
  EnsembleLaunch S = e->L;
  for(int m = 0; m < e->nmodels; m++) {
    const int n = e->L.offset[m + 1] - e->L.offset[m];
    const int k = std::max(1, std::min(n, (int) (n * sample_fraction + 0.5)));
    S.offset[m + 1] = S.offset[m] + k;
  }
  const int nv = ensemble_variant_count();
  cudaStream_t s = e->stream;
  for(galic_ctx *c : e->members) ECK(cudaStreamSynchronize(c->stream));
  double best_ms = 1e300;
  int best_v = 0;
  for(int v = 0; v < nv; v++) {
    double t = 1e300;
    for(int rep = 0; rep < 2; rep++) {
      ECK(cudaMemsetAsync(e->d_fx, 0, (size_t) e->nmodels * 4 * NG_COMMITTED * e->G * sizeof(FxWord), s));
      ECK(cudaMemsetAsync(e->d_next, 0, sizeof(int), s));
      ECK(cudaEventRecord(e->ev[1], s));
      ECK(launch_ensemble_fp32(S, v, persistent_grid(v, S.offset[e->nmodels], e->device), s));
      ECK(cudaEventRecord(e->ev[2], s));
      ECK(cudaStreamSynchronize(s));
      float ms = 0;
      ECK(cudaEventElapsedTime(&ms, e->ev[1], e->ev[2]));
      t = std::min(t, (double) ms);
    }
    if(ms_per_variant) ms_per_variant[v] = t;
    if(t < best_ms) {
      best_ms = t;
      best_v = v;
    }
  }
  // the sample runs overwrote orbit counts: the members' responses are stale
  for(int m = 0; m < e->nmodels; m++) e->members[m]->have_response = false;
  e->variant = best_v;
  if(best) *best = best_v;
  return efail(e, GALIC_OK);
}

extern "C" int galic_ensemble_last_timing(const galic_ensemble *e, double *ms_total, double *ms_orbit_kernel,
                                          long long *orbit_steps, int *graph_nodes)
{
  if(!e) return GALIC_ERR_INVALID_ARGUMENT;
  if(ms_total) *ms_total = e->last_ms_total;
  if(ms_orbit_kernel) *ms_orbit_kernel = e->last_ms_orbit;
  if(orbit_steps) *orbit_steps = e->last_steps;
  if(graph_nodes) *graph_nodes = (int) e->graph_nodes;
  return GALIC_OK;
}
