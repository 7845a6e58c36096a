// galic_ctx, the context that replaces GALIC's globals, and the helpers that
// api.cu shares with the ensemble layer (ensemble.cu).  Private to the
// library.
#ifndef GALIC_CONTEXT_CUH
#define GALIC_CONTEXT_CUH

#include <cuda_runtime.h>

#include <vector>

#include "galic_gpu.h"
#include "kernels.cuh"
#include "rep.cuh"

struct galic_ctx {
  galic_params_t prm;
  int status = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  int priority = 0;  // of the context's streams
  // second stream of galic_optimize_reps (the orbits of the next window of
  // repetitions) and its events: [0], [1] a half of the scratch committed,
  // [2] the context's stream reached the call's start, [3], [4] a half's
  // orbits done
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev2[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int *d_idx_all = nullptr;               // every particle index of a galic_optimize_reps call
  size_t idx_cap = 0;
  double *d_fit_hist = nullptr;           // [reps][4][7] fits after each repetition
  size_t fit_hist_cap = 0;
  unsigned long long *d_rep_stats = nullptr;  // orbit-steps total, worst orbit status
  DevModel dm{};
  int G = 0, Ns = 0, L = 0;
  // tables
  double2 *d_fg_acc = nullptr;
  double *d_fg_pot = nullptr, *d_vstream[4] = {nullptr, nullptr, nullptr, nullptr};
  double *d_cellsize = nullptr, *d_dist = nullptr;
  double *d_targets = nullptr;    // [4][6][Ns]
  double *d_committed = nullptr;  // [4][10][G]
  double *d_stacks = nullptr;     // [4][10][Ns]
  FxWord *d_fx = nullptr;         // [4][10][G]
  int *d_shift = nullptr;         // [4][10]
  double *d_fit = nullptr;        // [4][7] + raw [4][5]
  int *d_firstrun = nullptr;      // [4]
  unsigned long long *d_counters = nullptr;  // tries[4], changes[4], steps
  int *d_status = nullptr;
  int *d_next = nullptr;
  double *d_maxerr = nullptr;
  double pot_min = 0;
  bool have_fg = false, have_geom = false, have_response = false;
  bool have_targets[4] = {false, false, false, false};
  // particles
  int n = 0;
  double *d_pos = nullptr, *d_vel = nullptr, *d_mass = nullptr, *d_tint = nullptr, *d_vesc = nullptr;
  double *d_ptargets = nullptr, *d_vdisp = nullptr;
  int *d_type = nullptr, *d_orbits = nullptr;
  int *d_order = nullptr;  // orbit processing order of the batched kernels (by initial radius)
  // scratch of the per-orbit drop-ins and the repetition
  int scratch_orbits = 0;
  double *d_b_pos = nullptr, *d_b_vel = nullptr, *d_b_mass = nullptr, *d_b_time = nullptr, *d_grids = nullptr;
  double *d_b_tall = nullptr, *d_b_err = nullptr;
  int *d_b_type = nullptr, *d_b_norbit = nullptr, *d_b_status = nullptr;
  long long *d_b_steps = nullptr;
  int scratch_rep = 0;
  int *d_idx = nullptr, *d_accepted = nullptr, *d_acc_list = nullptr, *d_acc_n = nullptr;
  double *d_vel_try = nullptr, *d_F = nullptr, *d_inst_v = nullptr, *d_inst0 = nullptr, *d_fac = nullptr;
  Cell *d_inst_cell = nullptr;
  // diagnostics
  long long last_steps = 0;
  int last_launches = 0;
  double last_max_egy_err = 0;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  // FP32 form: per type a quad table, 4 float4 per force-grid cell (iz, iR):
  // DPotDR, DPotDz and Vstream[type] of the corners (iz,iR), (iz,iR+1),
  // (iz+1,iR), (iz+1,iR+1), then padding
  std::vector<double> h_dpotdr, h_dpotdz, h_vstream[4];
  float4 *d_tab32[4] = {nullptr, nullptr, nullptr, nullptr};
  float *d_cellsize32 = nullptr;
  bool tab32_dirty = true;
  std::vector<double> h_cellsize;
  double last_ms_total = 0, last_ms_orbit = 0;
  // bumped by every upload; an ensemble built over this context checks it
  unsigned generation = 0;
  // form of a galic_calc_all_shard awaiting galic_calc_all_finish, else -1
  int shard_form = -1;
  // pinned staging for the small per-call transfers (asynchronous copies
  // that do not go through the driver's shared pageable staging)
  char *h_stage = nullptr;
  size_t stage_cap = 0;
  // Jeans tables of get_disp_rtp per type (galic_set_dispersion): FG_Disp_r,
  // FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime, and the
  // largest magnitude of each (fixed-point range of the sampled energy maps)
  double *d_disp[4][5] = {};
  double disp_max[4][5] = {};
  bool have_disp[4] = {false, false, false, false};
  // target stacks written by the samplers: bit 0 DGs_MassTarget, bit 1 the
  // five energy-grid stacks; both make the type's targets complete
  unsigned target_parts[4] = {0, 0, 0, 0};
};

namespace galic_internal {
// galic_ctx_create with a stream priority (the serving loop's jobs)
int ctx_create(const galic_params_t *prm, int priority, galic_ctx **out);
// fixed-point shift of every committed grid of the context for `form`
void set_shifts(galic_ctx *ctx, int *shift, int form);
// FP32 force tables of the context, rebuilt after any table upload
int ensure_tab32(galic_ctx *ctx);
FitArgs make_fit_args(galic_ctx *ctx);
// keeps the device's default memory pool mapped between calls (once per device)
cudaError_t keep_device_pool(int device);
// installs particles whose arrays are on the device, stored type by type
int set_particles_device(galic_ctx *ctx, const int nt[4], const double tmass[4], const double *pos,
                         const double *vel, const double *tint, const double *vesc, const double *targets);
}  // namespace galic_internal

#endif
