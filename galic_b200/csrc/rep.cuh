// Arguments of one optimisation repetition on the device.
#ifndef GALIC_REP_CUH
#define GALIC_REP_CUH

#include <stdint.h>

#include "kernels.cuh"

struct RepArgs {
  int count;
  const int *idx;  // particles optimised in this repetition
  uint64_t seed;
  uint32_t rep_serial;
  // particles per repetition when idx spans a window of repetitions
  // (particle k draws from stream serial rep_serial + k / per_rep); 0: one
  int per_rep = 0;
  // particle state P[] (device)
  const double *p_pos;
  double *p_vel;
  const double *p_mass, *p_tint, *p_vesc, *p_targets;
  double *p_vdisp;
  const int *p_type;
  int *p_orbits;
  // 2*count orbits: [2k] old velocity, [2k+1] trial velocity
  double *b_pos, *b_vel, *b_mass, *b_time;
  int *b_type, *b_norbit;
  double *grids;  // 2*count x NF_ORBIT x Ngrid, unscaled (the kernels multiply by b_mass / b_tall)
  const double *b_tall;  // 2*count: each orbit's tall
  double *fac;           // 2*count: mass / tall of each orbit (k_accept, for the commit)
  double *vel_try;  // count x 3
  double *F;        // 2*count x 9: the stack terms of F_base, F_try (fit_fp64.cu:k_eval_terms)
  double *inst0;    // [4 types][4]: the committed instantaneous terms of the base evaluations
  int *accepted;    // count
  int *acc_list;    // count: the accepted positions k in increasing order (k_compact)
  int *acc_n;       // one per repetition of the window: the length of its acc_list
  double *inst_v;   // count x 4
  Cell *inst_cell;  // count
  unsigned long long *tries, *changes;  // [4]
  double fac_rs[4], fac_ts[4], fac_qs[4], fac_ps[4];
  int *status;
};

// quad32/cellsize32 non-null: the orbits of the repetition in the FP32 form
int launch_rep(const DevModel &M, const RepArgs &R, const FitArgs &f, const OrbitBatch &b, cudaStream_t s,
               const float4 *const *quad32 = nullptr, const float *cellsize32 = nullptr);
// the two halves of launch_rep: proposals and the old/trial orbits of R.count
// particles (which may span several repetitions, see per_rep), then the
// evaluation, acceptance and commit of ONE repetition whose arrays R points at
int launch_rep_orbits(const DevModel &M, const RepArgs &R, const OrbitBatch &b, cudaStream_t s,
                      const float4 *const *quad32 = nullptr, const float *cellsize32 = nullptr);
int launch_rep_commit(const DevModel &M, const RepArgs &R, const FitArgs &f, cudaStream_t s);
// R restricted to the `count` particles of window positions first ..
// first + count - 1 (G: bins per grid)
RepArgs rep_slice(const RepArgs &R, int first, int count, int G);

#endif
