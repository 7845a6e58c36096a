// Launch wrappers shared by the C-ABI layer (api.cu) and the kernel files.
#ifndef GALIC_KERNELS_CUH
#define GALIC_KERNELS_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "fixedpoint.cuh"
#include "galic_gpu.h"
#include "model.cuh"

// field order of the per-orbit grids: the argument order of
// produce_orbit_response_field_mod (orbit_response.c:155-157): m, r, t, q, p
enum { F_M = 0, F_R = 1, F_T = 2, F_Q = 3, F_P = 4, NF_ORBIT = 5 };
// committed per-type grids, in galic_grid_id order
enum { NG_COMMITTED = 10 };
// threads per CTA of the persistent orbit kernels
#define CALC_ALL_BLOCK_FP64 128
#define CALC_ALL_BLOCK_FP32 128
#ifndef GALIC_FP64_MIN_BLOCKS
// 4 CTAs of 128 threads per SM (128 registers, a few spilled) ran the
// halo + disk pass 10 % faster than 3 CTAs at 156 registers
#define GALIC_FP64_MIN_BLOCKS 4
#endif
#ifndef GALIC_FP32_MIN_BLOCKS
// 5 CTAs per SM (96 registers, none spilled; 5 x 31 KiB of queues) ran the
// FP32 pass 2 % faster than 4 (105 registers); 6 (80 registers, spills) 18 %
// slower
#define GALIC_FP32_MIN_BLOCKS 5
#endif
// target stacks per type: DGs_MassTarget, EGs_MassTarget, EGs_EgyTarget_{r,t,p,q}
enum { T_DGM = 0, T_EGM = 1, T_R = 2, T_T = 3, T_P = 4, T_Q = 5, NT_TARGET = 6 };

struct OrbitBatch {
  int count;
  const double *pos, *vel;    // count x 3
  const double *mass, *timespan;
  const int *type;
  double *grids;              // count x NF_ORBIT x DG_Ngrid (zeroed by the caller)
  double *tall;               // count
  int *norbit;                // count
  long long *steps;           // count
  double *egy_err;            // count
  int *status;                // count
  int with_egy;               // produce_orbit_response_field_mod (1) or _field (0)
};

struct CalcAllArgs {
  int n;                      // orbits of this launch: order[first + k * stride], k < n
  int first = 0, stride = 1;
  const double *pos, *vel, *mass, *tint;
  const int *type;
  const int *order;           // processing order (longest first)
  int *next;                  // work counter, zeroed by the caller
  FxWord *fx;                 // [4][NG_COMMITTED][Ngrid]
  const int *shift;           // [4][NG_COMMITTED]
  int *orbits;                // per particle
  unsigned long long *steps_total;
  double *max_egy_err;        // max relative energy error (as ordered bits)
  int *status;                // worst OrbitStatus seen
};

struct FitArgs {
  int L;                      // DG_MaxLevel == EG_MaxLevel
  int Ngrid, Nstack;
  const double *committed;    // [4][10][Ngrid]
  double *stacks;             // [4][10][Nstack]
  const double *targets;      // [4][6][Nstack]
  const double *dgs_distance; // [Nstack]
  double *fit;                // [4][7]
  int *firstrun;              // [4]
  double thr_d[4], thr_e[4], MType[4];
  int present[4], tovs[4];
  double R200_20, LowerDispLimit;
};

void launch_orbits_dense(const DevModel &M, const OrbitBatch &b, cudaStream_t s);
// the same orbits in the FP32 form (orbit_fp32.cu), with egy fields
void launch_orbits_dense_fp32(const DevModel &M64, const float4 *const quad[4], const float *cellsize32,
                              const OrbitBatch &b, cudaStream_t s);
void launch_scale_dense(const DevModel &M, const OrbitBatch &b, cudaStream_t s);
int launch_calc_all_fp64(const DevModel &M, const CalcAllArgs &a, int grid, int block, cudaStream_t s);
// particles first, first + stride, ... below n
void launch_instantaneous(const DevModel &M, int n, const double *pos, const double *vel, const double *mass,
                          const int *type, double *vdisp, FxWord *fx, const int *shift, int Ngrid, cudaStream_t s,
                          int first = 0, int stride = 1);
void launch_fx_finalize(const FxWord *fx, const int *shift, double *committed, int count, int Ngrid, cudaStream_t s);
int launch_global_fit(const FitArgs &f, cudaStream_t s);
cudaError_t prepare_fit_kernels();
int calc_all_occupancy(int block);
int calc_all_fp32_occupancy(int block);
int launch_calc_all_fp32(const DevModel &M64, const float4 *const quad[4], const float *cellsize32,
                         const CalcAllArgs &a, int grid, int block, cudaStream_t s);

// ---- ensemble of models in one persistent FP32 launch (orbit_fp32.cu)
#define GALIC_ENSEMBLE_MAX 64
struct EnsembleLaunch {
  int nmodels;
  int offset[GALIC_ENSEMBLE_MAX + 1];  // prefix sums of the models' orbit counts
  DevModel dm[GALIC_ENSEMBLE_MAX];
  const float4 *quad[GALIC_ENSEMBLE_MAX][4];
  const float *cellsize32[GALIC_ENSEMBLE_MAX];
  const void *members;  // device array of ensemble_member_bytes() per model
  int *next;
  FxWord *fx;           // [models * 4][NG_COMMITTED][Ngrid]
  const int *shift;     // [models * 4][NG_COMMITTED]
  unsigned long long *steps;
  double *maxerr;
  int *status;
};
int ensemble_variant_count();
int ensemble_variant(int v, int *block, int *min_blocks);
int ensemble_occupancy(int v);
size_t ensemble_member_bytes();
void ensemble_fill_member(void *dst, const DevModel &dm, const double *pos, const double *vel, const double *mass,
                          const double *tint, const int *type, const int *order, int *orbits);
cudaError_t launch_ensemble_fp32(const EnsembleLaunch &L, int v, int grid, cudaStream_t s);

#endif
