/*
 * galic_gpu.h - C ABI of the B200 (sm_100a) implementation of GALIC's
 * orbit-response hot path (libgalic_cuda.so).
 *
 * The reference (denisyurin/GALIC, C99 + MPI) keeps every input of the hot
 * path in globals: the run parameters in `All` (allvars.h:639-836), the
 * tabulated force grid FG_* (grid.c:204-230), the density/energy response
 * grids DG_* / EG_* and their stacks (grid.c:233-325) and the particle array
 * `P` (allvars.h:844-868).  This ABI replaces the globals by a context
 * handle: the caller uploads the same arrays once, in the reference's own
 * layouts, then calls entry points that replace the reference functions named
 * beside each declaration.  All pointers passed in or out are HOST pointers
 * unless a name says otherwise; every array uses the reference's index
 * convention:
 *   force grid  FG[iz * FG_Nbin + iR]                       (grid.c:78-80)
 *   response    grid[iz * DG_Nbin + iR]                     (orbit_response.c:283-286)
 *   stacks      stack[STACKOFFSET(l,i,j)], STACKOFFSET(l,i,j) =
 *               ((1<<2l)-1)/3 + i*2^l + j                   (allvars.h:160)
 *
 * Errors: every entry point returns a galic_status (0 = success) except the
 * per-orbit drop-ins, which return the reference's value (tall) and report a
 * failure as a negative return value plus galic_last_status().  Nothing
 * aborts and no kernel traps: the reference's terminate()/exit(1) paths
 * (orbit_response.c:450-456, main.c:432-433) become status codes.
 *
 * Threading: one context per host thread; a context is not reentrant, as the
 * reference's globals are not.
 */
#ifndef GALIC_GPU_H
#define GALIC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GALIC_OK = 0,
  GALIC_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or parameter */
  GALIC_ERR_STEP_CAP = 2,         /* an orbit exceeded the step cap (reference: >1e8 steps, exit(1)) */
  GALIC_ERR_CUDA = 3,             /* a CUDA runtime call failed */
  GALIC_ERR_NO_DEVICE = 4,        /* no CUDA device visible */
  GALIC_ERR_BUDGET = 5,           /* the request does not fit the HBM budget */
  GALIC_ERR_UNSUPPORTED = 6,      /* configuration the reference rejects with terminate() */
  GALIC_ERR_REJECTION_CAP = 7,    /* velocity proposal loop exceeded 100000 tries (main.c:432), or a
                                     sampler whose draws stopped landing inside Rmax */
  GALIC_ERR_OVERFLOW = 8,         /* a fixed-point response bin left its representable range */
  GALIC_ERR_STATE = 9             /* call out of order (e.g. fit requested before any response) */
} galic_status;

/* Compute forms of the orbit-response path. */
typedef enum {
  GALIC_FORM_FP64 = 0, /* plain FP64, bit-exact per orbit to the CPU restatement (the drop-in) */
  GALIC_FORM_FP32 = 1  /* FP32 integrate / FP64 merit: the batched throughput form */
} galic_form;

/*
 * Parameters of one galaxy model: the subset of the reference's `All`
 * (allvars.h:639-836) and grid globals (allvars.h:300-420) that the hot path
 * reads.  Arrays indexed by particle type use index 1 (halo), 2 (disk),
 * 3 (bulge); index 0 is unused, as in the reference's [6]-sized arrays.
 */
typedef struct galic_params {
  /* structure (structure.c:54-143, init.c:46-54) */
  double V200, M200, R200, G;
  double Halo_Mass, Halo_A, HaloStretch;
  double Disk_Mass;
  double Bulge_Mass, Bulge_A, BulgeStretch;
  /* orbit integration (orbit_response.c:16-26) */
  double TimeStepFactorOrbit, TimeStepFactorCellCross;
  /* optimisation (main.c:365-527, grid.c:1086-1151) */
  double LowerDispLimit, MaxVelInUnitsVesc;
  int SampleForceNhalo, SampleForceNdisk, SampleForceNbulge;
  int TypeOfVelocityStructure[4];
  int MinParticlesPerBinForDispersionMeasurement;
  int MinParticlesPerBinForDensityMeasurement;
  double MType[4];
  int NType[4];
  double fac_value_rs[4], fac_value_ts[4], fac_value_qs[4], fac_value_ps[4];
  /* grid geometry (grid.c:329-487) */
  int FG_Nbin, DG_MaxLevel, EG_MaxLevel;
  double FG_Rmin, FG_Fac, DG_Rmin, DG_Fac, EG_Rmin, EG_Fac;
} galic_params_t;

typedef struct galic_ctx galic_ctx;

/* ---------------------------------------------------------- context */

/* Creates a context on the current CUDA device and validates `prm`.
 * Replaces the reference's global set-up (forcegrid_allocate,
 * densitygrid_allocate, energygrid_allocate: grid.c:204-325). */
int galic_ctx_create(const galic_params_t *prm, galic_ctx **out);
void galic_ctx_destroy(galic_ctx *ctx);
int galic_last_status(const galic_ctx *ctx);
/* copy of the parameters the context was created with */
int galic_get_params(const galic_ctx *ctx, galic_params_t *out);
/* human-readable text of a status code */
const char *galic_status_string(int status);

/* Force grid: FG_Pot, FG_DPotDR, FG_DPotDz, each FG_Nbin^2 doubles
 * (grid.c:59-197, filled by forcedensitygrid_calculate grid.c:621-763). */
int galic_set_force_grid(galic_ctx *ctx, const double *pot, const double *dpotdr, const double *dpotdz);
/* FG_Vstream[type], FG_Nbin^2 doubles (disp_fields.c:118-132). */
int galic_set_vstream(galic_ctx *ctx, int type, const double *vstream);
/* DG_CellSize (DG_Ngrid doubles, grid.c:849) and DGs_Distance
 * (DG_Nstack doubles, grid.c:381-416). */
int galic_set_density_geometry(galic_ctx *ctx, const double *cellsize, const double *dgs_distance);
/* Target stacks of one type, each a full stack (DG_Nstack / EG_Nstack
 * doubles, already smoothed): DGs_MassTarget, EGs_MassTarget,
 * EGs_EgyTarget_{r,t,p,q} (grid.c:830-857, 941-1076). */
int galic_set_targets(galic_ctx *ctx, int type, const double *dgs_mass, const double *egs_mass,
                      const double *egs_r, const double *egs_t, const double *egs_p, const double *egs_q);
/* Particle state P[] (allvars.h:844-868): pos/vel are n x 3 doubles,
 * targets are n x 4 doubles (vr2_target, vt2_target, vp2_target,
 * vq2_target), type in {1,2,3}. */
int galic_set_particles(galic_ctx *ctx, int n, const double *pos, const double *vel, const double *mass,
                        const double *tint, const double *vesc, const int *type, const double *targets);
int galic_get_particles(galic_ctx *ctx, double *vel, int *orbits, double *vdisp /* n x 4: vr2,vt2,vp2,vq2 */);

/* ---------------------------------------------------------- per-orbit drop-ins */

/* Replaces produce_orbit_response_field_mod (orbit_response.c:155-491,
 * proto.h:142-145); same arguments after the context, q before p.  Output
 * grids are caller-owned host arrays of DG_Ngrid (= EG_Ngrid) doubles,
 * zeroed, filled and scaled by mass/tall by the callee.  Returns tall, or a
 * negative value on error (see galic_last_status). */
double galic_produce_orbit_response_field_mod(galic_ctx *ctx, double *pos, double *vel, int id, double *mfield,
                                              double *egyfield_r, double *egyfield_t, double *egyfield_q,
                                              double *egyfield_p, double mass, double timespan,
                                              int *orbitstaken, int type);
/* Replaces produce_orbit_response_field (orbit_response.c:33-151). */
double galic_produce_orbit_response_field(galic_ctx *ctx, double *pos, double *vel, int id, double *mfield,
                                          double mass, double timespan, int *orbitstaken);

/* ---------------------------------------------------------- batched hot path */

/* Replaces calc_all_response_fields (main.c:151-246) including its final
 * calc_global_fit (main.c:251-362): integrates every particle's orbit,
 * bins the time-averaged responses per type with exact fixed-point
 * accumulation, adds the instantaneous energy grid, and evaluates the fit. */
int galic_calc_all_response_fields(galic_ctx *ctx, int form);

/* calc_all_response_fields split for a model sharded over `world` ranks
 * (the reference's MPI layout, main.c:201-231 with the Allreduce of
 * main.c:259-285): galic_calc_all_shard integrates the orbits
 * order[rank + k * world] and the instantaneous energy of particles
 * rank, rank + world, ... into the context's fixed-point accumulators
 * (zeroed first); the caller sums the accumulators of all ranks elementwise
 * as 64-bit integers (galic_accumulators gives their device address and
 * count of int64 words: exact, so the sum equals a one-rank pass bit for bit)
 * and then calls galic_calc_all_finish on every rank, which converts them to
 * the committed grids and evaluates calc_global_fit.  Per-particle state
 * written by the pass (orbit counts, instantaneous dispersions) is valid for
 * the rank's own particles only. */
int galic_calc_all_shard(galic_ctx *ctx, int form, int rank, int world);
int galic_accumulators(galic_ctx *ctx, void **device_ptr, size_t *words);
int galic_calc_all_finish(galic_ctx *ctx);

/* One optimisation repetition: init_updates (main.c:844-874), optimize(n)
 * for n = idx[0..count-1] (main.c:365-527) and commit_updates
 * (main.c:808-841), which ends in calc_global_fit.  Proposals for idx[k] are
 * drawn from Philox stream (seed, idx[k], rep_serial).  All count
 * particles are evaluated against the committed state, as in the reference
 * (accepted changes only reach `_delta` grids until the commit).  form:
 * GALIC_FORM_FP64 integrates the old and trial orbits bit-exactly as the
 * CPU restatement; GALIC_FORM_FP32 integrates them in the FP32 form (the
 * merit function and the commit stay FP64). */
int galic_optimize_rep(galic_ctx *ctx, const int *idx, int count, uint64_t seed, uint32_t rep_serial, int form);

/* `reps` consecutive repetitions of `count` particles each: the loop body of
 * main.c:94-100 (init_updates, optimize_some_particles, commit_updates) run
 * reps times.  Repetition r optimises idx[r*count .. r*count+count-1] with
 * proposal streams (seed, n, rep_serial + r); the result equals reps calls of
 * galic_optimize_rep bit for bit.  The library integrates the old and trial
 * orbits of a window of repetitions in one launch (a proposal depends only
 * on P[n].Pos, the targets and its stream, and the old orbit on P[n].Vel,
 * which only n's own optimisation changes), then evaluates, accepts and
 * commits the repetitions in order; the orbits of the next window run on a
 * second stream meanwhile.  A window ends before a particle repeats and when
 * its per-orbit grids (2 x 5 x DG_Ngrid doubles per particle) would pass
 * window_bytes (0: 4 GiB; at least one repetition); two windows' grids are
 * held at once.  fits, when not NULL, receives the 4 x 7 galic_get_fit
 * values after every repetition ([reps][4][7]; GALIC logs them per
 * iteration, main.c:1220-1285).  No counterpart function in the reference:
 * it replaces the loop of main.c:94-100 (optimize_some_particles,
 * main.c:120-146, is the caller's choice of idx). */
int galic_optimize_reps(galic_ctx *ctx, const int *idx, int count, int reps, uint64_t seed, uint32_t rep_serial,
                        int form, size_t window_bytes, double *fits);

/* Merit values of the last calc_global_fit: per type (index 1..3)
 * S, Sdisp_r, Sdisp_t, Sdisp_p, Sdisp_q, Srelfac, Srelfac_count
 * (main.c:294-358): out is 4 x 7 doubles, row = type. */
int galic_get_fit(galic_ctx *ctx, double *out);
/* Counters of optimize (main.c:468, 505): tries[4], changes[4]. */
int galic_get_counters(galic_ctx *ctx, long long *tries, long long *changes);

/* Committed response grids of one type (DG_Ngrid doubles each), the
 * reference's DG_MassLoc, EG_EgyResponse{R,T,Q,P}LocS, EG_MassLoc,
 * EG_EgyResponse{R,T,P,Q}Loc; `which` selects one of them (galic_grid_id). */
typedef enum {
  GALIC_GRID_MASS_S = 0, GALIC_GRID_R_S, GALIC_GRID_T_S, GALIC_GRID_Q_S, GALIC_GRID_P_S,
  GALIC_GRID_MASS_I, GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I, GALIC_GRID_Q_I,
  GALIC_GRID_COUNT
} galic_grid_id;
int galic_get_response(galic_ctx *ctx, int type, int which, double *out);

/* Per-orbit step cap (reference: 1e8 steps, orbit_response.c:450, then
 * exit(1)); an orbit that exceeds it ends with GALIC_ERR_STEP_CAP. */
int galic_set_step_cap(galic_ctx *ctx, long long cap);

/* Total orbit steps taken by the last batched call (for throughput). */
long long galic_last_orbit_steps(const galic_ctx *ctx);
/* Device time of the last galic_calc_all_response_fields, measured with CUDA
 * events on the library's stream: the whole call and its orbit kernel (ms). */
int galic_last_timing(const galic_ctx *ctx, double *ms_total, double *ms_orbit_kernel);
/* Largest relative orbit energy error of the last batched call
 * (orbit_response.c:460-462; the reference only prints it above 0.5). */
double galic_last_max_energy_error(const galic_ctx *ctx);
/* Number of kernels launched by the last batched call. */
int galic_last_kernel_launches(const galic_ctx *ctx);

/* ---------------------------------------------------------- allocation-free variant */

/* No counterpart in the reference.  The orbit-response binning of
 * galic_calc_all_response_fields (time-averaged grids only, no fit) for
 * callers that cannot allocate device memory: a host framework that owns
 * every device allocation through its own pool, or a process with a
 * device-memory budget fixed in advance.  Every pointer named d_* is
 * caller-owned DEVICE memory:
 *   d_fg_acc2   FG_DPotDR / FG_DPotDz interleaved: [FG_Nbin^2][2]
 *   d_fg_pot    FG_Pot [FG_Nbin^2]
 *   d_vstream   FG_Vstream of types 1..3: [3][FG_Nbin^2]
 *   d_cellsize  DG_CellSize [DG_Ngrid]
 *   particles   d_pos/d_vel [n][3], d_mass, d_tint [n], d_type [n] in 1..3
 *   d_out       [3 types][5][DG_Ngrid]: DG_MassLoc, EG_EgyResponse{R,T,Q,P}LocS
 *   d_orbits    [n] orbit counts, may be NULL
 * phi_bound must be at least max|FG_Pot| (for example -min FG_Pot); it sets
 * the fixed-point range as the context path does, and a bound too small to
 * hold the bins gives GALIC_ERR_OVERFLOW.  A particle whose type is outside
 * 1..3, whose Tint is not positive and finite or whose mass is not finite is
 * skipped and the call returns GALIC_ERR_INVALID_ARGUMENT.  Step counts and
 * energy errors are not returned.  stream is a cudaStream_t (NULL = legacy
 * default stream); the call returns after the stream has finished.
 * Working memory is one file-scope device array of fixed size (3.75 MiB +
 * 256 B per device, kept until exit): DG_MaxLevel > 7 is rejected with
 * GALIC_ERR_BUDGET.  The first call on a device looks up the array's device
 * address; make it before any stream capture.  That address is stale after
 * cudaDeviceReset (reload the library).  Calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
int galic_orbit_responses_noalloc(const galic_params_t *prm, const double *d_fg_acc2, const double *d_fg_pot,
                                  const double *d_vstream, const double *d_cellsize, double phi_bound, int n,
                                  const double *d_pos, const double *d_vel, const double *d_mass,
                                  const double *d_tint, const int *d_type, double *d_out, int *d_orbits,
                                  void *stream);

/* ------------------------------------------------------- ensembles */

/* An ensemble advances up to 64 contexts (galaxy models of any particle
 * counts, same device, same DG_MaxLevel) together: one iteration is
 * calc_all_response_fields with its calc_global_fit (main.c:151-362) for
 * every member in the FP32 form, run as ONE persistent orbit launch over the
 * orbits of all members plus each member's read-out and merit kernels, and
 * replayed from a CUDA graph after the first call.  Each member's results
 * (galic_get_fit / galic_get_response / galic_get_particles on the member)
 * are identical to what galic_calc_all_response_fields(member,
 * GALIC_FORM_FP32) gives, whatever the other members and the tile variant.
 * No counterpart in the reference (one model per MPI job).  Uploading to a
 * member after galic_ensemble_create makes the ensemble return
 * GALIC_ERR_STATE; build a new one.  The members must outlive the ensemble. */
typedef struct galic_ensemble galic_ensemble;
int galic_ensemble_create(galic_ctx *const *members, int count, galic_ensemble **out);
void galic_ensemble_destroy(galic_ensemble *e);
int galic_ensemble_last_status(const galic_ensemble *e);
/* one iteration of every member */
int galic_ensemble_calc_all(galic_ensemble *e);
/* tile variants of the orbit kernel (threads per CTA, CTAs per SM asked of
 * the register allocator); returns their count, fills up to max entries */
int galic_ensemble_variants(int *block, int *min_blocks, int max);
int galic_ensemble_set_variant(galic_ensemble *e, int variant);
/* times every variant on the first sample_fraction of each member's orbits
 * (ms_per_variant may be NULL) and selects the fastest; the members'
 * responses must be recomputed afterwards */
int galic_ensemble_autotune(galic_ensemble *e, double sample_fraction, int *best, double *ms_per_variant);
/* device times of the last iteration (CUDA events in the graph), orbit-steps
 * summed over the members, and the number of nodes of the graph */
int galic_ensemble_last_timing(const galic_ensemble *e, double *ms_total, double *ms_orbit_kernel,
                               long long *orbit_steps, int *graph_nodes);

/* ------------------------------------------------------- serving */

/* One model-construction job: GALIC's run (main.c:69-107) from the point
 * where the grids and the initial particles exist.  Arrays are in the
 * layouts of the galic_set_* calls and must stay valid until the job is
 * done.  No counterpart in the reference (one model per MPI job). */
typedef struct {
  const galic_params_t *prm;
  const double *fg_pot, *fg_dpotdr, *fg_dpotdz;  /* FG_Nbin^2 each */
  const double *vstream[4];                      /* [1..3]; NULL = zero */
  const double *cellsize, *dgs_distance;         /* DG_Ngrid, DG_Nstack */
  const double *targets[4][6];                   /* [type 1..3]: DGs_Mass, EGs_Mass, r, t, p, q stacks */
  int n;
  const double *pos, *vel, *mass, *tint, *vesc, *ptargets;
  const int *type;
  int form;                  /* form of calc_all_response_fields and of the repetitions' orbits */
  int max_iterations;        /* All.MaximumNumberOfSteps */
  int reps_per_iteration;    /* All.IndepenentOptimizationsPerStep */
  double fraction_per_rep;   /* All.FractionToOptimizeIndependendly: n_per_cpu = 1 + f n (main.c:129) */
  double converge_rel;       /* stop after an iteration that lowers Sall by less than this fraction; 0 = never */
  uint64_t seed;             /* proposal streams (seed, particle, repetition) */
  const int *permutation;    /* optimisation order (main.c:137-139); NULL = 0..n-1 */
  double *vel_out;           /* n x 3 final velocities, or NULL */
} galic_job_t;

typedef struct {
  int status;                /* galic_status of the job */
  int iterations;
  long long reps;
  long long orbit_steps;     /* calc_all and every repetition */
  double sall_first, sall_last;  /* Sall (main.c:1270) summed over types, after calc_all / at the end */
  double fit[28];            /* galic_get_fit at the end */
  double t_submit, t_admit, t_first_response, t_done;  /* seconds since the server started */
} galic_job_result_t;

/* Worker threads run admitted jobs concurrently on the current device; a
 * queued job is admitted (first fit, in arrival order) when a worker is free
 * and its device footprint (galic_job_device_bytes) fits what the running
 * jobs leave of hbm_budget_bytes.  A job larger than the whole budget ends
 * with GALIC_ERR_BUDGET. */
typedef struct galic_server galic_server;
int galic_server_create(size_t hbm_budget_bytes, int workers, galic_server **out);
int galic_server_submit(galic_server *s, const galic_job_t *job, int *job_id);
/* waits up to timeout_s for the job; GALIC_ERR_STATE if it is not done */
int galic_server_wait(galic_server *s, int job_id, double timeout_s, galic_job_result_t *res);
int galic_server_stats(galic_server *s, size_t *peak_bytes, int *peak_running, int *queued, int *running);
/* finishes every submitted job, then stops the workers */
void galic_server_destroy(galic_server *s);
/* device bytes the server reserves for a job */
size_t galic_job_device_bytes(const galic_job_t *job);

/* ------------------------------------------------------- force-grid fill */

/* Parameters of the tree force-grid fill, from `All` and the grid globals. */
typedef struct {
  int FG_Nbin;            /* FG_Nbin (grid.c:204) */
  int MultipleDomains;    /* All.MultipleDomains (domain_toplevel.c:79) */
  double FG_Rmin, FG_Fac; /* FG_Rmin, FG_Fac (grid.c:466-470) */
  double G;               /* All.G (gravtree.c:456-463) */
  double ForceSoftening;  /* All.ForceSoftening = 2.8 * All.Softening (init.c:83) */
  double ErrTolTheta;     /* All.ErrTolTheta (forcetree_walk.c:109) */
  double TopNodeFactor;   /* All.TopNodeFactor (domain_toplevel.c:79) */
} galic_fill_params_t;

/* Diagnostics of one fill. */
typedef struct {
  double ms_walk;            /* device time of the tree walk (CUDA events) */
  double ms_total;           /* host time of the whole call */
  long long tree_items;      /* nodes + single-particle leaves of the tree */
  long long tree_nodes;      /* internal nodes (forcetree.c Tree_NumNodes) */
  long long interactions;    /* particle/node interactions summed over the probes */
  long long node_tests;      /* opening tests summed over the probes */
} galic_fill_stats_t;

/* Replaces the tree part of forcedensitygrid_calculate (grid.c:621-750):
 * places the FG_Nbin^2 x 8 massless probe points of grid.c:680-704 beside
 * the n sampled mass particles (pos[3n], mass[n], in the reference's P order:
 * halo, disk, bulge, as drawn by grid.c:662-678), runs gravity()
 * (gravtree.c:35-50) with one MPI rank, and writes the section-averaged
 * FG_DPotDR, FG_DPotDz, FG_Pot (FG_Nbin^2 each, [iz * FG_Nbin + iR]).  The
 * results are bit-identical to the single-rank reference.  stats may be
 * NULL.  Mass particles closer than DomainLen / 2^30 to one another (the
 * MAX_TREE_LEVEL case of forcetree.c:400-416) give GALIC_ERR_UNSUPPORTED. */
int galic_force_grid_fill(const galic_fill_params_t *fp, int n, const double *pos, const double *mass,
                          double *fg_dpotdr, double *fg_dpotdz, double *fg_pot, galic_fill_stats_t *stats);

/* peano_hilbert_key (peano.c:331-347) of the integer cell (x, y, z) with
 * `bits` bits per dimension (bits <= 21). */
uint64_t galic_peano_hilbert_key(int x, int y, int z, int bits);

/* ------------------------------------------------------- target sampling */

/* Component shapes and limits read by the coordinate samplers and by
 * get_disp_rtp (All.* of allvars.h:650-720). */
typedef struct {
  double Rmax;                  /* All.Rmax (grid.c:329-340) */
  double Halo_A, HaloStretch;   /* halo.c:17-40 */
  double Disk_Z0, Disk_H;       /* disk.c:17-50 */
  double Bulge_A, BulgeStretch; /* bulge.c:15-37 */
  double HaloBetaParameter, BulgeBetaParameter; /* get_beta_of_type, disp_fields.c:26-60 */
} galic_sample_params_t;

/* A position in a random stream.  GALIC draws every random number from one
 * sequential generator (random_generator, init.c:25-27).  This library's
 * stand-in is the Philox4x32-10 stream keyed by (seed, a, b) whose k-th
 * uniform double can be computed without the ones before it, so the
 * reference's sequential sampling loops are replayed in parallel and give
 * the same samples.  `position` is the index of the next uniform; every call
 * that draws advances it past the last uniform the reference loop would
 * have consumed. */
typedef struct {
  uint64_t seed;
  uint32_t a, b;
  uint64_t position;
} galic_stream_t;

/* Jeans tables of one type read by get_disp_rtp (disp_fields.c:66-198,
 * 375-398), each FG_Nbin^2 doubles laid out [iz * FG_Nbin + iR]
 * (FG_Disp_r: only its first FG_Nbin entries are read, by spherical radius
 * bin): FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime,
 * FG_tilted_vz2_prime.  A table that the type's velocity structure does
 * not read may be NULL (structure 0 and 1 read disp_r; 2 reads dispz and
 * dispphi; 3 reads tilted_vr2, tilted_vz2 and dispphi).  FG_Vstream[type]
 * comes from galic_set_vstream. */
int galic_set_dispersion(galic_ctx *ctx, int type, const double *disp_r, const double *dispz, const double *dispphi,
                         const double *tilted_vr2, const double *tilted_vz2);

/* Replaces densitygrid_sample_targetresponse (grid.c:536-617) with one rank.
 * For each type 1..3 with MType[type] > 0, in that order, draws coordinates
 * from `stream` as the reference's loop does until ntarget of them lie
 * inside Rmax (the reference's ntarget is SampleParticleCount / NTask + 1),
 * bins them bilinearly into the density grid, scales by MType / ntarget,
 * smooths the stack (grid.c:1247-1265) and stores it as the type's
 * DGs_MassTarget.  renormalize != 0 also applies the recalibration that
 * forcedensitygrid_calculate makes next (grid.c:862-880: the finest level
 * times MType / its sum, coarser levels unchanged).  Bins are exact
 * fixed-point sums (the reference sums in draw order; the two agree to
 * ~1e-13 relative).  GALIC_ERR_REJECTION_CAP when the samples stop landing
 * inside Rmax (the reference would loop for ever). */
int galic_sample_density_targets(galic_ctx *ctx, const galic_sample_params_t *sp, long long ntarget,
                                 galic_stream_t *stream, int renormalize);

/* Replaces calc_energy_grid_mass_maps (grid.c:941-1076) with one rank: as
 * above on the energy grid, each sample depositing its bilinear weights and
 * the weights times get_disp_rtp's four dispersions; stores EGs_MassTarget
 * and EGs_EgyTarget_{r,t,p,q} of every sampled type.  Needs
 * galic_set_dispersion for each sampled type. */
int galic_sample_energy_targets(galic_ctx *ctx, const galic_sample_params_t *sp, long long ntarget,
                                galic_stream_t *stream);

/* Copies the context's target stacks of one type (each Nstack doubles) to
 * host arrays; a NULL array is skipped. */
int galic_get_targets(galic_ctx *ctx, int type, double *dgs_mass, double *egs_mass, double *egs_r, double *egs_t,
                      double *egs_p, double *egs_q);

/* Replaces n calls of halo_get_fresh_coordinate (halo.c:17-40, type 1),
 * disk_get_fresh_coordinate (disk.c:17-50, type 2) or
 * bulge_get_fresh_coordinate (bulge.c:15-37, type 3): the mass-particle
 * positions that forcedensitygrid_calculate draws (grid.c:659-678), on the
 * current device.  pos: host array of 3n doubles. */
int galic_sample_positions(const galic_sample_params_t *sp, int type, long long n, galic_stream_t *stream,
                           double *pos);

/* ------------------------------------------------------- Jeans solvers */

/* Parameters of calculate_dispfield beyond galic_params_t and
 * galic_sample_params_t, indexed by type 1..3. */
typedef struct {
  double StreamingVelocityParameter[4]; /* All.{Halo,Disk,Bulge}StreamingVelocityParameter (disp_fields.c:570-575) */
  double DispersionRoverZratio[4];      /* All.{Halo,Disk,Bulge}DispersionRoverZratio (disp_fields.c:1051-1105) */
} galic_jeans_params_t;

/* The Jeans tables of one type, FG_Nbin^2 doubles each in [iz * FG_Nbin + iR]
 * (FG_Disp_r: its first FG_Nbin entries, by radius bin); NULL skips a table. */
typedef struct {
  double *disp_r, *dispz, *dispphi, *vstream;
  double *tilted_vz2, *tilted_vR2, *tilted_vz2_prime, *tilted_vR2_prime;
} galic_jeans_tables_t;

/* Replaces calculate_dispfield (disp_fields.c:502-1049): the spherical
 * Jeans equation with anisotropy beta (FG_Disp_r), the axisymmetric
 * f(E, Lz) solution (FG_DispZ, and FG_DispPhi / FG_Vstream) for every type
 * with particles, and for velocity structure 3 the method-of-lines solution
 * of the tilted (f(E, Lz, I3)) case (FG_tilted_*, and FG_DispPhi / FG_Vstream
 * again, VER_1_1 form).  Reads the context's force grid (galic_set_force_grid)
 * and the densities of halo.c / disk.c / bulge.c.  The results replace the
 * context's FG_Vstream and Jeans tables, as galic_set_vstream and
 * galic_set_dispersion would; out, when not NULL, is indexed by type (1..3)
 * and receives copies.  GALIC_ERR_UNSUPPORTED for velocity structure 3 with
 * a zero DispersionRoverZratio (the reference's terminate()). */
int galic_calculate_dispfield(galic_ctx *ctx, const galic_sample_params_t *sp, const galic_jeans_params_t *jp,
                              galic_jeans_tables_t *out);

/* ------------------------------------------------- particle initialisation */

/* The particle state initialize_particles writes (P[], allvars.h:844-868, and
 * permutation[], allvars.h:525-530), host arrays of NumPart entries (times 3
 * or 4 where noted), in P order; a NULL array is skipped. */
typedef struct {
  double *pos;       /* 3n: P[].Pos */
  double *vel;       /* 3n: P[].Vel */
  double *vel_theo;  /* 3n: P[].VelTheo (halo particles; 0 for the others) */
  double *mass;      /* n: P[].Mass */
  double *vesc;      /* n: P[].Vesc */
  double *tint;      /* n: P[].Tint */
  double *targets;   /* 4n: P[].vr2_target, vt2_target, vp2_target, vq2_target */
  int *type;         /* n: P[].Type */
  int *id;           /* n: P[].ID */
  int *permutation;  /* n: permutation[].index after the sort (set_particles.c:298-303) */
  int low_disp[4][4]; /* per type: particles whose r, t, p, q dispersion was raised to LowerDispLimit */
} galic_particles_out_t;

/* Replaces initialize_particles (set_particles.c:15-307) with one rank:
 * NType[t] particles of each type in P order (halo, disk, bulge), each with
 * its position (the type's *_get_fresh_coordinate), Vesc and Tint
 * (TorbitFac), for halo particles VelTheo from the Hernquist distribution
 * function (halo.c:168-184), the Jeans dispersion targets (get_disp_rtp,
 * raised to LowerDispLimit) and a velocity from three Gaussians redrawn while
 * faster than MaxVelInUnitsVesc Vesc; then one uniform per particle and the
 * permutation sorted by it.  The draws are those the reference's sequential
 * loop takes from `stream`, which comes back advanced past them.  Needs the
 * force grid and, per type with particles, FG_Vstream and the Jeans tables
 * (galic_set_vstream + galic_set_dispersion, or galic_calculate_dispfield).
 * The particles become the context's, as after galic_set_particles.
 * GALIC_ERR_UNSUPPORTED when more than 5 % of a type had a dispersion raised
 * to LowerDispLimit (the reference's endrun(), set_particles.c:261-282);
 * GALIC_ERR_REJECTION_CAP when a rejection loop on the draws' path ran past
 * 10^6 tries (where the reference would keep drawing). */
int galic_initialize_particles(galic_ctx *ctx, const galic_sample_params_t *sp, double TorbitFac,
                               galic_stream_t *stream, galic_particles_out_t *out);

/* ---------------------------------------------------------- output files */

/* Replaces write_file (io.c:906-1243) as output_particles calls it with one
 * rank and NumFilesPerSnapshot = 1 (io.c:460-540): a Gadget snapshot of
 * SnapFormat 1 or 2, the header followed by the blocks POS, VEL, ID, MASS
 * (types with mass_table[t] == 0; mass_table NULL: all zero, as GALIC never
 * sets All.MassTable) and VELT in single precision, particles grouped by type
 * in their order.  Host arrays as galic_particles_out_t holds them.  The
 * reference names the file OutputDir + OutputFile + "_%03d" (io.c:513). */
int galic_write_snapshot(const char *fname, int snap_format, int n, const double *pos, const double *vel,
                         const double *vel_theo, const double *mass, const int *id, const int *type,
                         const double *mass_table);
/* forcefield.dat (grid.c:789-823): FG_Nbin, FG_DPotDR, FG_DPotDz, FG_Pot, the
 * analytic halo's potential derivatives and potential at the grid points
 * (grid.c:766-786), and the points' R and z. */
int galic_write_forcefield(const char *fname, const galic_params_t *prm, const double *dpotdr, const double *dpotdz,
                           const double *pot);
/* densfield_<type>_<num>.dat of one type (io.c:36-460, without the optional
 * gnuplot output): the DG target stack level by level, the variable-
 * resolution (calc_smoothed_stack, grid.c:1217-1243) target and response,
 * the fine response, the DG and EG cell centres, and the variable-resolution
 * target and response of the energy-grid mass, r, t, p, q.  dgs_target: the
 * DG target stack; egs_targets: 5 EG target stacks (mass, r, t, p, q);
 * dg_mass_loc: the committed time-averaged DG mass grid; eg_loc: 5 committed
 * instantaneous EG grids (mass, r, t, p, q), which become the response stacks
 * as calc_global_fit builds them (main.c:259-289). */
int galic_write_density_field(const char *fname, const galic_params_t *prm, int type, const double *dgs_target,
                              const double *egs_targets, const double *dg_mass_loc, const double *eg_loc);
/* Replaces output_density_field (io.c:36-460) for dump number num: writes
 * outdir/densfield_<type>_<num>.dat for every type with particles from the
 * context's targets and committed grids. */
int galic_output_density_field(galic_ctx *ctx, const char *outdir, int num);

/* ---------------------------------------------------------- host helpers */

/* Grid geometry of forcedensitygrid_create (grid.c:329-480): from Halo_A,
 * the enclosed-mass fractions and the bin counts computes Rmax, DG_Rin,
 * the spacing factors and Rmin of the DG, FG and EG grids.
 * out: Rmax, DG_Rin, DG_Fac, DG_Rmin, FG_Fac, FG_Rmin, EG_Fac, EG_Rmin. */
int galic_grid_geometry(double halo_a, double outer_frac, double inner_frac, int fg_nbin, int dg_maxlevel,
                        int eg_maxlevel, double *out);
/* DGs_Distance stack (grid.c:381-416) and DG_CellSize/DG_CellVol
 * (grid.c:830-850) for DG_MaxLevel with spacing (dg_rmin, dg_fac). */
int galic_density_geometry(int dg_maxlevel, double dg_rmin, double dg_fac, double *dgs_distance,
                           double *cellsize, double *cellvol);
/* smooth_stack (grid.c:1247-1265) on a host stack, in place. */
void galic_smooth_stack(double *data, int maxlevel);

#ifdef __cplusplus
}
#endif
#endif
