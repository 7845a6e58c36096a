/*
 * galic_oracle.h - CPU restatement of GALIC's orbit-response hot path.
 *
 * TEST INFRASTRUCTURE: the checker for the CUDA kernels.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * oracle/liboracle.so; the product library never links it.
 *
 * Every function restates the reference function cited beside it, operation
 * for operation and in the same order, so that with `use_libm = 1` (glibc's
 * log/atan2/sin/cos/acos, like the reference) its outputs are bit-identical to
 * the reference's own C compiled in oracle/_ref (pinned by
 * tests/test_oracle_vs_reference.py and the golden fixtures), and with
 * `use_libm = 0` (the project's gmath.h functions, like the CUDA kernels) it
 * is the bit-exact per-orbit reference for the FP64 CUDA path.
 *
 * The reference's globals (All, FG_*, DG_*, EG_*, P, ...) live in an
 * orc_model; the per-type arrays are indexed by type 1..3 as in the
 * reference.
 */
#ifndef GALIC_ORACLE_H
#define GALIC_ORACLE_H

#include <stdint.h>
#include "galic_gpu.h"

typedef struct orc_model {
  galic_params_t p;
  int use_libm;
  long long step_cap; /* reference: 100000000 (orbit_response.c:450) */
  int FG_Ngrid, DG_Nbin, DG_Ngrid, DG_Nstack, EG_Nbin, EG_Ngrid, EG_Nstack;
  double log_FG_Fac, log_DG_Fac, log_EG_Fac;
  double *FG_Pot, *FG_DPotDR, *FG_DPotDz, *FG_Vstream[4];
  double *DG_CellSize, *DGs_Distance;
  double *DGs_MassTarget[4], *EGs_MassTarget[4];
  double *EGs_EgyTarget_r[4], *EGs_EgyTarget_t[4], *EGs_EgyTarget_p[4], *EGs_EgyTarget_q[4];
  /* committed local grids (main.c:151-246) */
  double *DG_MassLoc[4], *EG_RLocS[4], *EG_TLocS[4], *EG_QLocS[4], *EG_PLocS[4];
  double *EG_MassLoc[4], *EG_RLoc[4], *EG_TLoc[4], *EG_PLoc[4], *EG_QLoc[4];
  /* deltas of one repetition (main.c:844-874) */
  double *DG_MassLoc_d[4], *EG_RLocS_d[4], *EG_TLocS_d[4], *EG_QLocS_d[4], *EG_PLocS_d[4];
  double *EG_RLoc_d[4], *EG_TLoc_d[4], *EG_PLoc_d[4], *EG_QLoc_d[4];
  /* stacks of calc_global_fit (main.c:251-362) */
  double *DGs_MassResponse[4], *EGs_RS[4], *EGs_TS[4], *EGs_QS[4], *EGs_PS[4];
  double *EGs_MassResponse[4], *EGs_R[4], *EGs_T[4], *EGs_P[4], *EGs_Q[4];
  double S[4], Sdisp_r[4], Sdisp_t[4], Sdisp_p[4], Sdisp_q[4], Srelfac[4], Srelfac_count[4];
  int firstrun[4];
  long long tries[4], changes[4];
  /* particles (allvars.h:844-868) */
  int n;
  double *pos, *vel, *mass, *tint, *vesc, *targets, *vdisp;
  int *type, *orbits;
  long long steps_total;
} orc_model;

orc_model *orc_create(const galic_params_t *p, int use_libm);
void orc_destroy(orc_model *m);
void orc_set_step_cap(orc_model *m, long long cap);
void orc_set_force_grid(orc_model *m, const double *pot, const double *dpotdr, const double *dpotdz);
void orc_set_vstream(orc_model *m, int type, const double *v);
void orc_set_density_geometry(orc_model *m, const double *cellsize, const double *dgs_distance);
void orc_set_targets(orc_model *m, int type, const double *dgs_mass, const double *egs_mass, const double *egs_r,
                     const double *egs_t, const double *egs_p, const double *egs_q);
void orc_set_particles(orc_model *m, int n, const double *pos, const double *vel, const double *mass,
                       const double *tint, const double *vesc, const int *type, const double *targets);
void orc_get_particles(orc_model *m, double *vel, int *orbits, double *vdisp);

/* lookups */
void orc_forcegrid_acc(orc_model *m, const double *pos, double *acc);
double orc_forcegrid_pot(orc_model *m, const double *pos);
void orc_densitygrid_cell(orc_model *m, const double *pos, int *iR, int *iz, double *fR, double *fz);
double orc_vstream(orc_model *m, const double *pos, int type);

/* orbits; return tall, or -1 on step-cap hit.  info (may be NULL) receives
 * {steps, relative energy error}. */
double orc_orbit_mod(orc_model *m, const double *pos, const double *vel, double *mfield, double *egy_r,
                     double *egy_t, double *egy_q, double *egy_p, double mass, double timespan, int *orbitstaken,
                     int type, double *info);
double orc_orbit(orc_model *m, const double *pos, const double *vel, double *mfield, double mass, double timespan,
                 int *orbitstaken, double *info);

/* merit machinery */
void orc_smooth_stack(double *data, int maxlevel);
double orc_stack_difference(orc_model *m, const double *d1, const double *d2, int maxlevel, const double *ref1,
                            const double *ref2, double thresh, const double *dist, int flag);
double orc_stack_difference_mod(orc_model *m, const double *d1, const double *d2, int maxlevel, const double *ref1,
                                const double *ref2, double thresh, const double *dist, int flag);
double orc_eval_fit_mod(orc_model *m, int n, const double *vel, const double *m_new, const double *m_old,
                        const double *r_new, const double *r_old, const double *t_new, const double *t_old,
                        const double *q_new, const double *q_old, const double *p_new, const double *p_old);
int orc_calc_all(orc_model *m);
int orc_optimize_rep(orc_model *m, const int *idx, int count, uint64_t seed, uint32_t rep_serial);
void orc_get_fit(orc_model *m, double *out);
void orc_get_counters(orc_model *m, long long *tries, long long *changes);
void orc_get_response(orc_model *m, int type, int which, double *out);
long long orc_steps_total(orc_model *m);

/* grid geometry of forcedensitygrid_create (grid.c:329-480) */
int orc_grid_geometry(double halo_a, double outer_frac, double inner_frac, int fg_nbin, int dg_maxlevel,
                      int eg_maxlevel, double *out);
int orc_density_geometry(int dg_maxlevel, double dg_rmin, double dg_fac, double *dgs_distance, double *cellsize,
                         double *cellvol);

/* tree force-grid fill of forcedensitygrid_calculate (grid.c:621-750),
 * single rank; oracle_forcegrid.c */
uint64_t orc_peano_key(int x, int y, int z, int bits);
int orc_force_grid_fill(const galic_fill_params_t *fp, int n, const double *pos, const double *mass,
                        double *dpotdr, double *dpotdz, double *pot);

/* set-up sampling (grid.c:536-617, 659-678, 941-1076), one type, one rank;
 * oracle_sampling.c */
void orc_sample_positions(const galic_sample_params_t *sp, int type, long long n, galic_stream_t *stream,
                          int use_libm, double *pos);
void orc_sample_density(const galic_params_t *p, const galic_sample_params_t *sp, int type, long long ntarget,
                        galic_stream_t *stream, int use_libm, int renorm, double *stack);
void orc_sample_energy(const galic_params_t *p, const galic_sample_params_t *sp, int type, long long ntarget,
                       galic_stream_t *stream, int use_libm, const double *const *tab, double *stacks);

/* calculate_dispfield (disp_fields.c:502-1049); oracle_jeans.c.  out:
 * [4][8][FG_Nbin^2] (disp_r, dispz, dispphi, vstream, tilted_vz2, tilted_vR2,
 * tilted_vz2_prime, tilted_vR2_prime per type). */
int orc_calculate_dispfield(orc_model *m, const galic_sample_params_t *sp, const galic_jeans_params_t *jp,
                            double *out);

/* initialize_particles (set_particles.c:15-307), one rank; oracle_particles.c.
 * tab[t] = {FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime,
 * FG_tilted_vz2_prime, FG_Vstream} of type t. */
int orc_initialize_particles(orc_model *m, const galic_sample_params_t *sp, double TorbitFac,
                             const double *const *const *tab, galic_stream_t *stream, int use_libm, double *pos,
                             double *vel, double *vel_theo, double *mass, double *vesc, double *tint,
                             double *targets, int *type, int *id, int *perm, int *counts);

#endif
