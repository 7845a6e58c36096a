/*
 * ref_driver.c - ctypes entry points into GALIC's own reference C sources.
 *
 * TEST INFRASTRUCTURE.  This file is compiled together with the UNMODIFIED
 * reference sources (src/*.c of denisyurin/GALIC) and the project's
 * single-rank MPI / GSL stand-ins (oracle/shim/) into oracle/_ref/, by
 * oracle/Makefile.  It only sets the reference's globals from caller arrays
 * and calls reference functions; it computes nothing of its own.  Only the
 * tests, the golden-fixture script and bench.py's CPU-baseline leg load it.
 *
 * Each entry point names the reference function it drives.  The reference
 * keeps process-wide state (e.g. the static `firstrun` flags of
 * calc_global_fit, main.c:254), so callers run one scenario per process.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "allvars.h"
#include "proto.h"
#include "galic_gpu.h"

static int ref_ready = 0;

/* Sets All.* and the grid globals from p and allocates the grids with the
 * reference's own allocators (grid.c:204-325). */
int ref_setup(const galic_params_t *p)
{
  int t;
  if(ref_ready) return 1;
  ThisTask = 0;
  NTask = 1;
  PTask = 0;
  All.MaxMemSize = 3000;
  mymalloc_init();
  random_generator = gsl_rng_alloc(gsl_rng_ranlxd1);
  gsl_rng_set(random_generator, 42);

  All.V200 = p->V200;
  All.M200 = p->M200;
  All.R200 = p->R200;
  All.G = p->G;
  All.Halo_Mass = p->Halo_Mass;
  All.Halo_A = p->Halo_A;
  All.HaloStretch = p->HaloStretch;
  All.Disk_Mass = p->Disk_Mass;
  All.Bulge_Mass = p->Bulge_Mass;
  All.Bulge_A = p->Bulge_A;
  All.BulgeStretch = p->BulgeStretch;
  All.TimeStepFactorOrbit = p->TimeStepFactorOrbit;
  All.TimeStepFactorCellCross = p->TimeStepFactorCellCross;
  All.LowerDispLimit = p->LowerDispLimit;
  All.MaxVelInUnitsVesc = p->MaxVelInUnitsVesc;
  All.SampleForceNhalo = p->SampleForceNhalo;
  All.SampleForceNdisk = p->SampleForceNdisk;
  All.SampleForceNbulge = p->SampleForceNbulge;
  All.TypeOfHaloVelocityStructure = p->TypeOfVelocityStructure[1];
  All.TypeOfDiskVelocityStructure = p->TypeOfVelocityStructure[2];
  All.TypeOfBulgeVelocityStructure = p->TypeOfVelocityStructure[3];
  All.MinParticlesPerBinForDispersionMeasurement = p->MinParticlesPerBinForDispersionMeasurement;
  All.MinParticlesPerBinForDensityMeasurement = p->MinParticlesPerBinForDensityMeasurement;
  All.Halo_N = p->NType[1];
  All.Disk_N = p->NType[2];
  All.Bulge_N = p->NType[3];
  All.TotNumPart = (long long) p->NType[1] + p->NType[2] + p->NType[3];
  for(t = 0; t < 4; t++) {
    MType[t] = p->MType[t];
    NType[t] = p->NType[t];
    fac_value_rs[t] = p->fac_value_rs[t];
    fac_value_ts[t] = p->fac_value_ts[t];
    fac_value_qs[t] = p->fac_value_qs[t];
    fac_value_ps[t] = p->fac_value_ps[t];
  }

  FG_Nbin = p->FG_Nbin;
  DG_MaxLevel = p->DG_MaxLevel;
  EG_MaxLevel = p->EG_MaxLevel;
  forcegrid_allocate();
  densitygrid_allocate();
  energygrid_allocate();
  FG_Rmin = p->FG_Rmin;
  FG_Fac = p->FG_Fac;
  DG_Rmin = p->DG_Rmin;
  DG_Fac = p->DG_Fac;
  EG_Rmin = p->EG_Rmin;
  EG_Fac = p->EG_Fac;

  for(t = 1; t <= 3; t++) {
    memset(FG_Vstream[t], 0, FG_Ngrid * sizeof(double));
    memset(DGs_MassTarget[t], 0, DG_Nstack * sizeof(double));
    memset(EGs_MassTarget[t], 0, EG_Nstack * sizeof(double));
    memset(EGs_EgyTarget_r[t], 0, EG_Nstack * sizeof(double));
    memset(EGs_EgyTarget_t[t], 0, EG_Nstack * sizeof(double));
    memset(EGs_EgyTarget_p[t], 0, EG_Nstack * sizeof(double));
    memset(EGs_EgyTarget_q[t], 0, EG_Nstack * sizeof(double));
  }
  memset(FG_Pot, 0, FG_Ngrid * sizeof(double));
  memset(FG_DPotDR, 0, FG_Ngrid * sizeof(double));
  memset(FG_DPotDz, 0, FG_Ngrid * sizeof(double));
  ref_ready = 1;
  return 0;
}

int ref_dg_nstack(void) { return DG_Nstack; }
int ref_dg_ngrid(void) { return DG_Ngrid; }

void ref_set_force_grid(const double *pot, const double *dpotdr, const double *dpotdz)
{
  memcpy(FG_Pot, pot, FG_Ngrid * sizeof(double));
  memcpy(FG_DPotDR, dpotdr, FG_Ngrid * sizeof(double));
  memcpy(FG_DPotDz, dpotdz, FG_Ngrid * sizeof(double));
}

void ref_set_vstream(int type, const double *v) { memcpy(FG_Vstream[type], v, FG_Ngrid * sizeof(double)); }

void ref_set_density_geometry(const double *cellsize, const double *dgs_distance)
{
  memcpy(DG_CellSize, cellsize, DG_Ngrid * sizeof(double));
  memcpy(DGs_Distance, dgs_distance, DG_Nstack * sizeof(double));
}

void ref_set_targets(int type, const double *dgs_mass, const double *egs_mass, const double *egs_r,
                     const double *egs_t, const double *egs_p, const double *egs_q)
{
  memcpy(DGs_MassTarget[type], dgs_mass, DG_Nstack * sizeof(double));
  memcpy(EGs_MassTarget[type], egs_mass, EG_Nstack * sizeof(double));
  memcpy(EGs_EgyTarget_r[type], egs_r, EG_Nstack * sizeof(double));
  memcpy(EGs_EgyTarget_t[type], egs_t, EG_Nstack * sizeof(double));
  memcpy(EGs_EgyTarget_p[type], egs_p, EG_Nstack * sizeof(double));
  memcpy(EGs_EgyTarget_q[type], egs_q, EG_Nstack * sizeof(double));
}

/* Fills P[] the way initialize_particles leaves it (set_particles.c:42-161). */
void ref_set_particles(int n, const double *pos, const double *vel, const double *mass, const double *tint,
                       const double *vesc, const int *type, const double *targets)
{
  int i, k;
  NumPart = n;
  All.MaxPart = n;
  P = (struct particle_data *) mymalloc_movable(&P, "P", n * sizeof(struct particle_data));
  memset(P, 0, n * sizeof(struct particle_data));
  for(i = 0; i < n; i++) {
    for(k = 0; k < 3; k++) {
      P[i].Pos[k] = pos[3 * i + k];
      P[i].Vel[k] = vel[3 * i + k];
    }
    P[i].Mass = mass[i];
    P[i].Tint = tint[i];
    P[i].Vesc = vesc[i];
    P[i].Type = type[i];
    P[i].ID = i + 1;
    P[i].vr2_target = targets[4 * i + 0];
    P[i].vt2_target = targets[4 * i + 1];
    P[i].vp2_target = targets[4 * i + 2];
    P[i].vq2_target = targets[4 * i + 3];
  }
}

void ref_get_particles(double *vel, int *orbits, double *vdisp)
{
  int i, k;
  for(i = 0; i < NumPart; i++) {
    for(k = 0; k < 3; k++) vel[3 * i + k] = P[i].Vel[k];
    orbits[i] = P[i].Orbits;
    vdisp[4 * i + 0] = P[i].vr2;
    vdisp[4 * i + 1] = P[i].vt2;
    vdisp[4 * i + 2] = P[i].vp2;
    vdisp[4 * i + 3] = P[i].vq2;
  }
}

/* produce_orbit_response_field_mod (orbit_response.c:155-491) */
double ref_orbit_mod(double *pos, double *vel, double *m, double *r, double *t, double *q, double *pp,
                     double mass, double timespan, int *orbits, int type)
{
  return produce_orbit_response_field_mod(pos, vel, 0, m, r, t, q, pp, mass, timespan, orbits, type);
}

/* produce_orbit_response_field (orbit_response.c:33-151) */
double ref_orbit(double *pos, double *vel, double *m, double mass, double timespan, int *orbits)
{
  return produce_orbit_response_field(pos, vel, 0, m, mass, timespan, orbits);
}

/* forcegrid_get_acceleration / _potential (grid.c:59-197) */
void ref_forcegrid_acc(double *pos, double *acc) { forcegrid_get_acceleration(pos, acc); }
double ref_forcegrid_pot(double *pos) { return forcegrid_get_potential(pos); }
/* densitygrid_get_cell (grid.c:494-534) */
void ref_densitygrid_cell(double *pos, int *iR, int *iz, double *fR, double *fz)
{
  densitygrid_get_cell(pos, iR, iz, fR, fz);
}
/* get_vstream (disp_fields.c:118-132) */
double ref_vstream(double *pos, int type) { return get_vstream(pos, type); }

/* calc_all_response_fields (main.c:151-246), which ends in calc_global_fit */
void ref_calc_all(void) { calc_all_response_fields(); }

/* one repetition of main.c:96-100 over an explicit particle list */
void ref_optimize_rep(const int *idx, int count, unsigned long long seed, unsigned int rep_serial)
{
  int k;
  init_updates();
  for(k = 0; k < count; k++) {
    galic_shim_rng_stream(random_generator, seed, (unsigned int) idx[k], rep_serial);
    optimize(idx[k]);
  }
  commit_updates();
}

/* F of eval_fit_mod (main.c:1021-1217) for particle n with trial velocity
 * vel and the eight orbit grids. */
double ref_eval_fit_mod(int n, double *vel, double *m_new, double *m_old, double *r_new, double *r_old,
                        double *t_new, double *t_old, double *q_new, double *q_old, double *p_new, double *p_old)
{
  return eval_fit_mod(n, vel, m_new, m_old, r_new, r_old, t_new, t_old, q_new, q_old, p_new, p_old);
}

void ref_get_fit(double *out)
{
  int t;
  for(t = 0; t < 4; t++) {
    out[7 * t + 0] = S[t];
    out[7 * t + 1] = Sdisp_r[t];
    out[7 * t + 2] = Sdisp_t[t];
    out[7 * t + 3] = Sdisp_p[t];
    out[7 * t + 4] = Sdisp_q[t];
    out[7 * t + 5] = Srelfac[t];
    out[7 * t + 6] = Srelfac_count[t];
  }
}

void ref_get_counters(long long *tries, long long *changes)
{
  int t;
  for(t = 0; t < 4; t++) {
    tries[t] = Tries[t];
    changes[t] = Changes[t];
  }
}

/* committed per-type grids, numbered as galic_grid_id */
void ref_get_response(int type, int which, double *out)
{
  double *src = NULL;
  switch(which) {
    case GALIC_GRID_MASS_S: src = DG_MassLoc[type]; break;
    case GALIC_GRID_R_S: src = EG_EgyResponseRLocS[type]; break;
    case GALIC_GRID_T_S: src = EG_EgyResponseTLocS[type]; break;
    case GALIC_GRID_Q_S: src = EG_EgyResponseQLocS[type]; break;
    case GALIC_GRID_P_S: src = EG_EgyResponsePLocS[type]; break;
    case GALIC_GRID_MASS_I: src = EG_MassLoc[type]; break;
    case GALIC_GRID_R_I: src = EG_EgyResponseRLoc[type]; break;
    case GALIC_GRID_T_I: src = EG_EgyResponseTLoc[type]; break;
    case GALIC_GRID_P_I: src = EG_EgyResponsePLoc[type]; break;
    case GALIC_GRID_Q_I: src = EG_EgyResponseQLoc[type]; break;
  }
  if(src) memcpy(out, src, DG_Ngrid * sizeof(double));
}

/* smooth_stack (grid.c:1247-1265) and the stack metrics (grid.c:1086-1151) */
void ref_smooth_stack(double *data, int maxlevel) { smooth_stack(data, maxlevel); }
double ref_stack_difference(double *d1, double *d2, int maxlevel, double *ref1, double *ref2, double thresh,
                            double *dist, int flag)
{
  return calc_stack_difference(d1, d2, 0, 0, 0, maxlevel, ref1, ref2, thresh, dist, flag);
}
double ref_stack_difference_mod(double *d1, double *d2, int maxlevel, double *ref1, double *ref2, double thresh,
                                double *dist, int flag)
{
  return calc_stack_difference_mod(d1, d2, 0, 0, 0, maxlevel, ref1, ref2, thresh, dist, flag);
}

/* Grid geometry of forcedensitygrid_create (grid.c:329-487), run with an
 * analytic halo so that no tree or sampling work is done.  The reference
 * writes forcefield.dat / target_*.dat into OutputDir and forcetest.dat into
 * the working directory, so the call runs inside `outdir`.
 * out: Rmax, DG_Rin, DG_Fac, DG_Rmin, FG_Fac, FG_Rmin, EG_Fac, EG_Rmin. */
int ref_geometry(const char *outdir, double outer_frac, double inner_frac, double *out, double *dgs_distance,
                 double *cellsize, double *cellvol)
{
  char cwd[4096];
  if(!getcwd(cwd, sizeof(cwd))) return 1;
  if(chdir(outdir) != 0) return 2;
  strcpy(All.OutputDir, ".");
  All.OutermostBinEnclosedMassFraction = outer_frac;
  All.InnermostBinEnclosedMassFraction = inner_frac;
  All.SampleDensityFieldForTargetResponse = 0;
  int sh = All.SampleForceNhalo, sd = All.SampleForceNdisk, sb = All.SampleForceNbulge;
  double dm = All.Disk_Mass;
  All.SampleForceNhalo = All.SampleForceNdisk = All.SampleForceNbulge = 0;
  All.Disk_Mass = 0;
  forcedensitygrid_create();
  All.SampleForceNhalo = sh;
  All.SampleForceNdisk = sd;
  All.SampleForceNbulge = sb;
  All.Disk_Mass = dm;
  if(chdir(cwd) != 0) return 3;
  out[0] = All.Rmax;
  out[1] = DG_Rin;
  out[2] = DG_Fac;
  out[3] = DG_Rmin;
  out[4] = FG_Fac;
  out[5] = FG_Rmin;
  out[6] = EG_Fac;
  out[7] = EG_Rmin;
  memcpy(dgs_distance, DGs_Distance, DG_Nstack * sizeof(double));
  memcpy(cellsize, DG_CellSize, DG_Ngrid * sizeof(double));
  memcpy(cellvol, DG_CellVol, DG_Ngrid * sizeof(double));
  return 0;
}

/* ------------------------------------------------------------ force-grid fill */

/* extra parameters of the force-grid fill (All.* members, grid.c:621-757,
 * init.c:31-32, 78-84) */
typedef struct {
  double Softening, ErrTolTheta, TopNodeFactor, Disk_H, Disk_Z0, Rmax;
  int MultipleDomains, SampleForceNhalo, SampleForceNdisk, SampleForceNbulge;
  unsigned long long seed;
} ref_fill_params;

static void ref_fill_setup(const ref_fill_params *f)
{
  All.Softening = f->Softening;
  All.ForceSoftening = 2.8 * f->Softening; /* set_softenings, init.c:78-84 */
  All.ErrTolTheta = f->ErrTolTheta;
  All.TopNodeFactor = f->TopNodeFactor;
  All.MultipleDomains = f->MultipleDomains;
  All.TopNodeAllocFactor = 0.1; /* init.c:31-32 */
  All.BufferSize = 100;         /* MB, as in Model_*.param */
  All.BufferSizeGravity = 100;
  All.TreeAllocFactor = 0.8;
  All.Disk_H = f->Disk_H;
  All.Disk_Z0 = f->Disk_Z0;
  All.Rmax = f->Rmax;
  All.HaloStretch = 1.0;
  All.BulgeStretch = 1.0;
  All.SampleForceNhalo = f->SampleForceNhalo;
  All.SampleForceNdisk = f->SampleForceNdisk;
  All.SampleForceNbulge = f->SampleForceNbulge;
}

/* the mass-particle positions forcedensitygrid_calculate draws (grid.c:659-678)
 * for the same generator seed: halo, then disk, then bulge */
void ref_fill_positions(const ref_fill_params *f, double *pos)
{
  int i, n = 0;
  ref_fill_setup(f);
  gsl_rng_set(random_generator, f->seed);
  for(i = 0; i < f->SampleForceNhalo; i++, n++) halo_get_fresh_coordinate(&pos[3 * n]);
  for(i = 0; i < f->SampleForceNdisk; i++, n++) disk_get_fresh_coordinate(&pos[3 * n]);
  for(i = 0; i < f->SampleForceNbulge; i++, n++) bulge_get_fresh_coordinate(&pos[3 * n]);
}

/* forcedensitygrid_calculate (grid.c:621-891) with its tree force (gravity(),
 * gravtree.c:35-50); run inside outdir, which receives forcefield.dat,
 * forcetest.dat and target_*.dat */
int ref_force_fill(const char *outdir, const ref_fill_params *f, double *dpotdr, double *dpotdz, double *pot)
{
  char cwd[4096];
  if(!getcwd(cwd, sizeof(cwd))) return 1;
  if(chdir(outdir) != 0) return 2;
  strcpy(All.OutputDir, ".");
  ref_fill_setup(f);
  All.SampleDensityFieldForTargetResponse = 0;
  gsl_rng_set(random_generator, f->seed);
  forcedensitygrid_calculate();
  if(chdir(cwd) != 0) return 3;
  memcpy(dpotdr, FG_DPotDR, FG_Ngrid * sizeof(double));
  memcpy(dpotdz, FG_DPotDz, FG_Ngrid * sizeof(double));
  memcpy(pot, FG_Pot, FG_Ngrid * sizeof(double));
  return 0;
}

/* peano_hilbert_key (peano.c:331-347) */
unsigned long long ref_peano_key(int x, int y, int z, int bits) { return peano_hilbert_key(x, y, z, bits); }

/* ------------------------------------------------------- set-up sampling */

/* selects the stream of the reference's random_generator and its position */
void ref_rng_stream(unsigned long long seed, unsigned int a, unsigned int b, unsigned long long position)
{
  galic_shim_rng_stream(random_generator, seed, a, b);
  galic_shim_rng_seek(random_generator, position);
}
unsigned long long ref_rng_position(void) { return galic_shim_rng_position(random_generator); }

/* All.* that the samplers and get_disp_rtp read; SampleParticleCount =
 * ntarget - 1 with one rank (grid.c:558, grid.c:974) */
void ref_sample_setup(const galic_sample_params_t *sp, long long ntarget)
{
  All.Rmax = sp->Rmax;
  All.Halo_A = sp->Halo_A;
  All.HaloStretch = sp->HaloStretch;
  All.Disk_Z0 = sp->Disk_Z0;
  All.Disk_H = sp->Disk_H;
  All.Bulge_A = sp->Bulge_A;
  All.BulgeStretch = sp->BulgeStretch;
  All.HaloBetaParameter = sp->HaloBetaParameter;
  All.BulgeBetaParameter = sp->BulgeBetaParameter;
  All.SampleParticleCount = (int) (ntarget - 1);
}

/* FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime
 * of one type (FG_Ngrid doubles each; NULL leaves a table as it is) */
void ref_set_dispersion(int type, const double *disp_r, const double *dispz, const double *dispphi,
                        const double *tvr2, const double *tvz2)
{
  size_t b = FG_Ngrid * sizeof(double);
  if(disp_r) memcpy(FG_Disp_r[type], disp_r, b);
  if(dispz) memcpy(FG_DispZ[type], dispz, b);
  if(dispphi) memcpy(FG_DispPhi[type], dispphi, b);
  if(tvr2) memcpy(FG_tilted_vR2_prime[type], tvr2, b);
  if(tvz2) memcpy(FG_tilted_vz2_prime[type], tvz2, b);
}

/* densitygrid_sample_targetresponse (grid.c:536-617) */
void ref_sample_density(void) { densitygrid_sample_targetresponse(); }
/* calc_energy_grid_mass_maps (grid.c:941-1076) */
void ref_sample_energy(void) { calc_energy_grid_mass_maps(); }

/* the target stacks of one type (Nstack doubles each) */
void ref_get_targets(int type, double *dgs_mass, double *egs_mass, double *egs_r, double *egs_t, double *egs_p,
                     double *egs_q)
{
  memcpy(dgs_mass, DGs_MassTarget[type], DG_Nstack * sizeof(double));
  memcpy(egs_mass, EGs_MassTarget[type], EG_Nstack * sizeof(double));
  memcpy(egs_r, EGs_EgyTarget_r[type], EG_Nstack * sizeof(double));
  memcpy(egs_t, EGs_EgyTarget_t[type], EG_Nstack * sizeof(double));
  memcpy(egs_p, EGs_EgyTarget_p[type], EG_Nstack * sizeof(double));
  memcpy(egs_q, EGs_EgyTarget_q[type], EG_Nstack * sizeof(double));
}

/* n calls of the type's *_get_fresh_coordinate (halo.c:17, disk.c:17, bulge.c:15) */
void ref_fresh_positions(int type, long long n, double *pos)
{
  long long i;
  for(i = 0; i < n; i++) {
    if(type == 1)
      halo_get_fresh_coordinate(&pos[3 * i]);
    else if(type == 2)
      disk_get_fresh_coordinate(&pos[3 * i]);
    else
      bulge_get_fresh_coordinate(&pos[3 * i]);
  }
}

/* ------------------------------------------------------- Jeans solvers */

/* calculate_dispfield (disp_fields.c:502-1049) with the All.* it reads; its
 * sigma/pde output files go to outdir */
int ref_calculate_dispfield(const char *outdir, const galic_sample_params_t *sp, const galic_jeans_params_t *jp)
{
  ref_sample_setup(sp, 1);
  All.HaloStreamingVelocityParameter = jp->StreamingVelocityParameter[1];
  All.DiskStreamingVelocityParameter = jp->StreamingVelocityParameter[2];
  All.BulgeStreamingVelocityParameter = jp->StreamingVelocityParameter[3];
  All.HaloDispersionRoverZratio = jp->DispersionRoverZratio[1];
  All.DiskDispersionRoverZratio = jp->DispersionRoverZratio[2];
  All.BulgeDispersionRoverZratio = jp->DispersionRoverZratio[3];
  if(strlen(outdir) >= sizeof(All.OutputDir)) return 1;
  strcpy(All.OutputDir, outdir);
  /* tables the function leaves untouched read as zero */
  for(int t = 1; t <= 3; t++) {
    double *tab[8] = {FG_Disp_r[t], FG_DispZ[t], FG_DispPhi[t], FG_Vstream[t],
                      FG_tilted_vz2[t], FG_tilted_vR2[t], FG_tilted_vz2_prime[t], FG_tilted_vR2_prime[t]};
    for(int k = 0; k < 8; k++) memset(tab[k], 0, FG_Ngrid * sizeof(double));
  }
  calculate_dispfield();
  return 0;
}

/* the Jeans tables of one type: disp_r, dispz, dispphi, vstream, tilted_vz2,
 * tilted_vR2, tilted_vz2_prime, tilted_vR2_prime (FG_Ngrid doubles each) */
void ref_get_jeans(int type, double *out)
{
  double *src[8] = {FG_Disp_r[type], FG_DispZ[type], FG_DispPhi[type], FG_Vstream[type],
                    FG_tilted_vz2[type], FG_tilted_vR2[type], FG_tilted_vz2_prime[type], FG_tilted_vR2_prime[type]};
  for(int k = 0; k < 8; k++) memcpy(out + (size_t) k * FG_Ngrid, src[k], FG_Ngrid * sizeof(double));
}

/* ------------------------------------------------------- particle initialisation */

/* initialize_particles (set_particles.c:15-307) with TorbitFac and the
 * sampler shapes; its fit_*.txt files go to outdir.  Returns NumPart. */
int ref_initialize_particles(const char *outdir, const galic_sample_params_t *sp, double TorbitFac)
{
  ref_sample_setup(sp, 1);
  All.TorbitFac = TorbitFac;
  if(strlen(outdir) >= sizeof(All.OutputDir)) return -1;
  strcpy(All.OutputDir, outdir);
  initialize_particles();
  return NumPart;
}

/* P[] and permutation[] after initialize_particles */
void ref_get_init_particles(double *pos, double *vel, double *vel_theo, double *mass, double *vesc, double *tint,
                            double *targets, int *type, int *id, int *perm)
{
  for(int n = 0; n < NumPart; n++) {
    for(int k = 0; k < 3; k++) {
      pos[3 * n + k] = P[n].Pos[k];
      vel[3 * n + k] = P[n].Vel[k];
      vel_theo[3 * n + k] = P[n].VelTheo[k];
    }
    mass[n] = P[n].Mass;
    vesc[n] = P[n].Vesc;
    tint[n] = P[n].Tint;
    targets[4 * n] = P[n].vr2_target;
    targets[4 * n + 1] = P[n].vt2_target;
    targets[4 * n + 2] = P[n].vp2_target;
    targets[4 * n + 3] = P[n].vq2_target;
    type[n] = P[n].Type;
    id[n] = (int) P[n].ID;
    perm[n] = permutation[n].index;
  }
}

/* ------------------------------------------------------- output files */

/* output_particles (io.c:460-540) for dump 0 with one file of SnapFormat fmt:
 * writes prefix + "snap_000" (OutputDir is used as a prefix, io.c:513) */
void ref_output_particles(const char *prefix, int fmt)
{
  All.SnapFormat = fmt;
  All.NumFilesPerSnapshot = 1;
  All.NumFilesWrittenInParallel = 1;
  All.StepsBetweenDump = 1;
  All.BufferSize = 100;
  strcpy(All.OutputDir, prefix);
  strcpy(All.OutputFile, "snap");
  output_particles(0);
}

/* output_density_field (io.c:36-460) for dump 0: outdir/densfield_<type>_000.dat */
void ref_output_density_field(const char *outdir)
{
  All.StepsBetweenDump = 1;
  strcpy(All.OutputDir, outdir);
  output_density_field(0);
}
