/*
 * galic_oracle.c - CPU restatement of GALIC's orbit-response hot path.
 * TEST INFRASTRUCTURE (the checker of the CUDA kernels); see galic_oracle.h.
 *
 * Operation order follows the cited reference lines exactly; build with
 * -ffp-contract=off (oracle/Makefile).  All citations are into the
 * reference tree src/.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "galic_oracle.h"
#include "../galic_b200/csrc/gmath.h"
#include "../galic_b200/csrc/grng.h"

#define SO(l, i, j) ((((1 << (2 * (l))) - 1) / 3) + ((i) * (1 << (l))) + (j)) /* allvars.h:160 */
#define OFF(l, i, j) (((i) * (1 << (l))) + (j))                                /* allvars.h:161 */

/* the transcendental functions of the path, selectable per model */
static double m_log(const orc_model *m, double x) { return m->use_libm ? log(x) : gm_log(x); }
static double m_atan2(const orc_model *m, double y, double x) { return m->use_libm ? atan2(y, x) : gm_atan2(y, x); }
static double m_sin(const orc_model *m, double x) { return m->use_libm ? sin(x) : gm_sin(x); }
static double m_cos(const orc_model *m, double x) { return m->use_libm ? cos(x) : gm_cos(x); }
static double m_acos(const orc_model *m, double x) { return m->use_libm ? acos(x) : gm_acos(x); }

static double dmax(double a, double b) { return a > b ? a : b; } /* system.c:38 */
static double dmin(double a, double b) { return a < b ? a : b; } /* system.c:46 */
static double min_(double a, double b) { return a < b ? a : b; } /* grid.c:1078 */

static double *zalloc(size_t n) { return (double *) calloc(n ? n : 1, sizeof(double)); }

static int type_vel_structure(const orc_model *m, int type) { return m->p.TypeOfVelocityStructure[type]; }

orc_model *orc_create(const galic_params_t *p, int use_libm)
{
  orc_model *m = (orc_model *) calloc(1, sizeof(orc_model));
  int t;
  m->p = *p;
  m->use_libm = use_libm;
  m->step_cap = 100000000;
  m->FG_Ngrid = p->FG_Nbin * p->FG_Nbin;
  m->DG_Nbin = 1 << p->DG_MaxLevel;                                   /* grid.c:303 */
  m->DG_Ngrid = m->DG_Nbin * m->DG_Nbin;                              /* grid.c:306 */
  m->DG_Nstack = ((1 << (2 + 2 * p->DG_MaxLevel)) - 1) / 3;           /* grid.c:300 */
  m->EG_Nbin = 1 << p->EG_MaxLevel;                                   /* grid.c:239 */
  m->EG_Ngrid = m->EG_Nbin * m->EG_Nbin;
  m->EG_Nstack = ((1 << (2 + 2 * p->EG_MaxLevel)) - 1) / 3;           /* grid.c:238 */
  m->FG_Pot = zalloc(m->FG_Ngrid);
  m->FG_DPotDR = zalloc(m->FG_Ngrid);
  m->FG_DPotDz = zalloc(m->FG_Ngrid);
  m->DG_CellSize = zalloc(m->DG_Ngrid);
  m->DGs_Distance = zalloc(m->DG_Nstack);
  for(t = 1; t <= 3; t++) {
    m->FG_Vstream[t] = zalloc(m->FG_Ngrid);
    m->DGs_MassTarget[t] = zalloc(m->DG_Nstack);
    m->EGs_MassTarget[t] = zalloc(m->EG_Nstack);
    m->EGs_EgyTarget_r[t] = zalloc(m->EG_Nstack);
    m->EGs_EgyTarget_t[t] = zalloc(m->EG_Nstack);
    m->EGs_EgyTarget_p[t] = zalloc(m->EG_Nstack);
    m->EGs_EgyTarget_q[t] = zalloc(m->EG_Nstack);
    m->DG_MassLoc[t] = zalloc(m->DG_Ngrid);
    m->EG_RLocS[t] = zalloc(m->EG_Ngrid);
    m->EG_TLocS[t] = zalloc(m->EG_Ngrid);
    m->EG_QLocS[t] = zalloc(m->EG_Ngrid);
    m->EG_PLocS[t] = zalloc(m->EG_Ngrid);
    m->EG_MassLoc[t] = zalloc(m->EG_Ngrid);
    m->EG_RLoc[t] = zalloc(m->EG_Ngrid);
    m->EG_TLoc[t] = zalloc(m->EG_Ngrid);
    m->EG_PLoc[t] = zalloc(m->EG_Ngrid);
    m->EG_QLoc[t] = zalloc(m->EG_Ngrid);
    m->DG_MassLoc_d[t] = zalloc(m->DG_Ngrid);
    m->EG_RLocS_d[t] = zalloc(m->EG_Ngrid);
    m->EG_TLocS_d[t] = zalloc(m->EG_Ngrid);
    m->EG_QLocS_d[t] = zalloc(m->EG_Ngrid);
    m->EG_PLocS_d[t] = zalloc(m->EG_Ngrid);
    m->EG_RLoc_d[t] = zalloc(m->EG_Ngrid);
    m->EG_TLoc_d[t] = zalloc(m->EG_Ngrid);
    m->EG_PLoc_d[t] = zalloc(m->EG_Ngrid);
    m->EG_QLoc_d[t] = zalloc(m->EG_Ngrid);
    m->DGs_MassResponse[t] = zalloc(m->DG_Nstack);
    m->EGs_RS[t] = zalloc(m->EG_Nstack);
    m->EGs_TS[t] = zalloc(m->EG_Nstack);
    m->EGs_QS[t] = zalloc(m->EG_Nstack);
    m->EGs_PS[t] = zalloc(m->EG_Nstack);
    m->EGs_MassResponse[t] = zalloc(m->EG_Nstack);
    m->EGs_R[t] = zalloc(m->EG_Nstack);
    m->EGs_T[t] = zalloc(m->EG_Nstack);
    m->EGs_P[t] = zalloc(m->EG_Nstack);
    m->EGs_Q[t] = zalloc(m->EG_Nstack);
  }
  return m;
}

void orc_destroy(orc_model *m)
{
  int t;
  if(!m) return;
  free(m->FG_Pot); free(m->FG_DPotDR); free(m->FG_DPotDz); free(m->DG_CellSize); free(m->DGs_Distance);
  for(t = 1; t <= 3; t++) {
    double **a[] = {&m->FG_Vstream[t], &m->DGs_MassTarget[t], &m->EGs_MassTarget[t], &m->EGs_EgyTarget_r[t],
                    &m->EGs_EgyTarget_t[t], &m->EGs_EgyTarget_p[t], &m->EGs_EgyTarget_q[t], &m->DG_MassLoc[t],
                    &m->EG_RLocS[t], &m->EG_TLocS[t], &m->EG_QLocS[t], &m->EG_PLocS[t], &m->EG_MassLoc[t],
                    &m->EG_RLoc[t], &m->EG_TLoc[t], &m->EG_PLoc[t], &m->EG_QLoc[t], &m->DG_MassLoc_d[t],
                    &m->EG_RLocS_d[t], &m->EG_TLocS_d[t], &m->EG_QLocS_d[t], &m->EG_PLocS_d[t],
                    &m->EG_RLoc_d[t], &m->EG_TLoc_d[t], &m->EG_PLoc_d[t], &m->EG_QLoc_d[t],
                    &m->DGs_MassResponse[t], &m->EGs_RS[t], &m->EGs_TS[t], &m->EGs_QS[t], &m->EGs_PS[t],
                    &m->EGs_MassResponse[t], &m->EGs_R[t], &m->EGs_T[t], &m->EGs_P[t], &m->EGs_Q[t]};
    for(size_t k = 0; k < sizeof(a) / sizeof(a[0]); k++) free(*a[k]);
  }
  free(m->pos); free(m->vel); free(m->mass); free(m->tint); free(m->vesc); free(m->targets); free(m->vdisp);
  free(m->type); free(m->orbits);
  free(m);
}

void orc_set_step_cap(orc_model *m, long long cap) { m->step_cap = cap; }

void orc_set_force_grid(orc_model *m, const double *pot, const double *dpotdr, const double *dpotdz)
{
  memcpy(m->FG_Pot, pot, m->FG_Ngrid * sizeof(double));
  memcpy(m->FG_DPotDR, dpotdr, m->FG_Ngrid * sizeof(double));
  memcpy(m->FG_DPotDz, dpotdz, m->FG_Ngrid * sizeof(double));
}

void orc_set_vstream(orc_model *m, int type, const double *v) { memcpy(m->FG_Vstream[type], v, m->FG_Ngrid * sizeof(double)); }

void orc_set_density_geometry(orc_model *m, const double *cellsize, const double *dgs_distance)
{
  memcpy(m->DG_CellSize, cellsize, m->DG_Ngrid * sizeof(double));
  memcpy(m->DGs_Distance, dgs_distance, m->DG_Nstack * sizeof(double));
}

void orc_set_targets(orc_model *m, int type, const double *dgs_mass, const double *egs_mass, const double *egs_r,
                     const double *egs_t, const double *egs_p, const double *egs_q)
{
  memcpy(m->DGs_MassTarget[type], dgs_mass, m->DG_Nstack * sizeof(double));
  memcpy(m->EGs_MassTarget[type], egs_mass, m->EG_Nstack * sizeof(double));
  memcpy(m->EGs_EgyTarget_r[type], egs_r, m->EG_Nstack * sizeof(double));
  memcpy(m->EGs_EgyTarget_t[type], egs_t, m->EG_Nstack * sizeof(double));
  memcpy(m->EGs_EgyTarget_p[type], egs_p, m->EG_Nstack * sizeof(double));
  memcpy(m->EGs_EgyTarget_q[type], egs_q, m->EG_Nstack * sizeof(double));
}

void orc_set_particles(orc_model *m, int n, const double *pos, const double *vel, const double *mass,
                       const double *tint, const double *vesc, const int *type, const double *targets)
{
  free(m->pos); free(m->vel); free(m->mass); free(m->tint); free(m->vesc); free(m->targets); free(m->vdisp);
  free(m->type); free(m->orbits);
  m->n = n;
  m->pos = zalloc(3 * (size_t) n);
  m->vel = zalloc(3 * (size_t) n);
  m->mass = zalloc(n);
  m->tint = zalloc(n);
  m->vesc = zalloc(n);
  m->targets = zalloc(4 * (size_t) n);
  m->vdisp = zalloc(4 * (size_t) n);
  m->type = (int *) calloc(n ? n : 1, sizeof(int));
  m->orbits = (int *) calloc(n ? n : 1, sizeof(int));
  memcpy(m->pos, pos, 3 * (size_t) n * sizeof(double));
  memcpy(m->vel, vel, 3 * (size_t) n * sizeof(double));
  memcpy(m->mass, mass, n * sizeof(double));
  memcpy(m->tint, tint, n * sizeof(double));
  memcpy(m->vesc, vesc, n * sizeof(double));
  memcpy(m->targets, targets, 4 * (size_t) n * sizeof(double));
  memcpy(m->type, type, n * sizeof(int));
}

void orc_get_particles(orc_model *m, double *vel, int *orbits, double *vdisp)
{
  memcpy(vel, m->vel, 3 * (size_t) m->n * sizeof(double));
  memcpy(orbits, m->orbits, m->n * sizeof(int));
  memcpy(vdisp, m->vdisp, 4 * (size_t) m->n * sizeof(double));
}

/* ------------------------------------------------------------ analytic components */

/* halo_get_acceleration (halo.c:76-84) */
static void halo_acc(const orc_model *m, const double *pos, double *acc)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double fac = m->p.G * m->p.Halo_Mass / ((r + 1.0e-6 * m->p.Halo_A) * (r + m->p.Halo_A) * (r + m->p.Halo_A));
  acc[0] = -fac * pos[0];
  acc[1] = -fac * pos[1];
  acc[2] = -fac * pos[2];
}
/* halo_get_potential (halo.c:63-73) */
static double halo_pot(const orc_model *m, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return -m->p.G * m->p.Halo_Mass / (r + m->p.Halo_A);
}
/* bulge_get_acceleration (bulge.c:76-84) */
static void bulge_acc(const orc_model *m, const double *pos, double *acc)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double fac = m->p.G * m->p.Bulge_Mass / ((r + 1.0e-6 * m->p.Bulge_A) * (r + m->p.Bulge_A) * (r + m->p.Bulge_A));
  acc[0] = -fac * pos[0];
  acc[1] = -fac * pos[1];
  acc[2] = -fac * pos[2];
}
/* bulge_get_potential (bulge.c:63-73) */
static double bulge_pot(const orc_model *m, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return -m->p.G * m->p.Bulge_Mass / (r + m->p.Bulge_A);
}

static int fg_tabulated(const orc_model *m)
{
  return m->p.Disk_Mass > 0 || (m->p.Halo_Mass > 0 && m->p.SampleForceNhalo > 0) ||
         (m->p.Bulge_Mass > 0 && m->p.SampleForceNbulge > 0);
}

/* forcegrid_get_acceleration (grid.c:122-197) */
void orc_forcegrid_acc(orc_model *m, const double *pos, double *acc)
{
  const int N = m->p.FG_Nbin;
  if(fg_tabulated(m)) {
    double phi = m_atan2(m, pos[1], pos[0]);
    double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    double jdbl = m_log(m, R / m->p.FG_Rmin + 1.0) / m_log(m, m->p.FG_Fac);
    int jbin = (int) jdbl;
    double jfac = jdbl - jbin;
    double idbl = m_log(m, fabs(pos[2]) / m->p.FG_Rmin + 1.0) / m_log(m, m->p.FG_Fac);
    int ibin = (int) idbl;
    double ifac = idbl - ibin;
    if(ibin < N - 1 && jbin < N - 1) {
      const double *D = m->FG_DPotDR, *Z = m->FG_DPotDz;
      double accR = D[ibin * N + jbin] * (1 - ifac) * (1 - jfac) + D[ibin * N + (jbin + 1)] * (1 - ifac) * jfac +
                    D[(ibin + 1) * N + jbin] * ifac * (1 - jfac) + D[(ibin + 1) * N + (jbin + 1)] * ifac * jfac;
      double accz = Z[ibin * N + jbin] * (1 - ifac) * (1 - jfac) + Z[ibin * N + (jbin + 1)] * (1 - ifac) * jfac +
                    Z[(ibin + 1) * N + jbin] * ifac * (1 - jfac) + Z[(ibin + 1) * N + (jbin + 1)] * ifac * jfac;
      if(pos[2] < 0) accz = -accz;
      acc[0] = accR * m_cos(m, phi);
      acc[1] = accR * m_sin(m, phi);
      acc[2] = accz;
    } else {
      halo_acc(m, pos, acc);
      double fac = m->p.M200 / m->p.Halo_Mass;
      for(int k = 0; k < 3; k++) acc[k] *= fac;
    }
  } else {
    acc[0] = acc[1] = acc[2] = 0;
  }
  if(m->p.Halo_Mass > 0 && m->p.SampleForceNhalo == 0) {
    double a[3];
    halo_acc(m, pos, a);
    acc[0] += a[0];
    acc[1] += a[1];
    acc[2] += a[2];
  }
  if(m->p.Bulge_Mass > 0 && m->p.SampleForceNbulge == 0) {
    double a[3];
    bulge_acc(m, pos, a);
    acc[0] += a[0];
    acc[1] += a[1];
    acc[2] += a[2];
  }
}

/* forcegrid_get_potential (grid.c:59-113) */
double orc_forcegrid_pot(orc_model *m, const double *pos)
{
  const int N = m->p.FG_Nbin;
  double pot;
  if(fg_tabulated(m)) {
    double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    double jdbl = m_log(m, R / m->p.FG_Rmin + 1.0) / m_log(m, m->p.FG_Fac);
    int jbin = (int) jdbl;
    double jfac = jdbl - jbin;
    double idbl = m_log(m, fabs(pos[2]) / m->p.FG_Rmin + 1.0) / m_log(m, m->p.FG_Fac);
    int ibin = (int) idbl;
    double ifac = idbl - ibin;
    if(ibin < N - 1 && jbin < N - 1) {
      const double *P = m->FG_Pot;
      pot = P[ibin * N + jbin] * (1 - ifac) * (1 - jfac) + P[ibin * N + (jbin + 1)] * (1 - ifac) * jfac +
            P[(ibin + 1) * N + jbin] * ifac * (1 - jfac) + P[(ibin + 1) * N + (jbin + 1)] * ifac * jfac;
    } else
      pot = m->p.M200 / m->p.Halo_Mass * halo_pot(m, pos);
  } else
    pot = 0;
  if(m->p.Halo_Mass > 0 && m->p.SampleForceNhalo == 0) pot += halo_pot(m, pos);
  if(m->p.Bulge_Mass > 0 && m->p.SampleForceNbulge == 0) pot += bulge_pot(m, pos);
  return pot;
}

/* shared body of densitygrid_get_cell (grid.c:494-534), energygrid_get_cell
 * (grid.c:896-938, shift 0.5) and forcegrid_get_cell (grid.c:15-55, shift 0) */
static void get_cell(const orc_model *m, const double *pos, double rmin, double fac, int nbin, double shift,
                     int *iR, int *iz, double *fR, double *fz)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = fabs(pos[2]);
  double br, bz;
  if(shift != 0) {
    br = (m_log(m, r / rmin + 1.0) / m_log(m, fac)) - 0.5;
    bz = (m_log(m, z / rmin + 1.0) / m_log(m, fac)) - 0.5;
  } else {
    br = (m_log(m, r / rmin + 1.0) / m_log(m, fac));
    bz = (m_log(m, z / rmin + 1.0) / m_log(m, fac));
  }
  int binr, binz;
  if(br < 0) br = 0;
  if(bz < 0) bz = 0;
  binr = (int) br;
  *fR = br - binr;
  binz = (int) bz;
  *fz = bz - binz;
  if(binr >= nbin - 1) {
    binr = nbin - 2;
    *fR = 1;
  }
  if(binz >= nbin - 1) {
    binz = nbin - 2;
    *fz = 1;
  }
  *iR = binr;
  *iz = binz;
}

void orc_densitygrid_cell(orc_model *m, const double *pos, int *iR, int *iz, double *fR, double *fz)
{
  get_cell(m, pos, m->p.DG_Rmin, m->p.DG_Fac, m->DG_Nbin, 0.5, iR, iz, fR, fz);
}

/* get_vstream (disp_fields.c:118-132) */
double orc_vstream(orc_model *m, const double *pos, int type)
{
  int iz, iR;
  double fR, fz;
  const int N = m->p.FG_Nbin;
  const double *V = m->FG_Vstream[type];
  get_cell(m, pos, m->p.FG_Rmin, m->p.FG_Fac, N, 0.0, &iR, &iz, &fR, &fz);
  return V[iz * N + iR] * (1 - fR) * (1 - fz) + V[(iz + 1) * N + iR] * (1 - fR) * (fz) +
         V[iz * N + (iR + 1)] * (fR) * (1 - fz) + V[(iz + 1) * N + (iR + 1)] * (fR) * (fz);
}

/* get_timestep (orbit_response.c:16-26) */
static double get_timestep(const orc_model *m, const double *x, const double *v, const double *a, int icell)
{
  (void) x;
  double vv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double aa = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double torbit = m->p.V200 / aa;
  double tcross = m->DG_CellSize[icell] / vv;
  return dmin(m->p.TimeStepFactorOrbit * torbit, m->p.TimeStepFactorCellCross * tcross);
}

/* the velocity projections of orbit_response.c:222-273 (= 338-391) */
static void project(orc_model *m, int tovs, int type, const double *x, const double *v, double *vr2, double *vt2,
                    double *vq2, double *vp2)
{
  double r2, v_dot_x, q, q2, vq, v_dot_Q, t2, v_dot_T, vstr;
  double Z[] = {0, 0, -1};
  double T[3], Q[3];
  if(tovs == 2) {
    r2 = x[0] * x[0] + x[1] * x[1];
    v_dot_x = v[0] * x[0] + v[1] * x[1];
    *vr2 = v_dot_x * v_dot_x / r2;
    Q[0] = -x[1];
    Q[1] = x[0];
    q2 = Q[0] * Q[0] + Q[1] * Q[1];
    v_dot_Q = v[0] * Q[0] + v[1] * Q[1];
    q = sqrt(q2);
    vq = v_dot_Q / q;
    *vq2 = vq * vq;
    vstr = orc_vstream(m, x, type);
    *vp2 = (vq - vstr) * (vq - vstr);
    *vt2 = v[2] * v[2];
  } else {
    r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    v_dot_x = v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
    *vr2 = v_dot_x * v_dot_x / r2;
    Q[0] = x[1] * Z[2] - x[2] * Z[1];
    Q[1] = x[2] * Z[0] - x[0] * Z[2];
    Q[2] = x[0] * Z[1] - x[1] * Z[0];
    q2 = Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2];
    v_dot_Q = v[0] * Q[0] + v[1] * Q[1] + v[2] * Q[2];
    q = sqrt(q2);
    vq = v_dot_Q / q;
    *vq2 = vq * vq;
    vstr = orc_vstream(m, x, type);
    *vp2 = (vq - vstr) * (vq - vstr);
    T[0] = x[1] * Q[2] - x[2] * Q[1];
    T[1] = x[2] * Q[0] - x[0] * Q[2];
    T[2] = x[0] * Q[1] - x[1] * Q[0];
    t2 = T[0] * T[0] + T[1] * T[1] + T[2] * T[2];
    v_dot_T = v[0] * T[0] + v[1] * T[1] + v[2] * T[2];
    *vt2 = v_dot_T * v_dot_T / t2;
  }
}

/* produce_orbit_response_field_mod (orbit_response.c:155-491) */
double orc_orbit_mod(orc_model *m, const double *pos, const double *vel, double *mfield, double *egy_r,
                     double *egy_t, double *egy_q, double *egy_p, double mass, double timespan, int *orbitstaken,
                     int type, double *info)
{
  const int Nb = m->DG_Nbin;
  int tovs = type_vel_structure(m, type);
  int i, norbit, icell, flag = 0, iR, iz;
  double x[3], v[3], a[3], dt, tall, radsign_previous = 0, radsign, fR, fz;
  double vr2, vt2, vq2, vp2, mm[2][2];
  int irz[2][2];

  for(i = 0; i < 3; i++) {
    x[i] = pos[i];
    v[i] = vel[i];
  }
  for(i = 0; i < m->DG_Ngrid; i++) mfield[i] = 0;
  for(i = 0; i < m->EG_Ngrid; i++) egy_r[i] = egy_t[i] = egy_q[i] = egy_p[i] = 0;
  norbit = 0;
  tall = 0;
  orc_forcegrid_acc(m, x, a);
  orc_densitygrid_cell(m, x, &iR, &iz, &fR, &fz);
  icell = iz * Nb + iR;
  const int Norbits = 100000000;
  double E0 = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + orc_forcegrid_pot(m, x);
  long long steps = 0;

  do {
    dt = get_timestep(m, x, v, a, icell);
    if(0 < timespan)
      if(timespan < dt + tall) {
        dt = timespan - tall;
        flag = 1;
      }
    for(int half = 0; half < 2; half++) {
      if(half == 1) {
        for(i = 0; i < 3; i++) v[i] += 0.5 * dt * a[i];
        for(i = 0; i < 3; i++) x[i] += dt * v[i];
        orc_forcegrid_acc(m, x, a);
        for(i = 0; i < 3; i++) v[i] += 0.5 * dt * a[i];
        orc_densitygrid_cell(m, x, &iR, &iz, &fR, &fz);
        icell = iz * Nb + iR;
      }
      project(m, tovs, type, x, v, &vr2, &vt2, &vq2, &vp2);
      mm[0][0] = 0.5 * dt * (1 - fR) * (1 - fz);
      mm[1][0] = 0.5 * dt * (fR) * (1 - fz);
      mm[0][1] = 0.5 * dt * (1 - fR) * (fz);
      mm[1][1] = 0.5 * dt * (fR) * (fz);
      irz[0][0] = iz * Nb + iR;
      irz[1][0] = iz * Nb + (iR + 1);
      irz[0][1] = (iz + 1) * Nb + iR;
      irz[1][1] = (iz + 1) * Nb + (iR + 1);
      mfield[irz[0][0]] += mm[0][0];
      mfield[irz[1][0]] += mm[1][0];
      mfield[irz[0][1]] += mm[0][1];
      mfield[irz[1][1]] += mm[1][1];
      egy_r[irz[0][0]] += mm[0][0] * vr2;
      egy_r[irz[1][0]] += mm[1][0] * vr2;
      egy_r[irz[0][1]] += mm[0][1] * vr2;
      egy_r[irz[1][1]] += mm[1][1] * vr2;
      egy_t[irz[0][0]] += mm[0][0] * vt2;
      egy_t[irz[1][0]] += mm[1][0] * vt2;
      egy_t[irz[0][1]] += mm[0][1] * vt2;
      egy_t[irz[1][1]] += mm[1][1] * vt2;
      egy_q[irz[0][0]] += mm[0][0] * vq2;
      egy_q[irz[1][0]] += mm[1][0] * vq2;
      egy_q[irz[0][1]] += mm[0][1] * vq2;
      egy_q[irz[1][1]] += mm[1][1] * vq2;
      egy_p[irz[0][0]] += mm[0][0] * vp2;
      egy_p[irz[1][0]] += mm[1][0] * vp2;
      egy_p[irz[0][1]] += mm[0][1] * vp2;
      egy_p[irz[1][1]] += mm[1][1] * vp2;
    }
    tall += dt;
    radsign = v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
    if(radsign > 0 && radsign_previous < 0) norbit++;
    radsign_previous = radsign;
    steps++;
    if(steps > m->step_cap) {
      m->steps_total += steps;
      if(info) { info[0] = (double) steps; info[1] = -1; }
      return -1;
    }
  } while((timespan == 0 && norbit < Norbits) || (timespan != 0 && flag == 0));

  double E1 = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + orc_forcegrid_pot(m, x);
  double rel_egy_error = fabs((E1 - E0) / E0);
  double fac = mass / tall;
  for(i = 0; i < m->DG_Ngrid; i++) mfield[i] *= fac;
  for(i = 0; i < m->EG_Ngrid; i++) {
    egy_r[i] *= fac;
    egy_t[i] *= fac;
    egy_q[i] *= fac;
    egy_p[i] *= fac;
  }
  *orbitstaken = norbit;
  m->steps_total += steps;
  if(info) { info[0] = (double) steps; info[1] = rel_egy_error; }
  return tall;
}

/* produce_orbit_response_field (orbit_response.c:33-151) */
double orc_orbit(orc_model *m, const double *pos, const double *vel, double *mfield, double mass, double timespan,
                 int *orbitstaken, double *info)
{
  const int Nb = m->DG_Nbin;
  int i, norbit, icell, flag = 0, iR, iz;
  double x[3], v[3], a[3], dt, tall, radsign_previous = 0, radsign, fR, fz;
  for(i = 0; i < 3; i++) {
    x[i] = pos[i];
    v[i] = vel[i];
  }
  for(i = 0; i < m->DG_Ngrid; i++) mfield[i] = 0;
  norbit = 0;
  tall = 0;
  orc_forcegrid_acc(m, x, a);
  orc_densitygrid_cell(m, x, &iR, &iz, &fR, &fz);
  icell = iz * Nb + iR;
  const int Norbits = 100000000;
  double E0 = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + orc_forcegrid_pot(m, x);
  long long steps = 0;
  do {
    dt = get_timestep(m, x, v, a, icell);
    if(0 < timespan)
      if(timespan < dt + tall) {
        dt = timespan - tall;
        flag = 1;
      }
    mfield[iz * Nb + iR] += 0.5 * dt * (1 - fR) * (1 - fz);
    mfield[iz * Nb + (iR + 1)] += 0.5 * dt * (fR) * (1 - fz);
    mfield[(iz + 1) * Nb + iR] += 0.5 * dt * (1 - fR) * (fz);
    mfield[(iz + 1) * Nb + (iR + 1)] += 0.5 * dt * (fR) * (fz);
    for(i = 0; i < 3; i++) v[i] += 0.5 * dt * a[i];
    for(i = 0; i < 3; i++) x[i] += dt * v[i];
    orc_forcegrid_acc(m, x, a);
    for(i = 0; i < 3; i++) v[i] += 0.5 * dt * a[i];
    orc_densitygrid_cell(m, x, &iR, &iz, &fR, &fz);
    icell = iz * Nb + iR;
    mfield[iz * Nb + iR] += 0.5 * dt * (1 - fR) * (1 - fz);
    mfield[iz * Nb + (iR + 1)] += 0.5 * dt * (fR) * (1 - fz);
    mfield[(iz + 1) * Nb + iR] += 0.5 * dt * (1 - fR) * (fz);
    mfield[(iz + 1) * Nb + (iR + 1)] += 0.5 * dt * (fR) * (fz);
    tall += dt;
    radsign = v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
    if(radsign > 0 && radsign_previous < 0) norbit++;
    radsign_previous = radsign;
    steps++;
    if(steps > m->step_cap) {
      m->steps_total += steps;
      if(info) { info[0] = (double) steps; info[1] = -1; }
      return -1;
    }
  } while((timespan == 0 && norbit < Norbits) || (timespan != 0 && flag == 0));
  double E1 = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + orc_forcegrid_pot(m, x);
  double fac = mass / tall;
  for(i = 0; i < m->DG_Ngrid; i++) mfield[i] *= fac;
  *orbitstaken = norbit;
  m->steps_total += steps;
  if(info) { info[0] = (double) steps; info[1] = fabs((E1 - E0) / E0); }
  return tall;
}

/* ------------------------------------------------------------ merit machinery */

/* smooth_stack (grid.c:1247-1265) */
void orc_smooth_stack(double *data, int maxlevel)
{
  int l, i, j, n;
  for(l = maxlevel - 1; l >= 0; l--) {
    n = (1 << l);
    for(i = 0; i < n; i++)
      for(j = 0; j < n; j++)
        data[SO(l, i, j)] = data[SO(l + 1, 2 * i, 2 * j)] + data[SO(l + 1, 2 * i + 1, 2 * j)] +
                            data[SO(l + 1, 2 * i, 2 * j + 1)] + data[SO(l + 1, 2 * i + 1, 2 * j + 1)];
  }
}

/* calc_stack_difference (grid.c:1086-1112) */
static double stack_diff_rec(const orc_model *m, const double *d1, const double *d2, int l, int i, int j, int maxlevel,
                             const double *ref1, const double *ref2, double thresh, const double *dist, int flag)
{
  int s = SO(l, i, j);
  if(l >= maxlevel || ref1[s] < thresh) {
    if(flag) {
      if(ref1[s] > 0 && ref2[s] > 0)
        return fabs(d1[s] / ref1[s] - d2[s] / ref2[s]) / dmax((d2[s] / ref2[s]), m->p.LowerDispLimit);
      else
        return 0;
    } else
      return fabs(d1[s] - d2[s]) / min_(dist[s], m->p.R200 / 20.0);
  } else {
    double sum = 0;
    for(int ii = 2 * i; ii <= 2 * i + 1; ii++)
      for(int jj = 2 * j; jj <= 2 * j + 1; jj++)
        sum += stack_diff_rec(m, d1, d2, l + 1, ii, jj, maxlevel, ref1, ref2, thresh, dist, flag);
    return sum;
  }
}

/* calc_stack_difference_mod (grid.c:1115-1151) */
static double stack_diff_mod_rec(const orc_model *m, const double *d1, const double *d2, int l, int i, int j,
                                 int maxlevel, const double *ref1, const double *ref2, double thresh,
                                 const double *dist, int flag)
{
  int s = SO(l, i, j);
  if(l >= maxlevel || ref1[s] < thresh) {
    if(flag == 1) {
      if(ref1[s] > 0 && ref2[s] > 0)
        return fabs(d1[s] / ref1[s] - d2[s] / ref2[s]) / dmax((d2[s] / ref2[s]), m->p.LowerDispLimit);
      else
        return 0;
    } else if(flag == 2) {
      if(ref2[s] > 0)
        return fabs(d1[s] - d2[s]) * (ref1[s] / ref2[s]) / min_(dist[s], m->p.R200 / 20.0);
      else
        return 0;
    } else
      return fabs(d1[s] - d2[s]) / min_(dist[s], m->p.R200 / 20.0);
  } else {
    double sum = 0;
    for(int ii = 2 * i; ii <= 2 * i + 1; ii++)
      for(int jj = 2 * j; jj <= 2 * j + 1; jj++)
        sum += stack_diff_mod_rec(m, d1, d2, l + 1, ii, jj, maxlevel, ref1, ref2, thresh, dist, flag);
    return sum;
  }
}

double orc_stack_difference(orc_model *m, const double *d1, const double *d2, int maxlevel, const double *ref1,
                            const double *ref2, double thresh, const double *dist, int flag)
{
  return stack_diff_rec(m, d1, d2, 0, 0, 0, maxlevel, ref1, ref2, thresh, dist, flag);
}

double orc_stack_difference_mod(orc_model *m, const double *d1, const double *d2, int maxlevel, const double *ref1,
                                const double *ref2, double thresh, const double *dist, int flag)
{
  return stack_diff_mod_rec(m, d1, d2, 0, 0, 0, maxlevel, ref1, ref2, thresh, dist, flag);
}

/* energygrid_get_cell (grid.c:896-938) */
static void energygrid_cell(const orc_model *m, const double *pos, int *iR, int *iz, double *fR, double *fz)
{
  get_cell(m, pos, m->p.EG_Rmin, m->p.EG_Fac, m->EG_Nbin, 0.5, iR, iz, fR, fz);
}

/* add_to_energy_grid (main.c:877-917); egyMass may be NULL */
static void add_to_energy_grid(const orc_model *m, const double *pos, double mass, double vr2, double vt2,
                               double vp2, double vq2, double *egyMass, double *er, double *et, double *ep,
                               double *eq)
{
  int iR, iz;
  double fR, fz;
  const int L = m->p.EG_MaxLevel;
  energygrid_cell(m, pos, &iR, &iz, &fR, &fz);
  vr2 *= mass;
  vt2 *= mass;
  vp2 *= mass;
  vq2 *= mass;
  if(egyMass) {
    egyMass[OFF(L, iz, iR)] += (1 - fR) * (1 - fz) * mass;
    egyMass[OFF(L, iz, iR + 1)] += (fR) * (1 - fz) * mass;
    egyMass[OFF(L, iz + 1, iR)] += (1 - fR) * (fz) * mass;
    egyMass[OFF(L, iz + 1, iR + 1)] += (fR) * (fz) * mass;
  }
  er[OFF(L, iz, iR)] += (1 - fR) * (1 - fz) * vr2;
  er[OFF(L, iz, iR + 1)] += (fR) * (1 - fz) * vr2;
  er[OFF(L, iz + 1, iR)] += (1 - fR) * (fz) * vr2;
  er[OFF(L, iz + 1, iR + 1)] += (fR) * (fz) * vr2;
  et[OFF(L, iz, iR)] += (1 - fR) * (1 - fz) * vt2;
  et[OFF(L, iz, iR + 1)] += (fR) * (1 - fz) * vt2;
  et[OFF(L, iz + 1, iR)] += (1 - fR) * (fz) * vt2;
  et[OFF(L, iz + 1, iR + 1)] += (fR) * (fz) * vt2;
  ep[OFF(L, iz, iR)] += (1 - fR) * (1 - fz) * vp2;
  ep[OFF(L, iz, iR + 1)] += (fR) * (1 - fz) * vp2;
  ep[OFF(L, iz + 1, iR)] += (1 - fR) * (fz) * vp2;
  ep[OFF(L, iz + 1, iR + 1)] += (fR) * (fz) * vp2;
  eq[OFF(L, iz, iR)] += (1 - fR) * (1 - fz) * vq2;
  eq[OFF(L, iz, iR + 1)] += (fR) * (1 - fz) * vq2;
  eq[OFF(L, iz + 1, iR)] += (1 - fR) * (fz) * vq2;
  eq[OFF(L, iz + 1, iR + 1)] += (fR) * (fz) * vq2;
}

/* calc_disp_components_for_particle (disp_fields.c:200-372) */
static void disp_components(orc_model *m, int n, const double *vel, double *vr2, double *vt2, double *vp2,
                            double *vq2)
{
  int type = m->type[n];
  int tovs = type_vel_structure(m, type);
  const double *pos = &m->pos[3 * n];
  if(tovs == 0 || tovs == 1 || tovs == 3) {
    double phi = m_atan2(m, pos[1], pos[0]);
    double theta = m_acos(m, pos[2] / sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]));
    double er[3], ePhi[3], eTheta[3];
    er[0] = m_sin(m, theta) * m_cos(m, phi);
    er[1] = m_sin(m, theta) * m_sin(m, phi);
    er[2] = m_cos(m, theta);
    ePhi[0] = -m_sin(m, phi);
    ePhi[1] = m_cos(m, phi);
    ePhi[2] = 0;
    eTheta[0] = -m_cos(m, theta) * m_cos(m, phi);
    eTheta[1] = -m_cos(m, theta) * m_sin(m, phi);
    eTheta[2] = m_sin(m, theta);
    double vr = vel[0] * er[0] + vel[1] * er[1] + vel[2] * er[2];
    double vphi = vel[0] * ePhi[0] + vel[1] * ePhi[1] + vel[2] * ePhi[2];
    double vtheta = vel[0] * eTheta[0] + vel[1] * eTheta[1] + vel[2] * eTheta[2];
    double vstr = 0;
    if(tovs == 1 || tovs == 3) vstr = orc_vstream(m, pos, type);
    *vr2 = vr * vr;
    *vt2 = vtheta * vtheta;
    *vp2 = (vphi - vstr) * (vphi - vstr);
    *vq2 = vphi * vphi;
  } else if(tovs == 2) {
    double phi = m_atan2(m, pos[1], pos[0]);
    double eR[3], ePhi[3], eZ[3];
    eR[0] = m_cos(m, phi);
    eR[1] = m_sin(m, phi);
    eR[2] = 0;
    ePhi[0] = -m_sin(m, phi);
    ePhi[1] = m_cos(m, phi);
    ePhi[2] = 0;
    eZ[0] = 0;
    eZ[1] = 0;
    eZ[2] = 1;
    double vR = vel[0] * eR[0] + vel[1] * eR[1] + vel[2] * eR[2];
    double vphi = vel[0] * ePhi[0] + vel[1] * ePhi[1] + vel[2] * ePhi[2];
    double vZ = vel[0] * eZ[0] + vel[1] * eZ[1] + vel[2] * eZ[2];
    double vstr = orc_vstream(m, pos, type);
    *vr2 = vR * vR;
    *vt2 = vZ * vZ;
    *vp2 = (vphi - vstr) * (vphi - vstr);
    *vq2 = vphi * vphi;
  }
}

/* calc_global_fit (main.c:251-362) */
static void calc_global_fit(orc_model *m)
{
  const int DL = m->p.DG_MaxLevel, EL = m->p.EG_MaxLevel;
  const int doff = SO(DL, 0, 0), eoff = SO(EL, 0, 0);
  for(int type = 1; type <= 3; type++) {
    memcpy(&m->DGs_MassResponse[type][doff], m->DG_MassLoc[type], m->DG_Ngrid * sizeof(double));
    orc_smooth_stack(m->DGs_MassResponse[type], DL);
    memcpy(&m->EGs_RS[type][eoff], m->EG_RLocS[type], m->EG_Ngrid * sizeof(double));
    orc_smooth_stack(m->EGs_RS[type], EL);
    memcpy(&m->EGs_TS[type][eoff], m->EG_TLocS[type], m->EG_Ngrid * sizeof(double));
    orc_smooth_stack(m->EGs_TS[type], EL);
    memcpy(&m->EGs_QS[type][eoff], m->EG_QLocS[type], m->EG_Ngrid * sizeof(double));
    orc_smooth_stack(m->EGs_QS[type], EL);
    memcpy(&m->EGs_PS[type][eoff], m->EG_PLocS[type], m->EG_Ngrid * sizeof(double));
    orc_smooth_stack(m->EGs_PS[type], EL);
    memcpy(&m->EGs_MassResponse[type][eoff], m->EG_MassLoc[type], m->EG_Ngrid * sizeof(double));
    memcpy(&m->EGs_R[type][eoff], m->EG_RLoc[type], m->EG_Ngrid * sizeof(double));
    memcpy(&m->EGs_T[type][eoff], m->EG_TLoc[type], m->EG_Ngrid * sizeof(double));
    memcpy(&m->EGs_P[type][eoff], m->EG_PLoc[type], m->EG_Ngrid * sizeof(double));
    memcpy(&m->EGs_Q[type][eoff], m->EG_QLoc[type], m->EG_Ngrid * sizeof(double));
    orc_smooth_stack(m->EGs_MassResponse[type], EL);
    orc_smooth_stack(m->EGs_R[type], EL);
    orc_smooth_stack(m->EGs_T[type], EL);
    orc_smooth_stack(m->EGs_P[type], EL);
    orc_smooth_stack(m->EGs_Q[type], EL);

    double thr_d = m->p.MinParticlesPerBinForDensityMeasurement * m->p.MType[type] / m->p.NType[type];
    double thr_e = m->p.MinParticlesPerBinForDispersionMeasurement * m->p.MType[type] / m->p.NType[type];
    m->S[type] = orc_stack_difference(m, m->DGs_MassResponse[type], m->DGs_MassTarget[type], DL,
                                      m->DGs_MassTarget[type], NULL, thr_d, m->DGs_Distance, 0);
    m->S[type] *= 1.0 / m->DGs_MassTarget[type][0];
    m->Sdisp_r[type] = orc_stack_difference(m, m->EGs_R[type], m->EGs_EgyTarget_r[type], EL,
                                            m->EGs_MassResponse[type], m->EGs_MassTarget[type], thr_e, NULL, 1);
    m->Sdisp_t[type] = orc_stack_difference(m, m->EGs_T[type], m->EGs_EgyTarget_t[type], EL,
                                            m->EGs_MassResponse[type], m->EGs_MassTarget[type], thr_e, NULL, 1);
    m->Sdisp_p[type] = orc_stack_difference(m, m->EGs_P[type], m->EGs_EgyTarget_p[type], EL,
                                            m->EGs_MassResponse[type], m->EGs_MassTarget[type], thr_e, NULL, 1);
    m->Sdisp_q[type] = orc_stack_difference(m, m->EGs_Q[type], m->EGs_EgyTarget_q[type], EL,
                                            m->EGs_MassResponse[type], m->EGs_MassTarget[type], thr_e, NULL, 1);
    int tovs = type_vel_structure(m, type);
    if(tovs == 0 || tovs == 1) {
      m->Srelfac_count[type] = 3.0;
      m->Sdisp_q[type] = 0;
    } else
      m->Srelfac_count[type] = 4.0;
    if(m->firstrun[type] == 0) {
      m->Srelfac[type] = m->S[type] / ((m->Sdisp_r[type] + m->Sdisp_t[type] + m->Sdisp_p[type] + m->Sdisp_q[type]) /
                                       m->Srelfac_count[type]);
      m->firstrun[type] = 1;
    }
    m->Sdisp_r[type] *= m->Srelfac[type];
    m->Sdisp_t[type] *= m->Srelfac[type];
    m->Sdisp_p[type] *= m->Srelfac[type];
    m->Sdisp_q[type] *= m->Srelfac[type];
  }
}

static int type_present(const orc_model *m, int type) { return m->p.NType[type] != 0; }

/* calc_all_response_fields (main.c:151-246) */
int orc_calc_all(orc_model *m)
{
  int i, n, type;
  for(type = 1; type <= 3; type++) {
    if(!type_present(m, type)) continue;
    memset(m->DG_MassLoc[type], 0, m->DG_Ngrid * sizeof(double));
    memset(m->EG_RLocS[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_TLocS[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_QLocS[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_PLocS[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_MassLoc[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_RLoc[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_TLoc[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_PLoc[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_QLoc[type], 0, m->EG_Ngrid * sizeof(double));
  }
  double *mo = zalloc(m->DG_Ngrid), *ro = zalloc(m->EG_Ngrid), *to = zalloc(m->EG_Ngrid);
  double *qo = zalloc(m->EG_Ngrid), *po = zalloc(m->EG_Ngrid);
  int status = 0;
  for(n = 0; n < m->n; n++) {
    type = m->type[n];
    double tall = orc_orbit_mod(m, &m->pos[3 * n], &m->vel[3 * n], mo, ro, to, qo, po, m->mass[n], m->tint[n],
                                &m->orbits[n], type, NULL);
    if(tall < 0) { status = GALIC_ERR_STEP_CAP; break; }
    for(i = 0; i < m->DG_Ngrid; i++) m->DG_MassLoc[type][i] += mo[i];
    for(i = 0; i < m->EG_Ngrid; i++) {
      m->EG_RLocS[type][i] += ro[i];
      m->EG_TLocS[type][i] += to[i];
      m->EG_QLocS[type][i] += qo[i];
      m->EG_PLocS[type][i] += po[i];
    }
    double *vd = &m->vdisp[4 * n];
    disp_components(m, n, &m->vel[3 * n], &vd[0], &vd[1], &vd[2], &vd[3]);
    add_to_energy_grid(m, &m->pos[3 * n], m->mass[n], vd[0], vd[1], vd[2], vd[3], m->EG_MassLoc[type],
                       m->EG_RLoc[type], m->EG_TLoc[type], m->EG_PLoc[type], m->EG_QLoc[type]);
  }
  free(mo); free(ro); free(to); free(qo); free(po);
  if(status) return status;
  calc_global_fit(m);
  return 0;
}

/* eval_fit_mod (main.c:1021-1217) */
double orc_eval_fit_mod(orc_model *m, int n, const double *vel, const double *m_new, const double *m_old,
                        const double *r_new, const double *r_old, const double *t_new, const double *t_old,
                        const double *q_new, const double *q_old, const double *p_new, const double *p_old)
{
  int i, type = m->type[n];
  const int DL = m->p.DG_MaxLevel, EL = m->p.EG_MaxLevel;
  double value, value_rs, value_ts, value_qs, value_ps, value_r, value_t, value_p, value_q;
  double thr_d = m->p.MinParticlesPerBinForDensityMeasurement * m->p.MType[type] / m->p.NType[type];
  double thr_e = m->p.MinParticlesPerBinForDispersionMeasurement * m->p.MType[type] / m->p.NType[type];
  double *u = zalloc(m->DG_Nstack > m->EG_Nstack ? m->DG_Nstack : m->EG_Nstack);

  for(i = 0; i < m->DG_Ngrid; i++)
    u[SO(DL, 0, 0) + i] = m->DGs_MassResponse[type][SO(DL, 0, 0) + i] + m_new[i] - m_old[i];
  orc_smooth_stack(u, DL);
  value = orc_stack_difference(m, u, m->DGs_MassTarget[type], DL, m->DGs_MassTarget[type], NULL, thr_d,
                               m->DGs_Distance, 0);
  value *= 1.0 / m->p.MType[type];

  /* the stored offset uses DG_MaxLevel (main.c:1056); requires DG_MaxLevel == EG_MaxLevel */
  for(i = 0; i < m->EG_Ngrid; i++) u[SO(DL, 0, 0) + i] = m->EGs_RS[type][SO(EL, 0, 0) + i] + r_new[i] - r_old[i];
  orc_smooth_stack(u, EL);
  value_rs = orc_stack_difference_mod(m, u, m->EGs_EgyTarget_r[type], EL, m->DGs_MassTarget[type],
                                      m->EGs_EgyTarget_r[type], thr_d, m->DGs_Distance, 2) / m->p.MType[type];
  for(i = 0; i < m->EG_Ngrid; i++) u[SO(EL, 0, 0) + i] = m->EGs_TS[type][SO(EL, 0, 0) + i] + t_new[i] - t_old[i];
  orc_smooth_stack(u, EL);
  value_ts = orc_stack_difference_mod(m, u, m->EGs_EgyTarget_t[type], EL, m->DGs_MassTarget[type],
                                      m->EGs_EgyTarget_t[type], thr_d, m->DGs_Distance, 2) / m->p.MType[type];
  for(i = 0; i < m->EG_Ngrid; i++) u[SO(EL, 0, 0) + i] = m->EGs_QS[type][SO(EL, 0, 0) + i] + q_new[i] - q_old[i];
  orc_smooth_stack(u, EL);
  value_qs = orc_stack_difference_mod(m, u, m->EGs_EgyTarget_q[type], EL, m->DGs_MassTarget[type],
                                      m->EGs_EgyTarget_q[type], thr_d, m->DGs_Distance, 2) / m->p.MType[type];
  for(i = 0; i < m->EG_Ngrid; i++) u[SO(EL, 0, 0) + i] = m->EGs_PS[type][SO(EL, 0, 0) + i] + p_new[i] - p_old[i];
  orc_smooth_stack(u, EL);
  value_ps = orc_stack_difference_mod(m, u, m->EGs_EgyTarget_p[type], EL, m->DGs_MassTarget[type],
                                      m->EGs_EgyTarget_p[type], thr_d, m->DGs_Distance, 2) / m->p.MType[type];

  double vr2, vt2, vp2, vq2, mass = m->mass[n];
  disp_components(m, n, vel, &vr2, &vt2, &vp2, &vq2);
  double *vd = &m->vdisp[4 * n];
  double vr2_diff = (vr2 - vd[0]), vt2_diff = (vt2 - vd[1]), vp2_diff = (vp2 - vd[2]), vq2_diff = (vq2 - vd[3]);
  const int off = SO(EL, 0, 0);
  double *ur = zalloc(m->EG_Nstack), *ut = zalloc(m->EG_Nstack), *up = zalloc(m->EG_Nstack);
  double *uq = zalloc(m->EG_Nstack);
  for(i = 0; i < m->EG_Ngrid; i++) {
    ur[off + i] = m->EGs_R[type][off + i];
    ut[off + i] = m->EGs_T[type][off + i];
    up[off + i] = m->EGs_P[type][off + i];
    uq[off + i] = m->EGs_Q[type][off + i];
  }
  add_to_energy_grid(m, &m->pos[3 * n], mass, vr2_diff, vt2_diff, vp2_diff, vq2_diff, NULL, ur + off, ut + off,
                     up + off, uq + off);
  orc_smooth_stack(ur, EL);
  orc_smooth_stack(ut, EL);
  orc_smooth_stack(up, EL);
  orc_smooth_stack(uq, EL);
  value_r = orc_stack_difference(m, ur, m->EGs_EgyTarget_r[type], EL, m->EGs_MassResponse[type],
                                 m->EGs_MassTarget[type], thr_e, NULL, 1);
  value_t = orc_stack_difference(m, ut, m->EGs_EgyTarget_t[type], EL, m->EGs_MassResponse[type],
                                 m->EGs_MassTarget[type], thr_e, NULL, 1);
  value_p = orc_stack_difference(m, up, m->EGs_EgyTarget_p[type], EL, m->EGs_MassResponse[type],
                                 m->EGs_MassTarget[type], thr_e, NULL, 1);
  value_q = orc_stack_difference(m, uq, m->EGs_EgyTarget_q[type], EL, m->EGs_MassResponse[type],
                                 m->EGs_MassTarget[type], thr_e, NULL, 1);
  free(u); free(ur); free(ut); free(up); free(uq);
  int tovs = type_vel_structure(m, type);
  if(tovs == 0 || type == 2) value_q = 0; /* main.c:1195 */
  return value + m->Srelfac[type] / m->Srelfac_count[type] * (value_r + value_t + value_p + value_q) +
         (m->p.fac_value_rs[type] * value_rs + m->p.fac_value_ts[type] * value_ts +
          m->p.fac_value_ps[type] * value_ps + m->p.fac_value_qs[type] * value_qs) / 4;
}

/* init_updates (main.c:844-874) */
static void init_updates(orc_model *m)
{
  for(int type = 1; type <= 3; type++) {
    if(!type_present(m, type)) continue;
    memset(m->DG_MassLoc_d[type], 0, m->DG_Ngrid * sizeof(double));
    memset(m->EG_RLocS_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_TLocS_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_QLocS_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_PLocS_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_RLoc_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_TLoc_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_PLoc_d[type], 0, m->EG_Ngrid * sizeof(double));
    memset(m->EG_QLoc_d[type], 0, m->EG_Ngrid * sizeof(double));
  }
}

/* commit_updates (main.c:808-841) */
static void commit_updates(orc_model *m)
{
  int i;
  for(int type = 1; type <= 3; type++) {
    if(!type_present(m, type)) continue;
    for(i = 0; i < m->DG_Ngrid; i++) m->DG_MassLoc[type][i] += m->DG_MassLoc_d[type][i];
    for(i = 0; i < m->EG_Ngrid; i++) {
      m->EG_RLocS[type][i] += m->EG_RLocS_d[type][i];
      m->EG_TLocS[type][i] += m->EG_TLocS_d[type][i];
      m->EG_QLocS[type][i] += m->EG_QLocS_d[type][i];
      m->EG_PLocS[type][i] += m->EG_PLocS_d[type][i];
    }
    for(i = 0; i < m->EG_Ngrid; i++) {
      m->EG_RLoc[type][i] += m->EG_RLoc_d[type][i];
      m->EG_TLoc[type][i] += m->EG_TLoc_d[type][i];
      m->EG_PLoc[type][i] += m->EG_PLoc_d[type][i];
      m->EG_QLoc[type][i] += m->EG_QLoc_d[type][i];
    }
  }
  calc_global_fit(m);
}

/* optimize (main.c:365-527, VER_1_1); proposals from Philox stream (seed, n, rep_serial) */
static int optimize(orc_model *m, int n, uint64_t seed, uint32_t rep_serial)
{
  int i, k, orbits_try;
  int type = m->type[n];
  int tovs = type_vel_structure(m, type);
  const double *pos = &m->pos[3 * n];
  double *vel = &m->vel[3 * n];
  grng_t g;
  grng_init(&g, seed, (uint32_t) n, rep_serial);
  (void) grng_uniform(&g); /* dir_rnd, main.c:370 */

  double phi = m_atan2(m, pos[1], pos[0]);
  double R[3], T[3], Q[3];
  if(tovs == 2) {
    R[0] = m_cos(m, phi); R[1] = m_sin(m, phi); R[2] = 0;
    T[0] = -m_sin(m, phi); T[1] = m_cos(m, phi); T[2] = 0;
    Q[0] = 0; Q[1] = 0; Q[2] = 1;
  } else {
    double phi2 = m_atan2(m, pos[1], pos[0]);
    double theta = m_acos(m, pos[2] / sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]));
    R[0] = m_sin(m, theta) * m_cos(m, phi2); R[1] = m_sin(m, theta) * m_sin(m, phi2); R[2] = m_cos(m, theta);
    T[0] = -m_cos(m, theta) * m_cos(m, phi2); T[1] = -m_cos(m, theta) * m_sin(m, phi2); T[2] = m_sin(m, theta);
    Q[0] = -m_sin(m, phi2); Q[1] = m_cos(m, phi2); Q[2] = 0;
  }
  const double *tg = &m->targets[4 * n];
  double sigma_r = sqrt(tg[0]), sigma_t = sqrt(tg[1]), sigma_p = sqrt(tg[2]);
  double vstr = orc_vstream(m, pos, type);
  double vr_new, vt_new, vq_new, v_new[3], v2_new;
  int iter = 0;
  do {
    vr_new = grng_gaussian(&g, sigma_r);
    vt_new = grng_gaussian(&g, sigma_t);
    vq_new = vstr + grng_gaussian(&g, sigma_p);
    v_new[0] = vr_new * R[0] + vt_new * T[0] + vq_new * Q[0];
    v_new[1] = vr_new * R[1] + vt_new * T[1] + vq_new * Q[1];
    v_new[2] = vr_new * R[2] + vt_new * T[2] + vq_new * Q[2];
    v2_new = v_new[0] * v_new[0] + v_new[1] * v_new[1] + v_new[2] * v_new[2];
    iter++;
    if(iter > 100000) return GALIC_ERR_REJECTION_CAP;
  } while(sqrt(v2_new) >= m->p.MaxVelInUnitsVesc * m->vesc[n]);

  double vel_try[3];
  for(k = 0; k < 3; k++) vel_try[k] = v_new[k];
  const int G = m->DG_Ngrid, E = m->EG_Ngrid;
  double *mo = zalloc(G), *mn = zalloc(G), *ro = zalloc(E), *rn = zalloc(E), *to = zalloc(E), *tn = zalloc(E);
  double *qo = zalloc(E), *qn = zalloc(E), *po = zalloc(E), *pn = zalloc(E);
  double t1 = orc_orbit_mod(m, pos, vel, mo, ro, to, qo, po, m->mass[n], m->tint[n], &m->orbits[n], type, NULL);
  double t2 = orc_orbit_mod(m, pos, vel_try, mn, rn, tn, qn, pn, m->mass[n], m->tint[n], &orbits_try, type, NULL);
  int status = 0;
  if(t1 < 0 || t2 < 0) status = GALIC_ERR_STEP_CAP;
  if(!status) {
    double F_base = orc_eval_fit_mod(m, n, vel, mo, mo, ro, ro, to, to, qo, qo, po, po);
    double F_try = orc_eval_fit_mod(m, n, vel_try, mn, mo, rn, ro, tn, to, qn, qo, pn, po);
    m->tries[type]++;
    if(F_try < F_base) {
      for(k = 0; k < 3; k++) vel[k] = vel_try[k];
      m->orbits[n] = orbits_try;
      for(i = 0; i < G; i++) m->DG_MassLoc_d[type][i] += mn[i] - mo[i];
      for(i = 0; i < E; i++) {
        m->EG_RLocS_d[type][i] += rn[i] - ro[i];
        m->EG_TLocS_d[type][i] += tn[i] - to[i];
        m->EG_QLocS_d[type][i] += qn[i] - qo[i];
        m->EG_PLocS_d[type][i] += pn[i] - po[i];
      }
      double vr2, vt2, vp2, vq2;
      disp_components(m, n, vel_try, &vr2, &vt2, &vp2, &vq2);
      double *vd = &m->vdisp[4 * n];
      double vr2_diff = (vr2 - vd[0]), vt2_diff = (vt2 - vd[1]), vp2_diff = (vp2 - vd[2]), vq2_diff = (vq2 - vd[3]);
      add_to_energy_grid(m, pos, m->mass[n], vr2_diff, vt2_diff, vp2_diff, vq2_diff, NULL, m->EG_RLoc_d[type],
                         m->EG_TLoc_d[type], m->EG_PLoc_d[type], m->EG_QLoc_d[type]);
      vd[0] = vr2;
      vd[1] = vt2;
      vd[2] = vp2;
      vd[3] = vq2;
      m->changes[type]++;
    }
  }
  free(mo); free(mn); free(ro); free(rn); free(to); free(tn); free(qo); free(qn); free(po); free(pn);
  return status;
}

/* one repetition (main.c:96-100) over an explicit particle list */
int orc_optimize_rep(orc_model *m, const int *idx, int count, uint64_t seed, uint32_t rep_serial)
{
  init_updates(m);
  for(int k = 0; k < count; k++) {
    int st = optimize(m, idx[k], seed, rep_serial);
    if(st) return st;
  }
  commit_updates(m);
  return 0;
}

void orc_get_fit(orc_model *m, double *out)
{
  for(int t = 0; t < 4; t++) {
    out[7 * t + 0] = m->S[t];
    out[7 * t + 1] = m->Sdisp_r[t];
    out[7 * t + 2] = m->Sdisp_t[t];
    out[7 * t + 3] = m->Sdisp_p[t];
    out[7 * t + 4] = m->Sdisp_q[t];
    out[7 * t + 5] = m->Srelfac[t];
    out[7 * t + 6] = m->Srelfac_count[t];
  }
}

void orc_get_counters(orc_model *m, long long *tries, long long *changes)
{
  for(int t = 0; t < 4; t++) {
    tries[t] = m->tries[t];
    changes[t] = m->changes[t];
  }
}

void orc_get_response(orc_model *m, int type, int which, double *out)
{
  double *src = NULL;
  switch(which) {
    case GALIC_GRID_MASS_S: src = m->DG_MassLoc[type]; break;
    case GALIC_GRID_R_S: src = m->EG_RLocS[type]; break;
    case GALIC_GRID_T_S: src = m->EG_TLocS[type]; break;
    case GALIC_GRID_Q_S: src = m->EG_QLocS[type]; break;
    case GALIC_GRID_P_S: src = m->EG_PLocS[type]; break;
    case GALIC_GRID_MASS_I: src = m->EG_MassLoc[type]; break;
    case GALIC_GRID_R_I: src = m->EG_RLoc[type]; break;
    case GALIC_GRID_T_I: src = m->EG_TLoc[type]; break;
    case GALIC_GRID_P_I: src = m->EG_PLoc[type]; break;
    case GALIC_GRID_Q_I: src = m->EG_QLoc[type]; break;
  }
  if(src) memcpy(out, src, m->DG_Ngrid * sizeof(double));
}

long long orc_steps_total(orc_model *m) { return m->steps_total; }

/* ------------------------------------------------------------ grid geometry */

/* the Newton iteration of grid.c:358-372 (also 429-443, 461-475) */
static int solve_fac(double y, int nbin, double *fac_out)
{
  double fac = 1.02, dfac;
  int iter = 0;
  do {
    double f = log((pow(fac, nbin) - 1.0) / (y * (fac - 1.0)));
    double df = nbin / (fac - 1.0 / pow(fac, nbin - 1)) - 1.0 / (fac - 1.0);
    dfac = -f / df;
    fac += dfac;
    iter++;
    if(iter > 1000) return 1; /* MAXITER, allvars.h:270 */
  } while(fabs(dfac) > 1.0e-8 * fac);
  *fac_out = fac;
  return 0;
}

/* forcedensitygrid_create (grid.c:329-480) */
int orc_grid_geometry(double halo_a, double outer_frac, double inner_frac, int fg_nbin, int dg_maxlevel,
                      int eg_maxlevel, double *out)
{
  double fac = outer_frac;
  double Rmax = halo_a * (fac + sqrt(fac)) / (1 - fac);
  fac = inner_frac;
  double DG_Rin = halo_a * (fac + sqrt(fac)) / (1 - fac);
  double dgf, fgf, egf;
  if(solve_fac(Rmax / DG_Rin, 1 << dg_maxlevel, &dgf)) return 1;
  if(solve_fac(Rmax / DG_Rin, fg_nbin, &fgf)) return 1;
  if(solve_fac(Rmax / DG_Rin, 1 << eg_maxlevel, &egf)) return 1;
  out[0] = Rmax;
  out[1] = DG_Rin;
  out[2] = dgf;
  out[3] = DG_Rin / (dgf - 1.0);
  out[4] = fgf;
  out[5] = DG_Rin / (fgf - 1.0);
  out[6] = egf;
  out[7] = DG_Rin / (egf - 1.0);
  return 0;
}

/* DGs_Distance (grid.c:381-416) and DG_CellSize/DG_CellVol (grid.c:830-850) */
int orc_density_geometry(int L, double rmin, double fac, double *dist, double *cellsize, double *cellvol)
{
  int nbin = 1 << L, nstack = ((1 << (2 + 2 * L)) - 1) / 3;
  double *logR = zalloc(nstack), *logZ = zalloc(nstack);
  int i, j, k, l;
  for(k = 0; k < nbin; k++)
    for(j = 0; j < nbin; j++) {
      double z = rmin * 0.5 * (pow(fac, k) + pow(fac, k + 1) - 2.0);
      double R = rmin * 0.5 * (pow(fac, j) + pow(fac, j + 1) - 2.0);
      logR[SO(L, k, j)] = log(R);
      logZ[SO(L, k, j)] = log(z);
    }
  orc_smooth_stack(logR, L);
  orc_smooth_stack(logZ, L);
  for(l = L - 1; l >= 0; l--) {
    int n = (1 << l);
    int f = (1 << (L - l));
    for(i = 0; i < n; i++)
      for(j = 0; j < n; j++) {
        logR[SO(l, i, j)] /= (f * f);
        logZ[SO(l, i, j)] /= (f * f);
      }
  }
  for(l = L; l >= 0; l--) {
    int n = (1 << l);
    for(i = 0; i < n; i++)
      for(j = 0; j < n; j++)
        dist[SO(l, i, j)] = sqrt(pow(exp(logR[SO(l, i, j)]), 2) + pow(exp(logZ[SO(l, i, j)]), 2));
  }
  for(k = 0; k < nbin; k++)
    for(j = 0; j < nbin; j++) {
      i = k * nbin + j;
      double r1 = rmin * (pow(fac, j) - 1.0);
      double r2 = rmin * (pow(fac, j + 1) - 1.0);
      double z1 = rmin * (pow(fac, k) - 1.0);
      double z2 = rmin * (pow(fac, k + 1) - 1.0);
      double vol = M_PI * (r2 * r2 - r1 * r1) * (z2 - z1);
      vol *= 2;
      cellsize[i] = dmax(r2 - r1, z2 - z1);
      cellvol[i] = vol;
    }
  free(logR);
  free(logZ);
  return 0;
}
