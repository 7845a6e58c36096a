/*
 * oracle_sampling.c - CPU restatement of GALIC's set-up sampling:
 *   orc_sample_positions  {halo,disk,bulge}_get_fresh_coordinate
 *                         (halo.c:17-40, disk.c:17-50, bulge.c:15-37)
 *   orc_sample_density    one type of densitygrid_sample_targetresponse
 *                         (grid.c:536-617)
 *   orc_sample_energy     one type of calc_energy_grid_mass_maps
 *                         (grid.c:941-1076) with get_disp_rtp
 *                         (disp_fields.c:26-198, 375-398)
 *
 * TEST INFRASTRUCTURE: the checker for galic_b200/csrc/sampling.cu.  Only
 * tests/ and bench.py's CPU-baseline leg load it.
 *
 * The loops are the reference's, sequential, drawing from the same stream
 * stand-in (grng.h) the oracle's GSL shim gives the reference.  With
 * use_libm = 1 (glibc's log/exp/sin/cos/acos, like the reference) every
 * sample, the bins (summed in draw order) and the stream position are those
 * of GALIC's own functions; with use_libm = 0 (gmath.h, like the CUDA
 * kernels) every sample is bit-identical to the GPU's.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "galic_oracle.h"
#include "oracle_internal.h"

typedef struct {
  int use_libm;
} smath;

static double s_log(const smath *m, double x) { return m->use_libm ? log(x) : gm_log(x); }
static double s_exp(const smath *m, double x) { return m->use_libm ? exp(x) : gm_exp(x); }
static double s_sin(const smath *m, double x) { return m->use_libm ? sin(x) : gm_sin(x); }
static double s_cos(const smath *m, double x) { return m->use_libm ? cos(x) : gm_cos(x); }
static double s_acos(const smath *m, double x) { return m->use_libm ? acos(x) : gm_acos(x); }

static const double S_PI = 3.14159265358979323846; /* M_PI */

/* halo.c:17-40 */
static void halo_fresh(const smath *m, const galic_sample_params_t *sp, grng_t *g, double *pos)
{
  double r;
  do {
    double q = grng_uniform(g);
    if(q > 0)
      r = sp->Halo_A * (q + sqrt(q)) / (1 - q);
    else
      r = 0;
    double phi = grng_uniform(g) * S_PI * 2;
    double theta = s_acos(m, grng_uniform(g) * 2 - 1);
    pos[0] = r * s_sin(m, theta) * s_cos(m, phi);
    pos[1] = r * s_sin(m, theta) * s_sin(m, phi);
    pos[2] = r * s_cos(m, theta) / sp->HaloStretch;
    r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  } while(r > sp->Rmax);
}

/* disk.c:17-50 */
static void disk_fresh(const smath *m, const galic_sample_params_t *sp, grng_t *g, double *pos)
{
  double q, f, f_, R, R2, Rold, phi;
  do {
    q = grng_uniform(g);
    pos[2] = sp->Disk_Z0 / 2 * s_log(m, q / (1 - q));
    q = grng_uniform(g);
    R = 1.0;
    do {
      f = (1 + R) * s_exp(m, -R) + q - 1;
      f_ = -R * s_exp(m, -R);
      Rold = R;
      R = R - f / f_;
    } while(fabs(R - Rold) / R > 1e-7);
    R *= sp->Disk_H;
    phi = grng_uniform(g) * S_PI * 2;
    pos[0] = R * s_cos(m, phi);
    pos[1] = R * s_sin(m, phi);
    R2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2];
  } while(R2 > sp->Rmax * sp->Rmax);
}

/* bulge.c:15-37 */
static void bulge_fresh(const smath *m, const galic_sample_params_t *sp, grng_t *g, double *pos)
{
  double r;
  do {
    double q = grng_uniform(g);
    if(q > 0)
      r = sp->Bulge_A * (q + sqrt(q)) / (1 - q);
    else
      r = 0;
  } while(r > sp->Rmax);
  double phi = grng_uniform(g) * S_PI * 2;
  double theta = s_acos(m, grng_uniform(g) * 2 - 1);
  pos[0] = r * s_sin(m, theta) * s_cos(m, phi);
  pos[1] = r * s_sin(m, theta) * s_sin(m, phi);
  pos[2] = r * s_cos(m, theta) / sp->BulgeStretch;
}

/* the dispatch of grid.c:563-568 */
static void fresh(const smath *m, const galic_sample_params_t *sp, int type, grng_t *g, double *pos);
void orc_fresh(int use_libm, const galic_sample_params_t *sp, int type, grng_t *g, double *pos)
{
  smath m = {use_libm};
  fresh(&m, sp, type, g, pos);
}
static void fresh(const smath *m, const galic_sample_params_t *sp, int type, grng_t *g, double *pos)
{
  if(type == 1)
    halo_fresh(m, sp, g, pos);
  else if(type == 2)
    disk_fresh(m, sp, g, pos);
  else
    bulge_fresh(m, sp, g, pos);
}

static void stream_open(grng_t *g, const galic_stream_t *s)
{
  grng_init(g, s->seed, s->a, s->b);
  grng_seek(g, s->position);
}

/* n calls of the type's sampler */
void orc_sample_positions(const galic_sample_params_t *sp, int type, long long n, galic_stream_t *stream,
                          int use_libm, double *pos)
{
  smath m = {use_libm};
  grng_t g;
  stream_open(&g, stream);
  for(long long i = 0; i < n; i++) fresh(&m, sp, type, &g, &pos[3 * i]);
  stream->position = grng_position(&g);
}

/* densitygrid_get_cell (grid.c:494-534) and energygrid_get_cell
 * (grid.c:896-939): the same steps on their own geometry */
static void grid_cell(const smath *m, const double *pos, double Rmin, double Fac, int Nbin, int *iR, int *iz,
                      double *fR, double *fz)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = fabs(pos[2]);
  double br = (s_log(m, r / Rmin + 1.0) / s_log(m, Fac)) - 0.5;
  double bz = (s_log(m, z / Rmin + 1.0) / s_log(m, Fac)) - 0.5;
  int binr, binz;
  if(br < 0) br = 0;
  if(bz < 0) bz = 0;
  binr = (int) br;
  *fR = br - binr;
  binz = (int) bz;
  *fz = bz - binz;
  if(binr >= Nbin - 1) {
    binr = Nbin - 2;
    *fR = 1;
  }
  if(binz >= Nbin - 1) {
    binz = Nbin - 2;
    *fz = 1;
  }
  *iR = binr;
  *iz = binz;
}

/* scale by MType / nsum and smooth (grid.c:604-614 / 1050-1066) */
static void finish_stack(double *stack, int L, double mtype, long long ntarget)
{
  int off = ((1 << (2 * L)) - 1) / 3, G = 1 << (2 * L);
  double nsum = (double) ntarget;
  for(int i = 0; i < G; i++) stack[off + i] *= mtype / nsum;
  orc_smooth_stack(stack, L);
}

/* one type of densitygrid_sample_targetresponse (grid.c:536-617) with one
 * rank; renorm adds forcedensitygrid_calculate's recalibration
 * (grid.c:862-880).  stack: DG_Nstack doubles, overwritten. */
void orc_sample_density(const galic_params_t *p, const galic_sample_params_t *sp, int type, long long ntarget,
                        galic_stream_t *stream, int use_libm, int renorm, double *stack)
{
  smath m = {use_libm};
  const int L = p->DG_MaxLevel, N = 1 << L, G = N * N, off = ((1 << (2 * L)) - 1) / 3;
  double *mfield = calloc((size_t) G, sizeof(double));
  grng_t g;
  stream_open(&g, stream);
  long long count = 0;
  double pos[3];
  while(count < ntarget) {
    fresh(&m, sp, type, &g, pos);
    double r = sqrt(pos[0] * pos[0] + pos[2] * pos[2]);
    if(r < sp->Rmax) {
      int iR, iz;
      double fR, fz;
      grid_cell(&m, pos, p->DG_Rmin, p->DG_Fac, N, &iR, &iz, &fR, &fz);
      mfield[iz * N + iR] += (1 - fR) * (1 - fz);
      mfield[iz * N + (iR + 1)] += (fR) * (1 - fz);
      mfield[(iz + 1) * N + iR] += (1 - fR) * (fz);
      mfield[(iz + 1) * N + (iR + 1)] += (fR) * (fz);
      count++;
    }
  }
  stream->position = grng_position(&g);
  memset(stack, 0, (size_t) (((1 << (2 * (L + 1))) - 1) / 3) * sizeof(double));
  memcpy(stack + off, mfield, (size_t) G * sizeof(double));
  finish_stack(stack, L, p->MType[type], ntarget);
  if(renorm) {
    double msum = 0;
    for(int i = 0; i < G; i++) msum += stack[off + i];
    if(msum > 0)
      for(int i = 0; i < G; i++) stack[off + i] *= p->MType[type] / msum;
  }
  free(mfield);
}

/* forcegrid_get_cell (grid.c:15-55) */
static void fg_cell(const smath *m, const galic_params_t *p, const double *pos, int *iR, int *iz, double *fR,
                    double *fz)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = fabs(pos[2]);
  double br = (s_log(m, r / p->FG_Rmin + 1.0) / s_log(m, p->FG_Fac));
  double bz = (s_log(m, z / p->FG_Rmin + 1.0) / s_log(m, p->FG_Fac));
  int binr, binz;
  if(br < 0) br = 0;
  if(bz < 0) bz = 0;
  binr = (int) br;
  *fR = br - binr;
  binz = (int) bz;
  *fz = bz - binz;
  if(binr >= p->FG_Nbin - 1) {
    binr = p->FG_Nbin - 2;
    *fR = 1;
  }
  if(binz >= p->FG_Nbin - 1) {
    binz = p->FG_Nbin - 2;
    *fz = 1;
  }
  *iR = binr;
  *iz = binz;
}

/* the bilinear lookups of disp_fields.c:118-195 */
static double fg_interp(const smath *m, const galic_params_t *p, const double *T, const double *pos)
{
  int iz, iR;
  double fR, fz;
  fg_cell(m, p, pos, &iR, &iz, &fR, &fz);
  const int N = p->FG_Nbin;
  return T[iz * N + iR] * (1 - fR) * (1 - fz) + T[(iz + 1) * N + iR] * (1 - fR) * (fz) +
         T[iz * N + (iR + 1)] * (fR) * (1 - fz) + T[(iz + 1) * N + (iR + 1)] * (fR) * (fz);
}

/* get_radial_disp_spherical (disp_fields.c:375-398) */
static double radial_disp(const smath *m, const galic_params_t *p, const double *T, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double br = (s_log(m, r / p->FG_Rmin + 1.0) / s_log(m, p->FG_Fac));
  int binr;
  double fR;
  if(br < 0) br = 0;
  binr = (int) br;
  fR = br - binr;
  if(binr >= p->FG_Nbin - 1) {
    binr = p->FG_Nbin - 2;
    fR = 1;
  }
  return T[binr] * (1 - fR) + T[binr + 1] * (fR);
}

/* get_beta_of_type (disp_fields.c:26-60) */
static double beta_of(const galic_sample_params_t *sp, int type, const double *pos)
{
  double beta = 0, a = 0;
  if(type == 1) {
    beta = sp->HaloBetaParameter;
    a = sp->Halo_A;
  } else if(type == 3) {
    beta = sp->BulgeBetaParameter;
    a = sp->Bulge_A;
  }
  if(type != 2 && beta >= 1) {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    double dlogrhodr = -1.0 - 3.0 * r / (r + a);
    beta = -0.15 - 0.20 * dlogrhodr;
  }
  return beta;
}

/* get_disp_rtp (disp_fields.c:66-115); tab: disp_r, dispz, dispphi,
 * tilted_vr2, tilted_vz2, vstream */
static void disp_rtp(const smath *m, const galic_params_t *p, const galic_sample_params_t *sp, int type,
                     const double *const *tab, const double *pos, double *dr, double *dt, double *dp, double *dq);
void orc_disp_rtp(int use_libm, const galic_params_t *p, const galic_sample_params_t *sp, int type,
                  const double *const *tab, const double *pos, double *d)
{
  smath m = {use_libm};
  disp_rtp(&m, p, sp, type, tab, pos, &d[0], &d[1], &d[2], &d[3]);
}
double orc_vstream_tab(int use_libm, const galic_params_t *p, const double *vstream, const double *pos)
{
  smath m = {use_libm};
  return fg_interp(&m, p, vstream, pos);
}
static void disp_rtp(const smath *m, const galic_params_t *p, const galic_sample_params_t *sp, int type,
                     const double *const *tab, const double *pos, double *dr, double *dt, double *dp, double *dq)
{
  int tovs = p->TypeOfVelocityStructure[type];
  if(tovs == 0) {
    *dr = radial_disp(m, p, tab[0], pos);
    *dt = *dr;
    *dp = *dr;
    *dq = *dr;
  } else if(tovs == 1) {
    *dr = radial_disp(m, p, tab[0], pos);
    *dt = (1 - beta_of(sp, type, pos)) * (*dr);
    *dp = *dt;
    *dq = *dt;
  } else if(tovs == 2) {
    *dt = fg_interp(m, p, tab[1], pos);
    *dr = *dt;
    *dp = fg_interp(m, p, tab[2], pos);
    double vstr = tab[5] ? fg_interp(m, p, tab[5], pos) : 0.0;
    *dq = (*dp) + vstr * vstr;
  } else {
    *dr = fg_interp(m, p, tab[3], pos);
    *dt = fg_interp(m, p, tab[4], pos);
    *dp = fg_interp(m, p, tab[2], pos);
    double vstr = tab[5] ? fg_interp(m, p, tab[5], pos) : 0.0;
    *dq = (*dp) + vstr * vstr;
  }
}

/* one type of calc_energy_grid_mass_maps (grid.c:941-1076) with one rank.
 * tab: FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime,
 * FG_tilted_vz2_prime, FG_Vstream of the type (unread ones may be NULL).
 * stacks: 5 x EG_Nstack doubles (mass, r, t, p, q), overwritten. */
void orc_sample_energy(const galic_params_t *p, const galic_sample_params_t *sp, int type, long long ntarget,
                       galic_stream_t *stream, int use_libm, const double *const *tab, double *stacks)
{
  smath m = {use_libm};
  const int L = p->EG_MaxLevel, N = 1 << L, G = N * N, off = ((1 << (2 * L)) - 1) / 3;
  const int Ns = ((1 << (2 * (L + 1))) - 1) / 3;
  double *f[5];
  for(int k = 0; k < 5; k++) f[k] = calloc((size_t) G, sizeof(double));
  grng_t g;
  stream_open(&g, stream);
  long long count = 0;
  double pos[3];
  while(count < ntarget) {
    fresh(&m, sp, type, &g, pos);
    double r = sqrt(pos[0] * pos[0] + pos[2] * pos[2]);
    if(r < sp->Rmax) {
      int iR, iz;
      double fR, fz;
      grid_cell(&m, pos, p->EG_Rmin, p->EG_Fac, N, &iR, &iz, &fR, &fz);
      double d[4] = {0, 0, 0, 0};
      disp_rtp(&m, p, sp, type, tab, pos, &d[0], &d[1], &d[2], &d[3]);
      f[0][iz * N + iR] += (1 - fR) * (1 - fz);
      f[0][iz * N + (iR + 1)] += (fR) * (1 - fz);
      f[0][(iz + 1) * N + iR] += (1 - fR) * (fz);
      f[0][(iz + 1) * N + (iR + 1)] += (fR) * (fz);
      for(int k = 0; k < 4; k++) {
        f[k + 1][iz * N + iR] += (1 - fR) * (1 - fz) * d[k];
        f[k + 1][iz * N + (iR + 1)] += (fR) * (1 - fz) * d[k];
        f[k + 1][(iz + 1) * N + iR] += (1 - fR) * (fz) * d[k];
        f[k + 1][(iz + 1) * N + (iR + 1)] += (fR) * (fz) * d[k];
      }
      count++;
    }
  }
  stream->position = grng_position(&g);
  for(int k = 0; k < 5; k++) {
    double *st = stacks + (size_t) k * Ns;
    memset(st, 0, (size_t) Ns * sizeof(double));
    memcpy(st + off, f[k], (size_t) G * sizeof(double));
    finish_stack(st, L, p->MType[type], ntarget);
    free(f[k]);
  }
}
