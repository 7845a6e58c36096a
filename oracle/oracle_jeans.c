/*
 * oracle_jeans.c - CPU restatement of calculate_dispfield
 * (disp_fields.c:502-1049) with its helpers get_density_of_type
 * (disp_fields.c:11-24 with halo.c:43-54, disk.c:53-69, bulge.c:39-48),
 * get_beta_of_type (disp_fields.c:26-60), integrate_axisymmetric_jeans
 * (disp_fields.c:427-453), integrate_spherical_jeans_beta
 * (disp_fields.c:456-499), h_factor and h_over_R (disp_fields.c:1051-1105).
 *
 * TEST INFRASTRUCTURE: the checker for galic_b200/csrc/jeans.cu.  Only
 * tests/ and bench.py's CPU-baseline leg load it.
 *
 * The loops are the reference's, in its order.  With use_libm = 1 (glibc's
 * log/exp/sin/cos/atan/tan/pow) the tables are bit-identical to GALIC's own
 * calculate_dispfield; with use_libm = 0 the transcendental calls are the
 * project's (gmath.h; tan = sin/cos, atan(x) = atan2(x, 1), pow(x, 2) = x*x,
 * pow(x, 3) = x*x*x), as in the CUDA kernels.  The grid radii
 * FG_Rmin * (pow(FG_Fac, j) - 1) always come from the C library's pow: the
 * CUDA path computes that table on the host.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "galic_oracle.h"
#include "../galic_b200/csrc/gmath.h"

#define MIN_DENSITY 1e-25 /* allvars.h:201 */
static const double J_PI = 3.14159265358979323846;

typedef struct {
  orc_model *m;
  const galic_sample_params_t *sp;
  const galic_jeans_params_t *jp;
  int libm;
} jctx;

static double j_log(const jctx *c, double x) { return c->libm ? log(x) : gm_log(x); }
static double j_exp(const jctx *c, double x) { return c->libm ? exp(x) : gm_exp(x); }
static double j_sin(const jctx *c, double x) { return c->libm ? sin(x) : gm_sin(x); }
static double j_cos(const jctx *c, double x) { return c->libm ? cos(x) : gm_cos(x); }
static double j_tan(const jctx *c, double x) { return c->libm ? tan(x) : gm_sin(x) / gm_cos(x); }
static double j_atan(const jctx *c, double x) { return c->libm ? atan(x) : gm_atan2(x, 1.0); }
static double j_sq(const jctx *c, double x) { return c->libm ? pow(x, 2) : x * x; }
static double j_cube(const jctx *c, double x) { return c->libm ? pow(x, 3) : x * x * x; }

/* FG_Rmin * (pow(FG_Fac, j) - 1.0), the radius of force-grid line j */
static double fg_r(const jctx *c, int j) { return c->m->p.FG_Rmin * (pow(c->m->p.FG_Fac, j) - 1.0); }

/* get_density_of_type (disp_fields.c:11-24) */
static double density(const jctx *c, const double *pos, int type)
{
  const galic_params_t *p = &c->m->p;
  const galic_sample_params_t *sp = c->sp;
  double rho;
  if(type == 1) { /* halo.c:43-54 */
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + p->HaloStretch * p->HaloStretch * pos[2] * pos[2]);
    rho = p->HaloStretch * p->Halo_Mass / (2 * J_PI) * p->Halo_A / (r + 1.0e-6 * p->Halo_A) / j_cube(c, r + p->Halo_A);
  } else if(type == 2) { /* disk.c:53-69 */
    if(!(p->Disk_Mass > 0)) return 0;
    double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    double z = pos[2];
    rho = p->Disk_Mass / (4 * J_PI * sp->Disk_H * sp->Disk_H * sp->Disk_Z0) * j_exp(c, -R / sp->Disk_H) *
          j_sq(c, 2 / (j_exp(c, z / sp->Disk_Z0) + j_exp(c, -z / sp->Disk_Z0)));
  } else { /* bulge.c:39-48 */
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    rho = p->BulgeStretch * p->Bulge_Mass / (2 * J_PI) * p->Bulge_Mass / (r + 1.0e-6 * p->Bulge_A) /
          j_cube(c, r + p->Bulge_A);
  }
  if(fabs(rho) < MIN_DENSITY) rho = 0;
  return rho;
}

/* get_beta_of_type (disp_fields.c:26-60) */
static double beta_of(const jctx *c, const double *pos, int type)
{
  double beta = 0, a = 0;
  if(type == 1) {
    beta = c->sp->HaloBetaParameter;
    a = c->m->p.Halo_A;
  } else if(type == 3) {
    beta = c->sp->BulgeBetaParameter;
    a = c->m->p.Bulge_A;
  }
  if(type != 2 && beta >= 1) {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    double dlogrhodr = -1.0 - 3.0 * r / (r + a);
    beta = -0.15 - 0.20 * dlogrhodr;
  }
  return beta;
}

/* integrate_axisymmetric_jeans (disp_fields.c:427-453) */
static double integ_axi(const jctx *c, double zstart, double zend, double R, int type)
{
  int steps = 50, i;
  double dz = (zend - zstart) / steps;
  double sum = 0;
  for(i = 0; i < steps; i++) {
    double z0 = zstart + i * dz;
    double z1 = zstart + (i + 1) * dz;
    double pos0[3] = {R, 0, z0};
    double pos1[3] = {R, 0, z1};
    double acc0[3], acc1[3];
    orc_forcegrid_acc(c->m, pos0, acc0);
    double y0 = -acc0[2] * density(c, pos0, type);
    orc_forcegrid_acc(c->m, pos1, acc1);
    double y1 = -acc1[2] * density(c, pos1, type);
    sum += 0.5 * (y0 + y1) * dz;
  }
  return sum;
}

/* integrate_spherical_jeans_beta (disp_fields.c:456-499) */
static double integ_sph(const jctx *c, int type, double ystart, double rstart, double rend)
{
  int steps = 50, i;
  double dr = (rend - rstart) / steps;
  for(i = 0; i < steps; i++) {
    double r0 = rstart + i * dr;
    double r1 = rstart + (i + 1) * dr;
    double pos0[3] = {r0, 0, 0};
    double pos1[3] = {r1, 0, 0};
    double beta0 = beta_of(c, pos0, type);
    double beta1 = beta_of(c, pos1, type);
    double pos[3], acc[3];
    pos[0] = r0;
    pos[1] = 0;
    pos[2] = 0;
    double dens0 = density(c, pos, type);
    orc_forcegrid_acc(c->m, pos, acc);
    double acc0 = acc[0];
    pos[0] = r1;
    pos[1] = 0;
    pos[2] = 0;
    double dens1 = density(c, pos, type);
    orc_forcegrid_acc(c->m, pos, acc);
    double acc1 = acc[0];
    if(r1 > fabs(dr) && r0 > fabs(dr)) {
      double ypred = ystart + dr * (dens0 * acc0 - 2 * beta0 / r0 * ystart);
      ystart += dr * 0.5 * ((dens0 * acc0 - 2 * beta0 / r0 * ystart) + (dens1 * acc1 - 2 * beta1 / r1 * ypred));
    } else if(r0 > fabs(dr)) {
      ystart += dr * (dens0 * acc0 - 2 * beta0 / r0 * ystart);
    }
  }
  return ystart;
}

/* the denominator shared by h_factor, h_over_R and the tilted tables */
static double tilt_den(const jctx *c, double f, double alpha)
{
  return j_sq(c, j_cos(c, alpha)) - f * j_sq(c, j_sin(c, alpha)) +
         (1.0 + f) / 2.0 * j_sin(c, 2 * alpha) * j_tan(c, 2 * alpha);
}

/* h_factor (disp_fields.c:1051-1077) */
static double h_factor(const jctx *c, double R, double z, int type)
{
  double f = c->jp->DispersionRoverZratio[type], fac;
  if(R <= 1.0e-12 * z || R == 0)
    fac = 0;
  else {
    double alpha = j_atan(c, z / R);
    fac = ((f - 1) / 2 * j_tan(c, 2 * alpha)) / tilt_den(c, f, alpha);
  }
  return fac;
}

/* h_over_R (disp_fields.c:1079-1105); z > 0 on every call here */
static double h_over_r(const jctx *c, double R, double z, int type)
{
  double f = c->jp->DispersionRoverZratio[type], fac;
  if(R <= 1.0e-12 * z || R == 0)
    fac = (f - 1) / f;
  else {
    double alpha = j_atan(c, z / R);
    fac = ((f - 1) / 2 * j_tan(c, alpha) * j_tan(c, 2 * alpha)) / tilt_den(c, f, alpha);
  }
  return fac / z;
}

/* out: [4][8][FG_Nbin^2] = disp_r, dispz, dispphi, vstream, tilted_vz2,
 * tilted_vR2, tilted_vz2_prime, tilted_vR2_prime per type (type 0 unused);
 * tables of types the reference skips are left as they are.  Returns 0, or
 * 6 (GALIC_ERR_UNSUPPORTED) where the reference calls terminate(). */
int orc_calculate_dispfield(orc_model *m, const galic_sample_params_t *sp, const galic_jeans_params_t *jp,
                            double *out)
{
  jctx C = {m, sp, jp, m->use_libm};
  const jctx *c = &C;
  const int N = m->p.FG_Nbin;
  const size_t G = (size_t) N * N;
  int i, j, k, type;
#define T(t, w) (out + ((size_t) (t) * 8 + (w)) * G)
#define AA(i, j) ((i) * N + (j))

  /* spherical case (disp_fields.c:512-570) */
  for(type = 1; type <= 3; type++) {
    if(m->p.NType[type] == 0) continue;
    double *Disp_r = T(type, 0);
    double r1 = fg_r(c, N);
    double r2 = fg_r(c, N + 2);
    double y = integ_sph(c, type, 0.0, r2, r1);
    for(j = N - 1; j >= 0; j--) {
      r1 = fg_r(c, j);
      r2 = fg_r(c, j + 1);
      y = integ_sph(c, type, y, r2, r1);
      Disp_r[j] = y;
    }
    for(j = N - 1; j >= 0; j--) {
      r1 = fg_r(c, j);
      double pos[3] = {r1, 0, 0};
      double dens = density(c, pos, type);
      if(dens > 0)
        Disp_r[j] /= dens;
      else
        Disp_r[j] = 0;
    }
  }

  /* axisymmetric f(E, Lz) case (disp_fields.c:575-729) */
  for(type = 1; type <= 3; type++) {
    if(m->p.NType[type] == 0) continue;
    double *DispZ = T(type, 1), *DispPhi = T(type, 2), *Vstream = T(type, 3);
    double kParameter = jp->StreamingVelocityParameter[type];
    for(j = 0; j < N; j++) {
      double R = fg_r(c, j);
      double z1, z2;
      k = N;
      z1 = fg_r(c, k);
      double integ = integ_axi(c, z1, fg_r(c, 2 * N), R, type);
      for(k = N - 1; k >= 0; k--) {
        i = k * N + j;
        z1 = fg_r(c, k);
        z2 = fg_r(c, k + 1);
        integ += integ_axi(c, z1, z2, R, type);
        double pos[3] = {R, 0, z1};
        double dens = density(c, pos, type);
        if(dens > 0)
          DispZ[i] = integ / dens;
        else
          DispZ[i] = 0;
      }
    }
    for(k = N - 1; k >= 0; k--)
      for(j = 0; j < N; j++) {
        double z = fg_r(c, k);
        double R = fg_r(c, j);
        double pos[3], acc[3], R1, R2;
        int i1, i2;
        pos[0] = R;
        pos[1] = 0;
        pos[2] = z;
        orc_forcegrid_acc(m, pos, acc);
        i = k * N + j;
        if(j > 1 && j < N - 1) {
          R1 = fg_r(c, j - 1);
          i1 = k * N + j - 1;
          R2 = fg_r(c, j + 1);
          i2 = k * N + j + 1;
        } else if(j == 1) {
          R1 = fg_r(c, j);
          i1 = k * N + j;
          R2 = fg_r(c, j + 1);
          i2 = k * N + j + 1;
        } else if(j == 0) {
          R1 = fg_r(c, j + 1);
          i1 = k * N + j + 1;
          R2 = fg_r(c, j + 2);
          i2 = k * N + j + 2;
        } else {
          R1 = fg_r(c, j - 1);
          i1 = k * N + j - 1;
          R2 = fg_r(c, j);
          i2 = k * N + j;
        }
        pos[0] = R1;
        double dens1 = density(c, pos, type);
        pos[0] = R2;
        double dens2 = density(c, pos, type);
        double dlogDensSigma_dlogR = 0;
        if(dens1 * DispZ[i1] > 0 && dens2 * DispZ[i2] > 0)
          dlogDensSigma_dlogR = j_log(c, (dens2 * DispZ[i2]) / (dens1 * DispZ[i1])) / j_log(c, R2 / R1);
        double Vphi2 = DispZ[i] + R * (-acc[0]) + DispZ[i] * dlogDensSigma_dlogR;
        if(Vphi2 > 0) {
          double vstr = 0;
          if(Vphi2 >= DispZ[i]) vstr = kParameter * sqrt((Vphi2 - DispZ[i]));
          DispPhi[i] = Vphi2 - vstr * vstr;
          Vstream[i] = vstr;
        } else {
          DispPhi[i] = 0;
          Vstream[i] = 0;
        }
      }
  }

  /* tilted f(E, Lz, I3) case (disp_fields.c:733-1044), VER_1_1 */
  for(type = 1; type <= 3; type++) {
    if(m->p.NType[type] == 0) continue;
    if(m->p.TypeOfVelocityStructure[type] != 3) continue;
    double f = jp->DispersionRoverZratio[type];
    if(f == 0) return 6;
    double kParameter = jp->StreamingVelocityParameter[type];
    double *DispZ = T(type, 1), *DispPhi = T(type, 2), *Vstream = T(type, 3);
    double *tvz2 = T(type, 4), *tvR2 = T(type, 5), *tvz2p = T(type, 6), *tvR2p = T(type, 7);
    (void) DispZ;
    double *FG_q = calloc(G, sizeof(double));
    double *qprev = calloc((size_t) N, sizeof(double));
    for(k = N - 1; k >= 0; k--) {
      if(k == N - 1) {
        for(j = 0; j < N; j++) FG_q[AA(k, j)] = 0;
      } else {
        double z0 = fg_r(c, k + 1);
        double z1 = fg_r(c, k);
        double dz = (z1 - z0);
        int nsteps = 100, st;
        for(j = 0; j < N; j++) qprev[j] = FG_q[AA(k + 1, j)];
        for(st = 0; st < nsteps; st++) {
          double z = z0 + (dz / nsteps) * st;
          for(j = 0; j < N; j++) {
            double R1 = fg_r(c, j);
            double h1 = h_factor(c, R1, z, type);
            double pos[3], acc[3];
            pos[0] = R1;
            pos[1] = 0;
            pos[2] = z;
            double dens = density(c, pos, type);
            orc_forcegrid_acc(m, pos, acc);
            double p = -dens * acc[2];
            double dqdR;
            if(h1 > 0) {
              if(j == N - 1)
                dqdR = 0;
              else {
                double R2 = fg_r(c, j + 1);
                double h2 = h_factor(c, R2, z, type);
                double dR = R2 - R1;
                dqdR = (h2 * qprev[j + 1] - h1 * qprev[j]) / (dR) + qprev[j] * h_over_r(c, R1, z, type);
              }
              FG_q[AA(k, j)] = qprev[j] + (-p - dqdR) * (dz / nsteps);
            } else {
              if(j == 0) {
                double R2 = fg_r(c, j + 1);
                double h2 = h_factor(c, R2, z, type);
                double dR = R2 - R1;
                dqdR = (h2 * qprev[j + 1] - h1 * qprev[j]) / (dR) + qprev[j] * h_over_r(c, R1, z, type);
              } else {
                double R2 = fg_r(c, j - 1);
                double h2 = h_factor(c, R2, z, type);
                double dR = R2 - R1;
                dqdR = (h2 * qprev[j - 1] - h1 * qprev[j]) / (dR) + qprev[j] * h_over_r(c, R1, z, type);
              }
              FG_q[AA(k, j)] = qprev[j] + (-p - dqdR) * (dz / nsteps);
            }
          }
          for(j = 0; j < N; j++) qprev[j] = FG_q[AA(k, j)];
        }
      }
    }
    for(k = 0; k < N; k++)
      for(j = 0; j < N; j++) {
        double R = fg_r(c, j);
        double z = fg_r(c, k);
        double pos[3] = {R, 0, z};
        double dens = density(c, pos, type);
        if(dens > 0)
          tvz2[AA(k, j)] = FG_q[AA(k, j)] / dens;
        else
          tvz2[AA(k, j)] = 0;
        if(j > 0) {
          double alpha = j_atan(c, z / R);
          double vrvz = tvz2[AA(k, j)] * ((f - 1) / 2 * j_tan(c, 2 * alpha)) / tilt_den(c, f, alpha);
          double vr2 = tvz2[AA(k, j)] *
                       (f * j_sq(c, j_cos(c, alpha)) - j_sq(c, j_sin(c, alpha)) +
                        (1.0 + f) / 2.0 * j_sin(c, 2 * alpha) * j_tan(c, 2 * alpha)) /
                       tilt_den(c, f, alpha);
          double vr2_prime = vr2 * j_sq(c, j_cos(c, alpha)) + 2 * vrvz * j_sin(c, alpha) * j_cos(c, alpha) +
                             tvz2[AA(k, j)] * j_sq(c, j_sin(c, alpha));
          double vz2_prime = vr2 * j_sq(c, j_sin(c, alpha)) - 2 * vrvz * j_sin(c, alpha) * j_cos(c, alpha) +
                             tvz2[AA(k, j)] * j_sq(c, j_cos(c, alpha));
          tvR2[AA(k, j)] = vr2;
          tvz2p[AA(k, j)] = vz2_prime;
          tvR2p[AA(k, j)] = vr2_prime;
        } else {
          tvR2[AA(k, j)] = tvz2[AA(k, j)] / f;
          tvz2p[AA(k, j)] = tvR2[AA(k, j)];
          tvR2p[AA(k, j)] = tvz2[AA(k, j)];
        }
      }
    for(k = N - 1; k >= 0; k--)
      for(j = 0; j < N; j++) {
        double z = fg_r(c, k);
        double R = fg_r(c, j);
        double pos[3], acc[3];
        pos[0] = R;
        pos[1] = 0;
        pos[2] = z;
        double dens = density(c, pos, type);
        orc_forcegrid_acc(m, pos, acc);
        i = k * N + j;
        double Vphi2 = 0;
        if(dens > 0) {
          int j1 = (0 < j ? j - 1 : j);
          int j2 = (j < N - 1 ? j + 1 : j);
          int i1 = k * N + j1;
          int i2 = k * N + j2;
          double R1 = fg_r(c, j1);
          double R2 = fg_r(c, j2);
          pos[0] = R1;
          double dens1 = density(c, pos, type);
          pos[0] = R2;
          double dens2 = density(c, pos, type);
          Vphi2 = tvR2[i] + R / dens * (dens2 * tvR2[i2] - dens1 * tvR2[i1]) / (R2 - R1) + R * (-acc[0]) +
                  R / dens *
                      (dens2 * h_factor(c, R2, z, type) * tvz2[i2] - dens1 * h_factor(c, R1, z, type) * tvz2[i1]) /
                      (R2 - R1);
        }
        if(Vphi2 > 0) {
          double vstr = 0;
          if(Vphi2 >= tvR2[i]) vstr = kParameter * sqrt((Vphi2 - tvR2[i]));
          DispPhi[i] = Vphi2 - vstr * vstr;
          Vstream[i] = vstr;
        } else {
          DispPhi[i] = 0;
          Vstream[i] = 0;
        }
      }
    free(qprev);
    free(FG_q);
  }
#undef T
#undef AA
  return 0;
}
