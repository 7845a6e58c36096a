/*
 * oracle_particles.c - CPU restatement of initialize_particles
 * (set_particles.c:15-307) with halo_generate_v and the Hernquist
 * distribution function (halo.c:110-184), forcegrid_get_escape_speed
 * (grid.c:115-120) and the permutation sort (set_particles.c:298-303,
 * permutation_compare set_particles.c:309-316).
 *
 * TEST INFRASTRUCTURE: the checker for galic_b200/csrc/particles.cu.  Only
 * tests/ loads it.
 *
 * One sequential stream over all particles, in the reference's order.  With
 * use_libm = 1 (glibc's log/exp/sin/cos/acos/asin/atan2/pow) every particle
 * and the permutation are GALIC's own; with use_libm = 0 the transcendental
 * calls are gmath.h's (pow(x, 1.5) = x sqrt(x), pow(x, 2.5) = x x sqrt(x)),
 * as in the CUDA kernels.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "galic_oracle.h"
#include "oracle_internal.h"

static const double P_PI = 3.14159265358979323846; /* M_PI */

typedef struct {
  orc_model *m;
  const galic_sample_params_t *sp;
  int libm;
} pctx;

static double p_sin(const pctx *c, double x) { return c->libm ? sin(x) : gm_sin(x); }
static double p_cos(const pctx *c, double x) { return c->libm ? cos(x) : gm_cos(x); }
static double p_acos(const pctx *c, double x) { return c->libm ? acos(x) : gm_acos(x); }
static double p_asin(const pctx *c, double x) { return c->libm ? asin(x) : gm_asin(x); }
static double p_atan2(const pctx *c, double y, double x) { return c->libm ? atan2(y, x) : gm_atan2(y, x); }
static double p_pow15(const pctx *c, double x) { return c->libm ? pow(x, 1.5) : x * sqrt(x); }
static double p_pow25(const pctx *c, double x) { return c->libm ? pow(x, 2.5) : x * x * sqrt(x); }

/* halo_get_potential_from_radius (halo.c:69-73) */
static double halo_pot_r(const pctx *c, double r)
{
  return -c->m->p.G * c->m->p.Halo_Mass / (r + c->m->p.Halo_A);
}

/* halo_f_q (halo.c:136-147) */
static double halo_f_q(const pctx *c, double q)
{
  const galic_params_t *p = &c->m->p;
  double pre = (p->Halo_Mass / (p->Halo_A * p->Halo_A * p->Halo_A)) /
               (4 * P_PI * P_PI * P_PI * p_pow15(c, 2 * p->G * p->Halo_Mass / p->Halo_A));
  return pre * (3 * p_asin(c, q) + q * sqrt(1 - q * q) * (1 - 2 * q * q) * (8 * q * q * q * q - 8 * q * q - 3)) /
         p_pow25(c, 1 - q * q);
}

/* halo_f (halo.c:151-157) with halo_E_to_q (halo.c:113-116) */
static double halo_f(const pctx *c, double rad, double vel)
{
  double E = 0.5 * vel * vel + halo_pot_r(c, rad);
  double q = sqrt(-E * c->m->p.Halo_A / (c->m->p.G * c->m->p.Halo_Mass));
  return halo_f_q(c, q);
}

/* halo_generate_v (halo.c:168-184) */
static double halo_generate_v(const pctx *c, grng_t *g, double rad)
{
  double pot = halo_pot_r(c, rad);
  double v_max = sqrt(-2 * pot);
  double v_guess, x_aux;
  double f_max = v_max * v_max * halo_f(c, rad, 0);
  v_guess = grng_uniform(g) * v_max;
  x_aux = grng_uniform(g) * f_max;
  while(x_aux > v_guess * v_guess * halo_f(c, rad, v_guess)) {
    v_guess = grng_uniform(g) * v_max;
    x_aux = grng_uniform(g) * f_max;
  }
  return v_guess;
}

typedef struct {
  double rnd;
  int index;
} perm_t;

/* permutation_compare (set_particles.c:309-316) */
static int perm_compare(const void *a, const void *b)
{
  if(((const perm_t *) a)->rnd < ((const perm_t *) b)->rnd) return -1;
  if(((const perm_t *) a)->rnd > ((const perm_t *) b)->rnd) return +1;
  return 0;
}

/* initialize_particles (set_particles.c:15-307), one rank.  tab[t] =
 * {FG_Disp_r, FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime,
 * FG_Vstream} of type t.  Outputs (n = NType[1] + NType[2] + NType[3]):
 * pos, vel, vel_theo [3n]; mass, vesc, tint [n]; targets [4n]; type, id,
 * perm [n]; counts [4][4] (r, t, p, q raised to LowerDispLimit per type).
 * Returns 0, or 6 where the reference calls endrun() (set_particles.c:261-282). */
int orc_initialize_particles(orc_model *m, const galic_sample_params_t *sp, double TorbitFac,
                             const double *const *const *tab, galic_stream_t *stream, int use_libm, double *pos,
                             double *vel, double *vel_theo, double *mass, double *vesc, double *tint,
                             double *targets, int *type, int *id, int *perm, int *counts)
{
  pctx C = {m, sp, use_libm};
  const pctx *c = &C;
  const galic_params_t *p = &m->p;
  const int nt[4] = {0, p->NType[1], p->NType[2], p->NType[3]};
  const int N = nt[1] + nt[2] + nt[3];
  const double tmass[4] = {0, p->Halo_Mass, p->Disk_Mass, p->Bulge_Mass};
  grng_t g;
  grng_init(&g, stream->seed, stream->a, stream->b);
  grng_seek(&g, stream->position);
  memset(counts, 0, 16 * sizeof(int));
  memset(vel_theo, 0, 3 * (size_t) N * sizeof(double));
  int n = 0;
  for(int t = 1; t <= 3; t++)
    for(int i = 0; i < nt[t]; i++, n++) {
      type[n] = t;
      mass[n] = tmass[t] / nt[t];
      id[n] = n + 1;
    }
  for(n = 0; n < N; n++) {
    const int t = type[n];
    double *P = &pos[3 * n];
    orc_fresh(use_libm, sp, t, &g, P);
    vesc[n] = sqrt(-2.0 * orc_forcegrid_pot(m, P));
    double acc[3];
    orc_forcegrid_acc(m, P, acc);
    double a = sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
    double r = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    tint[n] = TorbitFac * 2 * P_PI * r / sqrt(r * a);
    if(t == 1) {
      double vr;
      do {
        vr = halo_generate_v(c, &g, r);
      } while(vr >= p->MaxVelInUnitsVesc * vesc[n]);
      double phi = grng_uniform(&g) * P_PI * 2;
      double theta = p_acos(c, grng_uniform(&g) * 2 - 1);
      vel_theo[3 * n] = vr * p_sin(c, theta) * p_cos(c, phi);
      vel_theo[3 * n + 1] = vr * p_sin(c, theta) * p_sin(c, phi);
      vel_theo[3 * n + 2] = vr * p_cos(c, theta);
    }
    const int tovs = p->TypeOfVelocityStructure[t];
    double d[4];
    orc_disp_rtp(use_libm, p, sp, t, tab[t], P, d);
    for(int k = 0; k < 4; k++)
      if(d[k] <= p->LowerDispLimit) {
        counts[4 * t + k]++;
        d[k] = p->LowerDispLimit;
      }
    for(int k = 0; k < 4; k++) targets[4 * n + k] = d[k];
    double vstr = orc_vstream_tab(use_libm, p, tab[t][5], P);
    double *V = &vel[3 * n];
    if(tovs == 0 || tovs == 1 || tovs == 3) {
      double sigmaR = sqrt(d[0]), sigmaT = sqrt(d[1]), sigmaP = sqrt(d[2]);
      double v, vr, vphi, vtheta;
      do {
        vr = grng_gaussian(&g, sigmaR);
        vtheta = grng_gaussian(&g, sigmaT);
        vphi = grng_gaussian(&g, sigmaP);
        vphi += vstr;
        v = sqrt(vr * vr + vphi * vphi + vtheta * vtheta);
      } while(p->MaxVelInUnitsVesc * vesc[n] < v);
      double phi = p_atan2(c, P[1], P[0]);
      double theta = p_acos(c, P[2] / sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]));
      double er[3], ePhi[3], eTheta[3];
      er[0] = p_sin(c, theta) * p_cos(c, phi);
      er[1] = p_sin(c, theta) * p_sin(c, phi);
      er[2] = p_cos(c, theta);
      ePhi[0] = -p_sin(c, phi);
      ePhi[1] = p_cos(c, phi);
      ePhi[2] = 0;
      eTheta[0] = -p_cos(c, theta) * p_cos(c, phi);
      eTheta[1] = -p_cos(c, theta) * p_sin(c, phi);
      eTheta[2] = p_sin(c, theta);
      for(int k = 0; k < 3; k++) V[k] = vr * er[k] + vphi * ePhi[k] + vtheta * eTheta[k];
    } else if(tovs == 2) {
      double sigmaR = sqrt(d[0]), sigmaT = sqrt(d[1]), sigmaP = sqrt(d[2]);
      double v, vR, vphi, vz;
      do {
        vR = grng_gaussian(&g, sigmaR);
        vz = grng_gaussian(&g, sigmaT);
        vphi = grng_gaussian(&g, sigmaP);
        vphi += vstr;
        v = sqrt(vR * vR + vphi * vphi + vz * vz);
      } while(v >= p->MaxVelInUnitsVesc * vesc[n]);
      double phi = p_atan2(c, P[1], P[0]);
      double eR[3], ePhi[3], eZ[3];
      eR[0] = p_cos(c, phi);
      eR[1] = p_sin(c, phi);
      eR[2] = 0;
      ePhi[0] = -p_sin(c, phi);
      ePhi[1] = p_cos(c, phi);
      ePhi[2] = 0;
      eZ[0] = 0;
      eZ[1] = 0;
      eZ[2] = 1;
      for(int k = 0; k < 3; k++) V[k] = vR * eR[k] + vphi * ePhi[k] + vz * eZ[k];
    }
  }
  int rc = 0;
  for(int t = 1; t <= 3; t++) {
    if(p->NType[t] == 0) continue;
    for(int k = 0; k < 4; k++)
      if((double) counts[4 * t + k] / p->NType[t] > 0.05) rc = 6;
  }
  perm_t *pm = malloc((size_t) (N > 0 ? N : 1) * sizeof(perm_t));
  for(n = 0; n < N; n++) {
    pm[n].rnd = grng_uniform(&g);
    pm[n].index = n;
  }
  qsort(pm, N, sizeof(perm_t), perm_compare);
  for(n = 0; n < N; n++) perm[n] = pm[n].index;
  free(pm);
  stream->position = grng_position(&g);
  return rc;
}
