/* Project-written stand-ins for the GSL routines GALIC's reference sources
 * link against.  CPU oracle test infrastructure only; nothing in the product
 * library uses this file.
 *  - gsl_rng_* / gsl_ran_gaussian draw from the project's Philox streams
 *    (galic_b200/csrc/grng.h), identical to the CUDA side.
 *  - gsl_integration_qag: adaptive Simpson quadrature (set-up only).
 *  - gsl_sf_bessel_{I0,I1,K0,K1}: trapezoid rule on the integral
 *    representations I_n(x) = (1/pi) int_0^pi e^{x cos t} cos(nt) dt and
 *    K_n(x) = int_0^inf e^{-x cosh t} cosh(nt) dt, both of which converge
 *    geometrically under the trapezoid rule (set-up only).
 */
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_sf_bessel.h"
#include "../../galic_b200/csrc/grng.h"

struct gsl_rng { grng_t g; };
static const gsl_rng_type ranlxd1_type = {"philox4x32-10 (oracle stand-in for ranlxd1)"};
const gsl_rng_type *gsl_rng_ranlxd1 = &ranlxd1_type;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T)
{
  (void) T;
  gsl_rng *r = (gsl_rng *) calloc(1, sizeof(gsl_rng));
  grng_init(&r->g, 0, 0, 0);
  return r;
}
void gsl_rng_free(gsl_rng *r) { free(r); }
void gsl_rng_set(const gsl_rng *r, unsigned long int seed) { grng_init(&((gsl_rng *) r)->g, seed, 0, 0); }
void galic_shim_rng_stream(gsl_rng *r, uint64_t seed, uint32_t a, uint32_t b) { grng_init(&r->g, seed, a, b); }
void galic_shim_rng_seek(gsl_rng *r, uint64_t position) { grng_seek(&r->g, position); }
uint64_t galic_shim_rng_position(const gsl_rng *r) { return grng_position(&r->g); }
double gsl_rng_uniform(const gsl_rng *r) { return grng_uniform(&((gsl_rng *) r)->g); }
double gsl_ran_gaussian(const gsl_rng *r, double sigma) { return grng_gaussian(&((gsl_rng *) r)->g, sigma); }

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{
  gsl_integration_workspace *w = (gsl_integration_workspace *) malloc(sizeof(*w));
  w->limit = n;
  return w;
}
void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }

static double simpson_rec(const gsl_function *f, double a, double b, double fa, double fm, double fb,
                          double whole, double eps, int depth)
{
  double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
  double flm = f->function(lm, f->params), frm = f->function(rm, f->params);
  double left = (m - a) / 6 * (fa + 4 * flm + fm), right = (b - m) / 6 * (fm + 4 * frm + fb);
  double diff = left + right - whole;
  if(depth <= 0 || fabs(diff) <= 15 * eps) return left + right + diff / 15;
  return simpson_rec(f, a, m, fa, flm, fm, left, eps / 2, depth - 1) +
         simpson_rec(f, m, b, fm, frm, fb, right, eps / 2, depth - 1);
}

int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs, double epsrel,
                        size_t limit, int key, gsl_integration_workspace *w, double *result, double *abserr)
{
  (void) limit; (void) key; (void) w;
  double fa = f->function(a, f->params), fb = f->function(b, f->params);
  double fm = f->function(0.5 * (a + b), f->params);
  double whole = (b - a) / 6 * (fa + 4 * fm + fb);
  double eps = epsabs > 0 ? epsabs : 1e-300;
  double r = simpson_rec(f, a, b, fa, fm, fb, whole, eps, 40);
  if(epsrel > 0) r = simpson_rec(f, a, b, fa, fm, fb, whole, fmax(eps, epsrel * fabs(r)), 40);
  *result = r;
  *abserr = fabs(r) * epsrel;
  return 0;
}

static double bessel_I(int n, double x)
{
  const int N = 400;
  double s = 0;
  for(int i = 0; i <= N; i++) {
    double t = M_PI * i / N;
    double w = (i == 0 || i == N) ? 0.5 : 1.0;
    s += w * exp(x * cos(t)) * cos(n * t);
  }
  return s / N;
}
static double bessel_K(int n, double x)
{
  const double h = 0.02;
  double s = 0;
  for(int i = 0; i < 4000; i++) {
    double t = i * h;
    double v = exp(-x * cosh(t)) * cosh(n * t);
    s += (i == 0 ? 0.5 : 1.0) * v;
    if(i > 10 && v < 1e-30 * s) break;
  }
  return s * h;
}
double gsl_sf_bessel_I0(double x) { return bessel_I(0, x); }
double gsl_sf_bessel_I1(double x) { return bessel_I(1, x); }
double gsl_sf_bessel_K0(double x) { return bessel_K(0, x); }
double gsl_sf_bessel_K1(double x) { return bessel_K(1, x); }
