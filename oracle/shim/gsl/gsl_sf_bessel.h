/* Stand-in for the modified Bessel functions used by structure.c:37-38
 * (set-up only).  CPU oracle test infrastructure only. */
#ifndef GALIC_ORACLE_GSL_SF_BESSEL_H
#define GALIC_ORACLE_GSL_SF_BESSEL_H
double gsl_sf_bessel_I0(double x);
double gsl_sf_bessel_I1(double x);
double gsl_sf_bessel_K0(double x);
double gsl_sf_bessel_K1(double x);
#endif
