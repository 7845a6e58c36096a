/* Stand-in for gsl_ran_gaussian (Marsaglia polar method, the method GSL
 * uses).  CPU oracle test infrastructure only. */
#ifndef GALIC_ORACLE_GSL_RANDIST_H
#define GALIC_ORACLE_GSL_RANDIST_H
#include "gsl_rng.h"
double gsl_ran_gaussian(const gsl_rng *r, double sigma);
#endif
