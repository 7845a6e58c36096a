/* Empty stand-in: GALIC includes this GSL header but uses nothing from it
 * on the oracle path.  CPU oracle test infrastructure only. */
#ifndef GALIC_ORACLE_gsl_spline_H
#define GALIC_ORACLE_gsl_spline_H
#endif
