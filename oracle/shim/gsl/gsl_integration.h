/* Stand-in for the GSL quadrature interface used by structure.c:148-177
 * (disk angular momentum, set-up only).  CPU oracle test infrastructure only. */
#ifndef GALIC_ORACLE_GSL_INTEGRATION_H
#define GALIC_ORACLE_GSL_INTEGRATION_H
#include <stddef.h>
typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
typedef struct { size_t limit; } gsl_integration_workspace;
enum { GSL_INTEG_GAUSS15 = 1, GSL_INTEG_GAUSS21, GSL_INTEG_GAUSS31, GSL_INTEG_GAUSS41,
       GSL_INTEG_GAUSS51, GSL_INTEG_GAUSS61 };
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace *w);
int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs, double epsrel,
                        size_t limit, int key, gsl_integration_workspace *w, double *result, double *abserr);
#endif
