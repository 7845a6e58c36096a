/* Stand-in for the parts of GSL's gsl_math.h that GALIC's reference sources
 * use (M_PI).  CPU oracle test infrastructure only. */
#ifndef GALIC_ORACLE_GSL_MATH_H
#define GALIC_ORACLE_GSL_MATH_H
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif
#endif
