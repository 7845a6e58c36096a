/* Stand-in for GSL's random-number interface as GALIC calls it
 * (init.c:25-27, gsl_rng_uniform everywhere).  Every generator draws from the
 * project's Philox4x32-10 streams (galic_b200/csrc/grng.h), so the CPU oracle
 * and the CUDA kernels see the same numbers.  CPU oracle test infrastructure
 * only. */
#ifndef GALIC_ORACLE_GSL_RNG_H
#define GALIC_ORACLE_GSL_RNG_H
#include <stdint.h>
typedef struct gsl_rng_type { const char *name; } gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_ranlxd1;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
double gsl_rng_uniform(const gsl_rng *r);
/* project extension: select the Philox stream (seed, a, b) for r */
void galic_shim_rng_stream(gsl_rng *r, uint64_t seed, uint32_t a, uint32_t b);
/* project extensions: move to / read the index of the next uniform */
void galic_shim_rng_seek(gsl_rng *r, uint64_t position);
uint64_t galic_shim_rng_position(const gsl_rng *r);
#endif
