/*
 * oracle_internal.h - helpers shared by the set-up restatements
 * (oracle_sampling.c, oracle_particles.c).  TEST INFRASTRUCTURE.
 */
#ifndef GALIC_ORACLE_INTERNAL_H
#define GALIC_ORACLE_INTERNAL_H

#include "galic_oracle.h"
#include "../galic_b200/csrc/gmath.h"
#include "../galic_b200/csrc/grng.h"

/* one call of the type's *_get_fresh_coordinate (halo.c:17-40, disk.c:17-50,
 * bulge.c:15-37) */
void orc_fresh(int use_libm, const galic_sample_params_t *sp, int type, grng_t *g, double *pos);
/* get_disp_rtp (disp_fields.c:66-115): d = {r, t, p, q}; tab = FG_Disp_r,
 * FG_DispZ, FG_DispPhi, FG_tilted_vR2_prime, FG_tilted_vz2_prime, FG_Vstream */
void orc_disp_rtp(int use_libm, const galic_params_t *p, const galic_sample_params_t *sp, int type,
                  const double *const *tab, const double *pos, double *d);
/* get_vstream (disp_fields.c:118-132) on the table vstream */
double orc_vstream_tab(int use_libm, const galic_params_t *p, const double *vstream, const double *pos);

#endif
