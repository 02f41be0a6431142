/*
 * mpcd_oracle.h -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * reference solvent timestep, used as the checker of the GPU library by the
 * tests, smoke() and the benchmark's CPU baseline.  Not part of the product.
 */
#ifndef MPCD_ORACLE_H
#define MPCD_ORACLE_H

#include <stdint.h>

#include "mpcd_gpu.h"

typedef struct oracle oracle_t;

oracle_t *oracle_create(const mpcd_config *cfg, int n, const double *Q,
                        const double *V, const double *U, const int *spid);
void oracle_destroy(oracle_t *o);
int oracle_step(oracle_t *o, uint32_t step);
int oracle_set_vdist(oracle_t *o, const int *vdist);
int oracle_get_particles(const oracle_t *o, double *Q, double *V, double *U);
int oracle_get_globals(const oracle_t *o, double *kbtnow, double *avnow);
int oracle_get_cells(const oracle_t *o, int *pop, double *mass, double *vcm,
                     double *cm);
double oracle_gndnst(const oracle_t *o);
int oracle_ncells(const oracle_t *o);
long oracle_escaped(const oracle_t *o);
long oracle_bounce_limit(const oracle_t *o);
int oracle_shifted_counts(const oracle_t *o, uint32_t step, int *pop);
int oracle_init_state(const mpcd_config *cfg, const mpcd_init_params *p, int max_attempts,
                      double *Q, double *V, double *U, int *spid, double *kbtnow);

#endif
