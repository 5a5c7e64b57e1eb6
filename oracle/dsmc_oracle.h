/*
 * dsmc_oracle.h - CPU restatement of the reference DSMC time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU leg of bench.py may load this library; the engine never does.
 *
 * The oracle restates, in plain C and in FP64, the reference routines of the
 * time step (src/Boundary.cpp, src/Geometry.cpp, src/Collision.cpp,
 * src/Sampling.cpp, src/Initialization.cpp, rng/ sources) under the engine's
 * stream and ordering contract:
 *   - every entity draws from its own keyed Philox stream (dsmc_philox.h):
 *     particle slot i in MoveParticles, strip s in BoundaryConditions,
 *     cell k*NY+l in CollideParticles, one stream for InitialConditions;
 *   - removal keeps the reference's swap-with-last order
 *     (src/Boundary.cpp:181-202, src/Geometry.cpp:231-247);
 *   - Indexing is followed by a stable reorder of the particles into cell
 *     order, so each step starts from a cell-sorted array.
 * Parity is pinned against the reference's own routines compiled under the
 * same contract (oracle/_ref) and against the reference tests' known answers.
 */
#ifndef DSMC_ORACLE_H
#define DSMC_ORACLE_H

#include <stdint.h>

#include "../include/dsmc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsmc_oracle dsmc_oracle;

int dsmc_oracle_setup(const dsmc_params *p, dsmc_derived *d);
dsmc_oracle *dsmc_oracle_create(const dsmc_params *p, const dsmc_derived *d, int64_t capacity);
void dsmc_oracle_destroy(dsmc_oracle *o);

int dsmc_oracle_init_cold(dsmc_oracle *o);
int dsmc_oracle_remove_inside_box(dsmc_oracle *o);
int dsmc_oracle_remove_outside_domain(dsmc_oracle *o);
int dsmc_oracle_stage_move(dsmc_oracle *o);
int dsmc_oracle_stage_boundary(dsmc_oracle *o);
int dsmc_oracle_stage_index(dsmc_oracle *o);
int dsmc_oracle_stage_collide(dsmc_oracle *o);
int dsmc_oracle_stage_sample(dsmc_oracle *o);
int dsmc_oracle_stage_end_step(dsmc_oracle *o);
int dsmc_oracle_step(dsmc_oracle *o);

int dsmc_oracle_get_counters(dsmc_oracle *o, dsmc_counters *c);
int64_t dsmc_oracle_np(dsmc_oracle *o);
int dsmc_oracle_get_particles(dsmc_oracle *o, double *x, double *y, double *vx, double *vy,
                              double *vz);
int dsmc_oracle_set_particles(dsmc_oracle *o, const double *x, const double *y, const double *vx,
                              const double *vy, const double *vz, int64_t n);
int dsmc_oracle_set_particles_raw(dsmc_oracle *o, const double *x, const double *y,
                                  const double *vx, const double *vy, const double *vz, int64_t n);
int dsmc_oracle_set_step(dsmc_oracle *o, int64_t step);
int dsmc_oracle_get_cell_starts(dsmc_oracle *o, int32_t *out);
int dsmc_oracle_get_fields(dsmc_oracle *o, double *out);
int dsmc_oracle_set_fields(dsmc_oracle *o, const double *in, int64_t sample_step);

int dsmc_oracle_intersect(dsmc_oracle *o, double x, double y, double dx, double dy, double *t,
                          double *nx, double *ny);
int dsmc_oracle_inside_box(dsmc_oracle *o, double x, double y);
int dsmc_oracle_scatter(dsmc_oracle *o, double *v, double nx, double ny, uint32_t kind,
                        uint32_t step, uint32_t entity);
int dsmc_oracle_generate(dsmc_oracle *o, const double *rect, double n_gas, double ux_gas,
                         double uy_gas, double t_gas, int move_flag, uint32_t kind, uint32_t step,
                         uint32_t entity);
int dsmc_oracle_collide_list(dsmc_oracle *o, double cell_volume, int n, const int32_t *ipc,
                             uint32_t kind, uint32_t step, uint32_t entity, int *nc);
int dsmc_oracle_elastic(dsmc_oracle *o, double *v1, double *v2, double cr, uint32_t kind,
                        uint32_t step, uint32_t entity);

#ifdef __cplusplus
}
#endif

#endif
