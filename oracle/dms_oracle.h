/*
 * dms_oracle.h — CPU oracle of the DaMaSCUS-SUN trajectory Monte Carlo (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference's hot path in the engine's units (km, s, km/s),
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker
 * of the CUDA engine.  Parity is pinned against the reference's own sources compiled in
 * oracle/_ref (see ref_driver.cpp) and against the reference's known-answer tests.
 *
 * Thread safety: all state lives in the dms_oracle object; distinct objects may be used from
 * distinct threads concurrently.
 */
#ifndef DMS_ORACLE_H
#define DMS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/dms.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dms_oracle dms_oracle;

dms_oracle* dms_oracle_create(const char* solar_model_path);
void dms_oracle_destroy(dms_oracle* o);
const char* dms_oracle_last_error(const dms_oracle* o);

/* DM particle, halo and an N x N total-rate grid (N = params->interpolation_points >= 2). */
int dms_oracle_set_point(dms_oracle* o, const dms_point_params* params);

/* Same query codes as dms_ref_query in ref_driver.cpp. */
double dms_oracle_query(dms_oracle* o, int what, double a, double b, double c);

/* Radial tables: n_nodes knots r [km]; fills (when non-null) GM [km^3/s^2], T [GeV],
 * v_esc^2 [km^2/s^2], n_e [1/km^3], and n_i [1/km^3] node-major (n_nodes x DMS_NUM_TARGETS). */
int dms_oracle_tables(const dms_oracle* o, double* r, double* gm, double* temperature_gev, double* vesc2, double* n_e, double* n_targets);
int dms_oracle_num_nodes(const dms_oracle* o);
/* Rate grid of the current point (N*N doubles, radius-major, 1/s). */
int dms_oracle_rate_grid(const dms_oracle* o, double* grid);
/* Replaces the current point's grid by n*n values (n must equal its interpolation_points). */
int dms_oracle_set_rate_grid(dms_oracle* o, const double* grid, uint32_t n);

/* Records plus the reflection-spectrum sample per trajectory (speed at 1 AU, cosine to the Sun's
 * velocity; NaN unless a recorded reflection), Parameter-point mode. */
int dms_oracle_run_reflections(dms_oracle* o, uint32_t seed, uint32_t point, uint64_t max_scatterings, double boundary_rsun,
                               uint64_t first, uint64_t count, dms_traj_record* records, double* reflection);

/* Records of trajectories started from caller-given events after the initial Kepler shift
 * (7 doubles per trajectory: t, x, v); the initial conditions still run for their draws. */
int dms_oracle_run_from_starts(dms_oracle* o, uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings,
                               double boundary_rsun, uint64_t first, uint64_t count, const double* starts,
                               dms_traj_record* records, double* trace, size_t trace_capacity, size_t* trace_length);

int dms_oracle_run_records(dms_oracle* o, uint32_t seed, uint32_t point, int capture_mode, uint64_t max_scatterings,
                           double boundary_rsun, uint64_t first, uint64_t count, dms_traj_record* records, double* hist_dt,
                           double* hist_v2dt, double* trace, size_t trace_capacity, size_t* trace_length);

#ifdef __cplusplus
}
#endif
#endif
