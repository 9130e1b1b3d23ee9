/*
 * fcc_oracle.h — CPU oracle of the Fourier contour cell time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++ restatement of the
 * FourierContourCells.jl CPU path (KernelAbstractions CPU backend,
 * BodyParallel layout, three separate synthesis/pullback products), used by
 * tests/ as the parity checker and by bench.py as the timed CPU baseline.
 * The product library (libfcc_b200) never links, loads or calls it.
 *
 * Parity pins: the reference's Philox4x32-10 known-answer vectors
 * (test/test_random.jl:4-11) and its golden trajectory
 * test/data/reference_N64.txt (test/test_dynamics.jl:53-70, atol 1e-10), both
 * carried as fixtures under tests/golden/.
 *
 * The ABI reuses the structs of include/fcc.h; functions carry the prefix
 * fcco_ and mirror the fcc_ functions of the same name.
 */
#ifndef FCC_ORACLE_H
#define FCC_ORACLE_H

#include "../include/fcc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fcco_sim fcco_sim;

fcc_status fcco_create(const fcc_params* params, const fcc_bodies_host* bodies, fcco_sim** out);
fcc_status fcco_destroy(fcco_sim* sim);
fcc_status fcco_step(fcco_sim* sim, int64_t n);
fcc_status fcco_update_neighbors(fcco_sim* sim, int32_t force);
fcc_status fcco_compute_gradients(fcco_sim* sim);
fcc_status fcco_get_state(fcco_sim* sim, fcc_bodies_host* out, int64_t* clock, double* t, int64_t* step);
fcc_status fcco_set_state(fcco_sim* sim, const fcc_bodies_host* in, int64_t clock);
fcc_status fcco_set_dt(fcco_sim* sim, double dt);
fcc_status fcco_get_gradients(fcco_sim* sim, const fcc_gradients_host* out);
fcc_status fcco_get_geometry(fcco_sim* sim, const fcc_geometry_host* out);
fcc_status fcco_neighbor_dims(fcco_sim* sim, int32_t* ncx, int32_t* ncy, int32_t* cap, int64_t* builds, int32_t* valid);
fcc_status fcco_get_neighbors(fcco_sim* sim, const fcc_neighbors_host* out);
fcc_status fcco_perimeters(fcco_sim* sim, int32_t type, double* out, int64_t* count);
fcc_status fcco_areas(fcco_sim* sim, int32_t type, double* out, int64_t* count);
fcc_status fcco_shape_index(fcco_sim* sim, int32_t type, double* out, int64_t* count);
fcc_status fcco_body_energy(fcco_sim* sim, double* out);
/* protrusion(sim; type): src/observables.jl:59-79 (NaN for self-parented bodies). */
fcc_status fcco_protrusion(fcco_sim* sim, int32_t type, double* out, int64_t* count);

/* Work counters of the last gradient evaluation: contact node/neighbour tests,
 * tests inside rmax (hits), and per body the smallest |d| over its hits
 * (near-ties of the Heaviside overlap; NULL skips). */
fcc_status fcco_contact_counters(fcco_sim* sim, int64_t* tests, int64_t* hits, double* min_abs_depth);

/* Philox4x32-10 (src/random.jl:25-36) on one counter/key. */
void fcco_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
fcc_status fcco_philox_noise(uint64_t seed, uint64_t draw, int64_t nbodies, int32_t precision, double* out);
fcc_status fcco_build_neighbors(int32_t precision, int64_t n, const double* x, const double* y,
                                const double* rmax, double Lx, double Ly, double cutoff, double range,
                                int32_t cap, int32_t* cellid, int32_t* perm, int32_t* start,
                                int32_t* stop, int32_t* idx, int32_t* count);

/* OpenMP threads used by the oracle (<= 0: all). Returns the count in use. */
int32_t fcco_set_threads(int32_t n);
const char* fcco_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
