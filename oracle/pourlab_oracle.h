/*
 * pourlab_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of PourLab's 3D reference solver (src/sim3d/solver3d.ts,
 * src/sim3d/vessel3d.ts, src/sim3d/presets3d.ts, src/sim/motion.ts, src/sim/rng.ts), used as the
 * checker of the CUDA engine and as the timed CPU baseline. The product never links or calls it.
 * It shares the plain-data types of include/pourlab.h so that both sides take the same config.
 *
 * Parity pins: the reference's committed goldens (benchmarks/run3d.json, benchmarks/gpu3d.json,
 * public/data/pour3d.bin.gz) — see tests/test_oracle_goldens.py.
 */
#ifndef POURLAB_ORACLE_H
#define POURLAB_ORACLE_H

#include "../include/pourlab.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct plo_sim plo_sim;

int plo_create(const pl_config* cfg, plo_sim** out);
void plo_destroy(plo_sim* s);
int plo_get_sizes(const plo_sim* s, pl_sizes* out);
double plo_stable_dt(plo_sim* s);
int plo_finished(const plo_sim* s);
int plo_step(plo_sim* s, double dt);
int plo_advance(plo_sim* s, double duration, pl_diagnostics* out);
int plo_set_tilt_target(plo_sim* s, double angle_deg, double time);
int plo_diagnostics(const plo_sim* s, pl_diagnostics* out);
int plo_discharged_fractions(const plo_sim* s, double out[3]);
int plo_read_particles(const plo_sim* s, double* x, double* y, double* z, double* vx, double* vy,
                       double* vz, uint8_t* status);
int plo_read_origin(const plo_sim* s, uint8_t* origin);
int plo_read_y0(const plo_sim* s, float* y0);
int plo_discharge_order(const plo_sim* s, int32_t* out, int32_t cap);
int plo_get_state(const plo_sim* s, pl_sim_state* st);
int plo_set_state(plo_sim* s, const pl_sim_state* st, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz,
                  const uint8_t* status);
int plo_get_field(const plo_sim* s, int32_t field, void* out, size_t count);

/* Pcg3D (solver3d.ts:827-974) on caller arrays of nx*ny*nz: returns iterations; *converged and
 * *residual as the reference's result record. q is overwritten. */
int plo_pcg_solve(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny,
                  int32_t nz, double tol, int32_t max_iter, int32_t* converged, double* residual);

/* APIC affine state per parcel id: 9 values (gradients of u, v, w). */
void plo_get_affine(const plo_sim* s, double* c9);
void plo_set_affine(plo_sim* s, const double* c9);
/* One dense n^3 snapshot of the Poisson batch (cells may carry PL_POISSON_PIN: diagonal + 1, the gauge
 * fix of src/sim/pressure.ts:232-268); FP64 MIC(0)-PCG as Pcg3D.solve. Returns the iterations. */
int plo_poisson_solve(const uint8_t* cell, const double* b, double* q, int32_t n, double tol, int32_t max_iter,
                      int32_t* converged, double* residual);
/* The same on a box of nx x ny x nz cells. */
int plo_poisson_solve_box(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny, int32_t nz,
                          double tol, int32_t max_iter, int32_t* converged, double* residual);

/* Geometry (vessel3d.ts:46-103) for unit tests. */
double plo_teapot_sdf(const pl_teapot* t, double x, double y, double z);
int plo_in_cavity(const pl_teapot* t, double x, double y, double z);
/* mulberry32 (src/sim/rng.ts:5-14): n draws from seed. */
void plo_rng(uint32_t seed, int32_t n, double* out);
/* Math.hypot as the JS engine evaluates it (normalise by the largest magnitude, Kahan-summed
 * squares, sqrt times the largest). */
double plo_js_hypot3(double a, double b, double c);

#ifdef __cplusplus
}
#endif

#endif
