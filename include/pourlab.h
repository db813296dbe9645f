/*
 * pourlab.h — C ABI of the B200 pour-substep engine (libpourlab_cuda.so).
 *
 * The engine simulates the 3D teapot pour of PourLab's src/sim3d solver: a half pot behind a
 * symmetry plane, FLIP/PIC parcels on a staggered MAC grid, two pressure-type solves per substep,
 * a target-volume pour controller, and per-layer accounting of the poured volume. Every entry
 * point below replaces one member of the reference's TypeScript surface; the citation after each
 * declaration names it (paths inside marcelpetrick/teapotFluidSimulation).
 *
 * Conventions
 *   - Status codes: 0 = ok, negative = error (PL_E_*). pl_last_error() returns a message for the
 *     last failing call on the calling thread. Non-convergence of a pressure solve is not an error:
 *     it is counted in pl_diagnostics.pressure_failures, as the reference counts it.
 *   - Ownership: a pl_sim owns all of its device memory; the caller owns every output buffer.
 *   - Threading: one handle per host thread. Calls are synchronous and not reentrant. Each handle
 *     runs on its own CUDA stream on the device that was current when it was created.
 *   - Units: SI (metres, seconds, m^3), angles in degrees where the name says deg.
 */
#ifndef POURLAB_H
#define POURLAB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PL_OK 0
#define PL_E_ARG (-1)      /* invalid argument or size */
#define PL_E_CUDA (-2)     /* a CUDA call failed (message names it) */
#define PL_E_TIMEOUT (-3)  /* a bounded device-side wait gave up */
#define PL_E_STATE (-4)    /* call not valid in the current state */
#define PL_E_NOMEM (-5)    /* device or host allocation failed */
#define PL_NONE 1          /* query has no value yet (e.g. fractions before any pour) */

/* Cell types (solver3d.ts:17-19) and parcel status (solver3d.ts:20-23). */
#define PL_AIR 0
#define PL_FLUID 1
#define PL_SOLID 2
#define PL_IN_POT 0
#define PL_DISCHARGED 1
#define PL_SPILLED 2
#define PL_LOST 3

/* Motion kinds and controller phases (src/sim/types.ts:57, src/sim/motion.ts:9). */
enum pl_motion_kind { PL_MOTION_STILL = 0, PL_MOTION_POUR = 1, PL_MOTION_TILT = 2, PL_MOTION_MANUAL = 3 };
enum pl_phase {
  PL_PHASE_WAIT = 0,
  PL_PHASE_TILT_IN = 1,
  PL_PHASE_HOLD = 2,
  PL_PHASE_RETURN = 3,
  PL_PHASE_REST = 4,
  PL_PHASE_DONE = 5,
  PL_PHASE_MANUAL = 6
};

/* Pressure preconditioner. MIC0 is the reference's MIC(0) (solver3d.ts:883-900, 955-973),
 * applied in wavefront order on the device; MG is a 3D geometric multigrid V-cycle (the 3D form
 * of src/sim/multigrid.ts with a red-black Gauss-Seidel smoother); CHEB is the Chebyshev
 * polynomial of the WebGPU port (src/gpu3d/shaders.ts:588-622). MG and CHEB run on one
 * 16-CTA thread-block cluster with the vectors in distributed shared memory, for systems up to
 * about 65k liquid cells (larger ones fall back to the single-block MIC(0) solve).
 * BOX_MG and LEARNED are the grid-scale solves, for any system size: the liquid system is embedded
 * in a dense power-of-two box around the grid and solved there by multigrid PCG (the Poisson
 * batch's Galerkin hierarchy) or by flexible CG with the network of pl_set_unet and that
 * multigrid as the fall-back, the whole solve a while-loop node of the substep's CUDA graph; the
 * density-correction system runs beside it on a second branch of the graph (multigrid). */
enum pl_preconditioner {
  PL_PRECOND_MIC0 = 0,
  PL_PRECOND_MG = 1,
  PL_PRECOND_CHEB = 2,
  PL_PRECOND_BOX_MG = 3,
  PL_PRECOND_LEARNED = 4
};
/* Arithmetic of the pressure solves: F64 keeps every solver vector in FP64; MIXED keeps the
 * Krylov and smoother vectors in FP32 with FP64 inner products, an FP64 solution and FP64
 * iterative refinement of the true residual. */
enum pl_solve_precision { PL_SOLVE_F64 = 0, PL_SOLVE_MIXED = 1 };
/* Particle-grid transfer. FLIP is the reference's FLIP/PIC blend with flip_ratio
 * (solver3d.ts:410-431, 607-624); APIC is the affine transfer of the 2D solver
 * (src/sim/solver.ts:543-590, 944-990) in 3D: each parcel carries the gradient of every velocity
 * component, P2G adds its affine term and G2P is the masked PIC sample plus the interpolant's
 * gradient (flip_ratio unused). */
enum pl_transfer { PL_TRANSFER_FLIP = 0, PL_TRANSFER_APIC = 1 };
/* Simulated domain. HALF is the reference's half pot behind the symmetry plane z = h
 * (solver3d.ts:9-10, 157, 756-760); FULL simulates both halves (the seeded half and its mirror image),
 * with no symmetry plane. */
enum pl_domain { PL_DOMAIN_HALF = 0, PL_DOMAIN_FULL = 1 };

/* Teapot3DConfig (src/sim3d/vessel3d.ts:9-20). */
typedef struct pl_teapot {
  double radius;          /* inner radius of the body (m) */
  double height;          /* inner height of the body (m) */
  double wall;            /* wall thickness (m) */
  double inlet_height;    /* spout inlet centre height (m) */
  double bore_radius;     /* spout bore radius (m) */
  double spout_angle_deg; /* spout elevation (deg) */
  double spout_length;    /* spout length (m) */
} pl_teapot;

/* MotionConfig (src/sim/types.ts:55-84). */
typedef struct pl_motion {
  int32_t kind; /* enum pl_motion_kind */
  int32_t repeats;
  double start_delay;
  double tilt_duration;
  double hold_angle_deg;
  double hold_tilt_rate;
  double max_angle_deg;
  double return_duration;
  double max_hold;
  double hold_time;
  double target_volume; /* m^3 */
  double anticipation;
  double repeat_gap;
  double settle_time;
} pl_motion;

/* Config3D (src/sim3d/solver3d.ts:25-43) plus the engine's own settings at the end. */
typedef struct pl_config {
  pl_teapot teapot;
  double h;              /* cell size (m) */
  double initial_volume; /* liquid volume of the whole pot (m^3) */
  pl_motion motion;
  double pivot[2]; /* tilt pivot in pot-local x, y (m) */
  double gravity;
  double flip_ratio;
  double density_correction;
  double cfl;
  double max_substep;
  double pressure_tolerance;
  int32_t pressure_max_iterations;
  uint32_t seed;
  double duration;
  /* engine settings (no counterpart in Config3D) */
  int32_t preconditioner;  /* enum pl_preconditioner */
  int32_t solve_precision; /* enum pl_solve_precision */
  int32_t device;          /* CUDA device ordinal; -1 = the calling thread's current device */
  int32_t solve_cluster;   /* CTAs of the cluster solves (1-16; 0 = 16), see pl_autotune_solver */
  int32_t solve_threads;   /* threads per CTA of the cluster solves (32-1024; 0 = 512) */
  int32_t transfer;        /* enum pl_transfer */
  int32_t domain;          /* enum pl_domain */
  int32_t reserved;
} pl_config;

/* Diagnostics3D (src/sim3d/solver3d.ts:45-60). */
typedef struct pl_diagnostics {
  double time;
  int64_t steps;
  double angle_deg;
  int32_t phase; /* enum pl_phase */
  int32_t particles;
  int32_t grid[3];
  int32_t pressure_iterations;   /* iterations of the last pressure solve */
  int32_t pressure_failures;     /* pressure solves that hit the iteration cap */
  int32_t correction_iterations; /* iterations of the last density-correction solve */
  double discharged_ml;
  double spilled_ml;
  double lost_ml;
  double in_pot_ml;
  double max_divergence; /* 1/s, after projection */
  double interior_density;
  int32_t liquid_cells; /* unknowns of the last pressure solve (engine extension) */
  int32_t reserved;
} pl_diagnostics;

/* Constructor-derived sizes (solver3d.ts:62-84, 116-228). */
typedef struct pl_sizes {
  int32_t n;  /* parcels in the simulated half */
  int32_t nx, ny, nz;
  double h;
  double parcel_volume; /* m^3 per parcel (half-pot volume / n) */
  double pivot_world[2];
  double fill_height;
  int32_t band_counts[3]; /* parcels per origin layer (bottom, middle, top) */
  int32_t step_copy_bytes; /* bytes pl_step copies to the device and back (the device scalar block) */
} pl_sizes;

/* PourController internal state (src/sim/motion.ts:21-38): enough to resume a run exactly. */
typedef struct pl_controller_state {
  int32_t phase; /* enum pl_phase */
  int32_t pour;
  double angle; /* rad */
  double phase_start;
  double start_angle;
  double start_rate;
  double last_rate;
  double flow_rate;
  double last_discharged;
  double target; /* rad, manual mode */
  double manual_rate;
} pl_controller_state;

/* Whole-simulation scalar state beside the parcel arrays (solver3d.ts:86-114). */
typedef struct pl_sim_state {
  double time;
  int64_t steps;
  double phi;   /* current pose angle (rad, = -tilt) */
  double omega; /* angular velocity of the last substep (rad/s) */
  int32_t counts[4];          /* parcels per status */
  int32_t discharged_by_origin[3];
  int32_t last_iterations;
  int32_t failures;
  int32_t reserved;
  double max_div;
  double interior;
  pl_controller_state controller;
} pl_sim_state;

/* Field selectors for pl_get_field (face fields are stored u, then v, then w). */
enum pl_field {
  PL_FIELD_CELL = 0,     /* u8[nx*ny*nz]: AIR/FLUID/SOLID of the last substep */
  PL_FIELD_VELOCITY = 1, /* f64[nu+nv+nw]: face velocity after projection and extrapolation */
  PL_FIELD_VELOCITY_PREV = 2, /* f64[nu+nv+nw]: particle-to-grid result (FLIP reference) */
  PL_FIELD_PRESSURE = 3,  /* f64[nx*ny*nz]: pressure of the last projection */
  PL_FIELD_CORRECTION = 4, /* f64[nu+nv+nw]: density-correction face velocity */
  PL_FIELD_VALID = 5,      /* u8[nu+nv+nw]: face valid mask before extrapolation */
  PL_FIELD_DENSITY = 6,    /* f64[nx*ny*nz]: particle density (sum of weights) */
  PL_FIELD_RHS = 7         /* f64[nx*ny*nz]: right-hand side of the last density solve */
};

/* ------------------------------------------------------------------ presets */

/* defaultTeapot3D() (src/sim3d/vessel3d.ts:22-32). */
void pl_default_teapot(pl_teapot* out);
/* defaultMotion() with maxHold 20 (src/sim/config.ts:168-186, src/sim3d/presets3d.ts:17). */
void pl_default_motion(pl_motion* out);
/* gentlePour3D(cellMm, seconds) (src/sim3d/presets3d.ts:9-26). */
void pl_gentle_pour(double cell_mm, double seconds, pl_config* out);

/* ------------------------------------------------------------------ lifetime */

typedef struct pl_sim pl_sim;

/* new Simulation3D(cfg) / new GpuSimulation3D(device, cfg)
 * (src/sim3d/solver3d.ts:116-228, src/gpu3d/solver.ts:108-124). Seeding, banding and grid sizing
 * run on the host in FP64 exactly as the reference constructor; the state then moves to the GPU. */
int pl_create(const pl_config* cfg, pl_sim** out);
/* The host part of that constructor alone, without a device: grid sizes, pivot, parcel volume and
 * band counts, and, where the pointers are not NULL, the seeded parcel positions (FP64, id order)
 * and origin layers (solver3d.ts:116-228). Call with NULL arrays first to learn n. */
int pl_plan(const pl_config* cfg, pl_sizes* out, double* x, double* y, double* z, uint8_t* origin);
/* GpuSimulation3D.destroy() (src/gpu3d/solver.ts:486-489). Accepts NULL. */
void pl_destroy(pl_sim* sim);
/* Message of the last failing call on this thread ("" if none). */
const char* pl_last_error(void);

/* ------------------------------------------------------------------ queries */

/* n, nx, ny, nz, h, parcelVolume, pivotWorld, fillHeight, bandCounts (solver3d.ts:62-84). */
int pl_get_sizes(const pl_sim* sim, pl_sizes* out);
/* stableDt() (solver3d.ts:268-278; src/gpu3d/solver.ts:256-263). Reads the device's max speed. */
int pl_stable_dt(pl_sim* sim, double* out);
/* get finished (solver3d.ts:264-266). */
int pl_finished(const pl_sim* sim);

/* ------------------------------------------------------------------ stepping */

/* step(dt) (solver3d.ts:288-309; src/gpu3d/solver.ts:304-370). dt <= 0 selects
 * min(stableDt(), duration - time), the default of GpuSimulation3D.step. Synchronous: the
 * controller and counters are current when it returns. */
int pl_step(pl_sim* sim, double dt);
/* advance(duration) (solver3d.ts:281-286; src/gpu3d/solver.ts:373-378): whole stable substeps
 * until duration has elapsed or the run is finished. The substep sequence runs on the device
 * (controller, stable dt and counters included) with no host round trip per substep.
 * out may be NULL. */
int pl_advance(pl_sim* sim, double duration, pl_diagnostics* out);
/* Wait for queued device work (GpuSimulation3D.sync, src/gpu3d/solver.ts:289-294). */
int pl_sync(pl_sim* sim);
/* Queue `count` stable substeps without waiting (the pipelined GpuSimulation3D.step,
 * src/gpu3d/solver.ts:296-370, with the controller on the device instead of one substep behind).
 * Substeps past the end of the run do nothing. pl_sync makes the host-side state current. */
int pl_enqueue_substeps(pl_sim* sim, int32_t count);
/* The CUDA stream (cudaStream_t) the handle runs on, for callers that order their own work
 * (timing events, buffer fills) with the engine's. */
void* pl_stream(const pl_sim* sim);

/* ------------------------------------------------------------------ stage timing */

/* Stages of one substep, in order. */
enum pl_stage {
  PL_STAGE_BIN = 0,      /* controller, binning, classification, liquid list */
  PL_STAGE_P2G = 1,      /* particle-to-grid, gravity, wall faces */
  PL_STAGE_PRESSURE = 2, /* pressure solve (setup + PCG) */
  PL_STAGE_EXTRAP = 3,   /* gradient update and two extrapolation layers */
  PL_STAGE_DENSITY = 4,  /* density, correction rhs, divergence check */
  PL_STAGE_CORRECTION = 5, /* density-correction solve */
  PL_STAGE_ADVECT = 6,   /* grid-to-particle, advection, collisions, accounting */
  PL_STAGES = 7
};
/* Record CUDA events between the stages of every substep (rebuilds the substep graph). The
 * density stage runs on a second stream beside the P2G face pass: its interval overlaps
 * PL_STAGE_P2G, which ends when both are done. The six other stages add up to the substep. */
int pl_enable_stage_timing(pl_sim* sim, int32_t on);
/* Device milliseconds per stage of the last completed substep (needs stage timing on). */
int pl_stage_times(pl_sim* sim, float ms[PL_STAGES]);

/* Host-side failure injection for tests (no counterpart in the solver; the reference injects
 * readback failures into its fake GPU, tests/fakeGpu.ts:26-33). PL_FAULT_ALLOC: the next `count`
 * device allocations of pl_create on this host thread fail as an out-of-memory cudaMalloc would
 * (pl_create returns PL_E_NOMEM and frees what it had set up); count 0 clears it. */
#define PL_FAULT_ALLOC 1
int pl_inject_fault(int32_t kind, int32_t count);
/* Polls before the binning scan's bounded look-back wait gives up (0: the default, 2^22). A wait
 * that gives up switches the rest of the substep off (the parcels keep their state) and the call
 * that synchronises reports PL_E_TIMEOUT; the handle stays in that error. For tests of the
 * bounded-wait path (no counterpart in the reference). */
int pl_set_wait_limit(pl_sim* sim, int32_t polls);
/* Launch-shape tuner of the cluster solves (no counterpart in the reference): runs `substeps`
 * substeps of cfg from its initial state for every candidate (cluster CTAs x threads per CTA) on a
 * scratch simulation and returns the shape with the smallest pressure + correction time, and that
 * time per substep. Set the result in pl_config.solve_cluster / solve_threads: results depend on
 * the shape only through the order of inner-product sums, so a fixed shape keeps runs bitwise
 * reproducible. */
int pl_autotune_solver(const pl_config* cfg, int32_t substeps, int32_t* best_cluster, int32_t* best_threads,
                       float* best_ms);

/* ------------------------------------------------------------------ controller */

/* controller.setTarget(angleDeg, time) (src/sim/motion.ts:40-44; used at
 * src/view3d/live.ts:262). Switches nothing by itself: the motion kind must be manual. */
int pl_set_tilt_target(pl_sim* sim, double angle_deg, double time);
/* controller.angleDeg and controller.phase (src/sim/motion.ts:156-158, 23). */
int pl_controller(const pl_sim* sim, double* angle_deg, int32_t* phase);

/* ------------------------------------------------------------------ results */

/* diagnostics() (solver3d.ts:796-814; src/gpu3d/solver.ts:380-399). */
int pl_get_diagnostics(pl_sim* sim, pl_diagnostics* out);
/* dischargedFractions() (solver3d.ts:817-823; src/gpu3d/solver.ts:402-406): shares of the
 * poured parcels by origin layer. Returns PL_NONE (out untouched) before anything poured. */
int pl_discharged_fractions(pl_sim* sim, double out[3]);
/* readParticles() (src/gpu3d/solver.ts:409-428): positions and velocities as xyzw float4
 * (w = 0) in parcel id order, status as u32. Any pointer may be NULL. */
int pl_read_particles(pl_sim* sim, float* pos4, float* vel4, uint32_t* status);
/* Same state in FP64 SoA (the arrays Simulation3D exposes: solver3d.ts:75-82). */
int pl_read_particles_f64(pl_sim* sim, double* x, double* y, double* z, double* vx, double* vy,
                          double* vz, uint8_t* status);
/* Simulation3D.origin (solver3d.ts:81): origin layer 0/1/2 per parcel id. */
int pl_read_origin(const pl_sim* sim, uint8_t* origin);
/* A recording frame (scripts/record3d.ts capture(), quantised as encodeRecording stores it,
 * src/view3d/format.ts:60): for every stride-th parcel in id order (k = 0, 1, ... for ids 0, stride,
 * 2 stride, ...), xyz3[3k + a] = max(0, min(65535, round(position_a / quantum))), positions in the
 * simulation frame as Float32, rounding halves up as Math.round does. xyz3 holds 3 * ceil(n / stride)
 * values. The quantisation runs on the device; 6 bytes per kept parcel cross to the host. */
int pl_read_quantized_positions(pl_sim* sim, int32_t stride, double quantum, uint16_t* xyz3);
/* readRenderPositions() (src/gpu3d/solver.ts:443-475; kernel src/gpu3d/shaders.ts:786-799):
 * packed xyz of the simulated half then its mirror image, 6*n floats (PL_DOMAIN_FULL: the xyz of
 * the n simulated parcels, 3*n floats), written by a device kernel into a device buffer and copied
 * to xyz6n. */
int pl_read_render_positions(pl_sim* sim, float* xyz6n);

/* ------------------------------------------------------------------ state (parity harness) */

/* Scalar state and parcel arrays in id order (FP64 SoA as in solver3d.ts:75-82). The engine
 * stores parcels in FP32, so pl_set_state rounds them. Any parcel pointer may be NULL on get. With
 * APIC, setting the parcels resets their affine vectors to zero. */
int pl_get_state(pl_sim* sim, pl_sim_state* st);
int pl_set_state(pl_sim* sim, const pl_sim_state* st, const double* x, const double* y,
                 const double* z, const double* vx, const double* vy, const double* vz,
                 const uint8_t* status);
/* APIC state (no counterpart in the 3D reference; the 2D solver's cux/cuy/cvx/cvy,
 * src/sim/solver.ts:91-94): per parcel id the gradients of u, v and w, 9 floats
 * (du/dx, du/dy, du/dz, dv/dx, ..., dw/dz). PL_E_STATE unless the transfer is APIC. */
int pl_get_affine(pl_sim* sim, float* c9);
int pl_set_affine(pl_sim* sim, const float* c9);
/* Copy one grid field of the last substep to host memory (enum pl_field); count is the number of
 * elements the caller's buffer holds. u8 fields are written as uint8_t, others as double. */
int pl_get_field(pl_sim* sim, int32_t field, void* out, size_t count);

/* ------------------------------------------------------------------ standalone pressure solve */

/* Pcg3D.solve(cell, b, q, tol, maxIter) (solver3d.ts:858-937) as a standalone call on
 * caller-provided device buffers: cell u8[nx*ny*nz], b and q f64[nx*ny*nz]. Runs the reference's
 * MIC(0) preconditioner in FP64 (preconditioner must be PL_PRECOND_MIC0 and precision
 * PL_SOLVE_F64; other values return PL_E_ARG) on stream (0 = legacy default stream) and writes
 * iterations, converged and the final max-norm residual to host memory after synchronising.
 * Scratch memory is allocated by the call and freed before it returns. */
int pl_pcg_solve_device(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny,
                        int32_t nz, double tol, int32_t max_iter, int32_t preconditioner,
                        int32_t precision, void* stream, int32_t* iterations, int32_t* converged,
                        double* residual);

/* No counterpart in the reference. The MIC(0), FP64 solve of pl_pcg_solve_device (same kernels,
 * same results) without any device allocation: its scratch is a fixed array in the library's
 * static device memory, one per device, sized for grids of up to PL_NOALLOC_MAX_CELLS cells
 * (about 30 MB); larger grids are rejected with PL_E_ARG. For hosts that own all device memory
 * (a pool or arena of their own, a budget that allows no allocation outside it) and so cannot
 * let a library call cudaMalloc/cudaFree. Runs on the current device. Every call looks up the
 * scratch's device address in the current context (no allocation); the first call in a context
 * loads the library module that holds the scratch (set-up), so make that first call before any
 * stream capture begins. The scratch stays with the device until the process exits; processes
 * that never call this entry point do not hold it. Calls that overlap on one device (two host
 * threads, or streams that run at once) share the scratch and race: serialise them. Nothing has
 * to be zeroed first. */
#define PL_NOALLOC_MAX_CELLS 262144
int pl_pcg_solve_device_noalloc(const uint8_t* cell, const double* b, double* q, int32_t nx,
                                int32_t ny, int32_t nz, double tol, int32_t max_iter, void* stream,
                                int32_t* iterations, int32_t* converged, double* residual);

/* ------------------------------------------------------------------ Poisson batch */

/* Batched isolated pressure solves (no counterpart in the reference as a batch: each snapshot is
 * Pcg3D.solve's system, solver3d.ts:858-973, on a dense n^3 grid). Cells are PL_AIR / PL_FLUID /
 * PL_SOLID, optionally with PL_POISSON_PIN on a FLUID cell: that cell's diagonal gets +1, the gauge fix
 * of a liquid component without air contact (src/sim/pressure.ts:232-268; the caller also removes the
 * component's rhs mean, as pl_poisson_generate does). FLUID cells on the grid border are not
 * unknowns. Snapshots are stored back to back, x fastest. */
#define PL_POISSON_PIN 4
enum pl_poisson_method {
  PL_POISSON_MIC0 = 0,   /* the reference's MIC(0) (solver3d.ts:883-900, 955-973), level-scheduled */
  PL_POISSON_MG = 1,     /* one V-cycle of 3D geometric multigrid (src/sim/multigrid.ts in 3D, RBGS) */
  PL_POISSON_LEARNED = 2 /* flexible CG with a pl_unet as preconditioner, MG fallback on a stall */
};
/* Synthetic workload on the host: snapshots first .. first+count-1 of n^3 cells (n a power of two in
 * [8, 512]): a solid cylinder wall (radius 60/128 n) and border, a liquid bottom slab (n/8) and 1-8
 * liquid spheres (radius 6-24 cells at n = 128) from mulberry32 (src/sim/rng.ts:5-14) seeded 1000 +
 * snapshot, AIR elsewhere; rhs = -div of a unit-variance Gaussian random face-velocity field
 * (standard deviation 8 cells at n = 128) on the unknowns, with the gauge fix applied. threads <= 0:
 * all hardware threads. cell: count * n^3 bytes, b: count * n^3 floats, or NULL for the masks alone
 * (no rhs and no gauge fix: the cheap part, whose unknowns give a snapshot's cost for sharding). */
int pl_poisson_generate(int32_t n, int32_t first, int32_t count, uint8_t* cell, float* b, int32_t threads);
/* The gauge fix on caller cells and rhs (host arrays, count snapshots of n^3): every 6-connected
 * component of unknowns without an AIR neighbour gets its rhs mean removed and its first cell (index
 * order) flagged PL_POISSON_PIN (fixEnclosedGauges, src/sim/pressure.ts:232-268). enclosed (may be
 * NULL) receives the number of such components per snapshot. */
int pl_poisson_gauge_fix(int32_t n, int32_t count, uint8_t* cell, float* b, int32_t* enclosed);
typedef struct pl_poisson pl_poisson;
/* Solver for `count` snapshots of n^3 cells with `method` and `precision` (PL_SOLVE_MIXED: FP32
 * vectors, FP64 inner products, norms, solution and true-residual refinement; PL_SOLVE_F64: all
 * FP64). Holds its device scratch until pl_poisson_destroy. */
int pl_poisson_create(int32_t n, int32_t count, int32_t method, int32_t precision, pl_poisson** out);
/* The same for boxes of nx x ny x nz cells (each a power of two in [8, 512]); the multigrid halves every
 * axis longer than 8 per level (semi-coarsening on thin boxes). */
int pl_poisson_create_box(int32_t nx, int32_t ny, int32_t nz, int32_t count, int32_t method, int32_t precision,
                          pl_poisson** out);
/* Solve every snapshot (device buffers: cell u8, b f32 and x f64, each count * cells) on stream with
 * the reference's stopping rule (max-norm residual <= max(tol * max|b|, 1e-14), at most max_iter
 * iterations); writes per-snapshot iterations, final max-norm residual and converged flag to host
 * arrays of count entries (any may be NULL). Synchronous. */
int pl_poisson_solve(pl_poisson* h, const uint8_t* cell, const float* b, double* x, double tol, int32_t max_iter,
                     void* stream, int32_t* iterations, double* residual, int32_t* converged);
/* The network of PL_POISSON_LEARNED (the caller keeps it alive while the solver uses it). */
typedef struct pl_unet pl_unet;
int pl_poisson_set_unet(pl_poisson* h, pl_unet* u);
/* Device bytes the solver holds. */
size_t pl_poisson_device_bytes(const pl_poisson* h);
/* Convergence record of one snapshot of the last pl_poisson_solve: the recurrence's max-norm residual
 * after each of its first PL_POISSON_HISTORY iterations (up to capacity entries written, recorded =
 * how many exist) and, for PL_POISSON_LEARNED, the iterations preconditioned by the network before any
 * fall-back to multigrid. (No counterpart in the reference; Pcg3D.solve returns only the totals.) */
#define PL_POISSON_HISTORY 64
int pl_poisson_history(const pl_poisson* h, int32_t snapshot, double* max_residual, int32_t capacity,
                       int32_t* recorded, int32_t* learned_iterations);
void pl_poisson_destroy(pl_poisson* h);

/* ------------------------------------------------------------------ learned preconditioner */

/* (pl_unet is declared with the Poisson batch above.) A 3-level 3D convolutional U-Net (16/32/64 channels, 3^3 kernels, BF16 weights and activations,
 * FP32 accumulation) that maps a residual r to an approximate correction z ~ A^-1 r on the liquid
 * cells of a box (no counterpart in the reference). Inputs: [r / max|r|, liquid mask, air mask];
 * output scaled by max|r| and zero off the liquid. Boxes are nx x ny x nz cells (multiples of 4), count
 * of them back to back, x fastest; cell u8 (PL_AIR / PL_FLUID / PL_SOLID), r, z, e f32, all device
 * buffers. Parameters are FP32 masters (per layer W[27][cin][cout] then the biases), trained by Adam
 * on the relative squared error sum_liquid (z - e)^2 / sum_liquid e^2, averaged over the boxes. */
int pl_unet_create(uint32_t seed, pl_unet** out);
/* Training loss: PL_UNET_LOSS_L2 (the default above) or PL_UNET_LOSS_ENERGY, the error in the operator's
 * energy norm, (z - e).A(z - e) / e.Ae per box (unknowns: liquid cells off the box border), the norm in
 * which a preconditioner's quality decides CG's convergence. */
enum pl_unet_loss { PL_UNET_LOSS_L2 = 0, PL_UNET_LOSS_ENERGY = 1 };
int pl_unet_set_loss(pl_unet* u, int32_t kind);
/* Convolution kernels: TCGEN05 (default; 5th-generation tensor cores, accumulator in tensor memory) or
 * MMA_SYNC (the warp-level tensor-core path, kept for comparison). Both compute the same convolutions
 * in BF16 with FP32 accumulation. */
enum pl_unet_conv { PL_UNET_CONV_TCGEN05 = 0, PL_UNET_CONV_MMA_SYNC = 1 };
int pl_unet_set_conv_kernel(pl_unet* u, int32_t kind);
/* 1 if a tensor-core convolution of this network gave up a bounded wait (its output is then invalid),
 * else 0. Synchronous. */
int pl_unet_error(pl_unet* u);
int32_t pl_unet_num_params(const pl_unet* u);
int pl_unet_get_params(pl_unet* u, float* host);
int pl_unet_set_params(pl_unet* u, const float* host); /* also resets the Adam moments */
int pl_unet_apply(pl_unet* u, const uint8_t* cell, const float* r, float* z, int32_t nx, int32_t ny, int32_t nz,
                  int32_t count, void* stream);
/* One Adam step (learning rate lr) on the boxes' (r, e) pairs; the loss before the step to *loss. */
int pl_unet_train_step(pl_unet* u, const uint8_t* cell, const float* r, const float* e, int32_t nx, int32_t ny,
                       int32_t nz, int32_t count, float lr, float* loss, void* stream);
/* The loss and its gradient with respect to every parameter (host array of pl_unet_num_params floats)
 * without a step. Synchronous. */
int pl_unet_gradient(pl_unet* u, const uint8_t* cell, const float* r, const float* e, int32_t nx, int32_t ny,
                     int32_t nz, int32_t count, float* loss, float* grad, void* stream);
void pl_unet_destroy(pl_unet* u);
/* The network of a simulation created with PL_PRECOND_LEARNED (required before its first substep;
 * the caller keeps it alive while the simulation uses it). Rebuilds the substep graph. */
int pl_set_unet(pl_sim* sim, pl_unet* u);

/* ------------------------------------------------------------------ ensembles */

/* Seeded pour configurations (no counterpart in the reference): count gentle pours at cell_mm, each
 * lasting `seconds`, drawn from a mulberry32 stream (src/sim/rng.ts) seeded with `seed`: fill
 * U[0.6, 1.0] L, peak tilt (motion.max_angle_deg) U[60, 110] degrees, tilt-in ramp
 * (motion.tilt_duration) U[4, 12] s; pour i gets seed + 1 + i as its seeding seed. The grid of each
 * follows from its fill and peak tilt (solver3d.ts:125-157), so an ensemble's grids are uneven. */
int pl_ensemble_configs(uint32_t seed, int32_t count, double cell_mm, double seconds, pl_config* out);
/* Many pours on one device: each pour a pl_sim with its own stream and substep graph; the calls below
 * launch the pours' substeps interleaved, so their small kernels run concurrently, with one host
 * synchronisation per pour per chunk. */
typedef struct pl_ensemble pl_ensemble;
int pl_ensemble_create(const pl_config* cfgs, int32_t count, pl_ensemble** out);
int32_t pl_ensemble_size(const pl_ensemble* e);
/* Member i (owned by the ensemble; every pl_* call on a pl_sim works on it). */
pl_sim* pl_ensemble_member(pl_ensemble* e, int32_t i);
/* Every pour advances by `duration` simulated seconds (advance(), solver3d.ts:281-286, per pour). */
int pl_ensemble_advance(pl_ensemble* e, double duration);
/* Every pour runs `substeps` stable substeps (those past its duration are no-ops). */
int pl_ensemble_enqueue(pl_ensemble* e, int32_t substeps);
void pl_ensemble_destroy(pl_ensemble* e);

#ifdef __cplusplus
}
#endif

#endif /* POURLAB_H */
