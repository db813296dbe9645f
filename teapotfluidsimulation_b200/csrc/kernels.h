// Launch helpers and sizes shared by kernels.cu, solver.cu and engine.cu.
#pragma once

#include "common.cuh"

namespace pl {

// 1024 threads x 2 bins (the same 2048-bin tile as 256 x 8, shorter per-thread chains): 4 mm whole pour
// 0.2839 ms per substep at 256 x 8, 0.2808 at 512 x 4, 0.2800 -> 0.2787 at 1024 x 2
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 2;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int SCAN_MAX_TILES = 4096;  // bins <= 8M
constexpr int DENSITY_BLOCKS = 148;
constexpr int SOLVER_THREADS = 1024;
constexpr int MAX_LEVELS = 2048;  // wavefronts i+j+k of the MIC(0) sweeps

// List-indexed scratch of the pressure solves (capacity = interior cells).
struct SolverWs {
  int cap;
  int* nb;        // 6 * cap: list index of the -x,+x,-y,+y,-z,+z neighbour or -1
  double* adiag;  // non-solid neighbour count
  int* wave;      // i + j + k
  int* order;     // list entries by wavefront
  int* lstart;    // MAX_LEVELS + 1 wavefront starts
  int* nlev;      // [0] wavefront count, [1] lowest wavefront
  double* pc;     // MIC(0) inverse-sqrt diagonal
  double* bp;     // pressure rhs (negative divergence)
  double *r, *z, *s, *as, *qv;
};

struct SolveArgs {
  const double* b;
  double* q;
  double tol;
  int max_iter;
  int is_correction;  // density solve: gated by corr_any, records corr_iters and the interior mean
  int factor;         // build the wavefront order and the MIC(0) factor first
  int fallback;       // run only when the cluster multigrid solve did not (mg_status == 0)
};

SolverWs solver_ws_carve(void* base, int cap);
size_t solver_ws_bytes(int cap);

void launch_stage_bin(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_stage_extrap(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_stage_density(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_stage_advect(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_pressure_solve(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_correction_solve(const Geo& g, const DevPtrs& P, cudaStream_t st);
// the two halves of the P2G stage, so that the density stage can run beside the faces
void launch_p2g_cells(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_p2g_faces(const Geo& g, const DevPtrs& P, cudaStream_t st);
// recording frames: every stride-th parcel's position quantised to u16 (format.ts:60)
void launch_quantize(const DevPtrs& P, int n, int stride, double quantum, uint16_t* out, cudaStream_t st);
struct PoissonImpl;
// grid-scale solves (PL_PRECOND_BOX_MG / PL_PRECOND_LEARNED): the liquid system in the dense box,
// solved by the Poisson batch's device-driven multigrid / learned PCG inside the substep graph
int launch_box_solves(const Geo& g, const DevPtrs& P, PoissonImpl* box, PoissonImpl* box2, cudaStream_t st,
                      cudaStream_t st2, cudaEvent_t fork, cudaEvent_t join, char* err, size_t errlen);
void launch_render(const Geo& g, const DevPtrs& P, cudaStream_t st);
void launch_export_correction(const Geo& g, const DevPtrs& P, float* out, cudaStream_t st);

// Standalone Pcg3D.solve on a caller's grid (pl_pcg_solve_device).
int standalone_pcg(const uint8_t* cell, const double* b, double* q, int nx, int ny, int nz, double tol,
                   int max_iter, int precond, int precision, cudaStream_t st, int* iterations, int* converged,
                   double* residual, char* err, size_t errlen);
// The same solve with fixed static scratch (pl_pcg_solve_device_noalloc); allocates nothing.
int standalone_pcg_noalloc(const uint8_t* cell, const double* b, double* q, int nx, int ny, int nz, double tol,
                           int max_iter, cudaStream_t st, int* iterations, int* converged, double* residual,
                           char* err, size_t errlen);

}  // namespace pl
