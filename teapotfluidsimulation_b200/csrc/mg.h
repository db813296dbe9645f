// Multigrid-preconditioned CG on one thread-block cluster (see mg.cu).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace pl {

constexpr int MG_MAX_LEVELS = 6;
constexpr int MG_CLUSTER = 16;           // CTAs per cluster (non-portable size, one per SM)
constexpr int MG_THREADS = 256;          // threads per CTA
constexpr int MG_SMEM = 224 * 1024;      // dynamic shared memory per CTA (227 KB less the static part)
constexpr int MG_COARSE_SWEEPS = 8;      // red-black sweeps each way on the coarsest level
constexpr unsigned MG_NONE = 0xffffffffu;

// Geometric hierarchy in global memory, rebuilt every substep from the cell types.
// Level 0 is the liquid list of the substep; level L+1 coarsens level L by 2 in each direction
// (a coarse cell is AIR if any child is AIR, else FLUID if any child is FLUID, else SOLID, and the
// border is SOLID: src/sim/multigrid.ts:58-80 in 3D).
struct MgLevel {
  int nx, ny, nz, cap;  // grid dims, capacity of the list-indexed arrays (= nx*ny*nz)
  uint8_t* type;        // [nx*ny*nz]
  int* lidx;            // [nx*ny*nz] list index or -1
  int* list;            // [cap] grid index of each liquid cell
  int* nb;              // [6*cap] neighbour list index (-x,+x,-y,+y,-z,+z) or -1
  int* nbp;             // [6*cap] parent (level L+1) list index of that neighbour or -1
  int* child;           // [8*cap] children (level L-1) list indices or -1 (L >= 1)
  int* parent;          // [cap] parent list index or -1
  float* adiag;         // [cap] non-solid neighbour count
};

struct MgWs {
  int nlev;
  MgLevel lv[MG_MAX_LEVELS];
  int* m;  // [MG_MAX_LEVELS] liquid cells per level (device)
};

struct MgArgs {
  const double* b;  // list-indexed rhs (level 0)
  double* q;        // list-indexed solution (level 0)
  double tol;
  int max_iter;
  int is_correction;
  int mixed;  // FP32 vectors with FP64 true-residual refinement
};

size_t mg_ws_bytes(const Geo& g, int* nlev_out);
MgWs mg_ws_carve(const Geo& g, void* base, const DevPtrs& P, const SolverWs& W);
void mg_configure();  // kernel attributes (cluster size, shared memory); call once per device
void launch_mg_setup(const Geo& g, const DevPtrs& P, const MgWs& M, cudaStream_t st);
void launch_mg_solve(const Geo& g, const DevPtrs& P, const MgWs& M, const MgArgs& a, cudaStream_t st);

}  // namespace pl
