// Pressure solves of the pour engine: Pcg3D.solve (solver3d.ts:858-973) on the liquid cells.
//
// The liquid system is small (thousands to tens of thousands of unknowns) and every iteration is a
// chain of dependent reductions, so one persistent thread block runs a whole solve: no kernel
// boundary and no host round trip per iteration. The preconditioner is the reference's MIC(0)
// factor itself. Its triangular sweeps are applied in wavefront order (all cells with equal
// i + j + k are independent, since every coupling of the lower factor goes to i-1, j-1 or k-1), so
// each cell is computed by exactly the reference's expression from the same operands: the factor
// and every preconditioner application agree with the FP64 reference bit for bit. Inner products
// are fixed-order tree reductions (deterministic; they differ from the reference's sequential sums
// only in rounding).
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "kernels.h"
#include "cheb.h"
#include "mg.h"
#include "poisson.h"
#include "pcg_block.cuh"

namespace pl {

SolverWs solver_ws_carve(void* base, int cap) {
  char* p = static_cast<char*>(base);
  size_t c = (size_t)cap;
  auto take = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~size_t(255);
    return r;
  };
  SolverWs w;
  w.cap = cap;
  w.adiag = (double*)take(c * 8);
  w.pc = (double*)take(c * 8);
  w.bp = (double*)take(c * 8);
  w.r = (double*)take(c * 8);
  w.z = (double*)take(c * 8);
  w.s = (double*)take(c * 8);
  w.as = (double*)take(c * 8);
  w.qv = (double*)take(c * 8);
  w.nb = (int*)take(c * 6 * 4);
  w.wave = (int*)take(c * 4);
  w.order = (int*)take(c * 4);
  w.lstart = (int*)take((MAX_LEVELS + 1) * 4);
  w.nlev = (int*)take(16);
  return w;
}

// Bytes of the carve above (256-byte aligned pieces).
size_t solver_ws_bytes(int cap) {
  size_t c = (size_t)cap;
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  return 8 * al(c * 8) + al(c * 24) + 2 * al(c * 4) + al((MAX_LEVELS + 1) * 4) + al(16);
}

// ---------------------------------------------------------------- setup (many blocks)

// Neighbour list indices, diagonal, wavefront and the pressure rhs of every liquid cell
// (solver3d.ts:869-881 and divergenceRhs, solver3d.ts:473-493). With tile_order, also the cluster
// solver's column-tile order: every block first forms the exclusive prefix of the (tile, plane)
// mask populations in shared memory (dynamic, ntx * nty * nz <= TILE_PLANES_MAX ints); a liquid cell's position is then
// its plane's prefix plus the liquid cells before it in its plane of the tile.
__global__ void k_solve_setup(Geo g, DevPtrs P, SolverWs W, int compute_rhs, int tile_order) {
  const SimScalars* sc = P.sc;
  if (!sc->active) return;
  extern __shared__ int s_pre[];
  __shared__ int s_warp[32];
  const int m = sc->m;
  const int nxy = g.nx * g.ny;
  const bool tiled = tile_order && g.tiled;
  if (tiled) {
    const int T = g.ntx * g.nty * g.nz;
    const int per = (T + blockDim.x - 1) / blockDim.x;
    const int e0 = threadIdx.x * per;
    int sum = 0;
    for (int q = 0; q < per; q++)
      if (e0 + q < T) sum += __popcll(P.tile_mask[e0 + q]);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < nw; w++) {
        int c = s_warp[w];
        s_warp[w] = acc;
        acc += c;
      }
    }
    __syncthreads();
    int run = s_warp[wid] + x - sum;
    for (int q = 0; q < per; q++)
      if (e0 + q < T) {
        s_pre[e0 + q] = run;
        run += __popcll(P.tile_mask[e0 + q]);
      }
    __syncthreads();
  }
  auto tpos = [&](int c) {
    const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / nxy;
    const int tp = ((j / TILE_W) * g.ntx + i / TILE_W) * g.nz + k;
    const int bit = (j % TILE_W) * TILE_W + i % TILE_W;
    return s_pre[tp] + __popcll(P.tile_mask[tp] & ((1ull << bit) - 1ull));
  };
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int c = P.list[t];
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / nxy;
    const int off[6] = {-1, 1, -g.nx, g.nx, -nxy, nxy};
    double d = 0;
    const int p = tiled ? tpos(c) : t;
    if (tile_order) P.tperm[p] = t;
#pragma unroll
    for (int e = 0; e < 6; e++) {
      int cc = c + off[e];
      const int li = P.lidx[cc];
      W.nb[e * W.cap + t] = li;
      if (tile_order) P.tnb[e * g.nc + p] = li < 0 ? -1 : (tiled ? tpos(cc) : li);
      if (P.cell[cc] != SOLID) d += 1;
    }
    W.adiag[t] = d;
    W.wave[t] = i + j + k;
    if (compute_rhs) {
      const float* u = P.u;
      int iu = i + (g.nx + 1) * (j + g.ny * k);
      int iv = g.nu + i + g.nx * (j + (g.ny + 1) * k);
      int iw = g.nu + g.nv + c;
      double dv = (double)u[iu + 1] - (double)u[iu] + (double)u[iv + g.nx] - (double)u[iv] +
                  (double)u[iw + nxy] - (double)u[iw];
      W.bp[t] = -dv;
    }
  }
}

__global__ void __launch_bounds__(SOLVER_THREADS) k_pcg(Geo g, DevPtrs P, SolverWs W, SolveArgs a) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  if (a.fallback && sc->mg_status) return;  // the cluster multigrid solve already ran
  __shared__ double s_red[64];
  __shared__ int s_lstart[MAX_LEVELS + 1];
  __shared__ int s_hist[MAX_LEVELS + 1];
  Reducer red{s_red, 0};
  const int m = sc->m;
  if (a.is_correction) {
    if (threadIdx.x == 0) {  // interior mean of the density ratios (solver3d.ts:670)
      double s = 0;
      int n = 0;
      for (int b = 0; b < DENSITY_BLOCKS; b++) {
        s += P.interior_part[b];
        n += P.interior_cnt_part[b];
      }
      sc->interior = n > 0 ? s / n : 1.0;
      sc->interior_count = n;
    }
    if (!sc->corr_any) {  // solver3d.ts:671: no solve, uc = vc = wc = 0
      if (threadIdx.x == 0) sc->corr_iters = 0;
      return;
    }
  }
  SolveOut o = pcg_block(W, m, a.b, a.q, a.tol, a.max_iter, a.factor != 0 || a.fallback != 0, red, s_lstart, s_hist);
  if (threadIdx.x == 0) {
    if (o.iterations < 0) {
      atomicOr(&sc->errors, ERR_SOLVER_SIZE);
      o.iterations = 0;
    }
    if (a.is_correction) {
      sc->corr_iters = o.iterations;
      sc->corr_residual = o.residual;
    } else {
      sc->last_iters = o.iterations;
      sc->last_residual = o.residual;
      if (!o.converged) sc->failures++;  // solver3d.ts:540
    }
  }
}

static SolverWs ws_of(const DevPtrs& P, int cap) { return solver_ws_carve(P.solver_ws, cap); }

// Liquid cells a cluster solve is sized for: a quarter more than the parcels fill at the seeding
// density of about 8 per cell (the liquid of a pour spreads, but it does not grow); a system above
// it goes to a launch sized for more, then to the wavefront solver.
static int cheb_m_bound(const Geo& g) { return std::min(g.nc, g.n * 5 / 32 + 64); }

// Pressure solve (project(), solver3d.ts:530-543). With the multigrid preconditioner the cluster
// solve runs first and the wavefront MIC(0) solve only if the cluster's shared memory could not
// hold the hierarchy (it then factors as usual).
void launch_pressure_solve(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  SolverWs W = ws_of(P, g.nc);
  const bool mg = g.precond == PL_PRECOND_MG, cheb = g.precond == PL_PRECOND_CHEB;
  const size_t pre_bytes = (cheb && g.tiled) ? size_t(g.ntx) * g.nty * g.nz * 4 : 0;
  k_solve_setup<<<DENSITY_BLOCKS, 256, pre_bytes, st>>>(g, P, W, 1, cheb ? 1 : 0);
  if (mg) {
    MgWs M = mg_ws_carve(g, P.mg_ws, P, W);
    launch_mg_setup(g, P, M, st);
    launch_mg_solve(g, P, M, MgArgs{W.bp, P.q, g.tol, g.max_iter, 0, g.precision == PL_SOLVE_MIXED}, st);
  } else if (cheb) {
    // both systems of the substep in one cluster launch: the density-correction rhs depends only on
    // the parcels and the cell types, so it is ready before the pressure solve
    ChebArgs c{W.bp, P.q, g.tol, g.max_iter, 0, g.precision == PL_SOLVE_MIXED, CHEB_DEGREE, CHEB_LO,
               g.solve_cluster, g.solve_threads, CHEB_SMEM, cheb_m_bound(g), 0};
    c.jobs = 2;
    c.b2 = P.rhs;
    c.q2 = P.qc;
    c.tol2 = 1e-4;  // solver3d.ts:673
    c.max_iter2 = 80;
    c.parallel = 1;
    launch_cheb_solve(g, P, W, c, st);
  }
  SolveArgs a{W.bp, P.q, g.tol, g.max_iter, 0, 1, (mg || cheb) ? 1 : 0};
  k_pcg<<<1, SOLVER_THREADS, 0, st>>>(g, P, W, a);
}

// Density-correction solve (solver3d.ts:671-674): tolerance 1e-4, at most 80 iterations. Runs after
// the pressure solve; its rhs (k_density) is computed before the pressure solve.
void launch_correction_solve(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  SolverWs W = ws_of(P, g.nc);
  const bool mg = g.precond == PL_PRECOND_MG, cheb = g.precond == PL_PRECOND_CHEB;
  if (mg) {
    MgWs M = mg_ws_carve(g, P.mg_ws, P, W);
    launch_mg_solve(g, P, M, MgArgs{P.rhs, P.qc, 1e-4, 80, 1, g.precision == PL_SOLVE_MIXED}, st);
  }  // the Chebyshev path solved this system in the pressure launch; only its fallback is left here
  SolveArgs a{P.rhs, P.qc, 1e-4, 80, 1, 0, (mg || cheb) ? 1 : 0};
  k_pcg<<<1, SOLVER_THREADS, 0, st>>>(g, P, W, a);
}

// ---------------------------------------------------------------- grid-scale solves (dense box)

// The liquid system in the power-of-two box: FLUID where the cell is on the liquid list, the grid's
// AIR / SOLID elsewhere, SOLID outside the grid (so the box operator is the liquid list's operator:
// diagonal = non-SOLID neighbours, -1 between liquid neighbours); b = rhs on the liquid cells (0 on an
// inactive substep, which the solve then finishes at once).
__global__ void k_box_embed(Geo g, DevPtrs P, const double* rhs, int with_cells, float* bout) {
  const long long nb = (long long)g.bx * g.by * g.bz;
  const bool act = P.sc->active != 0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nb; v += (long long)gridDim.x * blockDim.x) {
    const int i = int(v % g.bx), j = int((v / g.bx) % g.by), k = int(v / ((long long)g.bx * g.by));
    uint8_t t = SOLID;
    float b = 0.f;
    if (i < g.nx && j < g.ny && k < g.nz) {
      const int c = i + g.nx * (j + g.ny * k);
      const int li = P.lidx[c];
      if (li >= 0) {
        t = FLUID;
        if (act) b = float(rhs[li]);
      } else {
        t = P.cell[c] == SOLID ? SOLID : AIR;
      }
    }
    if (with_cells) P.box_cell[v] = t;
    bout[v] = b;
  }
}

// The box solution back on the liquid list, and the solve's outcome into the scalar block (the
// pressure solve counts a failure when it did not converge, solver3d.ts:540).
__global__ void k_box_finish(Geo g, DevPtrs P, const double* xbox, const double* out, double* q, int correction) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  const int m = sc->m;
  const int nxy = g.nx * g.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int c = P.list[t];
    const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / nxy;
    q[t] = xbox[i + (long long)g.bx * (j + (long long)g.by * k)];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int it = int(out[0]);
    const double res = out[2];
    if (correction) {
      sc->corr_iters = it;
      sc->corr_residual = res;
    } else {
      sc->last_iters = it;
      sc->last_residual = res;
      if (out[1] == 0) sc->failures++;
    }
  }
}

static unsigned box_blocks(const Geo& g) {
  const long long nb = (long long)g.bx * g.by * g.bz;
  return unsigned(std::min<long long>((nb + 255) / 256, 148 * 16));
}

// Both grid-scale solves of a substep. They are independent (the correction's rhs needs only the
// parcels and the cell types), so after the box's cell types are written the correction forks onto
// a second stream of the capture with its own solver and buffers (multigrid, tolerance 1e-4,
// solver3d.ts:673) and joins before the stream goes on: the graph runs the two solves side by side.
int launch_box_solves(const Geo& g, const DevPtrs& P, PoissonImpl* box, PoissonImpl* box2, cudaStream_t st,
                      cudaStream_t st2, cudaEvent_t fork, cudaEvent_t join, char* err, size_t errlen) {
  SolverWs W = ws_of(P, g.nc);
  k_solve_setup<<<DENSITY_BLOCKS, 256, 0, st>>>(g, P, W, 1, 0);
  k_box_embed<<<box_blocks(g), 256, 0, st>>>(g, P, W.bp, 1, P.box_b);
  cudaEventRecord(fork, st);
  cudaStreamWaitEvent(st2, fork, 0);
  // correction (second stream)
  k_box_embed<<<box_blocks(g), 256, 0, st2>>>(g, P, P.rhs, 0, P.box_b2);
  int rc = poisson_capture_setup(box2, P.box_cell, st2, err, errlen);
  if (!rc) rc = poisson_capture_solve(box2, P.box_b2, P.box_x2, 1e-4, 80, st2, err, errlen);
  if (!rc) {
    poisson_capture_result(box2, P.box_out2, st2);
    k_box_finish<<<DENSITY_BLOCKS, 256, 0, st2>>>(g, P, P.box_x2, P.box_out2, P.qc, 1);
  }
  cudaEventRecord(join, st2);
  // pressure (this stream)
  if (!rc) rc = poisson_capture_setup(box, P.box_cell, st, err, errlen);
  if (!rc) rc = poisson_capture_solve(box, P.box_b, P.box_x, g.tol, g.max_iter, st, err, errlen);
  if (!rc) {
    poisson_capture_result(box, P.box_out, st);
    k_box_finish<<<DENSITY_BLOCKS, 256, 0, st>>>(g, P, P.box_x, P.box_out, P.q, 0);
  }
  cudaStreamWaitEvent(st, join, 0);
  return rc;
}

// ---------------------------------------------------------------- standalone solve

int standalone_pcg(const uint8_t* cell, const double* b, double* q, int nx, int ny, int nz, double tol,
                   int max_iter, int precond, int precision, cudaStream_t st, int* iterations, int* converged,
                   double* residual, char* err, size_t errlen) {
  if (precond != PL_PRECOND_MIC0 || precision != PL_SOLVE_F64) {
    snprintf(err, errlen, "pl_pcg_solve_device: the standalone solve is MIC(0) in FP64 (preconditioner %d, "
             "precision %d requested)", precond, precision);
    return PL_E_ARG;
  }
  if (nx < 3 || ny < 3 || nz < 3 || nx + ny + nz > MAX_LEVELS) {
    snprintf(err, errlen, "pl_pcg_solve_device: grid %dx%dx%d out of range", nx, ny, nz);
    return PL_E_ARG;
  }
  // An error left pending by the caller's own earlier launches is reported as such and left in
  // place, so that the check after this call's launches sees only this call's launch errors.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "pl_pcg_solve_device: a CUDA error was already pending before the call: %s",
             cudaGetErrorString(e));
    return PL_E_CUDA;
  }
  const int nc = nx * ny * nz;
  size_t wsb = solver_ws_bytes(nc);
  size_t extra = (size_t)nc * 4 * 2 + (size_t)nc * 8 * 2 + 256;
  void* mem = nullptr;
  e = cudaMalloc(&mem, wsb + extra);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "cudaMalloc(%zu): %s", wsb + extra, cudaGetErrorString(e));
    return PL_E_NOMEM;
  }
  SolverWs W = solver_ws_carve(mem, nc);
  char* p = static_cast<char*>(mem) + wsb;
  int* lidx = (int*)p;
  int* list = lidx + nc;
  double* bl = (double*)(list + nc);  // 2 * nc ints from a 256-byte boundary: 8-byte aligned
  double* ql = bl + nc;
  int* small = (int*)(ql + nc);  // [0] m, [1..2] result
  double* resd = (double*)(small + 4);
  k_standalone_prep<<<1, 1024, 0, st>>>(cell, nx, ny, nz, lidx, list, small);
  k_standalone_setup<<<DENSITY_BLOCKS, 256, 0, st>>>(cell, b, nx, ny, lidx, list, small, W, bl);
  k_standalone_pcg<<<1, SOLVER_THREADS, 0, st>>>(W, small, bl, ql, tol, max_iter, small + 1, resd);
  k_standalone_scatter<<<(nc + 255) / 256, 256, 0, st>>>(lidx, ql, q, nc);
  int hres[3];
  double hr = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hres, small, 12, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hr, resd, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaError_t ef = cudaFree(mem);
  if (e != cudaSuccess || ef != cudaSuccess) {
    snprintf(err, errlen, "pl_pcg_solve_device: %s", cudaGetErrorString(e != cudaSuccess ? e : ef));
    return PL_E_CUDA;
  }
  if (iterations) *iterations = hres[1];
  if (converged) *converged = hres[2];
  if (residual) *residual = hr;
  return PL_OK;
}

}  // namespace pl
