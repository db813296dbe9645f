// Batched pressure-Poisson solves on dense n^3 grids: the isolated-solve workload of the pour engine
// (many independent snapshots of the same operator as Pcg3D, src/sim3d/solver3d.ts:858-973).
//
// Operator: for every unknown (FLUID, not on the grid border) the 7-point MAC Laplacian of Pcg3D:
// diagonal = number of non-SOLID neighbours, -1 to every FLUID neighbour; AIR is Dirichlet 0 and
// SOLID Neumann. A cell flagged PL_POISSON_PIN gets +1 on its diagonal: the gauge fix of a liquid
// component without air contact (src/sim/pressure.ts:232-268), which pl_poisson_generate applies.
//
// Layout: `count` snapshots back to back, each n^3 cells in x-fastest order; per level an
// unknown/neighbour code per cell (level 0 also a diagonal byte; coarse levels a diagonal and six link
// weights), and tiles of 256 cells (32 x 4 x 2 at n >= 32)
// with a flag "holds an unknown". Every kernel runs one CTA per active tile (a compact list in tile
// order built at set-up), so the work and the memory traffic follow the liquid, not the box, and
// neighbouring tiles run close together in time (their shared halo rows hit in L2).
//
// Solver: PCG with the reference's stopping rule (max-norm residual <= max(tol * max|b|, 1e-14),
// breakdown if s.As <= 0), all snapshots in lock step with per-snapshot alpha, beta and convergence;
// a converged snapshot's tiles drop out. Vectors are FP32 (PL_SOLVE_MIXED) or FP64 (PL_SOLVE_F64);
// inner products, norms and the solution are FP64, and a converged recursive residual is confirmed by
// the FP64 true residual b - A x (CG restarts from it if it misses: iterative refinement). Inner
// products are per-tile partials summed per snapshot in tile order (deterministic).
//
// Preconditioners:
//  - MG: one V-cycle of geometric multigrid on 2 x 2 x 2 aggregates (the level structure of
//    src/sim/multigrid.ts in 3D: coarsen by two per axis down to 8 cells, piecewise-constant
//    prolongation, sum restriction, red-black Gauss-Seidel smoothing) with Galerkin coarse operators
//    A_c = P^T A P instead of the reference's rediscretised levels: on these free-surface masks the
//    rediscretised coarse levels misplace the AIR and SOLID boundaries and the iteration count grows
//    with the grid (CPU prototype: 43 vs 15 iterations at 64^3), the Galerkin levels keep it nearly
//    flat. A coarse cell is an unknown if any child is; its link to a neighbour aggregate weighs the
//    number of fine links between them and its diagonal is the children's diagonals minus their
//    internal links. Two sweeps (red, black) before and (black, red) after the coarse correction,
//    which is over-relaxed by 1.5, and a palindromic sweep sequence on the coarsest level (8^3 per
//    snapshot, one CTA): the V-cycle is a symmetric operator, so CG stays valid.
//  - LEARNED: flexible CG (Polak-Ribiere beta) with the U-Net of unet.cu as the preconditioner
//    (z = the network's output for r), and the multigrid above as the fallback: a snapshot whose
//    max-norm residual falls less than 2x over 5 iterations (or that reaches 200 network iterations)
//    switches to multigrid and restarts CG from its FP64 true residual; every snapshot still ends on
//    the same max-norm rule.
//  - MIC0: the reference's MIC(0) factor and triangular sweeps (solver3d.ts:883-900, 955-973). A
//    cell depends only on its -x, -y, -z neighbours, so the planes i + j + k = d, processed in
//    increasing (forward) or decreasing (backward) order, give exactly the sequential result; one
//    launch per plane, captured in a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "common.cuh"
#include "poisson.h"
#include "unet.h"

namespace pl {

namespace {

constexpr int PMAXLEV = 8;
constexpr int PT = 256;  // cells per tile = threads per CTA
constexpr int RED_T = 256;
// Programmatic dependent launch inside the iteration loop: every kernel of the loop body first waits
// (in every CTA, before any early return) until its predecessor in the stream has completed and its
// writes are visible, then lets its own successor begin launching; the successor's launch and CTA
// set-up overlap this kernel's work. Waiting in every CTA keeps the ordering transitive. Launched
// without the attribute, both instructions do nothing.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
constexpr int COARSE_SWEEPS = 10;  // (red, black) pairs before and (black, red) pairs after: 40 half-sweeps
constexpr int MG_NU = 2;           // smoothing sweeps before and after the coarse correction
constexpr double MG_OMEGA = 1.5;   // over-relaxation of the coarse correction

// code bits: 0..5 neighbour (-x, +x, -y, +y, -z, +z) is an unknown; 6 this cell is an unknown
constexpr uint8_t C_SELF = 1u << 6;

struct TG {  // tiling of one level (every extent a power of two)
  int nx, ny, nz;     // cells per axis
  int rx, ry, rz;     // coarsening factor (1 or 2) from the finer level on each axis (1 on level 0)
  int tx, ty, tz;     // tile extent
  int px, py, pz;     // tiles per axis
  long long nc;       // cells per snapshot
  long long ntile;    // tiles per snapshot
  // base-2 logarithms for the index arithmetic (all indices fit in 32 bits: checked at creation)
  int lnx, lny, ltx, lty, lpx, lpy, lnt, lnc;
};

inline int ilog2(long long v) {
  int l = 0;
  while ((1ll << l) < v) l++;
  return l;
}

TG make_tg(int nx, int ny, int nz, int rx = 1, int ry = 1, int rz = 1) {
  TG t;
  t.nx = nx, t.ny = ny, t.nz = nz;
  t.rx = rx, t.ry = ry, t.rz = rz;
  t.tx = std::min(32, nx);
  t.ty = std::min(4, ny);
  t.tz = PT / (t.tx * t.ty);  // every extent is >= 8, so a tile always holds PT cells
  t.px = nx / t.tx;
  t.py = ny / t.ty;
  t.pz = nz / t.tz;
  t.nc = (long long)nx * ny * nz;
  t.ntile = (long long)t.px * t.py * t.pz;
  t.lnx = ilog2(nx);
  t.lny = ilog2(ny);
  t.ltx = ilog2(t.tx);
  t.lty = ilog2(t.ty);
  t.lpx = ilog2(t.px);
  t.lpy = ilog2(t.py);
  t.lnt = ilog2(t.ntile);
  t.lnc = ilog2(t.nc);
  return t;
}

// Cell of thread `tid` in global tile `gt` (snapshot-major); false for threads past a small tile.
__device__ __forceinline__ bool tile_cell(const TG& G, int gt, int tid, int& s, int& i, int& j, int& k, int& c) {
  if (tid >= G.tx * G.ty * G.tz) return false;
  s = gt >> G.lnt;
  const int lt = gt & ((1 << G.lnt) - 1);
  const int ti = lt & (G.px - 1), tj = (lt >> G.lpx) & (G.py - 1), tk = lt >> (G.lpx + G.lpy);
  i = (ti << G.ltx) + (tid & (G.tx - 1));
  j = (tj << G.lty) + ((tid >> G.ltx) & (G.ty - 1));
  k = (tk * G.tz) + (tid >> (G.ltx + G.lty));
  c = (s << G.lnc) + (((k << G.lny) + j) << G.lnx) + i;
  return true;
}

// Per-snapshot PCG state.
struct Snap {
  double bnorm, target;
  double rz, rz_old, alpha, beta, res;
  int it, done, converged, check, restarts, fresh;
  // learned preconditioning: 0 = the network, 1 = multigrid (after a stall); max |r| of the last
  // iterations (ring) for the stall test; iterations taken with the network
  int pre, learned_it;
  double hist[8];
  double rh[PL_POISSON_HISTORY];  // max |r| after iteration k + 1 (the first PL_POISSON_HISTORY iterations)
};

// First FP64 true-residual confirmation of an FP32-vector solve (not the learned one) at this multiple
// of the target; later confirmations and the acceptance use the target. 64 x 128^3 batch, MG-PCG at
// 1e-6: 1x 38.1 ms (13.7 iterations), 16x 33.7 ms (12.1), 64x 33.6 ms (12.0); MIC(0) 536 -> 495 ms.
constexpr double POISSON_FIRST_CHECK = 16.0;
constexpr int STALL_SPAN = 5;      // the network stalls when max|r| fell less than 2x over this many iterations
constexpr int LEARNED_CAP = 200;   // ... or after this many iterations with it

template <typename T>
struct Lvl {
  TG G;
  uint8_t *code, *diag, *flag;  // diag: level 0 only
  int* list;  // active global tile ids
  int nact;   // host copy after set-up
  T *x, *b;   // levels >= 1 (level 0 uses z and r)
  T *w, *dg;  // levels >= 1: six link weights (w[f * cells + c]) and the diagonal
};

// ---------------------------------------------------------------- set-up kernels

__device__ __forceinline__ uint8_t base_type(uint8_t t) { return t & 3; }

// Unknown/neighbour code, diagonal and tile flag of every cell of a level from its types.
__global__ void k_lvl_code(TG G, const uint8_t* type, uint8_t* code, uint8_t* diag, uint8_t* flag, int count) {
  const int gt = blockIdx.x;
  int s, i, j, k;
  int c;
  bool any = false;
  if (gt < (long long)count * G.ntile && tile_cell(G, gt, threadIdx.x, s, i, j, k, c)) {
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int nxy = nx * ny;
    const uint8_t t = type[c];
    const bool interior = i > 0 && j > 0 && k > 0 && i < nx - 1 && j < ny - 1 && k < nz - 1;
    uint8_t cd = 0, d = 0;
    if (interior && base_type(t) == FLUID) {
      const int off[6] = {-1, 1, -nx, nx, -nxy, nxy};
      const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
#pragma unroll
      for (int f = 0; f < 6; f++) {
        const uint8_t tn = base_type(type[c + off[f]]);
        if (tn != SOLID) d++;
        const bool nin = nb[f][0] > 0 && nb[f][1] > 0 && nb[f][2] > 0 && nb[f][0] < nx - 1 && nb[f][1] < ny - 1 &&
                         nb[f][2] < nz - 1;
        if (tn == FLUID && nin) cd |= uint8_t(1u << f);
      }
      cd |= C_SELF;
      if (t & PL_POISSON_PIN) d++;  // gauge fix (pressure.ts:265)
      any = true;
    }
    code[c] = cd;
    diag[c] = d;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0 && gt < (long long)count * G.ntile) flag[gt] = any ? 1 : 0;
}

// Galerkin coarse level l+1 from level l (A_c = P^T A P for rx x ry x rz aggregates): unknown if any
// child is; link weight to the aggregate across face f = sum of the children's links across it;
// diagonal = sum of the children's diagonals minus the links inside the aggregate. wf == nullptr:
// the fine level is level 0 (unit links from its code bits, diagonal bytes).
template <typename T>
__global__ void k_gal_coarsen(TG Gf, TG Gc, const uint8_t* codef, const uint8_t* diagf, const T* wf, const T* dgf,
                              uint8_t* codec, T* wc, T* dgc, uint8_t* flagc, int count) {
  const int gt = blockIdx.x;
  int s, i, j, k;
  int c;
  bool any = false;
  const int cellsf = int(count * Gf.nc), cellsc = int(count * Gc.nc);
  if (gt < (long long)count * Gc.ntile && tile_cell(Gc, gt, threadIdx.x, s, i, j, k, c)) {
    const int rx = Gc.rx, ry = Gc.ry, rz = Gc.rz;
    T w6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    T d = T(0);
    bool u = false;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int dx = q & 1, dy = (q >> 1) & 1, dz = q >> 2;
      if (dx >= rx || dy >= ry || dz >= rz) continue;
      const int cf = (s << Gf.lnc) + ((rz * k + dz) * Gf.ny + ry * j + dy) * Gf.nx + rx * i + dx;
      const uint8_t cd = codef[cf];
      if (!(cd & C_SELF)) continue;
      u = true;
      d += wf ? dgf[cf] : T(diagf[cf]);
      // the link leaves the aggregate (on an axis that is not coarsened both links leave)
      const int side[6] = {dx == 0, dx == rx - 1, dy == 0, dy == ry - 1, dz == 0, dz == rz - 1};
#pragma unroll
      for (int f = 0; f < 6; f++) {
        const T lw = wf ? wf[f * cellsf + cf] : ((cd >> f) & 1 ? T(1) : T(0));
        if (side[f]) w6[f] += lw;
        else d -= lw;  // an internal link: its two ends both lose it from the diagonal
      }
    }
    uint8_t cdc = 0;
    if (u) {
      cdc = C_SELF;
#pragma unroll
      for (int f = 0; f < 6; f++)
        if (w6[f] > T(0)) cdc |= uint8_t(1u << f);
      any = true;
    }
    codec[c] = cdc;
    dgc[c] = u ? d : T(1);
#pragma unroll
    for (int f = 0; f < 6; f++) wc[f * cellsc + c] = w6[f];
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0 && gt < (long long)count * Gc.ntile) flagc[gt] = any ? 1 : 0;
}

// Ordered compaction of the tile flags into the active-tile list (tile-id order, so consecutive CTAs
// work on neighbouring tiles and their halo rows are still in L2): per-chunk counts, one-block
// exclusive scan of the counts, then an in-order write per chunk.
constexpr int CHUNK = 1024;

__global__ void __launch_bounds__(CHUNK) k_compact_count(const uint8_t* flag, long long n, int* chunk_cnt) {
  const long long t = (long long)blockIdx.x * CHUNK + threadIdx.x;
  const int f = (t < n && flag[t]) ? 1 : 0;
  const int tot = __syncthreads_count(f);
  if (threadIdx.x == 0) chunk_cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(CHUNK) k_compact_scan(int* chunk_cnt, int nchunk, int* total) {
  __shared__ int sw[CHUNK / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < nchunk; base += CHUNK) {
    const int i = base + threadIdx.x;
    const int v = i < nchunk ? chunk_cnt[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sw[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = sw[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      sw[lane] = w;
    }
    __syncthreads();
    const int excl = carry + x - v + (wid > 0 ? sw[wid - 1] : 0);
    if (i < nchunk) chunk_cnt[i] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += sw[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(CHUNK) k_compact_write(const uint8_t* flag, long long n, const int* chunk_off,
                                                         int* list) {
  __shared__ int sw[CHUNK / 32];
  const long long t = (long long)blockIdx.x * CHUNK + threadIdx.x;
  const int f = (t < n && flag[t]) ? 1 : 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) sw[wid] = __popc(bal);
  __syncthreads();
  if (wid == 0) {
    int w = sw[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sw[lane] = w;
  }
  __syncthreads();
  if (f) {
    const int pos = chunk_off[blockIdx.x] + (wid > 0 ? sw[wid - 1] : 0) + __popc(bal & ((1u << lane) - 1u));
    list[pos] = int(t);
  }
}

// ---------------------------------------------------------------- stencil helpers

template <typename T>
__device__ __forceinline__ T nsum(const T* x, int c, uint8_t cd, int nx, int nxy) {
  T a = (cd & 1) ? x[c - 1] : T(0), b = (cd & 2) ? x[c + 1] : T(0);
  T e = (cd & 4) ? x[c - nx] : T(0), f = (cd & 8) ? x[c + nx] : T(0);
  T g = (cd & 16) ? x[c - nxy] : T(0), h = (cd & 32) ? x[c + nxy] : T(0);
  return ((a + b) + (e + f)) + (g + h);
}

// Weighted neighbour sum of a coarse level (link weights w[f * cells + c]).
template <typename T>
__device__ __forceinline__ T wsum(const T* x, const T* w, int cells, int c, uint8_t cd, int nx, int nxy) {
  T a = (cd & 1) ? w[c] * x[c - 1] : T(0), b = (cd & 2) ? w[cells + c] * x[c + 1] : T(0);
  T e = (cd & 4) ? w[2 * cells + c] * x[c - nx] : T(0), f = (cd & 8) ? w[3 * cells + c] * x[c + nx] : T(0);
  T g = (cd & 16) ? w[4 * cells + c] * x[c - nxy] : T(0), h = (cd & 32) ? w[5 * cells + c] * x[c + nxy] : T(0);
  return ((a + b) + (e + f)) + (g + h);
}

// Off-diagonal sum and diagonal of level (unit links and diagonal bytes when w is null).
template <typename T>
__device__ __forceinline__ void row_sum(const T* x, const uint8_t* diag, const T* w, const T* dg, int cells, int c,
                                        uint8_t cd, int nx, int nxy, T& off, T& d) {
  if (w) {
    off = wsum(x, w, cells, c, cd, nx, nxy);
    d = dg[c];
  } else {
    off = nsum(x, c, cd, nx, nxy);
    d = T(diag[c]);
  }
}

// ---------------------------------------------------------------- multigrid kernels

// Neighbour value x[n] of fine cell n = (i, j, k) of snapshot s with the coarse correction of its
// parent applied: x_fine + omega x_coarse(parent) where the parent is an unknown (the prolongation of
// multigrid.ts:150-156, over-relaxed), formed where it is read.
template <typename T>
__device__ __forceinline__ T prolonged(const T* x, const T* xc, const uint8_t* codec, const TG& Gc, int s, int n,
                                       int i, int j, int k) {
  const int cc = (s << Gc.lnc) + ((k >> (Gc.rz - 1)) * Gc.ny + (j >> (Gc.ry - 1))) * Gc.nx + (i >> (Gc.rx - 1));
  const T v = x[n];
  return (codec[cc] & C_SELF) ? v + T(MG_OMEGA) * xc[cc] : v;
}

// One red-black half-sweep of colour `color` ((i + j + k) & 1) on a level: x = (b + sum of the
// weighted unknown neighbours) / diagonal. first: the first half-sweep of a V-cycle from x = 0. The
// neighbours are all of the other colour, and the half-sweep after this one overwrites that colour
// without reading it, so two passes of the V-cycle are formed where this one reads them instead:
// - xc (the coarse level's solution, its codes codec and geometry Gc): the neighbours with the coarse
//   correction applied (the first post-smoothing half-sweep, in place of a prolongation pass);
// - nb_from_zero: the neighbours' values after a first half-sweep from x = 0, b / diagonal (the
//   second pre-smoothing half-sweep, in place of the first).
// One thread per cell of the colour (128 of a tile's 256 cells), two tiles per CTA.
// NB selects how the neighbours are read, one instantiation each so that the plain sweep keeps its
// own registers: 0 as stored, 1 with the coarse correction (xc), 2 as from x = 0 (nb_from_zero).
template <typename T, int NB>
__global__ void __launch_bounds__(PT) k_mg_smooth(TG G, const int* list, const uint8_t* code, const uint8_t* diag,
                                                   const T* w, const T* dg, int cells, T* x, const T* b,
                                                   int color, int first, const Snap* st, const int* nact,
                                                   const T* xc, const uint8_t* codec, TG Gc) {
  pdl_enter();
  const int ti = blockIdx.x * 2 + (threadIdx.x >> 7);
  if (ti >= *nact) return;
  const int gt = list[ti];
  const int s = gt >> G.lnt;
  if (st[s].done) return;
  const int u = threadIdx.x & 127;
  const int hx = G.ltx - 1;  // log2 of the colour's cells per tile row
  const int row = u >> hx;
  const int lt = gt & ((1 << G.lnt) - 1);
  const int ti_ = lt & (G.px - 1), tj = (lt >> G.lpx) & (G.py - 1), tk = lt >> (G.lpx + G.lpy);
  const int j = (tj << G.lty) + (row & (G.ty - 1));
  const int k = tk * G.tz + (row >> G.lty);
  const int i = (ti_ << G.ltx) + 2 * (u & ((1 << hx) - 1)) + ((color + j + k) & 1);
  const int c = (s << G.lnc) + (((k << G.lny) + j) << G.lnx) + i;
  const uint8_t cd = code[c];
  if (!(cd & C_SELF)) return;
  T off = T(0), d;
  if (NB == 0 && first) {
    d = w ? dg[c] : T(diag[c]);
  } else if constexpr (NB == 2) {
    const int nx = G.nx, nxy = G.nx * G.ny;
    auto z0 = [&](int n) { return b[n] / (w ? dg[n] : T(diag[n])); };
    const T va = (cd & 1) ? z0(c - 1) : T(0), vb = (cd & 2) ? z0(c + 1) : T(0);
    const T ve = (cd & 4) ? z0(c - nx) : T(0), vf = (cd & 8) ? z0(c + nx) : T(0);
    const T vg = (cd & 16) ? z0(c - nxy) : T(0), vh = (cd & 32) ? z0(c + nxy) : T(0);
    if (w) {  // wsum's terms and order
      const T a = (cd & 1) ? w[c] * va : T(0), bb = (cd & 2) ? w[cells + c] * vb : T(0);
      const T e = (cd & 4) ? w[2 * cells + c] * ve : T(0), f = (cd & 8) ? w[3 * cells + c] * vf : T(0);
      const T gg = (cd & 16) ? w[4 * cells + c] * vg : T(0), h = (cd & 32) ? w[5 * cells + c] * vh : T(0);
      off = ((a + bb) + (e + f)) + (gg + h);
      d = dg[c];
    } else {  // nsum's order
      off = ((va + vb) + (ve + vf)) + (vg + vh);
      d = T(diag[c]);
    }
  } else if constexpr (NB == 1) {
    const int nx = G.nx, nxy = G.nx * G.ny;
    const T va = (cd & 1) ? prolonged(x, xc, codec, Gc, s, c - 1, i - 1, j, k) : T(0);
    const T vb = (cd & 2) ? prolonged(x, xc, codec, Gc, s, c + 1, i + 1, j, k) : T(0);
    const T ve = (cd & 4) ? prolonged(x, xc, codec, Gc, s, c - nx, i, j - 1, k) : T(0);
    const T vf = (cd & 8) ? prolonged(x, xc, codec, Gc, s, c + nx, i, j + 1, k) : T(0);
    const T vg = (cd & 16) ? prolonged(x, xc, codec, Gc, s, c - nxy, i, j, k - 1) : T(0);
    const T vh = (cd & 32) ? prolonged(x, xc, codec, Gc, s, c + nxy, i, j, k + 1) : T(0);
    if (w) {  // wsum's terms and order
      const T a = (cd & 1) ? w[c] * va : T(0), bb = (cd & 2) ? w[cells + c] * vb : T(0);
      const T e = (cd & 4) ? w[2 * cells + c] * ve : T(0), f = (cd & 8) ? w[3 * cells + c] * vf : T(0);
      const T gg = (cd & 16) ? w[4 * cells + c] * vg : T(0), h = (cd & 32) ? w[5 * cells + c] * vh : T(0);
      off = ((a + bb) + (e + f)) + (gg + h);
      d = dg[c];
    } else {  // nsum's order
      off = ((va + vb) + (ve + vf)) + (vg + vh);
      d = T(diag[c]);
    }
  } else {
    row_sum(x, diag, w, dg, cells, c, cd, G.nx, G.nx * G.ny, off, d);
  }
  x[c] = (b[c] + off) / d;
}

// Coarse right-hand side: the sum of the unknown children's residuals b - A x (P^T r). The last
// pre-smoothing half-sweep updated the black cells from their red neighbours, so a black residual is
// zero up to rounding and only the red children ((i + j + k) even) are summed. Two tiles per CTA, two
// coarse cells per thread.
template <typename T>
__global__ void __launch_bounds__(PT) k_mg_restrict(TG Gf, TG Gc, const int* listc, const uint8_t* codef,
                                                     const uint8_t* diagf, const T* wf, const T* dgf, int cellsf,
                                                     const T* xf, const T* bf, const uint8_t* codec, T* bc,
                                                     const Snap* st, const int* nact) {
  pdl_enter();
  const int ti = blockIdx.x * 2 + (threadIdx.x >> 7);
  if (ti >= *nact) return;
  const int gt = listc[ti];
  if (st[gt >> Gc.lnt].done) return;
  const int rx = Gc.rx, ry = Gc.ry, rz = Gc.rz, nxf = Gf.nx, nxyf = Gf.nx * Gf.ny;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    int s, i, j, k, c;
    tile_cell(Gc, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
    if (!(codec[c] & C_SELF)) continue;
    const int fi = rx * i, fj = ry * j, fk = rz * k;
    const int base = (s << Gf.lnc) + (fk * Gf.ny + fj) * nxf + fi;
    T acc = T(0);
#pragma unroll
    for (int q2 = 0; q2 < 8; q2++) {
      const int dx = q2 & 1, dy = (q2 >> 1) & 1, dz = q2 >> 2;
      if (dx >= rx || dy >= ry || dz >= rz || ((fi + fj + fk + dx + dy + dz) & 1)) continue;
      const int cf = base + dx + dy * nxf + dz * nxyf;
      const uint8_t cd = codef[cf];
      if (!(cd & C_SELF)) continue;
      T off, d;
      row_sum(xf, diagf, wf, dgf, cellsf, cf, cd, nxf, nxyf, off, d);
      acc += bf[cf] - (d * xf[cf] - off);
    }
    bc[c] = acc;
  }
}

// Coarsest level (a Galerkin level), one CTA per snapshot, from x = 0: COARSE_SWEEPS (red, black) pairs
// then as many (black, red) pairs (palindromic, so symmetric).
template <typename T>
__global__ void __launch_bounds__(1024) k_mg_coarsest(TG G, const uint8_t* code, const T* w, const T* dg,
                                                       int cells, T* x, const T* b, const Snap* st) {
  pdl_enter();
  __shared__ T sx[512];
  const int s = blockIdx.x;
  if (st[s].done) return;
  const int nx = G.nx, nxy = G.nx * G.ny;
  const int ncell = int(G.nc);  // at most 512
  const int t = threadIdx.x;
  const int c = (s << G.lnc) + t;
  uint8_t cd = 0;
  T bb = T(0), d = T(1), w6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  int par = 0;
  if (t < ncell) {
    cd = code[c];
    d = dg[c];
    bb = b[c];
#pragma unroll
    for (int f = 0; f < 6; f++) w6[f] = w[f * cells + c];
    const int i = t % nx, j = (t / nx) % G.ny, k = t / nxy;
    par = (i + j + k) & 1;
    sx[t] = T(0);
  }
  __syncthreads();
  auto half = [&](int color) {
    T v = T(0);
    const bool act = t < ncell && (cd & C_SELF) && par == color;
    if (act) {
      T a = (cd & 1) ? w6[0] * sx[t - 1] : T(0), b2 = (cd & 2) ? w6[1] * sx[t + 1] : T(0);
      T e = (cd & 4) ? w6[2] * sx[t - nx] : T(0), f = (cd & 8) ? w6[3] * sx[t + nx] : T(0);
      T g = (cd & 16) ? w6[4] * sx[t - nxy] : T(0), h = (cd & 32) ? w6[5] * sx[t + nxy] : T(0);
      v = (bb + (((a + b2) + (e + f)) + (g + h))) / d;
    }
    __syncthreads();
    if (act) sx[t] = v;
    __syncthreads();
  };
  for (int q = 0; q < COARSE_SWEEPS; q++) {
    half(0);
    half(1);
  }
  for (int q = 0; q < COARSE_SWEEPS; q++) {
    half(1);
    half(0);
  }
  if (t < ncell) x[c] = sx[t];
}

// ---------------------------------------------------------------- MIC(0) kernels (plane d = i + j + k)

__device__ __forceinline__ int ilog2_dev(int v) { return 31 - __clz(v); }

// Factor (solver3d.ts:883-900) with a(c, c + e) = -1 iff both cells are unknowns.
template <typename T>
__global__ void k_mic_factor(TG G, const uint8_t* code, const uint8_t* diag, T* pc, int d, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = G.nx;
  if (t >= (count << (G.lny + ilog2_dev(G.nz)))) return;
  const int s = t >> (G.lny + ilog2_dev(G.nz)), j = t & (G.ny - 1), k = (t >> G.lny) & (G.nz - 1);
  const int i = d - j - k;
  if (i < 1 || i > nx - 2 || j < 1 || j > G.ny - 2 || k < 1 || k > G.nz - 2) return;
  const int n = nx, nxy = nx * G.ny;
  const int c = (s << G.lnc) + ((k << G.lny) + j) * nx + i;
  const uint8_t cd = code[c];
  if (!(cd & C_SELF)) return;
  const double tau = 0.97;
  const double ad = double(diag[c]);
  // a(c - e, c) = -1 when both are unknowns, and a neighbour's own +y/+z (etc.) coefficients likewise
  const double a1 = (cd & 1) ? -1.0 : 0.0, a2 = (cd & 4) ? -1.0 : 0.0, a3 = (cd & 16) ? -1.0 : 0.0;
  const double p1 = (cd & 1) ? double(pc[c - 1]) : 0.0, p2 = (cd & 4) ? double(pc[c - n]) : 0.0,
               p3 = (cd & 16) ? double(pc[c - nxy]) : 0.0;
  const uint8_t c1 = (cd & 1) ? code[c - 1] : 0, c2 = (cd & 4) ? code[c - n] : 0, c3 = (cd & 16) ? code[c - nxy] : 0;
  const double aj1 = (c1 & 8) ? -1.0 : 0.0, ak1 = (c1 & 32) ? -1.0 : 0.0;
  const double ai2 = (c2 & 2) ? -1.0 : 0.0, ak2 = (c2 & 32) ? -1.0 : 0.0;
  const double ai3 = (c3 & 2) ? -1.0 : 0.0, aj3 = (c3 & 8) ? -1.0 : 0.0;
  const double q1 = a1 * p1, q2 = a2 * p2, q3 = a3 * p3;
  double e = ad - q1 * q1 - q2 * q2 - q3 * q3 -
             tau * (a1 * (aj1 + ak1) * p1 * p1 + a2 * (ai2 + ak2) * p2 * p2 + a3 * (ai3 + aj3) * p3 * p3);
  if (e < 0.25 * ad) e = ad;
  pc[c] = T(e > 0 ? 1.0 / sqrt(e) : 0.0);
}

// Forward sweep (solver3d.ts:958-965): qv = (r + sum over unknown -x,-y,-z neighbours of pc qv) pc.
template <typename T>
__global__ void k_mic_fwd(TG G, const uint8_t* code, const T* pc, const T* r, T* qv, int d, int count,
                          const Snap* st) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = G.nx;
  if (t >= (count << (G.lny + ilog2_dev(G.nz)))) return;
  const int s = t >> (G.lny + ilog2_dev(G.nz)), j = t & (G.ny - 1), k = (t >> G.lny) & (G.nz - 1);
  const int i = d - j - k;
  if (i < 1 || i > nx - 2 || j < 1 || j > G.ny - 2 || k < 1 || k > G.nz - 2) return;
  if (st[s].done) return;
  const int n = nx, nxy = nx * G.ny;
  const int c = (s << G.lnc) + ((k << G.lny) + j) * nx + i;
  const uint8_t cd = code[c];
  if (!(cd & C_SELF)) return;
  T v = r[c];
  if (cd & 1) v += pc[c - 1] * qv[c - 1];
  if (cd & 4) v += pc[c - n] * qv[c - n];
  if (cd & 16) v += pc[c - nxy] * qv[c - nxy];
  qv[c] = v * pc[c];
}

// Backward sweep (solver3d.ts:966-972): z = (qv + pc * sum over unknown +x,+y,+z neighbours of z) pc.
template <typename T>
__global__ void k_mic_bwd(TG G, const uint8_t* code, const T* pc, const T* qv, T* z, int d, int count,
                          const Snap* st) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = G.nx;
  if (t >= (count << (G.lny + ilog2_dev(G.nz)))) return;
  const int s = t >> (G.lny + ilog2_dev(G.nz)), j = t & (G.ny - 1), k = (t >> G.lny) & (G.nz - 1);
  const int i = d - j - k;
  if (i < 1 || i > nx - 2 || j < 1 || j > G.ny - 2 || k < 1 || k > G.nz - 2) return;
  if (st[s].done) return;
  const int n = nx, nxy = nx * G.ny;
  const int c = (s << G.lnc) + ((k << G.lny) + j) * nx + i;
  const uint8_t cd = code[c];
  if (!(cd & C_SELF)) return;
  const T p = pc[c];
  T v = qv[c];
  if (cd & 2) v += p * z[c + 1];
  if (cd & 8) v += p * z[c + n];
  if (cd & 32) v += p * z[c + nxy];
  z[c] = v * p;
}

// ---------------------------------------------------------------- PCG kernels

// Reduction of a half CTA (128 threads, one tile) into that tile's partial: sum or maximum. Every
// thread of the CTA calls it; out is null for a half without a tile.
__device__ __forceinline__ void half_store(double v, double* out, bool is_max) {
  __shared__ double sw[PT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, y) : v + y;
  }
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if ((threadIdx.x & 127) == 0 && out) {
    const int w0 = (threadIdx.x >> 5);
    double a = sw[w0];
    for (int w = 1; w < 4; w++) a = is_max ? fmax(a, sw[w0 + w]) : a + sw[w0 + w];
    *out = a;
  }
  __syncthreads();
}

// The PCG kernels run two tiles per CTA (a half CTA per tile, two cells per thread) and leave one
// partial per tile.
#define PCG_TILE_PROLOGUE                                   \
  const int ti = blockIdx.x * 2 + (threadIdx.x >> 7);       \
  const bool has = ti < *nact;                              \
  const int gt = has ? list[ti] : 0;                        \
  const int snap = gt >> G.lnt;                             \
  const bool live = has && !st[snap].done;

// r = b, x = 0, p = 0, |b| max per snapshot.
template <typename T>
__global__ void __launch_bounds__(PT) k_pcg_init(TG G, const int* list, const uint8_t* code, const float* b, T* r,
                                                 double* x, T* p, double* part, const Snap* st, const int* nact) {
  PCG_TILE_PROLOGUE
  double v = 0;
  if (has) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int s, i, j, k, c;
      tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
      const bool u = code[c] & C_SELF;
      const double bv = u ? double(b[c]) : 0.0;
      r[c] = T(bv);
      x[c] = 0.0;
      p[c] = T(0);
      v = fmax(v, fabs(bv));
    }
  }
  (void)live;
  half_store(v, has ? &part[gt] : nullptr, true);
}

// Partial z.r per tile.
// Partial z.r per tile; with r_old (flexible CG) also z.r_old into part2.
template <typename T>
__global__ void __launch_bounds__(PT) k_pcg_rz(TG G, const int* list, const uint8_t* code, const T* r, const T* z,
                                               const T* rold, double* part, double* part2, const Snap* st, const int* nact) {
  pdl_enter();
  PCG_TILE_PROLOGUE
  double v = 0, v2 = 0;
  if (live) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int s, i, j, k, c;
      tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
      if (code[c] & C_SELF) {
        v += double(z[c]) * double(r[c]);
        if (rold) v2 += double(z[c]) * double(rold[c]);
      }
    }
  }
  half_store(v, live ? &part[gt] : nullptr, false);
  if (rold) half_store(v2, live ? &part2[gt] : nullptr, false);
}

// Learned preconditioning: z = the network's output zn on the snapshots that still use it.
template <typename T>
__global__ void __launch_bounds__(PT) k_select_pre(TG G, const int* list, const uint8_t* code, const float* zn, T* z,
                                                   const Snap* st, const int* nact) {
  pdl_enter();
  PCG_TILE_PROLOGUE
  if (!live || st[snap].pre) return;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    int s, i, j, k, c;
    tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
    if (code[c] & C_SELF) z[c] = T(zn[c]);
  }
}

// p = z + beta p_old into p_new and A p_new (neighbours' new p formed on the fly from z and p_old, which
// no CTA writes in this launch); partial p.Ap per tile.
template <typename T>
__global__ void __launch_bounds__(PT) k_pcg_pap(TG G, const int* list, const uint8_t* code, const uint8_t* diag,
                                                const T* z, const T* pold, T* pnew, T* ap, double* part,
                                                const Snap* st, const int* nact) {
  pdl_enter();
  PCG_TILE_PROLOGUE
  double v = 0;
  if (live) {
    const T beta = T(st[snap].beta);
    const int n = G.nx, nxy = G.nx * G.ny;
    auto pn = [&](int q) { return z[q] + beta * pold[q]; };
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int s, i, j, k, c;
      tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
      const uint8_t cd = code[c];
      if (!(cd & C_SELF)) continue;
      const T pc = pn(c);
      T a = (cd & 1) ? pn(c - 1) : T(0), b2 = (cd & 2) ? pn(c + 1) : T(0);
      T e = (cd & 4) ? pn(c - n) : T(0), f = (cd & 8) ? pn(c + n) : T(0);
      T g = (cd & 16) ? pn(c - nxy) : T(0), h = (cd & 32) ? pn(c + nxy) : T(0);
      const T apv = T(diag[c]) * pc - (((a + b2) + (e + f)) + (g + h));
      pnew[c] = pc;
      ap[c] = apv;
      v += double(pc) * double(apv);
    }
  }
  half_store(v, live ? &part[gt] : nullptr, false);
}

// x += alpha p, r -= alpha Ap; max |r| per tile.
template <typename T>
__global__ void __launch_bounds__(PT) k_pcg_update(TG G, const int* list, const uint8_t* code, double* x, const T* p,
                                                   T* r, const T* ap, T* rold, double* part, const Snap* st, const int* nact) {
  pdl_enter();
  PCG_TILE_PROLOGUE
  double v = 0;
  if (live) {
    const double a = st[snap].alpha;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int s, i, j, k, c;
      tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
      if (!(code[c] & C_SELF)) continue;
      x[c] += a * double(p[c]);
      if (rold) rold[c] = r[c];
      const T rv = r[c] - T(a) * ap[c];
      r[c] = rv;
      v = fmax(v, fabs(double(rv)));
    }
  }
  half_store(v, live ? &part[gt] : nullptr, true);
}

// FP64 true residual b - A x of the snapshots in their check state; it replaces r.
template <typename T>
__global__ void __launch_bounds__(PT) k_pcg_true(TG G, const int* list, const uint8_t* code, const uint8_t* diag,
                                                 const float* b, const double* x, T* r, double* part,
                                                 const Snap* st, const int* nact) {
  pdl_enter();
  PCG_TILE_PROLOGUE
  const bool chk = live && st[snap].check;
  double v = 0;
  if (chk) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int s, i, j, k, c;
      tile_cell(G, gt, (threadIdx.x & 127) + q * 128, s, i, j, k, c);
      const uint8_t cd = code[c];
      if (!(cd & C_SELF)) continue;
      const double rt = double(b[c]) - (double(diag[c]) * x[c] - nsum(x, c, cd, G.nx, G.nx * G.ny));
      r[c] = T(rt);
      v = fmax(v, fabs(rt));
    }
  }
  half_store(v, chk ? &part[gt] : nullptr, true);
}

// Per-snapshot scalar steps from the per-tile partials (summed or maximised in tile order: inactive
// tiles hold 0). phase 0: after init (max|b|: bnorm, target); 1: after z.r (beta); 2: after p.Ap
// (alpha, breakdown); 3: after the update (max|r|: convergence, check); 4: after a true residual.
__global__ void __launch_bounds__(RED_T) k_pcg_scalar(int phase, const double* part, const double* part2,
                                                      long long ntile, Snap* st, double tol, int max_iter, int learned,
                                                      double first_check) {
  pdl_enter();
  const int s = blockIdx.x;
  Snap& S = st[s];
  __shared__ double sw[RED_T / 32];
  if (phase != 0 && S.done) return;
  if (phase == 4 && !S.check) return;
  const bool is_max = phase == 0 || phase == 3 || phase == 4;
  double a = 0;
  for (long long t = threadIdx.x; t < ntile; t += RED_T) {
    const double v = part[(long long)s * ntile + t];
    a = is_max ? fmax(a, v) : a + v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, a, o);
    a = is_max ? fmax(a, v) : a + v;
  }
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double m = 0;
  for (int w = 0; w < RED_T / 32; w++) m = is_max ? fmax(m, sw[w]) : m + sw[w];
  if (phase == 1) {
    double m2 = 0;  // z . r_old (flexible CG): one thread sums the tile partials in tile order
    if (learned && !S.fresh)
      for (long long t = 0; t < ntile; t++) m2 += part2[(long long)s * ntile + t];
    S.rz_old = S.rz;
    S.rz = m;
    // Polak-Ribiere beta (z.(r - r_old) / z_old.r_old) keeps CG valid for a preconditioner that changes
    // from one iteration to the next (the network is not a fixed symmetric operator)
    S.beta = S.fresh ? 0.0 : (learned ? (m - m2) / S.rz_old : m / S.rz_old);
    S.fresh = 0;
    return;
  }
  if (phase == 2) {
    if (!(m > 0)) {  // breakdown (solver3d.ts:913)
      S.done = 1;
      S.converged = S.res <= S.target ? 1 : 0;
      return;
    }
    S.alpha = S.rz / m;
    return;
  }
  if (phase == 0) {
    S.bnorm = m;
    S.target = fmax(tol * m, 1e-14);
    S.res = m;
    S.it = 0;
    S.fresh = 1;
    S.check = 0;
    S.restarts = 0;
    S.converged = 0;
    S.pre = learned ? 0 : 1;
    S.learned_it = 0;
    for (int q = 0; q < 8; q++) S.hist[q] = m;
    S.done = (m < 1e-14) ? 1 : 0;  // solver3d.ts:901
    if (S.done) S.converged = 1;
    return;
  }
  if (phase == 3) {
    S.it++;
    S.res = m;
    if (S.it <= PL_POISSON_HISTORY) S.rh[S.it - 1] = m;
    if (!S.pre) {
      S.learned_it++;
      const double before = S.hist[(S.it - STALL_SPAN) & 7];
      if ((S.learned_it > STALL_SPAN && m > 0.5 * before) || S.learned_it >= LEARNED_CAP) {
        S.pre = 1;    // the network stalls: multigrid from here on, CG restarted from the true residual
        S.check = 1;
      }
    }
    S.hist[S.it & 7] = m;
    // the first confirmation at first_check times the target (FP32 vectors: the recursive residual
    // keeps falling after the true residual has stalled above the target); the later ones and the
    // acceptance at the target
    if (m <= (S.restarts == 0 ? S.target * first_check : S.target)) {
      S.check = 1;  // confirm with the true residual
    } else if (S.it >= max_iter) {
      S.done = 1;
      S.converged = 0;
    }
    return;
  }
  // phase 4: true residual of a checked snapshot
  S.check = 0;
  if (m <= S.target || S.restarts >= 4) {
    S.res = m;
    S.done = 1;
    S.converged = m <= S.target ? 1 : 0;
    return;
  }
  S.restarts++;
  S.fresh = 1;  // restart CG from the true residual
  if (S.it >= max_iter) {
    S.done = 1;
    S.converged = 0;
  }
}

__global__ void k_snap_result(const Snap* st, double* out) {
  out[0] = st[0].it;
  out[1] = st[0].converged;
  out[2] = st[0].res;
}

// Control of the iteration loop (a graph while-node): another pass while a snapshot is live, and never
// more than `cap` passes (every snapshot stops at its iteration cap well before; the count is a hard
// bound on the loop whatever the state holds).
__global__ void k_loop_next(const Snap* st, int count, int* passes, int cap, cudaGraphConditionalHandle h) {
  pdl_enter();
  int live = 0;
  for (int s = threadIdx.x; s < count; s += blockDim.x)
    if (!st[s].done) live = 1;
  live = __syncthreads_or(live);
  if (threadIdx.x == 0) {
    const int q = ++*passes;
    cudaGraphSetConditional(h, (live && q < cap) ? 1u : 0u);
  }
}

}  // namespace

// ---------------------------------------------------------------- host side

struct PoissonImpl {
  virtual ~PoissonImpl() {}
  UNetImpl* net = nullptr;  // learned preconditioning (PL_POISSON_LEARNED), owned by the caller
  virtual int solve(const uint8_t* cell, const float* b, double* x, double tol, int max_iter, cudaStream_t st,
                    int* iters, double* res, int* conv, char* err, size_t errlen) = 0;
  virtual int capture_setup(const uint8_t* cell, cudaStream_t st, char* err, size_t errlen) = 0;
  virtual int capture_solve(const float* b, double* x, double tol, int max_iter, cudaStream_t st, char* err,
                            size_t errlen) = 0;
  virtual void capture_result(double* out3, cudaStream_t st) = 0;
  size_t bytes = 0;
  std::vector<Snap> last;  // per-snapshot state at the end of the last solve
};

namespace {

template <typename T>
struct PoissonT : PoissonImpl {
  int count, method;
  int nlev = 0;
  Lvl<T> L[PMAXLEV];
  void* mem = nullptr;
  T *r = nullptr, *z = nullptr, *p = nullptr, *p1 = nullptr, *ap = nullptr, *pc = nullptr, *qv = nullptr;
  T* rold = nullptr;     // learned: r of the previous iteration (flexible beta)
  float* zn = nullptr;   // learned: the network's output
  const uint8_t* cell_in = nullptr;
  double *part = nullptr, *part2 = nullptr;
  Snap* st = nullptr;
  int* dcnt = nullptr;  // [PMAXLEV] active tile counters, then the loop's pass counter
  int* passes = nullptr;
  cudaStream_t side = nullptr;  // captures the loop body
  int* chunk = nullptr;  // per-chunk counts / offsets of the list compaction
  int* pinned = nullptr;
  cudaGraphExec_t iter_graph = nullptr;
  // A launch of the iteration loop's body: with programmatic stream serialisation (the kernels begin
  // with pdl_enter) while the body is being recorded, a plain launch otherwise.
  bool in_loop = false;
  template <typename... P, typename... A>
  void lk(void (*k)(P...), unsigned grid, unsigned block, cudaStream_t s, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = in_loop ? at : nullptr;
    cfg.numAttrs = in_loop ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<P>(args)...);
  }
  static unsigned grid2(int nact) { return unsigned(std::max(1, (nact + 1) / 2)); }  // two tiles per CTA
  // Device-driven mode: the active tile counts stay on the device (every launch is sized for all
  // tiles and its CTAs past the count return at once) and the iterations run as a graph while-loop,
  // so a whole solve can be captured into a caller's graph.
  bool devmode = false;
  int lim(int l) const { return devmode ? int(count * L[l].G.ntile) : L[l].nact; }
  bool any(int l) const { return devmode || L[l].nact > 0; }
  const int* nact_d(int l) const { return dcnt + l; }

  ~PoissonT() override {
    if (iter_graph) cudaGraphExecDestroy(iter_graph);
    if (side) cudaStreamDestroy(side);
    if (mem) cudaFree(mem);
    if (pinned) cudaFreeHost(pinned);
  }

  bool learned() const { return method == PL_POISSON_LEARNED; }

  // last MIC(0) plane: i + j + k of the far interior corner
  int dmax() const { return (L[0].G.nx - 2) + (L[0].G.ny - 2) + (L[0].G.nz - 2); }

  int init(int nx, int ny, int nz, int count_, int method_, char* err, size_t errlen) {
    count = count_, method = method_;
    // levels: halve every axis longer than 8 until none is (semi-coarsening keeps thin boxes going)
    int ex[3] = {nx, ny, nz}, rf[3] = {1, 1, 1};
    while (nlev < PMAXLEV) {
      L[nlev].G = make_tg(ex[0], ex[1], ex[2], rf[0], rf[1], rf[2]);
      nlev++;
      if (method == PL_POISSON_MIC0 || (ex[0] <= 8 && ex[1] <= 8 && ex[2] <= 8)) break;
      for (int a = 0; a < 3; a++) {
        rf[a] = ex[a] > 8 ? 2 : 1;
        ex[a] /= rf[a];
      }
    }
    std::vector<size_t> sizes;
    auto add = [&](size_t b) {
      sizes.push_back((b + 255) & ~size_t(255));
      return sizes.size() - 1;
    };
    const size_t C0 = size_t(count) * L[0].G.nc;
    size_t i_code[PMAXLEV], i_diag[PMAXLEV], i_flag[PMAXLEV], i_list[PMAXLEV], i_x[PMAXLEV], i_b[PMAXLEV],
        i_w[PMAXLEV], i_dg[PMAXLEV];
    for (int l = 0; l < nlev; l++) {
      const size_t cl = size_t(count) * L[l].G.nc, tl = size_t(count) * L[l].G.ntile;
      i_code[l] = add(cl);
      i_diag[l] = l == 0 ? add(cl) : 0;
      i_flag[l] = add(tl);
      i_list[l] = add(tl * 4);
      i_x[l] = l > 0 ? add(cl * sizeof(T)) : 0;
      i_b[l] = l > 0 ? add(cl * sizeof(T)) : 0;
      i_w[l] = l > 0 ? add(6 * cl * sizeof(T)) : 0;
      i_dg[l] = l > 0 ? add(cl * sizeof(T)) : 0;
    }
    const size_t i_r = add(C0 * sizeof(T)), i_z = add(C0 * sizeof(T)), i_p = add(C0 * sizeof(T)),
                 i_p1 = add(C0 * sizeof(T)), i_ap = add(C0 * sizeof(T));
    const size_t i_pc = method == PL_POISSON_MIC0 ? add(C0 * sizeof(T)) : 0;
    const size_t i_qv = method == PL_POISSON_MIC0 ? add(C0 * sizeof(T)) : 0;
    const size_t i_part = add(size_t(count) * L[0].G.ntile * 8);
    const size_t i_part2 = add(size_t(count) * L[0].G.ntile * 8);
    const size_t i_rold = learned() ? add(C0 * sizeof(T)) : 0;
    const size_t i_zn = learned() ? add(C0 * 4) : 0;
    const size_t i_st = add(size_t(count) * sizeof(Snap));
    const size_t i_cnt = add(2 * PMAXLEV * 4);
    const size_t i_chunk = add(size_t((size_t(count) * L[0].G.ntile + CHUNK - 1) / CHUNK) * 4);
    size_t total = 0;
    for (size_t s : sizes) total += s;
    cudaError_t e = cudaMalloc(&mem, total);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "pl_poisson_create: cudaMalloc(%zu): %s", total, cudaGetErrorString(e));
      mem = nullptr;
      return PL_E_NOMEM;
    }
    bytes = total;
    std::vector<char*> at(sizes.size());
    char* q = static_cast<char*>(mem);
    for (size_t s = 0; s < sizes.size(); s++) {
      at[s] = q;
      q += sizes[s];
    }
    for (int l = 0; l < nlev; l++) {
      L[l].code = (uint8_t*)at[i_code[l]];
      L[l].diag = l == 0 ? (uint8_t*)at[i_diag[l]] : nullptr;
      L[l].flag = (uint8_t*)at[i_flag[l]];
      L[l].list = (int*)at[i_list[l]];
      L[l].x = l > 0 ? (T*)at[i_x[l]] : nullptr;
      L[l].b = l > 0 ? (T*)at[i_b[l]] : nullptr;
      L[l].w = l > 0 ? (T*)at[i_w[l]] : nullptr;
      L[l].dg = l > 0 ? (T*)at[i_dg[l]] : nullptr;
    }
    r = (T*)at[i_r], z = (T*)at[i_z], p = (T*)at[i_p], p1 = (T*)at[i_p1], ap = (T*)at[i_ap];
    pc = method == PL_POISSON_MIC0 ? (T*)at[i_pc] : nullptr;
    qv = method == PL_POISSON_MIC0 ? (T*)at[i_qv] : nullptr;
    part = (double*)at[i_part];
    part2 = (double*)at[i_part2];
    rold = learned() ? (T*)at[i_rold] : nullptr;
    zn = learned() ? (float*)at[i_zn] : nullptr;
    st = (Snap*)at[i_st];
    dcnt = (int*)at[i_cnt];
    passes = dcnt + PMAXLEV;
    chunk = (int*)at[i_chunk];
    e = cudaMemset(mem, 0, total);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&pinned, 4 * (PMAXLEV + 1), cudaHostAllocDefault);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "pl_poisson_create: %s", cudaGetErrorString(e));
      return PL_E_CUDA;
    }
    return PL_OK;
  }

  // Level types, codes, Galerkin operators and active tile lists (counts left on the device).
  void build_levels(const uint8_t* cell, cudaStream_t s0) {
    for (int l = 0; l < nlev; l++) {
      const TG& G = L[l].G;
      const long long nt = (long long)count * G.ntile;
      if (l == 0)
        k_lvl_code<<<unsigned(nt), PT, 0, s0>>>(G, cell, L[0].code, L[0].diag, L[0].flag, count);
      else
        k_gal_coarsen<T><<<unsigned(nt), PT, 0, s0>>>(L[l - 1].G, G, L[l - 1].code, L[l - 1].diag, L[l - 1].w,
                                                      L[l - 1].dg, L[l].code, L[l].w, L[l].dg, L[l].flag, count);
    }
    cudaMemsetAsync(dcnt, 0, 2 * PMAXLEV * 4, s0);
    for (int l = 0; l < nlev; l++) {
      const long long nt = (long long)count * L[l].G.ntile;
      const int nchunk = int((nt + CHUNK - 1) / CHUNK);
      k_compact_count<<<nchunk, CHUNK, 0, s0>>>(L[l].flag, nt, chunk);
      k_compact_scan<<<1, CHUNK, 0, s0>>>(chunk, nchunk, dcnt + l);
      k_compact_write<<<nchunk, CHUNK, 0, s0>>>(L[l].flag, nt, chunk, L[l].list);
    }
  }

  // Host-driven set-up: the levels, their active tile counts read back, the MIC(0) factor.
  int setup(const uint8_t* cell, cudaStream_t s0) {
    build_levels(cell, s0);
    cudaMemcpyAsync(pinned, dcnt, 4 * PMAXLEV, cudaMemcpyDeviceToHost, s0);
    cudaError_t e = cudaStreamSynchronize(s0);
    if (e != cudaSuccess) return PL_E_CUDA;
    for (int l = 0; l < nlev; l++) L[l].nact = pinned[l];
    if (method == PL_POISSON_MIC0) {
      const TG& G = L[0].G;
      const long long thr = (long long)count * G.ny * G.nz;
      const unsigned blocks = unsigned((thr + 255) / 256);
      cudaMemsetAsync(pc, 0, size_t(count) * G.nc * sizeof(T), s0);
      for (int d = 3; d <= dmax(); d++) k_mic_factor<T><<<blocks, 256, 0, s0>>>(G, L[0].code, L[0].diag, pc, d, count);
    }
    return cudaGetLastError() == cudaSuccess ? PL_OK : PL_E_CUDA;
  }

  // z = M r (learned: the network's z on the snapshots that have not fallen back to multigrid)
  void precondition(cudaStream_t s0) {
    mg_or_mic0(s0);
    if (!learned()) return;
    char err[128];
    const TG& G = L[0].G;
    unet_apply(net, cell_in, reinterpret_cast<const float*>(r), zn, G.nx, G.ny, G.nz, count, s0, err, sizeof err);
    lk(k_select_pre<T>, grid2(lim(0)), PT, s0, G, L[0].list, L[0].code, zn, z, st, nact_d(0));
    // the network's correction, then red-black Gauss-Seidel sweeps from it: the network carries the
    // smooth part of the error, the sweeps the rough part (on a fallen-back snapshot they follow the
    // V-cycle's own post-smoothing)
    for (int q = 0; q < MG_NU; q++)
      for (int color = 0; color < 2; color++)
        lk(k_mg_smooth<T, 0>, grid2(lim(0)), PT, s0, G, L[0].list, L[0].code, L[0].diag, L[0].w, L[0].dg,
                                                        int(count * G.nc), z, r, color, 0, st, nact_d(0),
                                                        (const T*)nullptr, (const uint8_t*)nullptr, G);
  }

  void mg_or_mic0(cudaStream_t s0) {
    if (method == PL_POISSON_MIC0) {
      const TG& G = L[0].G;
      const long long thr = (long long)count * G.ny * G.nz;
      const unsigned blocks = unsigned((thr + 255) / 256);
      for (int d = 3; d <= dmax(); d++) k_mic_fwd<T><<<blocks, 256, 0, s0>>>(G, L[0].code, pc, r, qv, d, count, st);
      for (int d = dmax(); d >= 3; d--) k_mic_bwd<T><<<blocks, 256, 0, s0>>>(G, L[0].code, pc, qv, z, d, count, st);
      return;
    }
    auto X = [&](int l) { return l == 0 ? z : L[l].x; };
    auto B = [&](int l) -> const T* { return l == 0 ? r : L[l].b; };
    auto cells = [&](int l) { return (long long)count * L[l].G.nc; };
    // with_coarse: the neighbours read with level l + 1's correction applied (the first post-smoothing
    // half-sweep, in place of a prolongation pass); from_zero: the neighbours read as a first
    // half-sweep from x = 0 leaves them (the second pre-smoothing half-sweep, in place of the first)
    auto smooth = [&](int l, int color, int first, bool with_coarse = false, bool from_zero = false) {
      auto kern = with_coarse ? k_mg_smooth<T, 1> : from_zero ? k_mg_smooth<T, 2> : k_mg_smooth<T, 0>;
      lk(kern, grid2(lim(l)), PT, s0, L[l].G, L[l].list, L[l].code, L[l].diag, L[l].w, L[l].dg, cells(l), X(l),
         B(l), color, first, st, nact_d(l), with_coarse ? (const T*)L[l + 1].x : (const T*)nullptr,
         with_coarse ? (const uint8_t*)L[l + 1].code : (const uint8_t*)nullptr, with_coarse ? L[l + 1].G : L[l].G);
    };
    const int top = nlev - 1;
    static_assert(MG_NU >= 2, "the first pre-smoothing half-sweep is read on the fly by the second");
    for (int l = 0; l < top; l++) {
      if (!any(l)) continue;
      for (int q = 0; q < MG_NU; q++) {
        if (q > 0) smooth(l, 0, 0);
        smooth(l, 1, 0, false, q == 0);  // q == 0: colour 0 from x = 0, read on the fly
      }
      if (any(l + 1))
        lk(k_mg_restrict<T>, grid2(lim(l + 1)), PT, s0, L[l].G, L[l + 1].G, L[l + 1].list, L[l].code, L[l].diag,
                                                          L[l].w, L[l].dg, cells(l), X(l), B(l), L[l + 1].code,
                                                          L[l + 1].b, st, nact_d(l + 1));
    }
    if (any(top)) {
      if (top == 0 || L[top].G.nc > 512) {  // no level small enough for one CTA: plain red-black sweeps
        for (int q = 0; q < COARSE_SWEEPS; q++) {
          smooth(top, 0, q == 0);
          smooth(top, 1, 0);
        }
        for (int q = 0; q < COARSE_SWEEPS; q++) {
          smooth(top, 1, 0);
          smooth(top, 0, 0);
        }
      } else {
        lk(k_mg_coarsest<T>, count, 512, s0, L[top].G, L[top].code, L[top].w, L[top].dg, cells(top), X(top), B(top),
                                               st);
      }
    }
    for (int l = top - 1; l >= 0; l--) {
      if (!any(l)) continue;
      for (int q = 0; q < MG_NU; q++) {
        smooth(l, 1, 0, q == 0 && any(l + 1));  // q == 0: the coarse correction read on the fly
        smooth(l, 0, 0);
      }
    }
  }

  // Multiple of the target at which an FP32-vector solve first confirms with the FP64 true residual.
  double first_check() const { return sizeof(T) == 4 && !learned() ? POISSON_FIRST_CHECK : 1.0; }

  // One PCG iteration for every live snapshot (the loop body of solver3d.ts:912-935, with the
  // preconditioner first: z = M r, beta, p and Ap, alpha, update, convergence / true residual).
  void iteration(const float* b, double* x, double tol, int max_iter, T* pold, T* pnew, cudaStream_t s0) {
    const TG& G = L[0].G;
    const unsigned g0 = grid2(lim(0));
    const int* na = nact_d(0);
    precondition(s0);
    lk(k_pcg_rz<T>, g0, PT, s0, G, L[0].list, L[0].code, r, z, rold, part, part2, st, na);
    lk(k_pcg_scalar, count, RED_T, s0, 1, part, part2, G.ntile, st, tol, max_iter, learned(), first_check());
    lk(k_pcg_pap<T>, g0, PT, s0, G, L[0].list, L[0].code, L[0].diag, z, pold, pnew, ap, part, st, na);
    lk(k_pcg_scalar, count, RED_T, s0, 2, part, part2, G.ntile, st, tol, max_iter, learned(), first_check());
    lk(k_pcg_update<T>, g0, PT, s0, G, L[0].list, L[0].code, x, pnew, r, ap, rold, part, st, na);
    lk(k_pcg_scalar, count, RED_T, s0, 3, part, part2, G.ntile, st, tol, max_iter, learned(), first_check());
    lk(k_pcg_true<T>, g0, PT, s0, G, L[0].list, L[0].code, L[0].diag, b, x, r, part, st, na);
    lk(k_pcg_scalar, count, RED_T, s0, 4, part, part2, G.ntile, st, tol, max_iter, learned(), first_check());
  }

  // r = b, x = 0, p = p1 = 0 and the per-snapshot state (enqueued on s0, capturable).
  void start(const float* b, double* x, double tol, int max_iter, cudaStream_t s0) {
    const TG& G = L[0].G;
    // inactive tiles' partials stay 0 (tiles active in an earlier solve on other cells are not rewritten)
    cudaMemsetAsync(part, 0, size_t(count) * G.ntile * 8, s0);
    if (learned()) cudaMemsetAsync(part2, 0, size_t(count) * G.ntile * 8, s0);
    cudaMemsetAsync(x, 0, size_t(count) * G.nc * 8, s0);
    cudaMemsetAsync(p1, 0, size_t(count) * G.nc * sizeof(T), s0);
    if (learned()) cudaMemsetAsync(rold, 0, size_t(count) * G.nc * sizeof(T), s0);
    cudaMemsetAsync(passes, 0, 4, s0);
    if (any(0)) k_pcg_init<T><<<grid2(lim(0)), PT, 0, s0>>>(G, L[0].list, L[0].code, b, r, x, p, part, st, nact_d(0));
    k_pcg_scalar<<<count, RED_T, 0, s0>>>(0, part, part2, G.ntile, st, tol, max_iter, learned(), first_check());
  }

  // The iterations as a while-node of the graph being captured on s0: its body (two iterations, the
  // search direction alternating between p and p1, then the loop control) is captured on a private
  // stream into the node's body graph.
  int record_loop(const float* b, double* x, double tol, int max_iter, cudaStream_t s0, char* err, size_t errlen) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s0, &cs, nullptr, &cg, &deps, &nd);
    if (e == cudaSuccess && cs != cudaStreamCaptureStatusActive) e = cudaErrorStreamCaptureUnmatched;
    cudaGraphConditionalHandle h{};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, cg, deps, nd, &np);
    if (e == cudaSuccess && !side) e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      cudaGraph_t body = np.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
      if (e == cudaSuccess) {
        in_loop = true;
        iteration(b, x, tol, max_iter, p, p1, side);
        iteration(b, x, tol, max_iter, p1, p, side);
        lk(k_loop_next, 1, 256, side, st, count, passes, max_iter / 2 + 8, h);
        in_loop = false;
        e = cudaStreamEndCapture(side, &body);
      }
    }
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s0, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "pl_poisson: iteration loop: %s", cudaGetErrorString(e));
      return PL_E_CUDA;
    }
    return PL_OK;
  }

  // Device-driven use inside a caller's capture on s0: the levels of `cell` (once per cell layout),
  // then any number of solves on it. No host synchronisation; results stay in the snapshot state.
  int capture_setup(const uint8_t* cell, cudaStream_t s0, char* err, size_t errlen) override {
    if (method == PL_POISSON_MIC0) {
      snprintf(err, errlen, "pl_poisson: the device-driven solve is multigrid or learned");
      return PL_E_ARG;
    }
    devmode = true;
    cell_in = cell;
    build_levels(cell, s0);
    return PL_OK;
  }
  int capture_solve(const float* b, double* x, double tol, int max_iter, cudaStream_t s0, char* err,
                    size_t errlen) override {
    if (learned() && !net) {
      snprintf(err, errlen, "pl_poisson: the learned method needs a network");
      return PL_E_STATE;
    }
    start(b, x, tol, max_iter, s0);
    return record_loop(b, x, tol, max_iter, s0, err, errlen);
  }
  // The first snapshot's outcome (iterations, converged, max-norm residual) to device memory.
  void capture_result(double* out3, cudaStream_t s0) override { k_snap_result<<<1, 1, 0, s0>>>(st, out3); }

  struct SolveKey {
    const void *cell, *b, *x;
    double tol;
    int max_iter;
    int nact[PMAXLEV];
    bool operator==(const SolveKey& o) const {
      if (cell != o.cell || b != o.b || x != o.x || tol != o.tol || max_iter != o.max_iter) return false;
      for (int l = 0; l < PMAXLEV; l++)
        if (nact[l] != o.nact[l]) return false;
      return true;
    }
  };
  SolveKey cached{};

  int record_solve(const float* b, double* x, double tol, int max_iter, char* err, size_t errlen) {
    if (iter_graph) {
      cudaGraphExecDestroy(iter_graph);
      iter_graph = nullptr;
    }
    int rc = PL_OK;
    cudaGraph_t gph = nullptr;
    cudaStream_t cap = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      start(b, x, tol, max_iter, cap);
      rc = any(0) ? record_loop(b, x, tol, max_iter, cap, err, errlen) : PL_OK;
      e = cudaStreamEndCapture(cap, &gph);
      if (rc) e = cudaErrorUnknown;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&iter_graph, gph, 0);
    if (gph) cudaGraphDestroy(gph);
    if (cap) cudaStreamDestroy(cap);
    if (e != cudaSuccess) {
      if (iter_graph) cudaGraphExecDestroy(iter_graph);
      iter_graph = nullptr;
      if (!rc) snprintf(err, errlen, "pl_poisson_solve: solve graph: %s", cudaGetErrorString(e));
      return rc ? rc : PL_E_CUDA;
    }
    return PL_OK;
  }

  int solve(const uint8_t* cell, const float* b, double* x, double tol, int max_iter, cudaStream_t s0, int* iters,
            double* res, int* conv, char* err, size_t errlen) override {
    devmode = false;
    int rc = setup(cell, s0);
    if (rc) {
      snprintf(err, errlen, "pl_poisson_solve: set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
      return rc;
    }
    cell_in = cell;
    if (learned()) {
      if (!net) {
        snprintf(err, errlen, "pl_poisson_solve: the learned method needs a network (pl_poisson_set_unet)");
        return PL_E_STATE;
      }
      rc = unet_prepare(net, L[0].G.nx, L[0].G.ny, L[0].G.nz, count, err, errlen);  // before the capture
      if (rc) return rc;
    }
    // the whole solve as one graph (start, then the iteration loop), launched once; the instantiated
    // graph is kept for the next solve with the same buffers, rule and active-tile counts (the learned
    // method re-records: its network's workspace may move between solves)
    SolveKey key{cell, b, x, tol, max_iter, {}};
    for (int l = 0; l < nlev; l++) key.nact[l] = L[l].nact;
    cudaError_t e = cudaSuccess;
    if (!(iter_graph && !learned() && key == cached)) {
      rc = record_solve(b, x, tol, max_iter, err, errlen);
      if (rc) return rc;
      cached = key;
    }
    e = cudaGraphLaunch(iter_graph, s0);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "pl_poisson_solve: %s", cudaGetErrorString(e));
      return PL_E_CUDA;
    }
    std::vector<Snap> hs(count);
    e = cudaMemcpyAsync(hs.data(), st, sizeof(Snap) * count, cudaMemcpyDeviceToHost, s0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s0);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "pl_poisson_solve: %s", cudaGetErrorString(e));
      return PL_E_CUDA;
    }
    for (int s = 0; s < count; s++) {
      if (iters) iters[s] = hs[s].it;
      if (res) res[s] = hs[s].res;
      if (conv) conv[s] = hs[s].converged;
    }
    last = std::move(hs);
    return PL_OK;
  }
};

}  // namespace

// ---------------------------------------------------------------- workload generator (host)

namespace {

struct Mulberry {  // src/sim/rng.ts:5-14
  uint32_t a;
  double next() {
    a = a + 0x6d2b79f5u;
    uint32_t t = a;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return double(t ^ (t >> 14)) / 4294967296.0;
  }
};

// Counter-based uniform in (0, 1) (SplitMix64 finaliser of a key).
inline double uhash(uint64_t key) {
  uint64_t z = key + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double(z >> 11) + 0.5) / 9007199254740992.0;
}

}  // namespace

int gauge_fix_one(int n, uint8_t* cell, float* bout);

namespace {

void generate_one(int n, int snapshot, uint8_t* cell, float* bout) {
  const double sc = n / 128.0;
  const double R = 60.0 * sc, c0 = n / 2.0;
  const int slab = std::max(2, int(16 * sc));
  Mulberry rng{uint32_t(1000 + snapshot)};
  const int nsph = 1 + int(rng.next() * 8);
  double sph[8][4];
  for (int q = 0; q < nsph; q++) {
    const double rad = (6.0 + 18.0 * rng.next()) * sc;
    double cx, cz;
    do {
      cx = c0 + (2 * rng.next() - 1) * R;
      cz = c0 + (2 * rng.next() - 1) * R;
    } while ((cx - c0) * (cx - c0) + (cz - c0) * (cz - c0) > R * R);
    const double cy = slab + rng.next() * (n - 2.0 * slab);
    sph[q][0] = cx, sph[q][1] = cy, sph[q][2] = cz, sph[q][3] = rad;
  }
  const size_t nc = size_t(n) * n * n;
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) {
        const size_t c = (size_t(k) * n + j) * n + i;
        const double x = i + 0.5, y = j + 0.5, z = k + 0.5;
        uint8_t t;
        if (i == 0 || j == 0 || k == 0 || i == n - 1 || j == n - 1 || k == n - 1 ||
            (x - c0) * (x - c0) + (z - c0) * (z - c0) > R * R) {
          t = SOLID;
        } else {
          bool liq = j < slab;
          for (int q = 0; q < nsph && !liq; q++) {
            const double dx = x - sph[q][0], dy = y - sph[q][1], dz = z - sph[q][2];
            liq = dx * dx + dy * dy + dz * dz <= sph[q][3] * sph[q][3];
          }
          t = liq ? FLUID : AIR;
        }
        cell[c] = t;
      }
  if (!bout) return;  // the mask alone (its unknowns give the snapshot's cost for sharding)
  // Gaussian random face velocities: white noise smoothed by a separable Gaussian of standard
  // deviation 8 cells (at n = 128; scaled with n), unit variance; rhs = -div on the unknowns.
  const double sig = 8.0 * sc;
  const int rad = int(std::ceil(3 * sig));
  std::vector<double> w(2 * rad + 1);
  double w2 = 0;
  for (int q = -rad; q <= rad; q++) {
    w[q + rad] = std::exp(-double(q) * q / (2 * sig * sig));
    w2 += w[q + rad] * w[q + rad];
  }
  for (double& v : w) v /= std::sqrt(w2);  // unit variance per axis, so unit variance in 3D
  std::vector<float> div(nc, 0.f);
  for (int comp = 0; comp < 3; comp++) {
    const int sx = n + (comp == 0), sy = n + (comp == 1), sz = n + (comp == 2);
    const size_t nf = size_t(sx) * sy * sz;
    std::vector<float> f(nf), g(nf);
    for (size_t q = 0; q < nf; q++) {  // Box-Muller on two counter-based uniforms
      const uint64_t key = (uint64_t(uint32_t(snapshot)) << 40) ^ (uint64_t(comp) << 36) ^ (uint64_t(q) << 1);
      const double u1 = uhash(key), u2 = uhash(key | 1ull);
      f[q] = float(std::sqrt(-2.0 * std::log(u1)) * std::cos(2 * PI * u2));
    }
    auto pass = [&](const std::vector<float>& in, std::vector<float>& out, int axis) {
      const int ext[3] = {sx, sy, sz};
      const size_t stride[3] = {1, size_t(sx), size_t(sx) * sy};
      for (int k = 0; k < sz; k++)
        for (int j = 0; j < sy; j++)
          for (int i = 0; i < sx; i++) {
            const int pos[3] = {i, j, k};
            const size_t c = (size_t(k) * sy + j) * sx + i;
            double acc = 0;
            for (int q = -rad; q <= rad; q++) {
              int p = pos[axis] + q;
              p = p < 0 ? -p - 1 : p >= ext[axis] ? 2 * ext[axis] - p - 1 : p;  // mirror at the edges
              if (p < 0 || p >= ext[axis]) continue;
              acc += w[q + rad] * in[c + (long long)(p - pos[axis]) * (long long)stride[axis]];
            }
            out[c] = float(acc);
          }
    };
    pass(f, g, 0);
    pass(g, f, 1);
    pass(f, g, 2);
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
          const size_t c = (size_t(k) * n + j) * n + i;
          const size_t f0 = (size_t(k) * sy + j) * sx + i;
          const size_t f1 = f0 + (comp == 0 ? 1 : comp == 1 ? size_t(sx) : size_t(sx) * sy);
          div[c] += g[f1] - g[f0];
        }
  }
  // rhs on the unknowns, then the gauge fix
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) {
        const size_t c = (size_t(k) * n + j) * n + i;
        const bool unknown = cell[c] == FLUID && i > 0 && j > 0 && k > 0 && i < n - 1 && j < n - 1 && k < n - 1;
        bout[c] = unknown ? -div[c] : 0.f;
      }
  gauge_fix_one(n, cell, bout);
}

}  // namespace

// Gauge fix of one snapshot (src/sim/pressure.ts:232-268): every 6-connected component of unknowns
// without an AIR neighbour (a border FLUID cell counts as AIR: it is Dirichlet) has its rhs mean
// removed (FP64 sum in breadth-first order from its first cell in index order) and that first cell
// pinned. Returns the number of such components.
int gauge_fix_one(int n, uint8_t* cell, float* bout) {
  const size_t nc = size_t(n) * n * n;
  auto unknown = [&](size_t c, int i, int j, int k) {
    return (cell[c] & 3) == FLUID && i > 0 && j > 0 && k > 0 && i < n - 1 && j < n - 1 && k < n - 1;
  };
  std::vector<double> b(nc);
  for (size_t c = 0; c < nc; c++) b[c] = double(bout[c]);
  std::vector<int32_t> comp(nc, -1);
  std::vector<size_t> queue;
  queue.reserve(nc / 4);
  int label = 0, enclosed = 0;
  const long long offs[6] = {-1, 1, -(long long)n, (long long)n, -(long long)n * n, (long long)n * n};
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) {
        const size_t seed = (size_t(k) * n + j) * n + i;
        if (!unknown(seed, i, j, k) || comp[seed] >= 0) continue;
        queue.clear();
        queue.push_back(seed);
        comp[seed] = label;
        bool air = false;
        double sum = 0;
        for (size_t h = 0; h < queue.size(); h++) {
          const size_t c = queue[h];
          sum += b[c];
          const int ci = int(c % n), cj = int((c / n) % n), ck = int(c / (size_t(n) * n));
          for (int f = 0; f < 6; f++) {
            const size_t d = size_t((long long)c + offs[f]);
            const int di = ci + (f == 0 ? -1 : f == 1 ? 1 : 0), dj = cj + (f == 2 ? -1 : f == 3 ? 1 : 0),
                      dk = ck + (f == 4 ? -1 : f == 5 ? 1 : 0);
            if ((cell[d] & 3) == AIR || ((cell[d] & 3) == FLUID && !unknown(d, di, dj, dk))) air = true;
            else if (unknown(d, di, dj, dk) && comp[d] < 0) {
              comp[d] = label;
              queue.push_back(d);
            }
          }
        }
        if (!air) {
          const double mean = sum / double(queue.size());
          for (size_t c : queue) b[c] -= mean;
          cell[seed] |= PL_POISSON_PIN;
          enclosed++;
          for (size_t c : queue) bout[c] = float(b[c]);
        }
        label++;
      }
  return enclosed;
}

int poisson_generate(int n, int first, int count, uint8_t* cell, float* b, int threads) {
  const size_t nc = size_t(n) * n * n;
  if (threads < 1) threads = int(std::max(1u, std::thread::hardware_concurrency()));
  threads = std::min(threads, count);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++)
    pool.emplace_back([=]() {
      for (int s = t; s < count; s += threads)
        generate_one(n, first + s, cell + size_t(s) * nc, b ? b + size_t(s) * nc : nullptr);
    });
  for (auto& th : pool) th.join();
  return PL_OK;
}

PoissonImpl* poisson_create(int nx, int ny, int nz, int count, int method, int precision, char* err, size_t errlen,
                            int* rc) {
  PoissonImpl* h = nullptr;
  if (method == PL_POISSON_LEARNED && precision != PL_SOLVE_MIXED) {
    snprintf(err, errlen, "pl_poisson_create: the learned method runs with FP32 vectors (PL_SOLVE_MIXED)");
    *rc = PL_E_ARG;
    return nullptr;
  }
  if (precision == PL_SOLVE_F64) {
    auto* q = new PoissonT<double>();
    *rc = q->init(nx, ny, nz, count, method, err, errlen);
    h = q;
  } else {
    auto* q = new PoissonT<float>();
    *rc = q->init(nx, ny, nz, count, method, err, errlen);
    h = q;
  }
  if (*rc) {
    delete h;
    return nullptr;
  }
  return h;
}

int poisson_solve(PoissonImpl* h, const uint8_t* cell, const float* b, double* x, double tol, int max_iter,
                  cudaStream_t st, int* iters, double* res, int* conv, char* err, size_t errlen) {
  return h->solve(cell, b, x, tol, max_iter, st, iters, res, conv, err, errlen);
}

void poisson_destroy(PoissonImpl* h) { delete h; }

void poisson_set_unet(PoissonImpl* h, UNetImpl* u) { h->net = u; }

size_t poisson_bytes(const PoissonImpl* h) { return h ? h->bytes : 0; }

int poisson_capture_setup(PoissonImpl* h, const uint8_t* cell, cudaStream_t st, char* err, size_t errlen) {
  return h->capture_setup(cell, st, err, errlen);
}

int poisson_capture_solve(PoissonImpl* h, const float* b, double* x, double tol, int max_iter, cudaStream_t st,
                          char* err, size_t errlen) {
  return h->capture_solve(b, x, tol, max_iter, st, err, errlen);
}

void poisson_capture_result(PoissonImpl* h, double* out3, cudaStream_t st) { h->capture_result(out3, st); }

int poisson_history(const PoissonImpl* h, int snapshot, double* out, int capacity, int* recorded, int* learned_it) {
  if (snapshot < 0 || snapshot >= (int)h->last.size()) return PL_E_ARG;
  const Snap& S = h->last[snapshot];
  const int n = std::min(S.it, PL_POISSON_HISTORY);
  for (int k = 0; k < std::min(n, capacity); k++) out[k] = S.rh[k];
  if (recorded) *recorded = n;
  if (learned_it) *learned_it = S.learned_it;
  return PL_OK;
}

}  // namespace pl
