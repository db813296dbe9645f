// Multigrid-preconditioned CG for the pressure and density-correction solves, on one thread-block
// cluster of 16 CTAs (one per SM) with every solver vector in distributed shared memory.
//
// Why this shape: one substep's liquid system has 5k-15k unknowns, and a PCG iteration is a chain
// of ~14 dependent stencil phases. On one SM a 7-point phase over 11k cells is shared-memory
// bandwidth bound at ~2 us, and through L2 each dependent step costs ~0.5-1 us; a 16-CTA cluster
// spreads each phase over 16 SMs and synchronises with a hardware cluster barrier (~0.2-0.3 us),
// reading neighbour values across CTAs through DSMEM.
//
// Preconditioner: one V-cycle of geometric multigrid (the 3D form of src/sim/multigrid.ts: the same
// operator on every level, AIR neighbours Dirichlet and SOLID neighbours excluded, coarse type AIR if
// any child is AIR else FLUID if any child is FLUID, piecewise-constant prolongation). The smoother
// is red-black Gauss-Seidel: red then black before the coarse correction, black then red after it,
// and a palindromic sweep sequence on the coarsest level, so the V-cycle is a symmetric operator and
// CG stays valid. Restriction sums the children's residuals times 1/2 (the 3D counterpart of the
// 2D "sum = 4 x average": the coarse operator scales with the squared cell size). Because the last
// pre-smoothing half-sweep is black, black residuals are zero and only red children are restricted;
// prolongation is folded into the first post-smoothing half-sweep (black cells read their red
// neighbours plus the neighbours' coarse corrections), and the first pre-smoothing half-sweep from
// x = 0 is folded into the phase that produces the level's right-hand side.
//
// Stopping rule and bookkeeping are the reference's (solver3d.ts:858-937): max-norm residual
// <= max(tol * max|b|, 1e-14), breakdown if s.As <= 0. In FP32 mode (PL_SOLVE_MIXED) the vectors
// are FP32, inner products and the solution FP64, and a recursive-residual convergence is
// confirmed by the FP64 true residual b - A q; if that misses the target, CG restarts from it
// (iterative refinement).
#include <cooperative_groups.h>

#include <cstdio>

#include "mg.h"

namespace cg = cooperative_groups;

namespace pl {

// ---------------------------------------------------------------- workspace

static void mg_dims(const Geo& g, int dims[MG_MAX_LEVELS][3], int* nlev) {
  dims[0][0] = g.nx, dims[0][1] = g.ny, dims[0][2] = g.nz;
  int L = 1;
  while (L < MG_MAX_LEVELS) {
    int nx = (dims[L - 1][0] + 1) / 2, ny = (dims[L - 1][1] + 1) / 2, nz = (dims[L - 1][2] + 1) / 2;
    if (nx < 3 || ny < 3 || nz < 3) break;
    dims[L][0] = nx, dims[L][1] = ny, dims[L][2] = nz;
    L++;
  }
  *nlev = L;
}

static size_t al(size_t b) { return (b + 255) & ~size_t(255); }

size_t mg_ws_bytes(const Geo& g, int* nlev_out) {
  int dims[MG_MAX_LEVELS][3], nlev;
  mg_dims(g, dims, &nlev);
  size_t tot = al(MG_MAX_LEVELS * 4);
  for (int L = 0; L < nlev; L++) {
    size_t c = size_t(dims[L][0]) * dims[L][1] * dims[L][2];
    if (L > 0) tot += al(c) + al(c * 4) * 2 + al(c * 24) + al(c * 32);  // type, lidx, list, nb, child
    tot += al(c * 24) + al(c * 4) * 2;                                  // nbp, parent, adiag
  }
  if (nlev_out) *nlev_out = nlev;
  return tot;
}

MgWs mg_ws_carve(const Geo& g, void* base, const DevPtrs& P, const SolverWs& W) {
  int dims[MG_MAX_LEVELS][3];
  MgWs M{};
  mg_dims(g, dims, &M.nlev);
  char* p = static_cast<char*>(base);
  auto take = [&](size_t b) {
    char* r = p;
    p += al(b);
    return r;
  };
  M.m = (int*)take(MG_MAX_LEVELS * 4);
  for (int L = 0; L < M.nlev; L++) {
    MgLevel& lv = M.lv[L];
    lv.nx = dims[L][0], lv.ny = dims[L][1], lv.nz = dims[L][2];
    size_t c = size_t(lv.nx) * lv.ny * lv.nz;
    lv.cap = int(c);
    if (L == 0) {
      lv.type = P.cell;
      lv.lidx = P.lidx;
      lv.list = P.list;
      lv.nb = W.nb;  // stride W.cap = nc = c
      lv.child = nullptr;
    } else {
      lv.type = (uint8_t*)take(c);
      lv.lidx = (int*)take(c * 4);
      lv.list = (int*)take(c * 4);
      lv.nb = (int*)take(c * 24);
      lv.child = (int*)take(c * 32);
    }
    lv.nbp = (int*)take(c * 24);
    lv.parent = (int*)take(c * 4);
    lv.adiag = (float*)take(c * 4);
  }
  return M;
}

// ---------------------------------------------------------------- hierarchy build (one block)

// Order-preserving compaction of the cells with pred(c) over [0, n): list[pos] = c, lidx[c] = pos
// or -1. One block; returns the count to every thread.
template <class Pred>
__device__ int block_compact(int n, Pred pred, int* list, int* lidx, int* s_warp, int* s_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) *s_tot = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    int c = base + threadIdx.x;
    int f = c < n && pred(c) ? 1 : 0;
    int x = f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = lane < nw ? s_warp[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    int pos = *s_tot + x - f + (warp > 0 ? s_warp[warp - 1] : 0);
    if (c < n) {
      lidx[c] = f ? pos : -1;
      if (f) list[pos] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) *s_tot += s_warp[nw - 1];
    __syncthreads();
  }
  return *s_tot;
}

__global__ void __launch_bounds__(1024) k_mg_setup(Geo g, DevPtrs P, SolverWs W, MgWs M) {
  if (!P.sc->active) return;
  __shared__ int s_warp[32];
  __shared__ int s_tot;
  __shared__ int s_m[MG_MAX_LEVELS];
  if (threadIdx.x == 0) s_m[0] = P.sc->m;
  // coarse cell types and lists
  for (int L = 1; L < M.nlev; L++) {
    const MgLevel F = M.lv[L - 1];
    const MgLevel C = M.lv[L];
    const int nc = C.nx * C.ny * C.nz;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
      int i = c % C.nx, j = (c / C.nx) % C.ny, k = c / (C.nx * C.ny);
      uint8_t t;
      if (i == 0 || j == 0 || k == 0 || i == C.nx - 1 || j == C.ny - 1 || k == C.nz - 1) {
        t = SOLID;
      } else {
        bool air = false, liquid = false;
        for (int d = 0; d < 8; d++) {
          int fi = 2 * i + (d & 1), fj = 2 * j + ((d >> 1) & 1), fk = 2 * k + (d >> 2);
          if (fi >= F.nx || fj >= F.ny || fk >= F.nz) continue;
          uint8_t ft = F.type[fi + F.nx * (fj + F.ny * fk)];
          if (ft == AIR) air = true;
          else if (ft == FLUID) liquid = true;
        }
        t = air ? AIR : liquid ? FLUID : SOLID;
      }
      C.type[c] = t;
    }
    __syncthreads();
    int m = block_compact(nc, [&](int c) { return C.type[c] == FLUID; }, C.list, C.lidx, s_warp, &s_tot);
    if (threadIdx.x == 0) s_m[L] = m;
    __syncthreads();
  }
  // per-cell data: neighbours, diagonal, children, parent
  for (int L = 0; L < M.nlev; L++) {
    const MgLevel lv = M.lv[L];
    const int m = s_m[L];
    const int nxy = lv.nx * lv.ny;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
      int c = lv.list[t];
      int i = c % lv.nx, j = (c / lv.nx) % lv.ny, k = c / nxy;
      if (L == 0) {
        lv.adiag[t] = (float)W.adiag[t];
      } else {
        const int off[6] = {-1, 1, -lv.nx, lv.nx, -nxy, nxy};
        float d = 0;
        for (int e = 0; e < 6; e++) {
          lv.nb[e * lv.cap + t] = lv.lidx[c + off[e]];
          if (lv.type[c + off[e]] != SOLID) d += 1;
        }
        lv.adiag[t] = d;
        const MgLevel F = M.lv[L - 1];
        for (int dd = 0; dd < 8; dd++) {
          int fi = 2 * i + (dd & 1), fj = 2 * j + ((dd >> 1) & 1), fk = 2 * k + (dd >> 2);
          int ch = -1;
          if (fi < F.nx && fj < F.ny && fk < F.nz) ch = F.lidx[fi + F.nx * (fj + F.ny * fk)];
          lv.child[dd * lv.cap + t] = ch;
        }
      }
      int par = -1;
      if (L + 1 < M.nlev) {
        const MgLevel C = M.lv[L + 1];
        par = C.lidx[(i >> 1) + C.nx * ((j >> 1) + C.ny * (k >> 1))];
      }
      lv.parent[t] = par;
    }
  }
  __syncthreads();
  for (int L = 0; L < M.nlev; L++) {
    const MgLevel lv = M.lv[L];
    const int m = s_m[L];
    for (int t = threadIdx.x; t < m; t += blockDim.x)
      for (int e = 0; e < 6; e++) {
        int n = lv.nb[e * lv.cap + t];
        lv.nbp[e * lv.cap + t] = n >= 0 ? lv.parent[n] : -1;
      }
  }
  if (threadIdx.x < MG_MAX_LEVELS) M.m[threadIdx.x] = threadIdx.x < M.nlev ? s_m[threadIdx.x] : 0;
}

void launch_mg_setup(const Geo& g, const DevPtrs& P, const MgWs& M, cudaStream_t st) {
  SolverWs W = solver_ws_carve(P.solver_ws, g.nc);
  k_mg_setup<<<1, 1024, 0, st>>>(g, P, W, M);
}

// ---------------------------------------------------------------- cluster solve

// Where a level's cells live: rank r owns list indices [r * chunk, (r + 1) * chunk); the coarsest
// level lives entirely in rank 0.
struct Part {
  int m, chunk, own0, cnt;
};

__device__ __forceinline__ uint32_t pack_ref(const Part& p, int gi) {
  if (gi < 0) return MG_NONE;
  int r = gi / p.chunk;
  return (uint32_t(r) << 16) | uint32_t(gi - r * p.chunk);
}

// Shared-memory arrays of one level (identical offsets in every CTA of the cluster).
template <typename T>
struct LvSm {
  Part p;
  uint32_t* nb;   // [6][chunk]
  uint32_t* nbp;  // [6][chunk] (not on the coarsest level)
  uint32_t* ch;   // [8][chunk] (levels >= 1)
  float* adiag;
  uint8_t* red;   // 1 for red cells (i + j + k even)
  T* x;
  T* b;
};

template <typename T>
struct Sm {
  LvSm<T> lv[MG_MAX_LEVELS];
  T *r, *s0, *s1, *as;      // level-0 CG vectors (r is level 0's right-hand side)
  double* q;                // solution
  double* b64;              // FP64 rhs (true residual in FP32 mode)
  double* part;             // [2][MG_CLUSTER] reduction slots (used in rank 0)
  double* wpart;            // [MG_THREADS / 32] warp partials
};

template <typename T>
__device__ __forceinline__ T rd(const T* local, uint32_t ref, int me, cg::cluster_group& cl) {
  if (ref == MG_NONE) return T(0);
  int r = int(ref >> 16);
  int l = int(ref & 0xffffu);
  const T* p = (r == me) ? local : cl.map_shared_rank(const_cast<T*>(local), r);
  return p[l];
}

struct Red {
  double* part;
  double* wpart;
  int phase;
};

// Deterministic cluster-wide sum or max: warp shuffles, warps in order, ranks in order.
template <bool MAX>
__device__ double cluster_reduce(double v, Red& R, int me, int S, cg::cluster_group& cl) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = MAX ? dmax(v, w) : v + w;
  }
  if ((threadIdx.x & 31) == 0) R.wpart[threadIdx.x >> 5] = v;
  __syncthreads();
  double* slot = R.part + MG_CLUSTER * (R.phase & 1);
  R.phase++;
  if (threadIdx.x == 0) {
    double t = MAX ? 0.0 : 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) t = MAX ? dmax(t, R.wpart[w]) : t + R.wpart[w];
    double* dst = cl.map_shared_rank(slot, 0);
    dst[me] = t;
  }
  cl.sync();
  const double* src = cl.map_shared_rank(slot, 0);
  double t = 0;
  for (int r = 0; r < S; r++) t = MAX ? dmax(t, src[r]) : t + src[r];
  return t;
}

template <typename T>
__device__ __forceinline__ T nb_sum(const LvSm<T>& L, const T* xl, int t, int me, cg::cluster_group& cl) {
  const int ch = L.p.chunk;
  T s = 0;
#pragma unroll
  for (int e = 0; e < 6; e++) s += rd(xl, L.nb[e * ch + t], me, cl);
  return s;
}

// Right-hand side of a coarse level from its children's residuals (red children only), then the
// first pre-smoothing half-sweep from x = 0 (red cells: x = b / diag).
template <typename T>
__device__ void restrict_prered(Sm<T>& S, int L, int me, cg::cluster_group& cl) {
  LvSm<T>& C = S.lv[L];
  LvSm<T>& F = S.lv[L - 1];
  const T* fb = (L - 1 == 0) ? S.r : F.b;
  for (int t = threadIdx.x; t < C.p.cnt; t += blockDim.x) {
    T acc = 0;
#pragma unroll 1
    for (int d = 0; d < 8; d++) {
      uint32_t ref = C.ch[d * C.p.chunk + t];
      if (ref == MG_NONE) continue;
      int r = int(ref >> 16), l = int(ref & 0xffffu);
      const uint8_t* red = (r == me) ? F.red : cl.map_shared_rank(const_cast<uint8_t*>(F.red), r);
      if (!red[l]) continue;
      const T* fx = (r == me) ? F.x : cl.map_shared_rank(F.x, r);
      const T* fbb = (r == me) ? fb : cl.map_shared_rank(const_cast<T*>(fb), r);
      const float* fd = (r == me) ? F.adiag : cl.map_shared_rank(F.adiag, r);
      const uint32_t* fnb = (r == me) ? F.nb : cl.map_shared_rank(F.nb, r);
      T s = 0;
#pragma unroll
      for (int e = 0; e < 6; e++) s += rd(F.x, fnb[e * F.p.chunk + l], me, cl);
      acc += fbb[l] - T(fd[l]) * fx[l] + s;
    }
    T b = T(0.5) * acc;
    C.b[t] = b;
    C.x[t] = C.red[t] ? b / T(C.adiag[t]) : T(0);
  }
}

// Gauss-Seidel half-sweep over one colour; with `prolong`, neighbours add their parents' coarse
// correction first (the prolongation folded into the first post-smoothing half-sweep).
template <typename T>
__device__ void half_sweep(Sm<T>& S, int L, bool red_cells, bool prolong, int me, cg::cluster_group& cl) {
  LvSm<T>& V = S.lv[L];
  const T* b = (L == 0) ? S.r : V.b;
  const T* xc = prolong ? S.lv[L + 1].x : nullptr;
  const int ch = V.p.chunk;
  for (int t = threadIdx.x; t < V.p.cnt; t += blockDim.x) {
    if ((V.red[t] != 0) != red_cells) continue;
    T s = 0;
#pragma unroll
    for (int e = 0; e < 6; e++) {
      s += rd(V.x, V.nb[e * ch + t], me, cl);
      if (prolong) s += rd(xc, V.nbp[e * ch + t], me, cl);
    }
    V.x[t] = (b[t] + s) / T(V.adiag[t]);
  }
}

// Coarsest level: restriction, then a palindromic red-black sequence inside rank 0.
template <typename T>
__device__ void coarsest(Sm<T>& S, int L, int me, cg::cluster_group& cl) {
  restrict_prered(S, L, me, cl);
  if (me != 0) return;
  __syncthreads();
  for (int k = 0; k < MG_COARSE_SWEEPS; k++) {
    half_sweep(S, L, true, false, me, cl);
    __syncthreads();
    half_sweep(S, L, false, false, me, cl);
    __syncthreads();
  }
  for (int k = 0; k < MG_COARSE_SWEEPS; k++) {
    half_sweep(S, L, false, false, me, cl);
    __syncthreads();
    half_sweep(S, L, true, false, me, cl);
    __syncthreads();
  }
}

// One V-cycle on the current level-0 rhs S.r; level 0's red cells already hold r / diag.
// Returns the partial z.r over this rank's cells (z = level-0 x).
template <typename T>
__device__ double vcycle(Sm<T>& S, int nlev, int me, cg::cluster_group& cl) {
  const int last = nlev - 1;
  for (int L = 0; L < last; L++) {
    if (L > 0) {
      restrict_prered(S, L, me, cl);
      cl.sync();
    }
    half_sweep(S, L, false, false, me, cl);  // pre-smoothing, black
    cl.sync();
  }
  if (last > 0) {
    coarsest(S, last, me, cl);
    cl.sync();
  } else if (me == 0) {  // single level: smoothing only
    for (int k = 0; k < MG_COARSE_SWEEPS; k++) {
      half_sweep(S, 0, true, false, me, cl);
      __syncthreads();
      half_sweep(S, 0, false, false, me, cl);
      __syncthreads();
    }
  }
  double zr = 0;
  for (int L = last - 1; L >= 0; L--) {
    half_sweep(S, L, false, true, me, cl);  // post-smoothing, black, with prolongation
    cl.sync();
    half_sweep(S, L, true, false, me, cl);  // post-smoothing, red
    if (L > 0) cl.sync();
  }
  LvSm<T>& V = S.lv[0];
  for (int t = threadIdx.x; t < V.p.cnt; t += blockDim.x) zr += double(V.x[t]) * double(S.r[t]);
  return zr;
}

template <typename T>
__device__ Part make_part(int m, int S, int me, bool coarsest) {
  Part p;
  p.m = m;
  if (coarsest) {
    p.chunk = m > 0 ? m : 1;
    p.own0 = 0;
    p.cnt = me == 0 ? m : 0;
  } else {
    p.chunk = m > 0 ? (m + S - 1) / S : 1;
    p.own0 = me * p.chunk;
    int e = p.own0 + p.chunk;
    p.cnt = m > p.own0 ? (e < m ? e : m) - p.own0 : 0;
  }
  return p;
}

template <typename T>
__global__ void __launch_bounds__(MG_THREADS) k_mgpcg(Geo g, DevPtrs P, MgWs M, MgArgs a) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  if (a.is_correction) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // interior mean of the density ratios (solver3d.ts:670)
      double s = 0;
      int n = 0;
      for (int b = 0; b < DENSITY_BLOCKS; b++) {
        s += P.interior_part[b];
        n += P.interior_cnt_part[b];
      }
      sc->interior = n > 0 ? s / n : 1.0;
      sc->interior_count = n;
    }
    if (!sc->corr_any) {  // solver3d.ts:671
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->corr_iters = 0;
        sc->mg_status = 1;
      }
      return;
    }
  }
  cg::cluster_group cl = cg::this_cluster();
  const int NS = int(cl.num_blocks());
  const int me = int(cl.block_rank());
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Sm<T> S;  // the layout table itself lives in shared memory (indexed by level)
  __shared__ unsigned long long s_off;
  const int nlev = M.nlev;
  // ---- layout (identical in every rank)
  if (threadIdx.x == 0) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> void* {
      void* r = smem + off;
      off += (bytes + 15) & ~size_t(15);
      return r;
    };
    for (int L = 0; L < nlev; L++) {
      LvSm<T>& V = S.lv[L];
      V.p = make_part<T>(M.m[L], NS, me, L == nlev - 1);
      const size_t ch = V.p.chunk;
      V.x = (T*)take(ch * sizeof(T));
      V.b = (L == 0) ? nullptr : (T*)take(ch * sizeof(T));
      V.nb = (uint32_t*)take(ch * 24);
      V.nbp = (L < nlev - 1) ? (uint32_t*)take(ch * 24) : nullptr;
      V.ch = (L > 0) ? (uint32_t*)take(ch * 32) : nullptr;
      V.adiag = (float*)take(ch * 4);
      V.red = (uint8_t*)take(ch);
    }
    const size_t c0 = S.lv[0].p.chunk;
    S.r = (T*)take(c0 * sizeof(T));
    S.s0 = (T*)take(c0 * sizeof(T));
    S.s1 = (T*)take(c0 * sizeof(T));
    S.as = (T*)take(c0 * sizeof(T));
    S.q = (double*)take(c0 * 8);
    S.b64 = (double*)take(c0 * 8);
    S.part = (double*)take(2 * MG_CLUSTER * 8);
    S.wpart = (double*)take((MG_THREADS / 32) * 8);
    s_off = off;
  }
  __syncthreads();
  if (s_off > (unsigned long long)MG_SMEM) {  // uniform: every rank computes the same layout
    if (me == 0 && threadIdx.x == 0) sc->mg_status = 0;  // the wavefront solver takes over
    return;
  }
  // ---- load the hierarchy into the ranks' shared memory
  for (int L = 0; L < nlev; L++) {
    LvSm<T>& V = S.lv[L];
    const MgLevel& G = M.lv[L];
    const int ch = V.p.chunk;
    for (int t = threadIdx.x; t < V.p.cnt; t += blockDim.x) {
      int gi = V.p.own0 + t;
      int c = G.list[gi];
      int i = c % G.nx, j = (c / G.nx) % G.ny, k = c / (G.nx * G.ny);
      V.red[t] = ((i + j + k) & 1) == 0;
      V.adiag[t] = G.adiag[gi];
      V.x[t] = 0;
      for (int e = 0; e < 6; e++) {
        V.nb[e * ch + t] = pack_ref(V.p, G.nb[e * G.cap + gi]);
        if (L < nlev - 1) V.nbp[e * ch + t] = pack_ref(S.lv[L + 1].p, G.nbp[e * G.cap + gi]);
      }
      if (L > 0)
        for (int d = 0; d < 8; d++) V.ch[d * ch + t] = pack_ref(S.lv[L - 1].p, G.child[d * G.cap + gi]);
    }
  }
  Red R{S.part, S.wpart, 0};
  LvSm<T>& V0 = S.lv[0];
  double bmax = 0;
  for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) {
    double b = a.b[V0.p.own0 + t];
    S.b64[t] = b;
    S.r[t] = T(b);
    S.q[t] = 0;
    S.s0[t] = 0;
    S.s1[t] = 0;
    S.as[t] = 0;
    V0.x[t] = V0.red[t] ? T(b) / T(V0.adiag[t]) : T(0);
    bmax = dmax(bmax, fabs(b));
  }
  const double bnorm = cluster_reduce<true>(bmax, R, me, NS, cl);  // includes cl.sync()
  int iters = 0, converged = 1;
  double res = bnorm;
  const int m = V0.p.m;
  if (m > 0 && !(bnorm < 1e-14)) {
    const double target = dmax(a.tol * bnorm, 1e-14);
    double sigma = cluster_reduce<false>(vcycle(S, nlev, me, cl), R, me, NS, cl);
    double beta = 0;
    int parity = 0;
    int restarts = 0;
    converged = 0;
    int it = 1;
    for (; it <= a.max_iter; it++) {
      // s = z + beta s, As = A s (neighbours' s formed on the fly from the previous buffer)
      T* so = parity ? S.s1 : S.s0;
      T* sn = parity ? S.s0 : S.s1;
      const T tb = T(beta);
      double sp = 0;
      for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) {
        T st = V0.x[t] + tb * so[t];
        T acc = 0;
#pragma unroll
        for (int e = 0; e < 6; e++) {
          uint32_t ref = V0.nb[e * V0.p.chunk + t];
          acc += rd(V0.x, ref, me, cl) + tb * rd(so, ref, me, cl);
        }
        T as = T(V0.adiag[t]) * st - acc;
        sn[t] = st;
        S.as[t] = as;
        sp += double(st) * double(as);
      }
      parity ^= 1;
      double sas = cluster_reduce<false>(sp, R, me, NS, cl);
      if (!(sas > 0)) break;
      const double alpha = sigma / sas;
      const T ta = T(alpha);
      double rm = 0;
      for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) {
        S.q[t] += alpha * double(sn[t]);
        T rr = S.r[t] - ta * S.as[t];
        S.r[t] = rr;
        rm = dmax(rm, fabs(double(rr)));
        V0.x[t] = V0.red[t] ? rr / T(V0.adiag[t]) : T(0);
      }
      res = cluster_reduce<true>(rm, R, me, NS, cl);
      if (res <= target) {
        if (sizeof(T) == 8 || restarts >= 4) {
          converged = 1;
          break;
        }
        // FP32 vectors: confirm with the FP64 true residual b - A q
        double tm = 0;
        for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) {
          double acc = 0;
#pragma unroll
          for (int e = 0; e < 6; e++) acc += rd(S.q, V0.nb[e * V0.p.chunk + t], me, cl);
          double rt = S.b64[t] - (double(V0.adiag[t]) * S.q[t] - acc);
          tm = dmax(tm, fabs(rt));
          S.as[t] = T(rt);  // staged: r is overwritten only after every rank has read q
        }
        double tres = cluster_reduce<true>(tm, R, me, NS, cl);
        if (tres <= target) {
          res = tres;
          converged = 1;
          break;
        }
        restarts++;
        for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) {
          T rr = S.as[t];
          S.r[t] = rr;
          V0.x[t] = V0.red[t] ? rr / T(V0.adiag[t]) : T(0);
        }
        cl.sync();
        sigma = cluster_reduce<false>(vcycle(S, nlev, me, cl), R, me, NS, cl);
        beta = 0;
        continue;
      }
      double sn2 = cluster_reduce<false>(vcycle(S, nlev, me, cl), R, me, NS, cl);
      beta = sn2 / sigma;
      sigma = sn2;
    }
    iters = converged ? it : a.max_iter;
    if (!converged) converged = res <= target ? 1 : 0;
  }
  for (int t = threadIdx.x; t < V0.p.cnt; t += blockDim.x) a.q[V0.p.own0 + t] = S.q[t];
  if (me == 0 && threadIdx.x == 0) {
    if (a.is_correction) {
      sc->corr_iters = iters;
      sc->corr_residual = res;
    } else {
      sc->last_iters = iters;
      sc->last_residual = res;
      if (!converged) sc->failures++;
    }
    sc->mg_status = 1;
  }
  cl.sync();  // no rank leaves while another may still read its shared memory
}

void mg_configure() {
  cudaFuncSetAttribute(k_mgpcg<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM);
  cudaFuncSetAttribute(k_mgpcg<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM);
  cudaFuncSetAttribute(k_mgpcg<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(k_mgpcg<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

void launch_mg_solve(const Geo& g, const DevPtrs& P, const MgWs& M, const MgArgs& a, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(MG_CLUSTER);
  cfg.blockDim = dim3(MG_THREADS);
  cfg.dynamicSmemBytes = MG_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = MG_CLUSTER;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (a.mixed)
    cudaLaunchKernelEx(&cfg, k_mgpcg<float>, g, P, M, a);
  else
    cudaLaunchKernelEx(&cfg, k_mgpcg<double>, g, P, M, a);
}

}  // namespace pl
