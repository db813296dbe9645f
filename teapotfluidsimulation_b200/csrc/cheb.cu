// Chebyshev-polynomial-preconditioned CG on one thread-block cluster: the fast pressure solve.
//
// Preconditioner: z = p(D^-1 A) D^-1 r, `degree` Chebyshev steps for D^-1 A on [lo, 2] from z = 0
// (the WebGPU port's preconditioner, src/gpu3d/shaders.ts:588-622). The polynomial is positive on
// (0, 2], so the preconditioner is symmetric positive definite and CG stays valid; every step is one
// 7-point stencil with no inner products.
//
// Partition: the liquid cells in column-tile order (8 x 8 columns, then k, j, i; built by
// k_solve_setup) are split into `cluster` contiguous ranges, one per CTA, so each CTA owns a compact
// block and exchanges only its faces. Each thread owns up to CHEB_KMAX cells; their per-cell state
// (residuals, diagonal, solution, neighbour indices) stays in registers. Stencil vectors live in
// shared memory: own cells, a zero guard element, then one halo slot per remote cell that some own
// cell references (deduplicated: a remote cell has one slot however many own neighbours it has).
//
// Exchange (one "round" per stencil vector): the thread that computes a new value of a boundary cell
// stores it locally and writes it straight into the halo slot of every CTA that requested the cell
// with st.async, which also completes those bytes on that CTA's exchange mbarrier. A CTA then waits
// only for its own barrier (it expects one value per halo slot), so no round needs a cluster-wide
// barrier, and the halo traffic is one value per (boundary cell, requesting CTA). Two buffers and
// two barriers alternate by round parity: a CTA can run at most one round ahead of a neighbour,
// because it needs that neighbour's values of the previous round, which the neighbour sends only
// after it has read everything of the round before.
//
// Reductions are deterministic and also barrier-free: every CTA folds its warps' partials in warp
// order, sends the result to every other CTA's slot table (st.async on their reduction barrier), and
// sums the slots in rank order, its own partial in its own place.
//
// CG (Chronopoulos-Gear ordering): after z = M r each CTA forms w = A z from the exchanged z, and one
// reduction gives max|r|, z.r and z.w; s = z + beta s and A s = w + beta A s follow without another
// exchange, and s.As = z.w - beta z.r / alpha_prev. The stopping rule and bookkeeping are the
// reference's (solver3d.ts:858-937): max-norm residual <= max(tol * max|b|, 1e-14), breakdown if
// s.As <= 0, the same iteration count; like the WebGPU port the preconditioner runs before the
// convergence test so that max|r| and z.r share one reduction. With FP32 vectors (PL_SOLVE_MIXED) a
// recursive-residual convergence is confirmed by the FP64 true residual b - A q and CG restarts from
// it when it misses the target (iterative refinement).
//
// Every wait is bounded (CHEB_WAIT_LIMIT polls): a wait that gives up sets ERR_SOLVER_TIMEOUT and
// the solve still runs every round to the end, so no CTA is left waiting and none exits while
// another can still write into its shared memory.
#include <cooperative_groups.h>

#include <algorithm>

#include "cheb.h"

namespace cg = cooperative_groups;

namespace pl {

namespace {

constexpr int CHEB_WAIT_LIMIT = 1 << 20;
// First FP64 confirmation of an FP32-vector solve at this multiple of the target (4 mm pour, whole
// run: 4x, 16x and 64x cost 0.2915, 0.2884 and 0.2905 ms per substep, 1x 0.2998; each took one
// restart, with 20 instead of 21 preconditioner applications per solve at 16x).
constexpr double CHEB_FIRST_CHECK = 16.0;
constexpr int CHEB_MAX_DEGREE = 32;
constexpr int CHEB_BITMAP_WORDS = 1024;  // remote-reference bitmap over liquid positions (<= 32768)

__device__ __forceinline__ uint32_t s_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Shared::cluster address of the same shared-memory location in CTA `rank`.
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, int rank) {
  uint32_t o;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(o) : "r"(a), "r"(rank));
  return o;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// This CTA's arrival on its barrier, announcing the bytes the current phase receives.
__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of the given parity to complete; clears ok when the poll limit runs out, and
// once ok is clear no longer waits (so a failed solve runs its remaining rounds without stalling).
__device__ __forceinline__ void mbar_wait(uint32_t bar, uint32_t parity, bool& ok) {
  if (!ok) return;
  for (int i = 0; i < CHEB_WAIT_LIMIT; i++)
    if (mbar_try(bar, parity)) return;
  ok = false;
}

// Remote store that completes its bytes on the destination CTA's barrier.
__device__ __forceinline__ void st_async(uint32_t raddr, float v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(raddr),
               "r"(__float_as_uint(v)), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void st_async(uint32_t raddr, double v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];" ::"r"(raddr),
               "l"(__double_as_longlong(v)), "r"(rbar)
               : "memory");
}

// Plain shared-memory accesses at a byte offset into the dynamic shared memory. The round barriers
// (__syncthreads, and the mbarrier waits whose asm clobbers memory) keep them in place, and the
// compiler is free to issue a cell's six neighbour loads, and both cells' loads, back to back.
template <typename V>
__device__ __forceinline__ V ldsh(const char* smem, uint32_t off) {
  return *reinterpret_cast<const V*>(smem + off);
}
template <typename V>
__device__ __forceinline__ void stsh(char* smem, uint32_t off, V v) {
  *reinterpret_cast<V*>(smem + off) = v;
}

struct Cl {
  unsigned long long xbar[2];    // exchange barriers (round parity)
  unsigned long long rbar[2];    // reduction barriers (reduction parity)
  uint32_t rsmem[CHEB_CLUSTER];  // shared::cluster address of every rank's dynamic shared memory
  uint32_t rxbar[CHEB_CLUSTER];  // ... of every rank's xbar[0]
  uint32_t rrbar[CHEB_CLUSTER];  // ... of every rank's rbar[0]
  uint32_t rred[CHEB_CLUSTER];   // ... of every rank's red[0][0][0]
  double red[2][CHEB_CLUSTER][3];  // reduction slots: (max, sum, sum) from each rank
  double wpart[2][CHEB_MAX_THREADS / 32][3];
  double bcast[2][3];
  double coef[CHEB_MAX_DEGREE][2];  // Chebyshev step coefficients (c1, c2)
  float coef_f[CHEB_MAX_DEGREE][2];  // ... rounded to FP32 once (the FP32-vector solve's step arithmetic)
  int out_cnt[CHEB_CLUSTER];  // distinct remote cells this rank references in each owner
  int in_cnt[CHEB_CLUSTER];   // requests each rank sends to this rank
  int in_base[CHEB_CLUSTER];  // each referencing rank's halo slot of the first of this rank's cells it references
  int req_off[CHEB_CLUSTER];  // start of each referencing rank's entries in this rank's send list
  int nh;                     // halo slots of this rank
};

// Deterministic cluster-wide (max x, sum y, sum z). Xor butterflies leave the same bits in every
// lane (their additions pair the same operands in every lane), so: each warp reduces its lanes;
// warp 0 reduces the warp partials (lane w holds warp w's) into the CTA partial, sends it to every
// other rank's slot table (st.async on their reduction barrier), waits for theirs, and reduces the
// rank partials (lane q holds rank q's, its own in its own place) in the same fixed tree, so every
// rank gets the same bits; the result is broadcast through shared memory.
__device__ __forceinline__ void butterfly3(double& mx, double& s1, double& s2) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
}

__device__ double3 reduce3(double mx, double s1, double s2, Cl& C, int& rr, int me, int ns, bool& ok) {
  butterfly3(mx, s1, s2);
  const int sl = rr & 1;
  const uint32_t par = uint32_t(rr >> 1) & 1u;
  rr++;
  const int lane = int(threadIdx.x & 31), wid = int(threadIdx.x >> 5);
  if (lane == 0) {
    C.wpart[sl][wid][0] = mx;
    C.wpart[sl][wid][1] = s1;
    C.wpart[sl][wid][2] = s2;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = int(blockDim.x >> 5);
    double a = 0, b = 0, c = 0;  // all maxima reduced here are of non-negative values
    if (lane < nw) {
      a = C.wpart[sl][lane][0];
      b = C.wpart[sl][lane][1];
      c = C.wpart[sl][lane][2];
    }
    butterfly3(a, b, c);
    if (lane == 0) mbar_expect(s_addr(&C.rbar[sl]), uint32_t(ns - 1) * 24u);
    if (lane < ns && lane != me) {
      const uint32_t dst = C.rred[lane] + uint32_t((sl * CHEB_CLUSTER + me) * 24);
      const uint32_t bar = C.rrbar[lane] + uint32_t(sl * 8);
      st_async(dst, a, bar);
      st_async(dst + 8, b, bar);
      st_async(dst + 16, c, bar);
    }
    mbar_wait(s_addr(&C.rbar[sl]), par, ok);
    double x = 0, y = 0, z = 0;
    if (lane == me) {
      x = a;
      y = b;
      z = c;
    } else if (lane < ns) {
      x = C.red[sl][lane][0];
      y = C.red[sl][lane][1];
      z = C.red[sl][lane][2];
    }
    butterfly3(x, y, z);
    if (lane == 0) {
      C.bcast[sl][0] = x;
      C.bcast[sl][1] = y;
      C.bcast[sl][2] = z;
    }
  }
  __syncthreads();
  return make_double3(C.bcast[sl][0], C.bcast[sl][1], C.bcast[sl][2]);
}

// Element i of the shared-memory array at byte offset `off`.
template <typename V>
__device__ __forceinline__ V& sv(char* smem, uint32_t off, int i) {
  return reinterpret_cast<V*>(smem + off)[i];
}

}  // namespace

// K: cells per thread (1, 2 or 4; at most 1024 / K threads, so that the per-cell state stays in
// registers).
template <typename T, int K>
__global__ void __launch_bounds__(CHEB_MAX_THREADS / K, 1) k_chebpcg(Geo g, DevPtrs P, SolverWs W, ChebArgs a) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  if (a.gate && sc->mg_status) return;  // the launch before this one solved the system
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->t_solve[0] = globaltimer_ns();
  if (a.jobs == 1 && a.is_correction) {
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
    if (!sc->corr_any) {  // solver3d.ts:671: no solve, uc = vc = wc = 0
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->corr_iters = 0;
        sc->mg_status = 1;
      }
      return;
    }
  }
  cg::cluster_group cl = cg::this_cluster();
  const int ns = int(cl.num_blocks());
  const int me = int(cl.block_rank());
  const int nt = int(blockDim.x);
  const int tid = int(threadIdx.x);
  extern __shared__ __align__(16) char smem[];
  __shared__ Cl C;
  __shared__ int s_warp[CHEB_MAX_THREADS / 32];
  const int m = sc->m;
  const int chunk = m > 0 ? (m + ns - 1) / ns : 1;
  const int own0 = me * chunk;
  const int cnt = m > own0 ? min(own0 + chunk, m) - own0 : 0;
  const int guard = chunk;  // element [chunk] of every stencil vector is 0; halo slots follow it
  const int deg = a.degree;
  // uniform decisions: more cells per thread than registers hold, or a polynomial degree or a
  // liquid-cell count beyond the fixed tables: the wavefront solver takes over
  if ((chunk + nt - 1) / nt > K || deg < 1 || deg > CHEB_MAX_DEGREE || m > CHEB_BITMAP_WORDS * 32) {
    if (me == 0 && tid == 0) sc->mg_status = 0;
    return;
  }
  // bitmap of the referenced remote positions and its word prefix: a fixed place at the end of the
  // dynamic shared memory (the layout below stays clear of it)
  const uint32_t BM = uint32_t(a.smem_bytes) - CHEB_BITMAP_WORDS * 8;
  const uint32_t BMP = BM + CHEB_BITMAP_WORDS * 4;
  const int nwords = (m + 31) >> 5;
  if (tid == 0) {
    mbar_init(s_addr(&C.xbar[0]), 1);
    mbar_init(s_addr(&C.xbar[1]), 1);
    mbar_init(s_addr(&C.rbar[0]), 1);
    mbar_init(s_addr(&C.rbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // Chebyshev recurrence coefficients on [lo, 2]
    const double lo = a.cheb_lo, hi = 2.0;
    const double theta = (hi + lo) / 2, delta = (hi - lo) / 2, sigma1 = theta / delta;
    double rho = 1 / sigma1;
    for (int s = 1; s < deg; s++) {
      const double rhoN = 1 / (2 * sigma1 - rho);
      C.coef[s][0] = rhoN * rho;
      C.coef[s][1] = 2 * rhoN / delta;
      C.coef_f[s][0] = float(C.coef[s][0]);
      C.coef_f[s][1] = float(C.coef[s][1]);
      rho = rhoN;
    }
  }
  if (tid < ns) {
    C.rsmem[tid] = mapa_u32(s_addr(smem), tid);
    C.rxbar[tid] = mapa_u32(s_addr(&C.xbar[0]), tid);
    C.rrbar[tid] = mapa_u32(s_addr(&C.rbar[0]), tid);
    C.rred[tid] = mapa_u32(s_addr(&C.red[0][0][0]), tid);
    C.out_cnt[tid] = 0;
  }
  for (int w = tid; w < nwords; w += nt) sv<uint32_t>(smem, BM, w) = 0u;
  __syncthreads();
  // ---- own cells t_k = tid + k * nt at tile-order positions own0 + t_k
  int gnb[K][6];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int t = tid + k * nt;
#pragma unroll
    for (int f = 0; f < 6; f++) {
      const int gi = t < cnt ? P.tnb[f * g.nc + own0 + t] : -1;
      gnb[k][f] = gi;
      if (gi >= 0 && gi / chunk != me) atomicOr(&sv<uint32_t>(smem, BM, gi >> 5), 1u << (gi & 31));
    }
  }
  __syncthreads();
  // halo slot of a remote position = its rank among the referenced positions (so the slots of one
  // owner are contiguous and ordered by position)
  {
    const int per = (nwords + nt - 1) / nt;
    const int w0 = tid * per;
    int sum = 0;
    for (int q = 0; q < per; q++)
      if (w0 + q < nwords) sum += __popc(sv<uint32_t>(smem, BM, w0 + q));
    const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (tid == 0) {
      int acc = 0;
      for (int w = 0; w < nw; w++) {
        int c = s_warp[w];
        s_warp[w] = acc;
        acc += c;
      }
      C.nh = acc;
    }
    __syncthreads();
    int run = s_warp[wid] + x - sum;
    for (int q = 0; q < per; q++)
      if (w0 + q < nwords) {
        sv<int>(smem, BMP, w0 + q) = run;
        run += __popc(sv<uint32_t>(smem, BM, w0 + q));
      }
  }
  __syncthreads();
  auto hrank = [&](int gi) {  // referenced remote positions before gi
    if (gi >= m) return C.nh;
    const int w = gi >> 5;
    return sv<int>(smem, BMP, w) + __popc(sv<uint32_t>(smem, BM, w) & ((1u << (gi & 31)) - 1u));
  };
  if (tid < ns && tid != me) C.out_cnt[tid] = hrank(min((tid + 1) * chunk, m)) - hrank(min(tid * chunk, m));
  // Each rank's cells that a rank R references are exactly its cells with a neighbour owned by R (the
  // neighbour relation is symmetric), so every rank derives its own send list locally. R tells each
  // owner how many of its cells R references and R's halo slot of the first of them (R's slots for one
  // owner are consecutive and in position order).
  __syncthreads();
  if (tid < ns) {
    Cl* dst = cl.map_shared_rank(&C, tid);
    dst->in_cnt[me] = C.out_cnt[tid];
    dst->in_base[me] = tid == me ? 0 : hrank(min(tid * chunk, m));
  }
  // destination ranks of every own cell (bit R: a neighbour is owned by R), counted per warp and rank
  uint32_t dmask[K];
  const int lane = tid & 31, wid = tid >> 5, nwarps = nt >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    uint32_t mk = 0;
#pragma unroll
    for (int f = 0; f < 6; f++) {
      const int gi = gnb[k][f];
      if (gi >= 0 && gi / chunk != me) mk |= 1u << (gi / chunk);
    }
    dmask[k] = mk;
  }
  cl.sync();  // in_cnt / in_base complete everywhere; barrier initialisation visible to the cluster
  const int nh = C.nh;
  int incoming = 0;
  for (int r = 0; r < ns; r++) incoming += C.in_cnt[r];
  int rr = 0;  // reduction counter (advances identically in every thread)
  int e = 0;   // exchange-round counter (likewise)
  bool ok = true;
  // ---- layout (identical in every rank): byte offsets into the dynamic shared memory
  uint32_t off = 0;
  auto take = [&](size_t bytes) -> uint32_t {
    uint32_t r = off;
    off += uint32_t((bytes + 15) & ~size_t(15));
    return r;
  };
  const uint32_t WCNT = take(size_t(K) * CHEB_CLUSTER * (CHEB_MAX_THREADS / 32) * 4);  // per (k, rank, warp)
  const uint32_t SENDL = take(size_t(chunk) * 6 * 8);  // (own index | rank << 16, halo slot), by (rank, slot)
  const uint32_t NBOS = take(size_t(chunk) * 6 * 4);   // neighbour offsets by position, [f][own index]
  const uint32_t PERM = take(size_t(chunk) * 4);       // own index of each compute slot
  const uint32_t VEC0 = off;
  // per (k, rank, warp): cells of the warp's k-th group with a neighbour owned by the rank
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int r = 0; r < ns; r++) {
      const unsigned bal = __ballot_sync(0xffffffffu, (dmask[k] >> r) & 1u);
      if (lane == 0) sv<int>(smem, WCNT, (k * CHEB_CLUSTER + r) * (CHEB_MAX_THREADS / 32) + wid) = __popc(bal);
    }
  __syncthreads();
  // each rank's counts into exclusive offsets in (k, warp) order, i.e. in position order; a count that
  // disagrees with what the rank expects (it cannot, the relation being symmetric) is flagged
  double mismatch = 0;
  if (tid < ns) {
    int acc = 0;
    for (int k = 0; k < K; k++)
      for (int w = 0; w < nwarps; w++) {
        int& c = sv<int>(smem, WCNT, (k * CHEB_CLUSTER + tid) * (CHEB_MAX_THREADS / 32) + w);
        const int v = c;
        c = acc;
        acc += v;
      }
    if (tid != me && acc != C.in_cnt[tid]) mismatch = 1;
    if (tid == me && acc != 0) mismatch = 1;
    int o = 0;
    for (int r = 0; r < tid; r++) o += C.in_cnt[r];
    C.req_off[tid] = o;
  }
  // largest halo over the ranks (every rank's layout is the same) and the consistency flag, in one
  // cluster-wide reduction
  const double3 hm = reduce3(double(nh), mismatch, 0.0, C, rr, me, ns, ok);
  const int hcap = int(hm.x);
  const int n1 = chunk + 1 + hcap;  // own cells, guard, halo
  off = VEC0;
  const uint32_t DV0 = take(size_t(n1) * sizeof(T)), DV1 = take(size_t(n1) * sizeof(T));
  const uint32_t ZS = take(size_t(n1) * sizeof(T));
  const uint32_t QS = take(size_t(n1) * 8);
  if (off > BM || n1 > 65535 || hm.y != 0) {  // uniform decision: the wavefront solver takes over
    if (me == 0 && tid == 0) sc->mg_status = 0;
    cl.sync();
    return;
  }
  for (int i = tid; i < n1; i += nt) {
    sv<T>(smem, DV0, i) = sv<T>(smem, DV1, i) = sv<T>(smem, ZS, i) = T(0);
    sv<double>(smem, QS, i) = 0;
  }
  // Send list, ordered by (rank, halo slot): each round's send pass walks it, so consecutive threads
  // store to consecutive halo slots of one rank (coalesced remote stores: stores scattered over ranks
  // and slots cost several times more on the cluster network).
#pragma unroll
  for (int k = 0; k < K; k++)
    for (int r = 0; r < ns; r++) {
      const bool mine = (dmask[k] >> r) & 1u;
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      if (mine) {
        const int idx = sv<int>(smem, WCNT, (k * CHEB_CLUSTER + r) * (CHEB_MAX_THREADS / 32) + wid) +
                        __popc(bal & ((1u << lane) - 1u));
        sv<uint2>(smem, SENDL, C.req_off[r] + idx) =
            make_uint2(uint32_t(tid + k * nt) | (uint32_t(r) << 16), uint32_t(C.in_base[r] + idx));
      }
    }
  // byte offsets of the own cells' neighbours in a stencil vector of T (the guard for none), by position
  bool has[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    has[k] = tid + k * nt < cnt;
    if (has[k])
#pragma unroll
      for (int f = 0; f < 6; f++) {
        const int gi = gnb[k][f];
        const int li = gi < 0 ? guard : (gi / chunk == me ? gi - own0 : guard + 1 + hrank(gi));
        sv<uint32_t>(smem, NBOS, f * chunk + tid + k * nt) = uint32_t(li) * uint32_t(sizeof(T));
      }
  }
  // Compute slots: the boundary cells (those some rank holds in its halo) first, in position order, then
  // the interior cells, so that a round computes whole warps of boundary cells before its send pass
  // and the interior cells while the sends are in flight. Slot t_k = tid + k * nt computes own cell
  // oi[k]; the cells' values and the send lists stay by position.
  int brank[K], nbnd = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const bool b = has[k] && dmask[k] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, b);
    if (lane == 0) s_warp[wid] = __popc(bal);
    __syncthreads();
    int before = nbnd, tot = 0;
    for (int w = 0; w < nwarps; w++) {
      const int c = s_warp[w];
      before += w < wid ? c : 0;
      tot += c;
    }
    brank[k] = before + __popc(bal & ((1u << lane) - 1u));
    nbnd += tot;
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < K; k++)
    if (has[k]) {
      const int t = tid + k * nt;
      sv<int>(smem, PERM, dmask[k] != 0 ? brank[k] : nbnd + t - brank[k]) = t;
    }
  __syncthreads();
  int oi[K];
  bool bnd[K];
  uint32_t nbo[K][6];
#pragma unroll
  for (int k = 0; k < K; k++) {
    oi[k] = has[k] ? sv<int>(smem, PERM, tid + k * nt) : 0;
    bnd[k] = has[k] && tid + k * nt < nbnd;
#pragma unroll
    for (int f = 0; f < 6; f++) nbo[k][f] = has[k] ? sv<uint32_t>(smem, NBOS, f * chunk + oi[k]) : 0u;
  }
  __syncthreads();
  // ---- per-thread state of the owned cells (the exchange data serves every job of the launch)
  T r[K], z[K], res[K], as[K], sown[K], cdown[K], idg[K], dg[K], w[K];
  double q[K], b64[K];
  int li_own[K];  // liquid-list index of each own cell
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int li = has[k] ? P.tperm[own0 + oi[k]] : 0;
    li_own[k] = li;
    const double d = has[k] ? W.adiag[li] : 1.0;
    dg[k] = T(d);
    idg[k] = T(1) / T(d);
  }
  const uint32_t xb0 = s_addr(&C.xbar[0]);
  // Store v (a T) as this thread's own cell k of the vector at byte offset voff (the round's send pass
  // carries it to the requesting ranks).
  auto put = [&](uint32_t voff, int k, T v) { stsh<T>(smem, voff + uint32_t(oi[k]) * uint32_t(sizeof(T)), v); };
  // The same for an FP64 vector (the solution q in the FP32 refinement).
  auto put64 = [&](uint32_t voff, int k, double v) { stsh<double>(smem, voff + uint32_t(oi[k]) * 8u, v); };
  // End of an exchange round of the vector at byte offset voff, values of V: once every own value of
  // the round is stored, the send pass stores each requested value into its halo slot of the
  // requesting rank on that rank's barrier of this round; then warp 0 alone polls this rank's barrier
  // (every halo slot received) and the CTA barrier after it orders every thread's reads of the round's
  // own and received values after both (cheaper than 16 warps polling).
  auto round_end = [&](uint32_t voff, auto vtype) {
    using V = decltype(vtype);
    __syncthreads();
    const uint32_t bo = uint32_t(e & 1) * 8u;
    for (int i = tid; i < incoming; i += nt) {
      const uint2 en = sv<uint2>(smem, SENDL, i);
      const int rk = int(en.x >> 16);
      const V v = ldsh<V>(smem, voff + (en.x & 0xffffu) * uint32_t(sizeof(V)));
      st_async(C.rsmem[rk] + voff + (uint32_t(guard + 1) + en.y) * uint32_t(sizeof(V)), v, C.rxbar[rk] + bo);
    }
    const uint32_t bar = xb0 + bo;
    if (tid == 0) mbar_expect(bar, uint32_t(nh) * uint32_t(sizeof(V)));
    if (tid < 32) mbar_wait(bar, uint32_t(e >> 1) & 1u, ok);
    __syncthreads();
    e++;
  };
  // Sum of the six neighbour values of own cell k in the vector at byte offset voff (pairwise: three
  // dependent additions).
  auto nsum = [&](uint32_t voff, int k) -> T {
    const T x0 = ldsh<T>(smem, voff + nbo[k][0]), x1 = ldsh<T>(smem, voff + nbo[k][1]);
    const T x2 = ldsh<T>(smem, voff + nbo[k][2]), x3 = ldsh<T>(smem, voff + nbo[k][3]);
    const T x4 = ldsh<T>(smem, voff + nbo[k][4]), x5 = ldsh<T>(smem, voff + nbo[k][5]);
    return ((x0 + x1) + (x2 + x3)) + (x4 + x5);
  };
  // A Chebyshev round whose output is the vector at byte offset out: cell(k) computes and stores this
  // thread's own cell k. The boundary cells come first; one CTA barrier later the send pass stores them
  // into the holding ranks' halos, and the interior cells are computed while those stores are in flight;
  // then warp 0 waits for this rank's halo and a CTA barrier orders the round's reads after it.
  auto cheb_round = [&](uint32_t out, auto&& cell) {
#pragma unroll
    for (int k = 0; k < K; k++)
      if (bnd[k]) cell(k);
    __syncthreads();
    const uint32_t bo = uint32_t(e & 1) * 8u;
    for (int i = tid; i < incoming; i += nt) {
      const uint2 en = sv<uint2>(smem, SENDL, i);
      const int rk = int(en.x >> 16);
      const T v = ldsh<T>(smem, out + (en.x & 0xffffu) * uint32_t(sizeof(T)));
      st_async(C.rsmem[rk] + out + (uint32_t(guard + 1) + en.y) * uint32_t(sizeof(T)), v, C.rxbar[rk] + bo);
    }
#pragma unroll
    for (int k = 0; k < K; k++)
      if (has[k] && !bnd[k]) cell(k);
    const uint32_t bar = xb0 + bo;
    if (tid == 0) mbar_expect(bar, uint32_t(nh) * uint32_t(sizeof(T)));
    if (tid < 32) mbar_wait(bar, uint32_t(e >> 1) & 1u, ok);
    __syncthreads();
    e++;
  };
  const T itheta = T(2.0 / (2.0 + a.cheb_lo));
  // z = p(D^-1 A) D^-1 r, published (own cells and halo) in ZS
  auto precondition = [&]() {
    uint32_t out = deg > 1 ? ((e & 1) ? DV1 : DV0) : ZS;
    cheb_round(out, [&](int k) {
      const T d = r[k] * idg[k] * itheta;
      cdown[k] = d;
      z[k] = d;
      res[k] = r[k];
      put(out, k, d);
    });
    uint32_t last = out;
    for (int s = 1; s < deg; s++) {
      const T c1 = sizeof(T) == 4 ? T(C.coef_f[s][0]) : T(C.coef[s][0]);
      const T c2 = sizeof(T) == 4 ? T(C.coef_f[s][1]) : T(C.coef[s][1]);
      const bool final_step = s + 1 == deg;
      out = final_step ? ZS : ((e & 1) ? DV1 : DV0);
      cheb_round(out, [&](int k) {
        const T acc = nsum(last, k);
        const T rs = res[k] - (dg[k] * cdown[k] - acc);
        res[k] = rs;
        const T d = c1 * cdown[k] + c2 * rs * idg[k];
        cdown[k] = d;
        z[k] += d;
        put(out, k, final_step ? z[k] : d);
      });
      last = out;
    }
  };
  // w = A z from the published z; partial z.r and z.w
  auto apply_z = [&](double* zr, double* zw) {
    double pr = 0, pw = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!has[k]) continue;
      w[k] = dg[k] * z[k] - nsum(ZS, k);
      pr += double(z[k]) * double(r[k]);
      pw += double(z[k]) * double(w[k]);
    }
    *zr = pr;
    *zw = pw;
  };
  const int cid = int(blockIdx.x) / ns;  // cluster of the launch (two when the jobs run in parallel)
  const int job0 = a.parallel ? cid : 0, job1 = a.parallel ? cid + 1 : a.jobs;
  for (int job = job0; job < job1; job++) {
  // job 0: the launch's first system (pressure, or the one system of a single-job launch); job 1:
  // the density correction of the same substep (same liquid cells, so the same exchange tables)
  const bool corr = job == 1 || a.is_correction;
  const double* jb = job == 0 ? a.b : a.b2;
  double* jq = job == 0 ? a.q : a.q2;
  const double jtol = job == 0 ? a.tol : a.tol2;
  const int jmax = job == 0 ? a.max_iter : a.max_iter2;
  if (job == 1) {
    if (me == 0 && tid == 0) {  // interior mean of the density ratios (solver3d.ts:670)
      if (!a.parallel) sc->t_solve[1] = globaltimer_ns();
      double s = 0;
      int n = 0;
      for (int b = 0; b < DENSITY_BLOCKS; b++) {
        s += P.interior_part[b];
        n += P.interior_cnt_part[b];
      }
      sc->interior = n > 0 ? s / n : 1.0;
      sc->interior_count = n;
    }
    if (!sc->corr_any) {  // solver3d.ts:671: no solve, uc = vc = wc = 0 (uniform: set before the launch)
      if (me == 0 && tid == 0) sc->corr_iters = 0;
      break;
    }
  }
  double bmax = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    b64[k] = has[k] ? jb[li_own[k]] : 0.0;
    r[k] = T(b64[k]);
    q[k] = 0;
    z[k] = res[k] = as[k] = sown[k] = cdown[k] = w[k] = T(0);
    bmax = dmax(bmax, fabs(b64[k]));
  }
  const double bnorm = reduce3(bmax, 0.0, 0.0, C, rr, me, ns, ok).x;
  int iters = 0, converged = 1;
  double res_norm = bnorm;
  if (m > 0 && !(bnorm < 1e-14)) {
    const double target = dmax(jtol * bnorm, 1e-14);
    converged = 0;
    int restarts = 0;
    bool fresh = true;
    double gamma, delta, gamma_prev = 1, alpha_prev = 1;
    {
      double zr, zw;
      precondition();
      apply_z(&zr, &zw);
      const double3 g3 = reduce3(0.0, zr, zw, C, rr, me, ns, ok);
      gamma = g3.y;
      delta = g3.z;
    }
    int it = 1;
    for (; it <= jmax; it++) {
      double beta = 0, sas = delta;
      if (!fresh) {
        beta = gamma / gamma_prev;
        sas = delta - beta * gamma / alpha_prev;
      }
      if (!(sas > 0)) break;  // breakdown (solver3d.ts:913)
      const double alpha = gamma / sas;
      const T tb = T(beta), ta = T(alpha);
      double rm = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (!has[k]) continue;
        sown[k] = z[k] + tb * sown[k];
        as[k] = w[k] + tb * as[k];
        q[k] += alpha * double(sown[k]);
        r[k] = r[k] - ta * as[k];
        rm = dmax(rm, fabs(double(r[k])));
      }
      double zr, zw;
      precondition();
      apply_z(&zr, &zw);
      const double3 g3 = reduce3(rm, zr, zw, C, rr, me, ns, ok);  // max|r|, z.r, z.w in one round
      res_norm = g3.x;
      // With FP32 vectors the recursive residual keeps falling after the FP64 true residual has
      // stalled above the target, so the first confirmation comes early, at CHEB_FIRST_CHECK times the
      // target, and the restart from the true residual finishes the solve; every later confirmation,
      // and the acceptance itself, use the target.
      const double trigger = sizeof(T) == 4 && restarts == 0 ? target * CHEB_FIRST_CHECK : target;
      if (res_norm <= trigger) {
        if constexpr (sizeof(T) == 8) {
          converged = 1;
          break;
        }
        if (restarts >= 4) {
          converged = 1;
          break;
        }
        // FP32 vectors: confirm with the FP64 true residual b - A q
#pragma unroll
        for (int k = 0; k < K; k++)
          if (has[k]) put64(QS, k, q[k]);
        round_end(QS, 0.0);
        double tm = 0;
        T rt[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          rt[k] = T(0);
          if (!has[k]) continue;
          constexpr uint32_t sc8 = 8 / sizeof(T);  // FP64 offsets from the T offsets
          const double acc =
              ((ldsh<double>(smem, QS + nbo[k][0] * sc8) + ldsh<double>(smem, QS + nbo[k][1] * sc8)) +
               (ldsh<double>(smem, QS + nbo[k][2] * sc8) + ldsh<double>(smem, QS + nbo[k][3] * sc8))) +
              (ldsh<double>(smem, QS + nbo[k][4] * sc8) + ldsh<double>(smem, QS + nbo[k][5] * sc8));
          const double rd = b64[k] - (double(dg[k]) * q[k] - acc);
          tm = dmax(tm, fabs(rd));
          rt[k] = T(rd);
        }
        const double tres = reduce3(tm, 0.0, 0.0, C, rr, me, ns, ok).x;
        if (tres <= target) {
          res_norm = tres;
          converged = 1;
          break;
        }
        restarts++;
#pragma unroll
        for (int k = 0; k < K; k++) r[k] = rt[k];
        precondition();
        apply_z(&zr, &zw);
        const double3 h3 = reduce3(0.0, zr, zw, C, rr, me, ns, ok);
        gamma = h3.y;
        delta = h3.z;
        fresh = true;
        continue;
      }
      gamma_prev = gamma;
      gamma = g3.y;
      delta = g3.z;
      alpha_prev = alpha;
      fresh = false;
    }
    iters = converged ? it : jmax;
    if (!converged) converged = res_norm <= target ? 1 : 0;
  }
#pragma unroll
  for (int k = 0; k < K; k++)
    if (has[k]) jq[li_own[k]] = q[k];
  if (me == 0 && tid == 0) {
    if (corr) {
      sc->corr_iters = iters;
      sc->corr_residual = res_norm;
    } else {
      sc->last_iters = iters;
      sc->last_residual = res_norm;
      if (!converged) sc->failures++;
    }
  }
  }  // jobs
  if (!ok) atomicOr(&sc->errors, ERR_SOLVER_TIMEOUT);  // (exchange waits run in warp 0)
  if (me == 0 && tid == 0) {
    if (cid == 0) {
      const unsigned long long t = globaltimer_ns();
      sc->t_solve[2] = t;
      // one system, or two overlapping ones: the launch's time stays with the solve stage
      if (a.jobs < 2 || a.parallel || !sc->corr_any) sc->t_solve[1] = t;
    }
    sc->mg_status = 1;
  }
  cl.sync();  // no rank leaves while another may still address its shared memory
  // after a wait gave up anywhere in the cluster, stores of skipped rounds may still be in flight:
  // let them land before the shared memory is released
  if (tid == 0 && (*reinterpret_cast<volatile int*>(&sc->errors) & ERR_SOLVER_TIMEOUT))
    for (int i = 0; i < 100; i++) __nanosleep(10000);
}

namespace {

template <typename T, int K>
void configure_one() {
  cudaFuncSetAttribute(k_chebpcg<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, CHEB_SMEM);
  cudaFuncSetAttribute(k_chebpcg<T, K>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

template <int K>
void launch_k(const Geo& g, const DevPtrs& P, const SolverWs& W, const ChebArgs& a, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.cluster * (a.parallel ? 2 : 1));
  cfg.blockDim = dim3(std::min(a.threads, CHEB_MAX_THREADS / K));
  cfg.dynamicSmemBytes = a.smem_bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = a.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (a.mixed)
    cudaLaunchKernelEx(&cfg, k_chebpcg<float, K>, g, P, W, a);
  else
    cudaLaunchKernelEx(&cfg, k_chebpcg<double, K>, g, P, W, a);
}

void launch_cells(int K, const Geo& g, const DevPtrs& P, const SolverWs& W, const ChebArgs& a, cudaStream_t st) {
  if (K == 1)
    launch_k<1>(g, P, W, a, st);
  else if (K == 2)
    launch_k<2>(g, P, W, a, st);
  else
    launch_k<4>(g, P, W, a, st);
}

// Cells the launch with K cells per thread can hold.
int capacity(const ChebArgs& a, int K) { return a.cluster * std::min(a.threads, CHEB_MAX_THREADS / K) * K; }

}  // namespace

void cheb_configure() {
  configure_one<double, 1>();
  configure_one<double, 2>();
  configure_one<double, 4>();
  configure_one<float, 1>();
  configure_one<float, 2>();
  configure_one<float, 4>();
}

// The launch sized for a.m_bound liquid cells, then (gated on the device) one with four cells per
// thread for a pour that exceeds it; the wavefront solver launched after these takes any system
// neither could hold.
void launch_cheb_solve(const Geo& g, const DevPtrs& P, const SolverWs& W, const ChebArgs& a, cudaStream_t st) {
  int K = 1;
  while (K < CHEB_KMAX && capacity(a, K) < a.m_bound) K *= 2;
  launch_cells(K, g, P, W, a, st);
  if (K < CHEB_KMAX && capacity(a, CHEB_KMAX) > capacity(a, K)) {
    ChebArgs b = a;
    b.gate = 1;
    launch_cells(CHEB_KMAX, g, P, W, b, st);
  }
}

}  // namespace pl
