// Chebyshev-polynomial-preconditioned CG on one 16-CTA thread-block cluster: the fast pressure solve.
//
// Preconditioner: z = p(D^-1 A) D^-1 r, `degree` Chebyshev steps for D^-1 A on [lo, 2] from z = 0
// (the WebGPU port's preconditioner, src/gpu3d/shaders.ts:588-622). The polynomial is positive on
// (0, 2], so the preconditioner is symmetric positive definite and CG stays valid; every step is one
// 7-point stencil with no inner products. On these free-surface systems it needs about as many
// stencil applications as the best geometric multigrid variants while using a single level, so
// each CG iteration is `degree + 1` cluster phases and there is no hierarchy to build.
//
// Layout: the liquid list (index order) is split into 16 contiguous ranges, one per CTA; every
// vector lives in the owning CTA's shared memory and neighbour values are read through DSMEM.
// A neighbour reference is (rank << 16 | local index); missing neighbours point at a guard element
// that is always 0, so stencils have no branches. Reductions are deterministic: warps in order,
// then each CTA's partial is written into every CTA's slot table and each CTA sums the 16 slots in
// rank order from its own shared memory.
//
// Stopping rule and bookkeeping: the reference's (solver3d.ts:858-937), max-norm residual
// <= max(tol * max|b|, 1e-14), breakdown if s.As <= 0; like the WebGPU port the preconditioner
// runs before the convergence test so that max|r| and z.r share one reduction. With FP32 vectors
// (PL_SOLVE_MIXED) a recursive-residual convergence is confirmed by the FP64 true residual
// b - A q and CG restarts from it when it misses the target (iterative refinement).
#include <cooperative_groups.h>

#include <type_traits>

#include "cheb.h"

namespace cg = cooperative_groups;

namespace pl {

namespace {

struct Cl {
  char* base[CHEB_CLUSTER];  // generic address of every rank's dynamic shared memory
  double2 slot[2][CHEB_CLUSTER];
  double2 wpart[CHEB_MAX_THREADS / 32];
};

// Deterministic cluster-wide (max of x, sum of y) in one barrier: warp shuffles, warps in order,
// then this CTA's partial into slot `me` of every rank and each rank sums the slots in rank order.
__device__ double2 reduce2(double mx, double sm, Cl& C, int& phase, int me, int ns, cg::cluster_group& cl) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
  }
  if ((threadIdx.x & 31) == 0) C.wpart[threadIdx.x >> 5] = make_double2(mx, sm);
  __syncthreads();
  const int sl = phase & 1;
  phase++;
  if (threadIdx.x < ns) {
    double2 t = make_double2(0.0, 0.0);
    for (int w = 0; w < int(blockDim.x >> 5); w++) {
      t.x = dmax(t.x, C.wpart[w].x);
      t.y += C.wpart[w].y;
    }
    Cl* dst = cl.map_shared_rank(&C, int(threadIdx.x));
    dst->slot[sl][me] = t;
  }
  cl.sync();
  double2 t = make_double2(0.0, 0.0);
  for (int r = 0; r < ns; r++) {
    t.x = dmax(t.x, C.slot[sl][r].x);
    t.y += C.slot[sl][r].y;
  }
  return t;
}

}  // namespace

// Element i of the shared-memory vector at byte offset `off` (explicitly in the shared state space).
template <typename T>
__device__ __forceinline__ T& sv(char* smem, uint32_t off, int i) {
  return reinterpret_cast<T*>(smem + off)[i];
}

template <typename T>
__global__ void __launch_bounds__(CHEB_MAX_THREADS) k_chebpcg(Geo g, DevPtrs P, SolverWs W, ChebArgs a) {
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
  extern __shared__ __align__(16) char smem[];
  __shared__ Cl C;
  __shared__ int s_warp[CHEB_MAX_THREADS / 32];
  __shared__ int s_nh;
  const int m = sc->m;
  const int chunk = m > 0 ? (m + ns - 1) / ns : 1;
  const int own0 = me * chunk;
  const int cnt = m > own0 ? min(own0 + chunk, m) - own0 : 0;
  const int guard = chunk;  // element [chunk] of every vector is 0; halo entries follow it
  if (threadIdx.x < ns) C.base[threadIdx.x] = (char*)cl.map_shared_rank((void*)smem, int(threadIdx.x));
  int phase = 0;  // reduction slot parity (advances identically in every thread)
  // ---- halo size: references to cells owned by other ranks (one slot per reference)
  int myrem = 0;
  for (int t = threadIdx.x; t < cnt; t += blockDim.x)
    for (int e = 0; e < 6; e++) {
      int gi = W.nb[e * W.cap + own0 + t];
      myrem += (gi >= 0 && gi / chunk != me) ? 1 : 0;
    }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = myrem;
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
    s_nh = acc;
  }
  __syncthreads();
  int hslot = s_warp[wid] + x - myrem;
  const int nh = s_nh;
  const int hcap = int(reduce2(double(nh), 0.0, C, phase, me, ns, cl).x);
  // ---- layout (identical in every rank): byte offsets into the dynamic shared memory
  uint32_t off = 0;
  auto take = [&](size_t bytes) -> uint32_t {
    uint32_t r = off;
    off += uint32_t((bytes + 15) & ~size_t(15));
    return r;
  };
  const int n1 = chunk + 1 + hcap;  // own cells, guard, halo
  const int no = chunk + 1;
  const uint32_t Q = take(size_t(n1) * 8), B64 = take(size_t(no) * 8);
  const uint32_t R = take(size_t(no) * sizeof(T)), Z = take(size_t(n1) * sizeof(T));
  const uint32_t RES = take(size_t(no) * sizeof(T)), AS = take(size_t(no) * sizeof(T));
  const uint32_t S0 = take(size_t(n1) * sizeof(T)), S1 = take(size_t(n1) * sizeof(T));
  const uint32_t D0 = take(size_t(n1) * sizeof(T)), D1 = take(size_t(n1) * sizeof(T));
  const uint32_t IDG = take(size_t(no) * sizeof(T)), DG = take(size_t(no) * 4);
  const uint32_t NB = take(size_t(no) * 12), HS = take(size_t(hcap) * 4 + 4);
  if (off > uint32_t(a.smem_bytes) || n1 > 65535) {  // uniform decision: the wavefront solver takes over
    if (me == 0 && threadIdx.x == 0) sc->mg_status = 0;
    cl.sync();
    return;
  }
  auto nbi = [&](int e, int t) -> int { return sv<uint16_t>(smem, NB, e * no + t); };
  // ---- load
  for (int i = threadIdx.x; i < n1; i += blockDim.x) {  // guard and halo slots start at zero
    sv<double>(smem, Q, i) = 0;
    sv<T>(smem, Z, i) = sv<T>(smem, S0, i) = sv<T>(smem, S1, i) = T(0);
    sv<T>(smem, D0, i) = sv<T>(smem, D1, i) = T(0);
  }
  double bmax = 0;
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
    const int gi0 = own0 + t;
    for (int e = 0; e < 6; e++) {
      int gi = W.nb[e * W.cap + gi0];
      int li;
      if (gi < 0) {
        li = guard;
      } else {
        int rk = gi / chunk;
        if (rk == me) {
          li = gi - own0;
        } else {
          sv<uint32_t>(smem, HS, hslot) = (uint32_t(rk) << 16) | uint32_t(gi - rk * chunk);
          li = guard + 1 + hslot;
          hslot++;
        }
      }
      sv<uint16_t>(smem, NB, e * no + t) = uint16_t(li);
    }
    float d = float(W.adiag[gi0]);
    sv<float>(smem, DG, t) = d;
    sv<T>(smem, IDG, t) = T(1) / T(d);
    double bv = a.b[gi0];
    sv<double>(smem, B64, t) = bv;
    sv<T>(smem, R, t) = T(bv);
    bmax = dmax(bmax, fabs(bv));
  }
  // Copy the other ranks' current values of the vector at `voff` into this rank's halo slots.
  // Each thread issues the DSMEM loads of up to PULL_UNROLL slots before storing any of them, so
  // their latencies overlap instead of forming one chain per slot.
  auto pull = [&](uint32_t voff, auto tag) {
    using V = decltype(tag);
    constexpr int U = PULL_UNROLL;
    const int nt = blockDim.x;
    for (int h0 = threadIdx.x; h0 < nh; h0 += U * nt) {
      V v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int h = h0 + u * nt;
        if (h < nh) {
          uint32_t src = sv<uint32_t>(smem, HS, h);
          v[u] = reinterpret_cast<const V*>(C.base[src >> 16] + voff)[src & 0xffffu];
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int h = h0 + u * nt;
        if (h < nh) sv<V>(smem, voff, guard + 1 + h) = v[u];
      }
    }
  };
  const double bnorm = reduce2(bmax, 0.0, C, phase, me, ns, cl).x;  // its barrier publishes the loads
  const double lo = a.cheb_lo, hi = 2.0;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2;
  const double sigma1 = theta / delta;
  const int deg = a.degree;
  int iters = 0, converged = 1;
  double res_norm = bnorm;
  if (m > 0 && !(bnorm < 1e-14)) {
    const double target = dmax(a.tol * bnorm, 1e-14);
    converged = 0;
    int cur = 0;  // current direction buffer
    int cdb = 0;  // current Chebyshev buffer
    double sigma = 0, beta = 0;
    int restarts = 0;
    bool fresh = true;  // s restarts from z
    const T itheta = T(1.0 / theta);
    // z = p(D^-1 A) D^-1 r on own cells; returns partial z.r and max|r|
    auto precondition = [&](double* zr_out, double* rmax_out) {
      {
        const uint32_t CD = cdb ? D1 : D0;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
          T rt = sv<T>(smem, R, t);
          T d = rt * sv<T>(smem, IDG, t) * itheta;
          sv<T>(smem, CD, t) = d;
          sv<T>(smem, Z, t) = d;
          sv<T>(smem, RES, t) = rt;
        }
      }
      double rho = 1 / sigma1;
      for (int k = 1; k < deg; k++) {
        cl.sync();  // neighbours' previous direction is published
        const uint32_t CO = cdb ? D1 : D0, CN = cdb ? D0 : D1;
        pull(CO, T(0));
        __syncthreads();
        const double rhoN = 1 / (2 * sigma1 - rho);
        const T c1 = T(rhoN * rho), c2 = T(2 * rhoN / delta);
        // two cells per pass: every load of both is issued before the first store
        const int nt = blockDim.x;
        for (int t0 = threadIdx.x; t0 < cnt; t0 += 2 * nt) {
          const int t1 = t0 + nt;
          const bool h1 = t1 < cnt;
          const int u1 = h1 ? t1 : t0;
          T a0 = sv<T>(smem, CO, nbi(0, t0)) + sv<T>(smem, CO, nbi(1, t0)) + sv<T>(smem, CO, nbi(2, t0)) +
                 sv<T>(smem, CO, nbi(3, t0)) + sv<T>(smem, CO, nbi(4, t0)) + sv<T>(smem, CO, nbi(5, t0));
          T a1 = sv<T>(smem, CO, nbi(0, u1)) + sv<T>(smem, CO, nbi(1, u1)) + sv<T>(smem, CO, nbi(2, u1)) +
                 sv<T>(smem, CO, nbi(3, u1)) + sv<T>(smem, CO, nbi(4, u1)) + sv<T>(smem, CO, nbi(5, u1));
          T c00 = sv<T>(smem, CO, t0), c01 = sv<T>(smem, CO, u1);
          T r0 = sv<T>(smem, RES, t0), r1 = sv<T>(smem, RES, u1);
          T g0 = T(sv<float>(smem, DG, t0)), g1 = T(sv<float>(smem, DG, u1));
          T i0 = sv<T>(smem, IDG, t0), i1 = sv<T>(smem, IDG, u1);
          T z0 = sv<T>(smem, Z, t0), z1 = sv<T>(smem, Z, u1);
          T rs0 = r0 - (g0 * c00 - a0), rs1 = r1 - (g1 * c01 - a1);
          T d0 = c1 * c00 + c2 * rs0 * i0, d1 = c1 * c01 + c2 * rs1 * i1;
          sv<T>(smem, RES, t0) = rs0;
          sv<T>(smem, CN, t0) = d0;
          sv<T>(smem, Z, t0) = z0 + d0;
          if (h1) {
            sv<T>(smem, RES, t1) = rs1;
            sv<T>(smem, CN, t1) = d1;
            sv<T>(smem, Z, t1) = z1 + d1;
          }
        }
        cdb ^= 1;
        rho = rhoN;
      }
      double zr = 0, rm = 0;
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        T rt = sv<T>(smem, R, t);
        zr += double(sv<T>(smem, Z, t)) * double(rt);
        rm = dmax(rm, fabs(double(rt)));
      }
      *zr_out = zr;
      *rmax_out = rm;
    };
    int it = 1;
    {
      double zr, rm;
      precondition(&zr, &rm);
      sigma = reduce2(0.0, zr, C, phase, me, ns, cl).y;
    }
    for (; it <= a.max_iter; it++) {
      // s = z + beta s; As = A s (neighbours' s formed on the fly from their z and old s)
      const T tb = T(fresh ? 0.0 : beta);
      const uint32_t SO = cur ? S1 : S0, SN = cur ? S0 : S1;
      pull(Z, T(0));
      if (!fresh) pull(SO, T(0));
      __syncthreads();
      double sp = 0;
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        T st = sv<T>(smem, Z, t) + tb * sv<T>(smem, SO, t);
        T acc = 0;
#pragma unroll
        for (int e = 0; e < 6; e++) {
          const int li = nbi(e, t);
          acc += sv<T>(smem, Z, li) + tb * sv<T>(smem, SO, li);
        }
        T av = T(sv<float>(smem, DG, t)) * st - acc;
        sv<T>(smem, SN, t) = st;
        sv<T>(smem, AS, t) = av;
        sp += double(st) * double(av);
      }
      cur ^= 1;
      fresh = false;
      const double sas = reduce2(0.0, sp, C, phase, me, ns, cl).y;
      if (!(sas > 0)) break;
      const double alpha = sigma / sas;
      const T ta = T(alpha);
      const uint32_t SC = cur ? S1 : S0;  // the direction just formed
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        sv<double>(smem, Q, t) += alpha * double(sv<T>(smem, SC, t));
        sv<T>(smem, R, t) = sv<T>(smem, R, t) - ta * sv<T>(smem, AS, t);
      }
      double zr, rm;
      precondition(&zr, &rm);
      const double2 both = reduce2(rm, zr, C, phase, me, ns, cl);  // max|r| and z.r in one barrier
      res_norm = both.x;
      if (res_norm <= target) {
        if (sizeof(T) == 8 || restarts >= 4) {
          converged = 1;
          break;
        }
        // FP32 vectors: confirm with the FP64 true residual b - A q
        pull(Q, double(0));
        __syncthreads();
        double tm = 0;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
          double acc = 0;
#pragma unroll
          for (int e = 0; e < 6; e++) acc += sv<double>(smem, Q, nbi(e, t));
          double rt = sv<double>(smem, B64, t) - (double(sv<float>(smem, DG, t)) * sv<double>(smem, Q, t) - acc);
          tm = dmax(tm, fabs(rt));
          sv<T>(smem, AS, t) = T(rt);
        }
        double tres = reduce2(tm, 0.0, C, phase, me, ns, cl).x;
        if (tres <= target) {
          res_norm = tres;
          converged = 1;
          break;
        }
        restarts++;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) sv<T>(smem, R, t) = sv<T>(smem, AS, t);
        precondition(&zr, &rm);
        sigma = reduce2(0.0, zr, C, phase, me, ns, cl).y;
        fresh = true;
        continue;
      }
      beta = both.y / sigma;
      sigma = both.y;
    }
    iters = converged ? it : a.max_iter;
    if (!converged) converged = res_norm <= target ? 1 : 0;
  }
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) a.q[own0 + t] = sv<double>(smem, Q, t);
  if (me == 0 && threadIdx.x == 0) {
    if (a.is_correction) {
      sc->corr_iters = iters;
      sc->corr_residual = res_norm;
    } else {
      sc->last_iters = iters;
      sc->last_residual = res_norm;
      if (!converged) sc->failures++;
    }
    sc->mg_status = 1;
  }
  cl.sync();  // no rank leaves while another may still read its shared memory
}

void cheb_configure() {
  cudaFuncSetAttribute(k_chebpcg<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, CHEB_SMEM);
  cudaFuncSetAttribute(k_chebpcg<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, CHEB_SMEM);
  cudaFuncSetAttribute(k_chebpcg<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(k_chebpcg<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

void launch_cheb_solve(const Geo& g, const DevPtrs& P, const SolverWs& W, const ChebArgs& a, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.cluster);
  cfg.blockDim = dim3(a.threads);
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
    cudaLaunchKernelEx(&cfg, k_chebpcg<float>, g, P, W, a);
  else
    cudaLaunchKernelEx(&cfg, k_chebpcg<double>, g, P, W, a);
}

}  // namespace pl
