// Chebyshev-polynomial-preconditioned CG on one thread-block cluster: the fast pressure solve.
//
// Preconditioner: z = p(D^-1 A) D^-1 r, `degree` Chebyshev steps for D^-1 A on [lo, 2] from z = 0
// (the WebGPU port's preconditioner, src/gpu3d/shaders.ts:588-622). The polynomial is positive on
// (0, 2], so the preconditioner is symmetric positive definite and CG stays valid; every step is one
// 7-point stencil with no inner products. On these free-surface systems it needs about as many
// stencil applications as the best geometric multigrid variants while using a single level, so a
// CG iteration is `degree + 1` cluster phases and there is no hierarchy to build.
//
// Layout: the liquid list (index order) is split into `cluster` contiguous ranges, one per CTA, and
// each thread owns up to CHEB_KMAX cells of its CTA's range. Everything a cell needs only for itself
// (residuals, inverse diagonal, solution, neighbour indices) stays in the owning thread's registers;
// the stencil vectors (Chebyshev direction, z, CG direction, and q in FP32 mode) live in shared
// memory, own cells first, then a zero guard element, then one halo slot per reference to a cell of
// another CTA. A CTA never reads another CTA's shared memory while solving: whenever a thread
// computes a new value of a stencil vector it stores it locally and also writes it straight into the
// halo slots that reference it in other CTAs (DSMEM stores, which need no round trip), and the
// cluster barrier that ends the phase publishes both. The destinations of each cell are learnt once,
// in the prologue, from the other CTAs' requests. Vectors are double-buffered where a phase writes
// what the same phase reads.
//
// Reductions are deterministic: per-thread partials in cell order, warps in order, then each CTA's
// partial is written into every CTA's slot table and each CTA sums the slots in rank order.
//
// Stopping rule and bookkeeping: the reference's (solver3d.ts:858-937), max-norm residual
// <= max(tol * max|b|, 1e-14), breakdown if s.As <= 0; like the WebGPU port the preconditioner
// runs before the convergence test so that max|r| and z.r share one reduction. With FP32 vectors
// (PL_SOLVE_MIXED) a recursive-residual convergence is confirmed by the FP64 true residual
// b - A q and CG restarts from it when it misses the target (iterative refinement).
#include <cooperative_groups.h>

#include "cheb.h"

namespace cg = cooperative_groups;

namespace pl {

namespace {

struct Cl {
  char* base[CHEB_CLUSTER];  // generic address of every rank's dynamic shared memory
  double2 slot[2][CHEB_CLUSTER];
  double2 wpart[CHEB_MAX_THREADS / 32];
  int out_cnt[CHEB_CLUSTER];  // requests this rank sends to each owner
  int in_cnt[CHEB_CLUSTER];   // requests each rank sends to this rank
  int out_pos[CHEB_CLUSTER];  // running position of this rank's requests in each owner's table
  int nh;
  int hcap;
};

// Deterministic cluster-wide (max of x, sum of y) in one barrier.
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

// Element i of the shared-memory array at byte offset `off`.
template <typename V>
__device__ __forceinline__ V& sv(char* smem, uint32_t off, int i) {
  return reinterpret_cast<V*>(smem + off)[i];
}

}  // namespace

template <typename T>
__global__ void __launch_bounds__(CHEB_MAX_THREADS) k_chebpcg(Geo g, DevPtrs P, SolverWs W, ChebArgs a) {
  constexpr int K = CHEB_KMAX;
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
  const int nt = int(blockDim.x);
  extern __shared__ __align__(16) char smem[];
  __shared__ Cl C;
  __shared__ int s_warp[CHEB_MAX_THREADS / 32];
  const int m = sc->m;
  const int chunk = m > 0 ? (m + ns - 1) / ns : 1;
  const int own0 = me * chunk;
  const int cnt = m > own0 ? min(own0 + chunk, m) - own0 : 0;
  const int guard = chunk;  // element [chunk] of every stencil vector is 0; halo slots follow it
  if ((chunk + nt - 1) / nt > K) {  // uniform: more cells per thread than registers hold
    if (me == 0 && threadIdx.x == 0) sc->mg_status = 0;
    return;
  }
  if (threadIdx.x < ns) {
    C.base[threadIdx.x] = (char*)cl.map_shared_rank((void*)smem, int(threadIdx.x));
    C.out_cnt[threadIdx.x] = 0;
    C.out_pos[threadIdx.x] = 0;
  }
  __syncthreads();
  int phase = 0;  // reduction slot parity (advances identically in every thread)
  // ---- own cells: t_k = threadIdx.x + k * nt
  int gnb[K][6];  // neighbour list indices (prologue only)
  int myrem = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int t = threadIdx.x + k * nt;
#pragma unroll
    for (int e = 0; e < 6; e++) {
      int gi = t < cnt ? W.nb[e * W.cap + own0 + t] : -1;
      gnb[k][e] = gi;
      if (gi >= 0 && gi / chunk != me) {
        myrem++;
        atomicAdd(&C.out_cnt[gi / chunk], 1);
      }
    }
  }
  // halo slots: block-exclusive scan of the per-thread remote counts
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = nt >> 5;
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
    C.nh = acc;
  }
  // tell every owner how many requests it gets from this rank
  if (threadIdx.x < ns) {
    Cl* dst = cl.map_shared_rank(&C, int(threadIdx.x));
    dst->in_cnt[me] = C.out_cnt[threadIdx.x];
  }
  __syncthreads();
  int hslot = s_warp[wid] + x - myrem;
  int incoming = 0;
  cl.sync();  // in_cnt complete everywhere
  for (int r = 0; r < ns; r++) incoming += C.in_cnt[r];
  const double2 caps = reduce2(double(C.nh), double(0), C, phase, me, ns, cl);
  const int hcap = int(caps.x);
  int inmax = int(reduce2(double(incoming), 0.0, C, phase, me, ns, cl).x);
  // ---- layout (identical in every rank): byte offsets into the dynamic shared memory
  uint32_t off = 0;
  auto take = [&](size_t bytes) -> uint32_t {
    uint32_t r = off;
    off += uint32_t((bytes + 15) & ~size_t(15));
    return r;
  };
  const int n1 = chunk + 1 + hcap;  // own cells, guard, halo
  const uint32_t CD0 = take(size_t(n1) * sizeof(T)), CD1 = take(size_t(n1) * sizeof(T));
  const uint32_t ZS = take(size_t(n1) * sizeof(T));
  const uint32_t S0 = take(size_t(n1) * sizeof(T)), S1 = take(size_t(n1) * sizeof(T));
  const uint32_t QS = take(size_t(n1) * 8);
  const uint32_t DCNT = take(size_t(chunk) * 4);
  const uint32_t DST = take(size_t(chunk) * 24);       // up to 6 destinations per own cell
  const uint32_t REQ = take(size_t(inmax) * 8 + 8);  // (own local index, rank << 16 | slot)
  if (off > uint32_t(a.smem_bytes) || n1 > 65535) {  // uniform decision: the wavefront solver takes over
    if (me == 0 && threadIdx.x == 0) sc->mg_status = 0;
    cl.sync();
    return;
  }
  // my requests' offset in each owner's table: the requests of lower ranks come first
  if (threadIdx.x < ns) {
    const Cl* own = cl.map_shared_rank(&C, int(threadIdx.x));
    int o = 0;
    for (int r = 0; r < me; r++) o += own->in_cnt[r];
    C.out_pos[threadIdx.x] = o;
  }
  for (int i = threadIdx.x; i < n1; i += nt) {
    sv<T>(smem, CD0, i) = sv<T>(smem, CD1, i) = sv<T>(smem, ZS, i) = T(0);
    sv<T>(smem, S0, i) = sv<T>(smem, S1, i) = T(0);
    sv<double>(smem, QS, i) = 0;
  }
  for (int i = threadIdx.x; i < chunk; i += nt) sv<int>(smem, DCNT, i) = 0;
  __syncthreads();
  // ---- requests: for each reference to another rank's cell, a halo slot here and an entry there
  uint32_t nbl[K][3];  // local indices, two 16-bit halves per word
#pragma unroll
  for (int k = 0; k < K; k++) {
    int li[6];
#pragma unroll
    for (int e = 0; e < 6; e++) {
      const int gi = gnb[k][e];
      if (gi < 0) {
        li[e] = guard;
      } else {
        const int rk = gi / chunk;
        if (rk == me) {
          li[e] = gi - own0;
        } else {
          const int h = hslot++;
          li[e] = guard + 1 + h;
          const int pos = atomicAdd(&C.out_pos[rk], 1);
          char* owner = C.base[rk];
          reinterpret_cast<uint2*>(owner + REQ)[pos] = make_uint2(uint32_t(gi - rk * chunk), (uint32_t(me) << 16) | uint32_t(h));
        }
      }
    }
    nbl[k][0] = uint32_t(li[0]) | (uint32_t(li[1]) << 16);
    nbl[k][1] = uint32_t(li[2]) | (uint32_t(li[3]) << 16);
    nbl[k][2] = uint32_t(li[4]) | (uint32_t(li[5]) << 16);
  }
  cl.sync();  // every request is in its owner's table
  for (int i = threadIdx.x; i < incoming; i += nt) {
    const uint2 rq = sv<uint2>(smem, REQ, i);
    const int p = atomicAdd(&sv<int>(smem, DCNT, int(rq.x)), 1);
    sv<uint32_t>(smem, DST, p * chunk + int(rq.x)) = rq.y;
  }
  __syncthreads();
  // ---- per-thread state of the owned cells
  T r[K], z[K], res[K], as[K], sown[K], cdown[K], idg[K], dg[K];
  double q[K], b64[K];
  int ndst[K];
  double bmax = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int t = threadIdx.x + k * nt;
    const bool ok = t < cnt;
    const double d = ok ? W.adiag[own0 + t] : 1.0;
    dg[k] = T(d);
    idg[k] = T(1) / T(d);
    b64[k] = ok ? a.b[own0 + t] : 0.0;
    r[k] = T(b64[k]);
    q[k] = 0;
    z[k] = res[k] = as[k] = sown[k] = cdown[k] = T(0);
    ndst[k] = ok ? sv<int>(smem, DCNT, t) : 0;
    bmax = dmax(bmax, fabs(b64[k]));
  }
  // Store v as own cell t_k of the vector at `voff` and into the halo slots that reference it.
  auto put = [&](uint32_t voff, int k, auto v) {
    using V = decltype(v);
    const int t = threadIdx.x + k * nt;
    sv<V>(smem, voff, t) = v;
    for (int j = 0; j < ndst[k]; j++) {
      const uint32_t d = sv<uint32_t>(smem, DST, j * chunk + t);
      reinterpret_cast<V*>(C.base[d >> 16] + voff)[guard + 1 + int(d & 0xffffu)] = v;
    }
  };
  auto nsum = [&](uint32_t voff, int k) -> T {
    const uint32_t w0 = nbl[k][0], w1 = nbl[k][1], w2 = nbl[k][2];
    return sv<T>(smem, voff, w0 & 0xffff) + sv<T>(smem, voff, w0 >> 16) + sv<T>(smem, voff, w1 & 0xffff) +
           sv<T>(smem, voff, w1 >> 16) + sv<T>(smem, voff, w2 & 0xffff) + sv<T>(smem, voff, w2 >> 16);
  };
  const double bnorm = reduce2(bmax, 0.0, C, phase, me, ns, cl).x;
  const double lo = a.cheb_lo, hi = 2.0;
  const double theta = (hi + lo) / 2, delta = (hi - lo) / 2;
  const double sigma1 = theta / delta;
  const int deg = a.degree;
  int iters = 0, converged = 1;
  double res_norm = bnorm;
  if (m > 0 && !(bnorm < 1e-14)) {
    const double target = dmax(a.tol * bnorm, 1e-14);
    converged = 0;
    int cur = 0;  // CG direction buffer holding the current s
    double sigma = 0, beta = 0;
    int restarts = 0;
    bool fresh = true;  // s restarts from z
    const T itheta = T(1.0 / theta);
    // z = p(D^-1 A) D^-1 r; ends with z in ZS (own and halo), returns partial z.r and max|r|
    auto precondition = [&](double* zr_out, double* rmax_out) {
      int cdb = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (threadIdx.x + k * nt >= cnt) continue;
        const T d = r[k] * idg[k] * itheta;
        cdown[k] = d;
        z[k] = d;
        res[k] = r[k];
        if (deg > 1) put(CD0, k, d);
      }
      double rho = 1 / sigma1;
      for (int s = 1; s < deg; s++) {
        cl.sync();  // the previous direction is published (own cells and halos)
        const uint32_t CO = cdb ? CD1 : CD0, CN = cdb ? CD0 : CD1;
        const double rhoN = 1 / (2 * sigma1 - rho);
        const T c1 = T(rhoN * rho), c2 = T(2 * rhoN / delta);
        T acc[K];
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = (threadIdx.x + k * nt < cnt) ? nsum(CO, k) : T(0);
#pragma unroll
        for (int k = 0; k < K; k++) {
          if (threadIdx.x + k * nt >= cnt) continue;
          const T rs = res[k] - (dg[k] * cdown[k] - acc[k]);
          res[k] = rs;
          const T d = c1 * cdown[k] + c2 * rs * idg[k];
          cdown[k] = d;
          z[k] += d;
          if (s + 1 < deg) put(CN, k, d);
        }
        cdb ^= 1;
        rho = rhoN;
      }
      double zr = 0, rm = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (threadIdx.x + k * nt >= cnt) continue;
        put(ZS, k, z[k]);
        zr += double(z[k]) * double(r[k]);
        rm = dmax(rm, fabs(double(r[k])));
      }
      *zr_out = zr;
      *rmax_out = rm;
    };
    int it = 1;
    {
      double zr, rm;
      precondition(&zr, &rm);
      sigma = reduce2(0.0, zr, C, phase, me, ns, cl).y;  // its barrier publishes z
    }
    for (; it <= a.max_iter; it++) {
      // s = z + beta s and As = A s, the neighbours' s formed from their published z and old s
      const T tb = T(fresh ? 0.0 : beta);
      const uint32_t SO = cur ? S1 : S0, SN = cur ? S0 : S1;
      double sp = 0;
      T az[K], aso[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        const bool ok = threadIdx.x + k * nt < cnt;
        az[k] = ok ? nsum(ZS, k) : T(0);
        aso[k] = ok ? nsum(SO, k) : T(0);
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (threadIdx.x + k * nt >= cnt) continue;
        const T st = z[k] + tb * sown[k];
        const T av = dg[k] * st - (az[k] + tb * aso[k]);
        sown[k] = st;
        as[k] = av;
        put(SN, k, st);
        sp += double(st) * double(av);
      }
      cur ^= 1;
      fresh = false;
      const double sas = reduce2(0.0, sp, C, phase, me, ns, cl).y;
      if (!(sas > 0)) break;
      const double alpha = sigma / sas;
      const T ta = T(alpha);
#pragma unroll
      for (int k = 0; k < K; k++) {
        q[k] += alpha * double(sown[k]);
        r[k] = r[k] - ta * as[k];
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
#pragma unroll
        for (int k = 0; k < K; k++)
          if (threadIdx.x + k * nt < cnt) put(QS, k, q[k]);
        cl.sync();
        double tm = 0;
        T rt[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
          rt[k] = T(0);
          if (threadIdx.x + k * nt >= cnt) continue;
          const uint32_t w0 = nbl[k][0], w1 = nbl[k][1], w2 = nbl[k][2];
          const double acc = sv<double>(smem, QS, w0 & 0xffff) + sv<double>(smem, QS, w0 >> 16) +
                             sv<double>(smem, QS, w1 & 0xffff) + sv<double>(smem, QS, w1 >> 16) +
                             sv<double>(smem, QS, w2 & 0xffff) + sv<double>(smem, QS, w2 >> 16);
          const double rd = b64[k] - (double(dg[k]) * q[k] - acc);
          tm = dmax(tm, fabs(rd));
          rt[k] = T(rd);
        }
        const double tres = reduce2(tm, 0.0, C, phase, me, ns, cl).x;
        if (tres <= target) {
          res_norm = tres;
          converged = 1;
          break;
        }
        restarts++;
#pragma unroll
        for (int k = 0; k < K; k++) r[k] = rt[k];
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
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int t = threadIdx.x + k * nt;
    if (t < cnt) a.q[own0 + t] = q[k];
  }
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
  cl.sync();  // no rank leaves while another may still write into its shared memory
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
