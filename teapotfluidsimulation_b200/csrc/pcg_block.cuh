// The single-block MIC(0)-PCG solve (Pcg3D.solve, solver3d.ts:858-973) and the standalone solve's
// kernels, shared by the translation units that launch them: solver.cu (the engine's wavefront
// MIC(0) solve and pl_pcg_solve_device) and noalloc.cu (pl_pcg_solve_device_noalloc). Everything
// here has internal linkage, so each unit compiles its own copy into its own device module.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace pl {
namespace {

// ---------------------------------------------------------------- block reductions

struct Reducer {
  double* buf;  // 2 x 32 doubles in shared memory
  int phase;
  // Deterministic block sum / max: xor-butterfly inside each warp (every lane ends with the same
  // bits), then every thread folds the warp partials in warp order. Two alternating buffers make
  // one barrier per reduction sufficient.
  __device__ double sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    double* b = buf + 32 * (phase & 1);
    phase++;
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; w++) t += b[w];
    return t;
  }
  __device__ double max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    double* b = buf + 32 * (phase & 1);
    phase++;
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; w++) t = dmax(t, b[w]);
    return t;
  }
  __device__ int imin(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = ::min(v, __shfl_xor_sync(0xffffffffu, v, o));
    double* b = buf + 32 * (phase & 1);
    phase++;
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = (double)v;
    __syncthreads();
    int t = 0x7fffffff;
    int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; w++) t = ::min(t, (int)b[w]);
    return t;
  }
  __device__ int imax(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = ::max(v, __shfl_xor_sync(0xffffffffu, v, o));
    double* b = buf + 32 * (phase & 1);
    phase++;
    if ((threadIdx.x & 31) == 0) b[threadIdx.x >> 5] = (double)v;
    __syncthreads();
    int t = -0x7fffffff;
    int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; w++) t = ::max(t, (int)b[w]);
    return t;
  }
};

// ---------------------------------------------------------------- MIC(0) pieces

struct Coef {  // the reference's coefficient arrays around one liquid cell (all -1 or 0)
  int xm, xp, ym, yp, zm, zp;
};

__device__ __forceinline__ Coef nbrs(const SolverWs& W, int t) {
  Coef c;
  c.xm = W.nb[t];
  c.xp = W.nb[W.cap + t];
  c.ym = W.nb[2 * W.cap + t];
  c.yp = W.nb[3 * W.cap + t];
  c.zm = W.nb[4 * W.cap + t];
  c.zp = W.nb[5 * W.cap + t];
  return c;
}
__device__ __forceinline__ double cf(int idx) { return idx >= 0 ? -1.0 : 0.0; }
__device__ __forceinline__ double at(const double* v, int idx) { return idx >= 0 ? v[idx] : 0.0; }

// MIC(0) diagonal of one cell (solver3d.ts:884-900), tau = 0.97, from its three predecessors.
__device__ __forceinline__ double mic_pc(const SolverWs& W, int t) {
  const double tau = 0.97;
  Coef n = nbrs(W, t);
  double ai_m = cf(n.xm), aj_m = cf(n.ym), ak_m = cf(n.zm);
  // coefficients of the predecessors: aj[c-1], ak[c-1], ai[c-nx], ak[c-nx], ai[c-nxy], aj[c-nxy]
  double aj_x = n.xm >= 0 ? cf(W.nb[3 * W.cap + n.xm]) : 0.0;
  double ak_x = n.xm >= 0 ? cf(W.nb[5 * W.cap + n.xm]) : 0.0;
  double ai_y = n.ym >= 0 ? cf(W.nb[W.cap + n.ym]) : 0.0;
  double ak_y = n.ym >= 0 ? cf(W.nb[5 * W.cap + n.ym]) : 0.0;
  double ai_z = n.zm >= 0 ? cf(W.nb[W.cap + n.zm]) : 0.0;
  double aj_z = n.zm >= 0 ? cf(W.nb[3 * W.cap + n.zm]) : 0.0;
  double pi = at(W.pc, n.xm), pj = at(W.pc, n.ym), pk = at(W.pc, n.zm);
  double adiag = W.adiag[t];
  double e1 = DMUL(ai_m, pi), e2 = DMUL(aj_m, pj), e3 = DMUL(ak_m, pk);
  double tx = DMUL(DMUL(DMUL(ai_m, DADD(aj_x, ak_x)), pi), pi);
  double ty = DMUL(DMUL(DMUL(aj_m, DADD(ai_y, ak_y)), pj), pj);
  double tz = DMUL(DMUL(DMUL(ak_m, DADD(ai_z, aj_z)), pk), pk);
  double e = DSUB(DSUB(DSUB(DSUB(adiag, DMUL(e1, e1)), DMUL(e2, e2)), DMUL(e3, e3)), DMUL(tau, DADD(DADD(tx, ty), tz)));
  if (e < DMUL(0.25, adiag)) e = adiag;
  return e > 0 ? 1.0 / sqrt(e) : 0.0;
}

// y = A x on one cell (solver3d.ts:939-953), reference term order.
__device__ __forceinline__ double apply_a(const SolverWs& W, const double* x, int t) {
  Coef n = nbrs(W, t);
  double y = DMUL(W.adiag[t], x[t]);
  y = DADD(y, DMUL(cf(n.xp), at(x, n.xp)));
  y = DADD(y, DMUL(cf(n.xm), at(x, n.xm)));
  y = DADD(y, DMUL(cf(n.yp), at(x, n.yp)));
  y = DADD(y, DMUL(cf(n.ym), at(x, n.ym)));
  y = DADD(y, DMUL(cf(n.zp), at(x, n.zp)));
  y = DADD(y, DMUL(cf(n.zm), at(x, n.zm)));
  return y;
}

// z = M^-1 r with the MIC(0) factor (solver3d.ts:955-973): forward sweep over wavefronts in
// increasing order, backward sweep in decreasing order; one barrier per wavefront.
__device__ void mic_apply(const SolverWs& W, const double* r, double* z, int nlev, const int* lstart) {
  for (int L = 0; L < nlev; L++) {
    int a = lstart[L], b = lstart[L + 1];
    for (int idx = a + threadIdx.x; idx < b; idx += blockDim.x) {
      int t = W.order[idx];
      Coef n = nbrs(W, t);
      double v = r[t];
      v = DSUB(v, DMUL(DMUL(cf(n.xm), at(W.pc, n.xm)), at(W.qv, n.xm)));
      v = DSUB(v, DMUL(DMUL(cf(n.ym), at(W.pc, n.ym)), at(W.qv, n.ym)));
      v = DSUB(v, DMUL(DMUL(cf(n.zm), at(W.pc, n.zm)), at(W.qv, n.zm)));
      W.qv[t] = DMUL(v, W.pc[t]);
    }
    __syncthreads();
  }
  for (int L = nlev - 1; L >= 0; L--) {
    int a = lstart[L], b = lstart[L + 1];
    for (int idx = a + threadIdx.x; idx < b; idx += blockDim.x) {
      int t = W.order[idx];
      Coef n = nbrs(W, t);
      double pct = W.pc[t];
      double v = W.qv[t];
      v = DSUB(v, DMUL(DMUL(cf(n.xp), pct), at(z, n.xp)));
      v = DSUB(v, DMUL(DMUL(cf(n.yp), pct), at(z, n.yp)));
      v = DSUB(v, DMUL(DMUL(cf(n.zp), pct), at(z, n.zp)));
      z[t] = DMUL(v, pct);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- the solve (one block)

struct SolveOut {
  int iterations, converged;
  double residual;
};

// Pcg3D.solve body (solver3d.ts:858-937) for m liquid cells with workspace W.
__device__ SolveOut pcg_block(const SolverWs& W, int m, const double* b, double* q, double tol, int max_iter,
                              bool factor, Reducer& red, int* s_lstart, int* s_hist) {
  SolveOut out{0, 1, 0.0};
  const int tid = threadIdx.x, nt = blockDim.x;
  double bmax = 0;
  for (int t = tid; t < m; t += nt) {
    q[t] = 0;
    bmax = dmax(bmax, fabs(b[t]));
  }
  double bnorm = red.max(bmax);
  if (m == 0 || bnorm < 1e-14) {
    out.residual = bnorm;
    return out;
  }
  int nlev;
  if (factor) {
    // wavefront order: counting sort of the liquid cells by i + j + k
    int wlo = 0x7fffffff, whi = -0x7fffffff;
    for (int t = tid; t < m; t += nt) {
      int w = W.wave[t];
      wlo = ::min(wlo, w);
      whi = ::max(whi, w);
    }
    wlo = red.imin(wlo);
    whi = red.imax(whi);
    nlev = whi - wlo + 1;
    if (nlev > MAX_LEVELS) {  // cannot happen for grids with nx + ny + nz <= MAX_LEVELS
      out.converged = 0;
      out.iterations = -1;
      return out;
    }
    for (int L = tid; L <= nlev; L += nt) s_hist[L] = 0;
    __syncthreads();
    for (int t = tid; t < m; t += nt) atomicAdd(&s_hist[W.wave[t] - wlo], 1);
    __syncthreads();
    if (tid == 0) {
      int acc = 0;
      for (int L = 0; L < nlev; L++) {
        int c = s_hist[L];
        s_lstart[L] = acc;
        s_hist[L] = acc;
        acc += c;
      }
      s_lstart[nlev] = acc;
      W.nlev[0] = nlev;
      W.nlev[1] = wlo;
    }
    __syncthreads();
    for (int t = tid; t < m; t += nt) {
      int pos = atomicAdd(&s_hist[W.wave[t] - wlo], 1);
      W.order[pos] = t;
    }
    for (int L = tid; L <= nlev; L += nt) W.lstart[L] = s_lstart[L];
    __syncthreads();
    // MIC(0) factor, wavefront by wavefront
    for (int L = 0; L < nlev; L++) {
      for (int idx = s_lstart[L] + tid; idx < s_lstart[L + 1]; idx += nt) {
        int t = W.order[idx];
        W.pc[t] = mic_pc(W, t);
      }
      __syncthreads();
    }
  } else {
    nlev = W.nlev[0];
    for (int L = tid; L <= nlev; L += nt) s_lstart[L] = W.lstart[L];
    __syncthreads();
  }
  double* r = W.r;
  double* z = W.z;
  double* s = W.s;
  double* as = W.as;
  for (int t = tid; t < m; t += nt) r[t] = b[t];
  __syncthreads();
  mic_apply(W, r, z, nlev, s_lstart);
  double part = 0;
  for (int t = tid; t < m; t += nt) {
    s[t] = z[t];
    part = DADD(part, DMUL(z[t], r[t]));
  }
  double sigma = red.sum(part);  // also orders the s writes before the first apply_a
  const double target = dmax(tol * bnorm, 1e-14);
  double res = bnorm;
  for (int it = 1; it <= max_iter; it++) {
    double sp = 0;
    for (int t = tid; t < m; t += nt) {
      double a = apply_a(W, s, t);
      as[t] = a;
      sp = DADD(sp, DMUL(s[t], a));
    }
    double sas = red.sum(sp);
    if (!(sas > 0)) break;
    double alpha = sigma / sas;
    double rm = 0;
    for (int t = tid; t < m; t += nt) {
      q[t] = DADD(q[t], DMUL(alpha, s[t]));
      double rr = DSUB(r[t], DMUL(alpha, as[t]));
      r[t] = rr;
      rm = dmax(rm, fabs(rr));
    }
    res = red.max(rm);
    if (res <= target) {
      out.iterations = it;
      out.converged = 1;
      out.residual = res;
      return out;
    }
    mic_apply(W, r, z, nlev, s_lstart);
    double zp = 0;
    for (int t = tid; t < m; t += nt) zp = DADD(zp, DMUL(z[t], r[t]));
    double sn = red.sum(zp);
    double beta = sn / sigma;
    for (int t = tid; t < m; t += nt) s[t] = DADD(z[t], DMUL(beta, s[t]));
    sigma = sn;
    __syncthreads();
  }
  out.iterations = max_iter;
  out.converged = res <= target ? 1 : 0;
  out.residual = res;
  return out;
}

// ---------------------------------------------------------------- standalone solve kernels

// Liquid list of a caller's cell grid (index order) and the neighbour data, single block.
__global__ void k_standalone_prep(const uint8_t* cell, int nx, int ny, int nz, int* lidx, int* list, int* m_out) {
  // Sequential-order compaction by one block: chunked block scan over the grid.
  __shared__ int s_tot;
  __shared__ int s_warp[32];
  const int nc = nx * ny * nz;
  if (threadIdx.x == 0) s_tot = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nc; base += blockDim.x) {
    int c = base + threadIdx.x;
    int f = 0;
    if (c < nc) {
      int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
      bool interior = i > 0 && j > 0 && k > 0 && i < nx - 1 && j < ny - 1 && k < nz - 1;
      f = (interior && cell[c] == FLUID) ? 1 : 0;
    }
    int x = f;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = lane < nw ? s_warp[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    int pos = s_tot + x - f + (warp > 0 ? s_warp[warp - 1] : 0);
    if (c < nc) {
      lidx[c] = f ? pos : -1;
      if (f) list[pos] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_tot += s_warp[nw - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *m_out = s_tot;
}

__global__ void k_standalone_setup(const uint8_t* cell, const double* b, int nx, int ny, const int* lidx,
                                   const int* list, const int* m_ptr, SolverWs W, double* bl) {
  const int m = *m_ptr;
  const int nxy = nx * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int c = list[t];
    int i = c % nx, j = (c / nx) % ny, k = c / nxy;
    const int off[6] = {-1, 1, -nx, nx, -nxy, nxy};
    double d = 0;
    for (int e = 0; e < 6; e++) {
      W.nb[e * W.cap + t] = lidx[c + off[e]];
      if (cell[c + off[e]] != SOLID) d += 1;
    }
    W.adiag[t] = d;
    W.wave[t] = i + j + k;
    bl[t] = b[c];
  }
}

__global__ void __launch_bounds__(SOLVER_THREADS) k_standalone_pcg(SolverWs W, const int* m_ptr, const double* bl,
                                                                    double* ql, double tol, int max_iter,
                                                                    int* result, double* residual) {
  __shared__ double s_red[64];
  __shared__ int s_lstart[MAX_LEVELS + 1];
  __shared__ int s_hist[MAX_LEVELS + 1];
  Reducer red{s_red, 0};
  SolveOut o = pcg_block(W, *m_ptr, bl, ql, tol, max_iter, true, red, s_lstart, s_hist);
  if (threadIdx.x == 0) {
    result[0] = o.iterations;
    result[1] = o.converged;
    *residual = o.residual;
  }
}

__global__ void k_standalone_scatter(const int* lidx, const double* ql, double* q, int nc) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  int t = lidx[c];
  q[c] = t >= 0 ? ql[t] : 0.0;
}

}  // namespace
}  // namespace pl
