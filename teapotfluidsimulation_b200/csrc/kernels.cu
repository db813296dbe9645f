// Per-substep kernels of the pour engine except the pressure solver (solver.cu).
//
// Order inside one substep (engine.cu builds it into a CUDA graph):
//   k_controller      1 thread: stable dt, pour controller, pose (solver3d.ts:268-292)
//   k_bin_count       parcels -> bin key (cell, or a removed-parcel bin) + atomic count
//   k_scan_classify   one decoupled look-back scan over the bins: bin starts, cell types
//                     (solver3d.ts:313-336), the liquid-cell list and its size
//   k_bin_place       parcels -> (id, slot) at start[key] + atomic rank
//   k_bin_permute     canonical in-bin order by id, gather parcels into the sorted layout
//   k_p2g             one thread per face: deterministic gather of the weighted sums over the
//                     sorted parcels of the 18 neighbouring cells, normalise, gravity, wall
//                     velocity, valid mask (solver3d.ts:410-471, 545-562)
//   [pressure solve]  solver.cu
//   k_grad_ext1       u -= grad q and the first extrapolation layer (solver3d.ts:496-528, 565-605)
//   k_ext2            second extrapolation layer
//   k_density         density per liquid cell, correction rhs, interior statistics, max
//                     divergence (solver3d.ts:627-670, 473-493)
//   [correction solve] solver.cu
//   k_advect          FLIP/PIC grid-to-particle update, RK2 advection with the correction
//                     velocity, SDF collision, symmetry plane, discharge and spill accounting
//                     (solver3d.ts:607-624, 677-794)
// Every kernel returns at once when the controller marked the substep inactive, so a batch of
// graph launches can overshoot the end of an advance() call without changing the state.
#include <cstdio>

#include "common.cuh"
#include "controller.cuh"
#include "kernels.h"

namespace pl {

// ---------------------------------------------------------------- controller

__global__ void k_controller(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  bool forced = sc->force_step != 0;
  bool finished = sc->time >= g.duration - 1e-9;  // solver3d.ts:264-266
  bool active = forced || (sc->time < sc->end_time - 1e-12 && !finished);  // solver3d.ts:283
  sc->active = active ? 1 : 0;
  if (!active) return;
  // stableDt (solver3d.ts:268-278) from the max speed of the last advection
  double m = __longlong_as_double((long long)sc->max_speed_bits);
  double speed = sqrt(m) + sqrt(5 * g.h * g.gravity) + fabs(sc->omega) * g.R;
  double dt = dmin(g.max_substep, (g.cfl * g.h) / speed);
  dt = dmin(dt, g.duration - sc->time);  // solver3d.ts:284
  if (forced && sc->forced_dt > 0) dt = sc->forced_dt;
  sc->force_step = 0;
  sc->forced_dt = 0;
  // step(dt) (solver3d.ts:288-292)
  double discharged = sc->counts[DISCHARGED] * g.parcel_volume * 2;
  double tilt1 = ctl_advance(sc->motion, sc->ctl, sc->time + dt, dt, discharged);
  double phi1 = -tilt1;
  sc->omega = (phi1 - sc->phi) / dt;
  sc->dt = dt;
  sc->phi1 = phi1;
  sc->c0 = cos(sc->phi);
  sc->s0 = sin(sc->phi);
  sc->c1 = cos(phi1);
  sc->s1 = sin(phi1);
  // per-substep counters
  sc->max_speed_bits = 0;
  sc->max_div_bits = 0;
  sc->corr_any = 0;
  sc->corr_iters = 0;
  sc->scan_tile = 0;
  // commit the pose and clock (solver3d.ts:306-308); kernels of this substep read phi0 from c0/s0
  sc->phi = phi1;
  sc->time += dt;
  sc->steps += 1;
}

// ---------------------------------------------------------------- binning

// Bin key and FP64-derived cell fractions of a parcel. The cell is floor(x / h) in FP64 on the
// FP32 position (the oracle evaluates the same expression), clamped into the interior cells.
__device__ __forceinline__ int parcel_bin(const Geo& g, float4 p, float4* frac, int* outlier) {
  double gx = (double)p.x / g.h, gy = (double)p.y / g.h, gz = (double)p.z / g.h;
  double fx = floor(gx), fy = floor(gy), fz = floor(gz);
  double cx = dmin(dmax(fx, 1.0), (double)(g.nx - 2));
  double cy = dmin(dmax(fy, 1.0), (double)(g.ny - 2));
  double cz = dmin(dmax(fz, 1.0), (double)(g.nz - 2));
  *outlier = (cx != fx || cy != fy || cz != fz) ? 1 : 0;
  int ix = (int)cx, iy = (int)cy, iz = (int)cz;
  int key = ix + g.nx * (iy + g.ny * iz);
  frac->x = (float)dmin(dmax(gx - cx, 0.0), 1.0);
  frac->y = (float)dmin(dmax(gy - cy, 0.0), 1.0);
  frac->z = (float)dmin(dmax(gz - cz, 0.0), 1.0);
  frac->w = __int_as_float(key);
  return key;
}

__global__ void k_bin_count(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < SCAN_MAX_TILES) P.scan_state[s] = 0ull;
  if (g.tiled && s < g.ntx * g.nty * g.nz) P.tile_mask[s] = 0ull;
  if (s >= g.n) return;
  float4 p = P.pos_home[s];
  float4 v = P.vel_home[s];
  int status = __float_as_int(v.w) & 0xff;
  int id = __float_as_int(p.w);
  int key;
  if (status == IN_POT) {
    float4 fr;
    int outl;
    key = parcel_bin(g, p, &fr, &outl);
    if (outl) atomicAdd(&P.sc->outliers, 1);
    P.frac_tmp[s] = fr;
  } else {
    key = g.nc + (id & (REMOVED_BINS - 1));
    P.frac_tmp[s] = make_float4(0.f, 0.f, 0.f, __int_as_float(key));
  }
  P.key[s] = key;
  P.rank[s] = atomicAdd(&P.cnt[key], 1);
}

// Cell type (solver3d.ts:313-336): border or inside the walls at the current pose -> SOLID, else
// FLUID when an in-pot parcel is in it, else AIR. The SDF runs in FP64 with the reference's
// operation order so the classification matches the FP64 reference exactly.
__device__ __forceinline__ uint8_t classify_cell(const Geo& g, const SimScalars* sc, int c, bool occupied) {
  int i = c % g.nx;
  int j = (c / g.nx) % g.ny;
  int k = c / (g.nx * g.ny);
  if (i == 0 || j == 0 || k == 0 || i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1) return SOLID;
  double loc[3];
  to_local(g, sc->c0, sc->s0, DMUL(i + 0.5, g.h), DMUL(j + 0.5, g.h), DMUL(k + 0.5, g.h), loc);
  if (teapot_sdf(g, loc[0], loc[1], loc[2]) < 0) return SOLID;
  return occupied ? FLUID : AIR;
}

// Scan descriptors: bit 62-63 flag (1 aggregate, 2 inclusive prefix), bits 32-61 liquid cells,
// bits 0-31 parcels.
constexpr unsigned long long DESC_AGG = 1ull << 62, DESC_INC = 2ull << 62, DESC_VAL = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_classify(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  __shared__ int s_tile;
  __shared__ unsigned long long s_warp[SCAN_THREADS / 32];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(&sc->scan_tile, 1);
  __syncthreads();
  const int tile = s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b0 = tile * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  unsigned long long val[SCAN_ITEMS];
  uint8_t typ[SCAN_ITEMS];
  unsigned long long local = 0;
#pragma unroll
  for (int e = 0; e < SCAN_ITEMS; e++) {
    int b = b0 + e;
    unsigned long long v = 0;
    typ[e] = AIR;
    if (b < g.nbins) {
      int cn = P.cnt[b];
      P.cnt[b] = 0;
      v = (unsigned long long)(unsigned)cn;
      if (b < g.nc) {
        typ[e] = classify_cell(g, sc, b, cn > 0);
        if (typ[e] == FLUID) {
          v += 1ull << 32;
          if (g.tiled) {
            const int i = b % g.nx, j = (b / g.nx) % g.ny, k = b / (g.nx * g.ny);
            const int tp = ((j / TILE_W) * g.ntx + i / TILE_W) * g.nz + k;
            atomicOr(&P.tile_mask[tp], 1ull << ((j % TILE_W) * TILE_W + i % TILE_W));
          }
        }
      }
    }
    val[e] = v;
    local += v;
  }
  // block exclusive scan of the per-thread totals
  unsigned long long x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned long long w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < SCAN_THREADS / 32) s_warp[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  unsigned long long thread_excl = x - local + (warp > 0 ? s_warp[warp - 1] : 0ull);
  unsigned long long aggregate = s_warp[SCAN_THREADS / 32 - 1];
  // decoupled look-back (bounded waits)
  if (threadIdx.x == 0) {
    unsigned long long* desc = P.scan_state;
    if (tile == 0) {
      atomicExch(&desc[0], DESC_INC | aggregate);
      s_prefix = 0;
    } else {
      atomicExch(&desc[tile], DESC_AGG | aggregate);
      unsigned long long excl = 0;
      int j = tile - 1;
      int spins = 0;
      while (j >= 0) {
        unsigned long long d = ld_volatile_u64(&desc[j]);
        if ((d >> 62) == 0) {
          if (++spins > SPIN_LIMIT) {
            atomicOr(&sc->errors, ERR_SCAN_TIMEOUT);
            break;
          }
          continue;
        }
        excl += d & DESC_VAL;
        if ((d >> 62) == 2) break;
        j--;
      }
      atomicExch(&desc[tile], DESC_INC | (excl + aggregate));
      s_prefix = excl;
    }
  }
  __syncthreads();
  unsigned long long run = s_prefix + thread_excl;
#pragma unroll
  for (int e = 0; e < SCAN_ITEMS; e++) {
    int b = b0 + e;
    if (b < g.nbins) {
      P.start[b] = (int)(run & 0xffffffffull);
      if (b < g.nc) {
        int lpos = (int)((run >> 32) & 0x3fffffffull);
        P.cell[b] = typ[e];
        if (typ[e] == FLUID) {
          P.list[lpos] = b;
          P.lidx[b] = lpos;
        } else {
          P.lidx[b] = -1;
        }
        if (b == g.nc - 1) sc->m = lpos + (typ[e] == FLUID ? 1 : 0);
      }
    }
    run += val[e];
  }
}

__global__ void k_bin_place(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  int key = P.key[s];
  int id = __float_as_int(P.pos_home[s].w);
  P.placed[P.start[key] + P.rank[s]] = make_int2(id, s);
}

// In-bin order by parcel id (canonical, so the layout and every sum over it is deterministic):
// the rank of an entry is the number of entries of its bin with a smaller id.
__global__ void k_bin_permute(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  int2 e = P.placed[i];
  int key = P.key[e.y];
  int b0 = P.start[key], b1 = P.start[key + 1];
  int r = 0;
  for (int j = b0; j < b1; j++) r += P.placed[j].x < e.x ? 1 : 0;
  int dst = b0 + r;
  P.pos_sorted[dst] = P.pos_home[e.y];
  P.vel_sorted[dst] = P.vel_home[e.y];
  P.frac_sorted[dst] = P.frac_tmp[e.y];
}

// ---------------------------------------------------------------- particle-to-grid

// Weight along one axis of a parcel in cell `cell` with FP64-derived fraction f for a node at
// `node`; offset 0 (face axis) or 1/2 (cell-centred axis) as in solver3d.ts:352-360.
__device__ __forceinline__ double axis_weight(int node, int cell, float f, bool half) {
  int base = cell;
  double fr = f;
  if (half) {
    if (f >= 0.5f) {
      fr = (double)f - 0.5;
    } else {
      base = cell - 1;
      fr = (double)f + 0.5;
    }
  }
  int d = node - base;
  return d == 0 ? 1.0 - fr : d == 1 ? fr : -1.0;
}

__global__ void k_p2g(Geo g, DevPtrs P) {
  const SimScalars* sc = P.sc;
  if (!sc->active) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nf) return;
  Face F = decode_face(g, f);
  const int fc[3] = {F.i, F.j, F.k};
  const int nn[3] = {g.nx, g.ny, g.nz};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    lo[a] = max(fc[a] - 1, 1);
    hi[a] = min(a == F.comp ? fc[a] : fc[a] + 1, nn[a] - 2);
  }
  double sw = 0, swv = 0;
  for (int cz = lo[2]; cz <= hi[2]; cz++)
    for (int cy = lo[1]; cy <= hi[1]; cy++)
      for (int cx = lo[0]; cx <= hi[0]; cx++) {
        int c = cx + g.nx * (cy + g.ny * cz);
        int p0 = P.start[c], p1 = P.start[c + 1];
        for (int p = p0; p < p1; p++) {
          float4 fr = P.frac_sorted[p];
          double wx = axis_weight(F.i, cx, fr.x, F.comp != 0);
          double wy = axis_weight(F.j, cy, fr.y, F.comp != 1);
          double wz = axis_weight(F.k, cz, fr.z, F.comp != 2);
          if (wx < 0 || wy < 0 || wz < 0) continue;
          double w = wx * wy * wz;
          const float* vel = reinterpret_cast<const float*>(&P.vel_sorted[p]);
          sw += w;
          swv += w * (double)vel[F.comp];
        }
      }
  double val = sw > 1e-9 ? swv / sw : 0.0;  // solver3d.ts:429
  P.uprev[f] = (float)val;
  // cells on the two sides of the face
  int ia = F.i - (F.comp == 0), ja = F.j - (F.comp == 1), ka = F.k - (F.comp == 2);
  uint8_t a = cell_at(g, P.cell, ia, ja, ka);
  uint8_t b = cell_at(g, P.cell, F.i, F.j, F.k);
  // gravity on v faces next to liquid (solver3d.ts:433-443)
  if (F.comp == 1 && F.j >= 1 && F.j < g.ny && (a == FLUID || b == FLUID)) val -= g.gravity * sc->dt;
  // moving-wall velocity on faces touching solid (solver3d.ts:446-471)
  if (a == SOLID || b == SOLID) {
    if (F.comp == 0)
      val = -sc->omega * ((F.j + 0.5) * g.h - g.pwy);
    else if (F.comp == 1)
      val = sc->omega * ((F.i + 0.5) * g.h - g.pwx);
    else
      val = 0.0;
  }
  P.u[f] = (float)val;
  P.valid[f] = (a == SOLID || b == SOLID || a == FLUID || b == FLUID) ? 1 : 0;  // solver3d.ts:545-562
}

// ---------------------------------------------------------------- projection update + extrapolation

__device__ __forceinline__ double q_at(const DevPtrs& P, const double* ql, int c) {
  int t = P.lidx[c];
  return t >= 0 ? ql[t] : 0.0;
}

// Gradient term of face (comp, i, j, k) of potential ql: applyGradient (solver3d.ts:496-528).
__device__ __forceinline__ double grad_term(const Geo& g, const DevPtrs& P, const double* ql, int comp, int i,
                                            int j, int k) {
  if (comp == 0 && (i < 1 || i >= g.nx)) return 0.0;
  if (comp == 1 && (j < 1 || j >= g.ny)) return 0.0;
  if (comp == 2 && (k < 1 || k >= g.nz)) return 0.0;
  int b = i + g.nx * (j + g.ny * k);
  int a = comp == 0 ? b - 1 : comp == 1 ? b - g.nx : b - g.nx * g.ny;
  uint8_t ca = P.cell[a], cb = P.cell[b];
  if (ca == SOLID || cb == SOLID || (ca != FLUID && cb != FLUID)) return 0.0;
  return -(q_at(P, ql, b) - q_at(P, ql, a));
}

__device__ __forceinline__ double projected(const Geo& g, const DevPtrs& P, int comp, int i, int j, int k, int sx,
                                            int sy) {
  int f = comp_base(g, comp) + i + sx * (j + sy * k);
  return (double)P.u[f] + grad_term(g, P, P.q, comp, i, j, k);
}

__global__ void k_grad_ext1(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nf) return;
  Face F = decode_face(g, f);
  if (P.valid[f]) {
    P.uext[f] = (float)projected(g, P, F.comp, F.i, F.j, F.k, F.sx, F.sy);
    P.vext[f] = 1;
    return;
  }
  // first layer (solver3d.ts:574-594): average of the valid neighbours of the same component
  double s = 0;
  int n = 0;
  const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma unroll
  for (int d = 0; d < 6; d++) {
    int i = F.i + off[d][0], j = F.j + off[d][1], k = F.k + off[d][2];
    if (i < 0 || j < 0 || k < 0 || i >= F.sx || j >= F.sy || k >= F.sz) continue;
    int nf = f + off[d][0] + F.sx * (off[d][1] + F.sy * off[d][2]);
    if (!P.valid[nf]) continue;
    s += projected(g, P, F.comp, i, j, k, F.sx, F.sy);
    n++;
  }
  if (n > 0) {
    P.uext[f] = (float)(s / n);
    P.vext[f] = 1;
  } else {
    P.uext[f] = P.u[f];
    P.vext[f] = 0;
  }
}

__global__ void k_ext2(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nf) return;
  if (P.vext[f]) {
    P.u[f] = P.uext[f];
    return;
  }
  Face F = decode_face(g, f);
  double s = 0;
  int n = 0;
  const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma unroll
  for (int d = 0; d < 6; d++) {
    int i = F.i + off[d][0], j = F.j + off[d][1], k = F.k + off[d][2];
    if (i < 0 || j < 0 || k < 0 || i >= F.sx || j >= F.sy || k >= F.sz) continue;
    int nf = f + off[d][0] + F.sx * (off[d][1] + F.sy * off[d][2]);
    if (!P.vext[nf]) continue;
    s += (double)P.uext[nf];
    n++;
  }
  P.u[f] = n > 0 ? (float)(s / n) : P.uext[f];
}

// ---------------------------------------------------------------- density correction rhs

__global__ void __launch_bounds__(256) k_density(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  const int m = sc->m;
  __shared__ double s_sum[8];
  __shared__ int s_cnt[8];
  double isum = 0;
  int icnt = 0;
  int any = 0;
  double maxd = 0;
  const int nxy = g.nx * g.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int c = P.list[t];
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / nxy;
    // density: trilinear weights of parcels in the 27 neighbouring cells (solver3d.ts:633-642)
    double dens = 0;
    for (int cz = max(k - 1, 1); cz <= min(k + 1, g.nz - 2); cz++)
      for (int cy = max(j - 1, 1); cy <= min(j + 1, g.ny - 2); cy++)
        for (int cx = max(i - 1, 1); cx <= min(i + 1, g.nx - 2); cx++) {
          int cc = cx + g.nx * (cy + g.ny * cz);
          int p0 = P.start[cc], p1 = P.start[cc + 1];
          for (int p = p0; p < p1; p++) {
            float4 fr = P.frac_sorted[p];
            double wx = axis_weight(i, cx, fr.x, true);
            double wy = axis_weight(j, cy, fr.y, true);
            double wz = axis_weight(k, cz, fr.z, true);
            if (wx < 0 || wy < 0 || wz < 0) continue;
            dens += wx * wy * wz;
          }
        }
    P.density[t] = dens;
    double ratio = dens / 8;
    const uint8_t* cl = P.cell;
    bool interior = cl[c - 1] != AIR && cl[c + 1] != AIR && cl[c - g.nx] != AIR && cl[c + g.nx] != AIR &&
                    cl[c - nxy] != AIR && cl[c + nxy] != AIR;
    if (interior) {
      icnt++;
      isum += ratio;
    }
    double r = 0;
    if (g.kappa > 0 && (ratio > 1 || interior)) {
      r = (g.kappa * (ratio - 1) * g.h) / sc->dt;
      any = 1;
    }
    P.rhs[t] = r;
    // divergence after projection (solver3d.ts:473-493, 542)
    const float* u = P.u;
    int iu = i + (g.nx + 1) * (j + g.ny * k);
    int iv = g.nu + i + g.nx * (j + (g.ny + 1) * k);
    int iw = g.nu + g.nv + c;
    double d = (double)u[iu + 1] - (double)u[iu] + (double)u[iv + g.nx] - (double)u[iv] + (double)u[iw + nxy] -
               (double)u[iw];
    maxd = dmax(maxd, fabs(d));
  }
  // deterministic per-block partial sums (fixed shuffle tree, then warps in order)
  for (int o = 16; o > 0; o >>= 1) {
    isum += __shfl_down_sync(0xffffffffu, isum, o);
    icnt += __shfl_down_sync(0xffffffffu, icnt, o);
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_sum[warp] = isum;
    s_cnt[warp] = icnt;
  }
  if (any) atomicOr(&sc->corr_any, 1);
  if (maxd > 0) atomicMax(&sc->max_div_bits, (unsigned long long)__double_as_longlong(maxd));
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    int n = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) {
      s += s_sum[w];
      n += s_cnt[w];
    }
    P.interior_part[blockIdx.x] = s;
    P.interior_cnt_part[blockIdx.x] = n;
  }
}

// ---------------------------------------------------------------- advection

struct Sten {
  int base, sx, sxy;
  double fx, fy, fz;
};

// solver3d.ts:339-362 for component comp (0/1/2 = u/v/w faces)
__device__ __forceinline__ Sten face_stencil(const Geo& g, int comp, double x, double y, double z) {
  double ox = comp == 0 ? 0.0 : 0.5, oy = comp == 1 ? 0.0 : 0.5, oz = comp == 2 ? 0.0 : 0.5;
  int sx = g.nx + (comp == 0), sy = g.ny + (comp == 1), sz = g.nz + (comp == 2);
  double gx = x / g.h - ox, gy = y / g.h - oy, gz = z / g.h - oz;
  double i = dmax(0.0, dmin((double)(sx - 2), floor(gx)));
  double j = dmax(0.0, dmin((double)(sy - 2), floor(gy)));
  double k = dmax(0.0, dmin((double)(sz - 2), floor(gz)));
  Sten s;
  s.fx = dmax(0.0, dmin(1.0, gx - i));
  s.fy = dmax(0.0, dmin(1.0, gy - j));
  s.fz = dmax(0.0, dmin(1.0, gz - k));
  s.sx = sx;
  s.sxy = sx * sy;
  s.base = comp_base(g, comp) + (int)i + sx * ((int)j + sy * (int)k);
  return s;
}

__device__ __forceinline__ int corner(const Sten& s, int c) {
  return s.base + (c & 1) + ((c & 2) ? s.sx : 0) + ((c & 4) ? s.sxy : 0);
}
__device__ __forceinline__ double corner_w(const Sten& s, int c) {
  double wx = (c & 1) ? s.fx : 1 - s.fx;
  double wy = (c & 2) ? s.fy : 1 - s.fy;
  double wz = (c & 4) ? s.fz : 1 - s.fz;
  return wx * wy * wz;
}

// sample() without a valid mask (solver3d.ts:386-408)
__device__ __forceinline__ double sample(const Geo& g, const float* field, int comp, double x, double y, double z) {
  Sten s = face_stencil(g, comp, x, y, z);
  double all = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) all += corner_w(s, c) * (double)field[corner(s, c)];
  return all;
}

// sample() with the valid mask (solver3d.ts:386-408)
__device__ __forceinline__ double sample_valid(const Geo& g, const float* field, const uint8_t* valid, int comp,
                                               double x, double y, double z) {
  Sten s = face_stencil(g, comp, x, y, z);
  double acc = 0, ws = 0, all = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    int idx = corner(s, c);
    double w = corner_w(s, c);
    double fv = (double)field[idx];
    all += w * fv;
    if (valid[idx]) {
      acc += w * fv;
      ws += w;
    }
  }
  return ws > 1e-9 ? acc / ws : all;
}

// Correction velocity uc at face corners: the gradient of the correction potential evaluated on
// the fly (applyGradient into zeroed uc,vc,wc: solver3d.ts:629-631, 674).
__device__ __forceinline__ double sample_corr(const Geo& g, const DevPtrs& P, int comp, double x, double y,
                                              double z) {
  Sten s = face_stencil(g, comp, x, y, z);
  int sx = g.nx + (comp == 0), sy = g.ny + (comp == 1);
  double all = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    int local = corner(s, c) - comp_base(g, comp);
    int i = local % sx, j = (local / sx) % sy, k = local / (sx * sy);
    all += corner_w(s, c) * grad_term(g, P, P.qc, comp, i, j, k);
  }
  return all;
}

__device__ __forceinline__ void set_status(SimScalars* sc, int from, int to) {  // solver3d.ts:790-794
  atomicSub(&sc->counts[from], 1);
  atomicAdd(&sc->counts[to], 1);
}

__global__ void k_advect(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.n) return;
  float4 pos = P.pos_sorted[p];
  float4 vel = P.vel_sorted[p];
  int meta = __float_as_int(vel.w);
  int st = meta & 0xff;
  const double dt = sc->dt;
  if (st == DISCHARGED || st == SPILLED) {  // solver3d.ts:693-702
    if ((double)pos.y > -1) {
      double vy = (double)vel.y - g.gravity * dt;
      vel.y = (float)vy;
      pos.x = (float)((double)pos.x + (double)vel.x * dt);
      pos.y = (float)((double)pos.y + (double)vel.y * dt);
      pos.z = (float)((double)pos.z + (double)vel.z * dt);
    }
    P.pos_home[p] = pos;
    P.vel_home[p] = vel;
    return;
  }
  if (st != IN_POT) {
    P.pos_home[p] = pos;
    P.vel_home[p] = vel;
    return;
  }
  const double x0 = pos.x, y0 = pos.y, z0 = pos.z;
  double vx = vel.x, vy = vel.y, vz = vel.z;
  // gridToParticles (solver3d.ts:607-624): FLIP/PIC blend with valid-masked samples
  {
    const float* U = P.u;
    const float* UP = P.uprev;
    const uint8_t* V = P.valid;
    double un = sample_valid(g, U, V, 0, x0, y0, z0);
    double vn = sample_valid(g, U, V, 1, x0, y0, z0);
    double wn = sample_valid(g, U, V, 2, x0, y0, z0);
    double uo = sample_valid(g, UP, V, 0, x0, y0, z0);
    double vo = sample_valid(g, UP, V, 1, x0, y0, z0);
    double wo = sample_valid(g, UP, V, 2, x0, y0, z0);
    double a = g.flip;
    vx = (1 - a) * un + a * (vx + un - uo);
    vy = (1 - a) * vn + a * (vy + vn - vo);
    vz = (1 - a) * wn + a * (vz + wn - wo);
  }
  // advect (solver3d.ts:704-787)
  double loc0[3], loc1[3], out[3];
  to_local(g, sc->c0, sc->s0, x0, y0, z0, loc0);
  const float* U = P.u;
  double u1 = sample(g, U, 0, x0, y0, z0);
  double v1 = sample(g, U, 1, x0, y0, z0);
  double w1 = sample(g, U, 2, x0, y0, z0);
  double xm = x0 + 0.5 * dt * u1, ym = y0 + 0.5 * dt * v1, zm = z0 + 0.5 * dt * w1;
  double x1 = x0 + dt * sample(g, U, 0, xm, ym, zm);
  double y1 = y0 + dt * sample(g, U, 1, xm, ym, zm);
  double z1 = z0 + dt * sample(g, U, 2, xm, ym, zm);
  if (g.kappa > 0 && sc->corr_any) {
    x1 += dt * sample_corr(g, P, 0, x0, y0, z0);
    y1 += dt * sample_corr(g, P, 1, x0, y0, z0);
    z1 += dt * sample_corr(g, P, 2, x0, y0, z0);
  }
  const double c1 = sc->c1, s1 = sc->s1;
  const double margin = 0.1 * g.h, eps = 1e-4;
  to_local(g, c1, s1, x1, y1, z1, loc1);
  double d = teapot_sdf(g, loc1[0], loc1[1], loc1[2]);
  if (d < margin) {
    double gx = teapot_sdf(g, loc1[0] + eps, loc1[1], loc1[2]) - teapot_sdf(g, loc1[0] - eps, loc1[1], loc1[2]);
    double gy = teapot_sdf(g, loc1[0], loc1[1] + eps, loc1[2]) - teapot_sdf(g, loc1[0], loc1[1] - eps, loc1[2]);
    double gz = teapot_sdf(g, loc1[0], loc1[1], loc1[2] + eps) - teapot_sdf(g, loc1[0], loc1[1], loc1[2] - eps);
    double gl = js_hypot3(gx, gy, gz);
    if (!(gl != 0)) gl = 1;
    double push = margin - d;
    loc1[0] += (gx / gl) * push;
    loc1[1] += (gy / gl) * push;
    loc1[2] += (gz / gl) * push;
    to_world(g, c1, s1, loc1[0], loc1[1], loc1[2], out);
    x1 = out[0];
    y1 = out[1];
    z1 = out[2];
    double nwx = (c1 * gx - s1 * gy) / gl;
    double nwy = (s1 * gx + c1 * gy) / gl;
    double nwz = gz / gl;
    double wvx = -sc->omega * (y1 - g.pwy);
    double wvy = sc->omega * (x1 - g.pwx);
    double rn = (vx - wvx) * nwx + (vy - wvy) * nwy + vz * nwz;
    if (rn < 0) {
      vx -= rn * nwx;
      vy -= rn * nwy;
      vz -= rn * nwz;
    }
  }
  if (z1 < g.h) {  // symmetry plane
    z1 = 2 * g.h - z1;
    vz = fabs(vz);
  }
  vel.x = (float)vx;
  vel.y = (float)vy;
  vel.z = (float)vz;
  if (!isfinite(x1 + y1 + z1)) {
    set_status(sc, IN_POT, LOST);
    vel.w = __int_as_float((meta & ~0xff) | LOST);
    P.pos_home[p] = pos;
    P.vel_home[p] = vel;
    return;
  }
  pos.x = (float)x1;
  pos.y = (float)y1;
  pos.z = (float)z1;
  // status tests on the stored (FP32) position, as the next substep will see it
  x1 = pos.x;
  y1 = pos.y;
  z1 = pos.z;
  to_local(g, c1, s1, x1, y1, z1, loc1);
  double s0d = (loc0[0] - g.tipx) * g.dx + (loc0[1] - g.tipy) * g.dy;
  double s1d = (loc1[0] - g.tipx) * g.dx + (loc1[1] - g.tipy) * g.dy;
  int new_st = IN_POT;
  if (s0d < 0 && s1d >= 0) {
    double rx = loc1[0] - g.tipx - s1d * g.dx;
    double ry = loc1[1] - g.tipy - s1d * g.dy;
    if (js_hypot3(rx, ry, loc1[2]) < g.bore + 3 * g.wall) new_st = DISCHARGED;
  }
  if (new_st == IN_POT) {
    double r = js_hypot2(loc1[0], loc1[2]);
    bool inside_body = r < g.radius + 2 * g.wall && loc1[1] > -2 * g.wall;
    bool near_spout = loc1[0] > 0 && loc1[0] < g.tipx + 0.03;
    double lo = g.h * 1.01;
    bool at_edge = x1 <= lo || y1 <= lo || x1 >= (g.nx - 1) * g.h || y1 >= (g.ny - 1) * g.h ||
                   z1 >= (g.nz - 1) * g.h;
    if ((!inside_body && !near_spout) || at_edge) new_st = SPILLED;
  }
  if (new_st != IN_POT) {
    set_status(sc, IN_POT, new_st);
    if (new_st == DISCHARGED) atomicAdd(&sc->by_origin[(meta >> 8) & 0xff], 1);
    vel.w = __int_as_float((meta & ~0xff) | new_st);
  } else {
    double sp = vx * vx + vy * vy + vz * vz;  // stableDt (solver3d.ts:269-274) of the next substep
    atomicMax(&sc->max_speed_bits, (unsigned long long)__double_as_longlong(sp));
  }
  P.pos_home[p] = pos;
  P.vel_home[p] = vel;
}

// ---------------------------------------------------------------- render positions

// writePositions (src/gpu3d/shaders.ts:786-799): xyz of the simulated half then its mirror image,
// indexed by parcel id; parcels that fell out of the domain are moved far below the view.
__global__ void k_render(Geo g, DevPtrs P) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.n) return;
  float4 p = P.pos_home[s];
  int id = __float_as_int(p.w);
  float x = p.x, y = p.y, z = p.z;
  if (y < 0.0005f) y = -100.0f;
  int m = id + g.n;
  P.render[3 * id] = x;
  P.render[3 * id + 1] = y;
  P.render[3 * id + 2] = z;
  P.render[3 * m] = x;
  P.render[3 * m + 1] = y;
  P.render[3 * m + 2] = (float)(2.0 * g.h) - z;
}

// Correction face velocity for export: uc = -grad qc on applicable faces, 0 elsewhere.
__global__ void k_export_correction(Geo g, DevPtrs P, float* out) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nf) return;
  Face F = decode_face(g, f);
  out[f] = P.sc->corr_any ? (float)grad_term(g, P, P.qc, F.comp, F.i, F.j, F.k) : 0.0f;
}

// ---------------------------------------------------------------- launchers

static inline int blocks(int n, int t) { return (n + t - 1) / t; }

void launch_stage_bin(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_controller<<<1, 1, 0, st>>>(g, P);
  k_bin_count<<<blocks(max(max(g.n, SCAN_MAX_TILES), g.tiled ? g.ntx * g.nty * g.nz : 0), 256), 256, 0, st>>>(g, P);
  k_scan_classify<<<blocks(g.nbins, SCAN_TILE), SCAN_THREADS, 0, st>>>(g, P);
  k_bin_place<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
  k_bin_permute<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
}

void launch_stage_p2g(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_p2g<<<blocks(g.nf, 256), 256, 0, st>>>(g, P);
}

void launch_stage_extrap(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_grad_ext1<<<blocks(g.nf, 256), 256, 0, st>>>(g, P);
  k_ext2<<<blocks(g.nf, 256), 256, 0, st>>>(g, P);
}

void launch_stage_density(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_density<<<DENSITY_BLOCKS, 256, 0, st>>>(g, P);
}

void launch_stage_advect(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_advect<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
}

void launch_render(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_render<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
}

void launch_export_correction(const Geo& g, const DevPtrs& P, float* out, cudaStream_t st) {
  k_export_correction<<<blocks(g.nf, 256), 256, 0, st>>>(g, P, out);
}

}  // namespace pl
