// Per-substep kernels of the pour engine except the pressure solver (solver.cu).
//
// Order inside one substep (engine.cu builds it into a CUDA graph):
//   k_controller      1 thread: stable dt, pour controller, pose (solver3d.ts:268-292)
//   k_bin_count       parcels -> bin key (cell, or a removed-parcel bin) + atomic count; cells ->
//                     SOLID/AIR by the border and SDF test
//   k_scan_classify   one decoupled look-back scan over the bins: bin starts, FLUID cells
//                     (solver3d.ts:313-336), occupancy, the liquid-cell list and its size
//   k_bin_place       parcels -> (id, slot) at start[key] + atomic rank
//   k_bin_permute     canonical in-bin order by id, gather parcels into the sorted layout
//   k_p2g_cells       one thread per (occupied cell, component): node partial sums of the cell's
//                     parcels (velocity components and density)
//   k_p2g             one thread per face: deterministic fixed-order sum of the partials of the
//                     18 neighbouring cells, normalise, gravity, wall velocity, valid mask
//                     (solver3d.ts:410-471, 545-562)
//   k_density         density per liquid cell, correction rhs, interior statistics
//                     (solver3d.ts:627-670): it depends only on the parcels and the cell types, so
//                     it runs before the solves
//   [pressure solve, correction solve]  solver.cu / cheb.cu (one cluster launch for both)
//   k_grad_ext1       u -= grad q, the first extrapolation layer, max divergence after projection,
//                     the correction face velocity -grad qc (solver3d.ts:496-528, 565-605, 473-493,
//                     674)
//   k_ext2            second extrapolation layer
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

// One thread. Every field is read once up front (independent loads, one L2 round trip) and the
// controller runs on local copies. The pose at the start of this substep is the last substep's new
// pose, whose cosine and sine that substep already formed: they are reused when the pose's bits are
// the ones they were formed for (the host setting a state clears that), so only the new pose's two
// transcendentals stay on this kernel's path.
__global__ void k_controller(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  const int force_step = sc->force_step;
  const double time = sc->time, end_time = sc->end_time, forced_dt = sc->forced_dt;
  const unsigned long long msb = sc->max_speed_bits;
  const double omega0 = sc->omega, phi = sc->phi, c1p = sc->c1, s1p = sc->s1;
  const unsigned long long phi_trig = sc->phi_trig_bits;
  const int ndis = sc->counts[DISCHARGED];
  const long long steps = sc->steps;
  const pl_motion motion = sc->motion;
  DevController ctl = sc->ctl;
  const bool forced = force_step != 0;
  const bool finished = time >= g.duration - 1e-9;  // solver3d.ts:264-266
  const bool active = forced || (time < end_time - 1e-12 && !finished);  // solver3d.ts:283
  sc->active = active ? 1 : 0;
  if (!active) return;
  // stableDt (solver3d.ts:268-278) from the max speed of the last advection
  double m = __longlong_as_double((long long)msb);
  double speed = sqrt(m) + sqrt(5 * g.h * g.gravity) + fabs(omega0) * g.R;
  double dt = dmin(g.max_substep, (g.cfl * g.h) / speed);
  dt = dmin(dt, g.duration - time);  // solver3d.ts:284
  if (forced && forced_dt > 0) dt = forced_dt;
  // step(dt) (solver3d.ts:288-292)
  double discharged = ndis * g.parcel_volume * g.vol_factor;
  double tilt1 = ctl_advance(motion, ctl, time + dt, dt, discharged);
  double phi1 = -tilt1;
  const bool reuse = (unsigned long long)__double_as_longlong(phi) == phi_trig;
  const double c0 = reuse ? c1p : cos(phi), s0 = reuse ? s1p : sin(phi);
  const double c1 = cos(phi1), s1 = sin(phi1);
  sc->force_step = 0;
  sc->forced_dt = 0;
  sc->ctl = ctl;
  sc->omega = (phi1 - phi) / dt;
  sc->dt = dt;
  sc->phi1 = phi1;
  sc->c0 = c0;
  sc->s0 = s0;
  sc->c1 = c1;
  sc->s1 = s1;
  sc->phi_trig_bits = (unsigned long long)__double_as_longlong(phi1);
  // per-substep counters
  sc->max_speed_bits = 0;
  sc->max_div_bits = 0;
  sc->corr_any = 0;
  sc->corr_iters = 0;
  sc->scan_tile = 0;
  // commit the pose and clock (solver3d.ts:306-308); kernels of this substep read phi0 from c0/s0
  sc->phi = phi1;
  sc->time = time + dt;
  sc->steps = steps + 1;
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

// Solid part of the cell classification (solver3d.ts:313-322): border or inside the walls at the
// current pose -> SOLID, else AIR; the scan then marks occupied non-solid cells FLUID. The SDF runs
// in FP64 with the reference's operation order so the classification matches the FP64 reference
// exactly.
__device__ __forceinline__ uint8_t solid_or_air(const Geo& g, const SimScalars* sc, int c) {
  int i = c % g.nx;
  int j = (c / g.nx) % g.ny;
  int k = c / (g.nx * g.ny);
  if (i == 0 || j == 0 || k == 0 || i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1) return SOLID;
  double loc[3];
  to_local(g, sc->c0, sc->s0, DMUL(i + 0.5, g.h), DMUL(j + 0.5, g.h), DMUL(k + 0.5, g.h), loc);
  return teapot_sdf(g, loc[0], loc[1], loc[2]) < 0 ? SOLID : AIR;
}

// One thread per parcel and per cell: the parcel's bin key and rank in its bin, and the cell's solid
// test (independent work in one launch so the SDF evaluations use the whole GPU).
__global__ void k_bin_count(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < SCAN_MAX_TILES) P.scan_state[s] = 0ull;
  if (g.tiled && s < g.ntx * g.nty * g.nz) P.tile_mask[s] = 0ull;
  if (s < brick_count(g)) P.brick_occ[s] = 0;  // brick_count <= nc
  if (s == 0) P.sc->n_occ_solid = 0;
  if (s < g.nc) P.cell[s] = solid_or_air(g, P.sc, s);
  if (s >= g.n) return;
  float4 p = P.pos_home[s];
  float4 v = P.vel_home[s];
  int status = __float_as_int(v.w) & 0xff;
  int id = __float_as_int(p.w);
  int key;
  // A non-finite in-pot parcel is in no cell: the reference's classify and particle-to-grid index its
  // typed arrays with NaN, which reads undefined and writes nothing (solver3d.ts:329-335, 339-431);
  // advection then marks it LOST (solver3d.ts:761-764). It waits in a removed-parcel bin.
  if (status == IN_POT && isfinite(p.x + p.y + p.z)) {
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

// Scan descriptors: bit 62-63 flag (1 aggregate, 2 inclusive prefix), bits 32-61 liquid cells,
// bits 0-31 parcels.
constexpr unsigned long long DESC_AGG = 1ull << 62, DESC_INC = 2ull << 62, DESC_VAL = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_classify(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  constexpr int NW = SCAN_THREADS / 32;
  __shared__ int s_tile;
  __shared__ unsigned long long s_seg[SCAN_ITEMS * NW];  // segment totals, then their exclusive prefixes
  __shared__ unsigned long long s_agg;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(&sc->scan_tile, 1);
  __syncthreads();
  const int tile = s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Striped ownership: item e of a thread is bin tile * SCAN_TILE + e * SCAN_THREADS + threadIdx.x, so
  // every load and store of the bin and cell arrays is coalesced. A warp's 32 bins of one item are a
  // segment of consecutive bins; segment (e, warp) precedes segment (e, warp + 1) and (e + 1, 0).
  const int b0 = tile * SCAN_TILE + threadIdx.x;
  unsigned long long val[SCAN_ITEMS], incl[SCAN_ITEMS];
  uint8_t typ[SCAN_ITEMS];
#pragma unroll
  for (int e = 0; e < SCAN_ITEMS; e++) {
    int b = b0 + e * SCAN_THREADS;
    unsigned long long v = 0;
    typ[e] = AIR;
    if (b < g.nbins) {
      int cn = P.cnt[b];
      P.cnt[b] = 0;
      v = (unsigned long long)(unsigned)cn;
      if (b < g.nc) {
        const uint8_t base = P.cell[b];  // SOLID or AIR from k_bin_count (solver3d.ts:313-336)
        typ[e] = base == SOLID ? SOLID : cn > 0 ? FLUID : AIR;
        if (cn > 0 && base == SOLID) P.occ_solid[atomicAdd(&sc->n_occ_solid, 1)] = b;
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
    // inclusive scan of the warp's segment
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    incl[e] = x;
    if (lane == 31) s_seg[e * NW + warp] = x;
  }
  __syncthreads();
  // exclusive scan of the SCAN_ITEMS * NW segment totals (two per lane of warp 0), in bin order
  if (warp == 0) {
    static_assert(SCAN_ITEMS * NW == 64, "two segments per lane");
    const unsigned long long a0 = s_seg[2 * lane], a1 = s_seg[2 * lane + 1];
    unsigned long long x = a0 + a1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const unsigned long long ex = x - a0 - a1;
    s_seg[2 * lane] = ex;
    s_seg[2 * lane + 1] = ex + a0;
    if (lane == 31) s_agg = x;
  }
  __syncthreads();
  const unsigned long long aggregate = s_agg;
  // decoupled look-back (bounded waits), one warp reading 32 predecessor descriptors at a time: the
  // exclusive prefix is the sum of the aggregates back to the nearest inclusive prefix
  if (warp == 0) {
    unsigned long long* desc = P.scan_state;
    if (tile == 0) {
      if (lane == 0) {
        atomicExch(&desc[0], DESC_INC | aggregate);
        s_prefix = 0;
      }
    } else {
      if (lane == 0) atomicExch(&desc[tile], DESC_AGG | aggregate);
      unsigned long long excl = 0;
      int top = tile - 1;  // highest predecessor not yet summed
      int spins = 0;
      const int limit = sc->spin_limit > 0 ? sc->spin_limit : SPIN_LIMIT;
      bool failed = false;
      while (top >= 0) {
        const int j = top - lane;
        const unsigned long long d = j >= 0 ? ld_volatile_u64(&desc[j]) : DESC_INC;  // below tile 0: prefix 0
        // nearest predecessor (lowest lane) holding an inclusive prefix; the lanes up to it are needed
        const unsigned inc = __ballot_sync(0xffffffffu, (d >> 62) == 2);
        const unsigned pend = __ballot_sync(0xffffffffu, (d >> 62) == 0);
        const int first = inc ? __ffs(inc) - 1 : 31;
        const unsigned need = first == 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (pend & need) {  // a needed descriptor is not published yet
          if (++spins > limit) {
            failed = true;
            break;
          }
          continue;
        }
        unsigned long long v = lane <= first ? (d & DESC_VAL) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (inc) break;
        top -= 32;
      }
      if (lane == 0) {
        if (failed) atomicOr(&sc->errors, ERR_SCAN_TIMEOUT);
        atomicExch(&desc[tile], DESC_INC | (excl + aggregate));
        s_prefix = excl;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < SCAN_ITEMS; e++) {
    const int b = b0 + e * SCAN_THREADS;
    const unsigned long long run = s_prefix + s_seg[e * NW + warp] + incl[e] - val[e];  // exclusive prefix
    if (b < g.nbins) {
      P.start[b] = (int)(run & 0xffffffffull);
      if (b < g.nc) {
        int lpos = (int)((run >> 32) & 0x3fffffffull);
        P.cell[b] = typ[e];
        P.occ[b] = (val[e] & 0xffffffffull) != 0 ? 1 : 0;
        if (typ[e] == FLUID) {
          P.list[lpos] = b;
          P.lidx[b] = lpos;
        } else {
          P.lidx[b] = -1;
        }
        if (b == g.nc - 1) sc->m = lpos + (typ[e] == FLUID ? 1 : 0);
      }
    }
  }
}

__global__ void k_bin_place(Geo g, DevPtrs P) {
  if (!P.sc->active) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  // A look-back that gave up left partial bin starts (each at most the true start, so every write of
  // the scan stayed in bounds). Nothing after it may use them: the substep is switched off here, every
  // later kernel returns at its active check, and the parcels keep their state before the substep.
  if (P.sc->errors & ERR_SCAN_TIMEOUT) {
    if (s == 0) P.sc->active = 0;
    return;
  }
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
  if (g.apic)
#pragma unroll
    for (int a = 0; a < 3; a++) P.aff_sorted[a * g.n + dst] = P.aff_home[a * g.n + e.y];
}

// ---------------------------------------------------------------- particle-to-grid

// The cell-partials pass: 128-thread blocks, 148 per component, so that the four components' blocks
// (four per SM at its register count) are resident at once and stride over the occupied cells.
constexpr int P2G_CELL_THREADS = 128, P2G_CELL_BLOCKS = 148;

// Weights along one axis of a parcel with FP64-derived cell fraction f for the nodes at offsets -1,
// 0, +1 from its cell: on a face axis (offset 0) the nodes 0 and +1; on a cell-centred axis (offset
// 1/2) the nodes (-1, 0) or (0, +1) by which half of the cell the parcel is in (solver3d.ts:352-360).
// Nodes the parcel does not touch get weight 0.
__device__ __forceinline__ void axis_w3(float f, bool half, double w[3]) {
  if (!half) {
    w[0] = 0.0;
    w[1] = 1.0 - (double)f;
    w[2] = (double)f;
  } else if (f >= 0.5f) {
    const double fr = (double)f - 0.5;
    w[0] = 0.0;
    w[1] = 1.0 - fr;
    w[2] = fr;
  } else {
    const double fr = (double)f + 0.5;
    w[0] = 1.0 - fr;
    w[1] = fr;
    w[2] = 0.0;
  }
}

// Node partials of one cell: for every node a parcel of the cell can touch, the sum over the cell's
// parcels (in their canonical order) of the trilinear weight w = wx * wy * wz and of w times the
// velocity component (COMP 0..2, particlesToGrid, solver3d.ts:410-431), or of w alone (COMP 3, the
// density of densityCorrection, solver3d.ts:633-642). A node's full sum is then a fixed-order sum of
// at most 18 (velocity) or 27 (density) partials, so the face and density gathers issue independent
// loads instead of walking every parcel of the neighbourhood. With APIC the velocity carried to a node
// is the parcel's affine field there, v + c . (x_node - x_p) (src/sim/solver.ts:553-587 in 3D).
template <int COMP, bool APIC>
__device__ __forceinline__ void cell_moments(const Geo& g, const DevPtrs& P, int c, int p0, int p1) {
  constexpr bool hx = COMP != 0, hy = COMP != 1, hz = COMP != 2;
  double sw[27], swv[27];
#pragma unroll
  for (int q = 0; q < 27; q++) sw[q] = swv[q] = 0.0;
  const int ci = c % g.nx, cj = (c / g.nx) % g.ny, ck = c / (g.nx * g.ny);
  // the next parcel's fraction and velocity are loaded while this one is summed
  float4 fr_next = P.frac_sorted[p0];
  float v_next = COMP < 3 ? reinterpret_cast<const float*>(&P.vel_sorted[p0])[COMP] : 0.f;
  for (int p = p0; p < p1; p++) {
    const float4 fr = fr_next;
    const double v = (double)v_next;
    if (p + 1 < p1) {
      fr_next = P.frac_sorted[p + 1];
      if (COMP < 3) v_next = reinterpret_cast<const float*>(&P.vel_sorted[p + 1])[COMP];
    }
    double wx[3], wy[3], wz[3];
    axis_w3(fr.x, hx, wx);
    axis_w3(fr.y, hy, wy);
    axis_w3(fr.z, hz, wz);
    // APIC: the affine field at the node offsets, v + cx dx + cy dy + cz dz per axis term
    double ax[3] = {0, 0, 0}, ay[3] = {0, 0, 0}, az[3] = {0, 0, 0};
    if (APIC && COMP < 3) {
      const float4 ps = P.pos_sorted[p];
      const float4 ca = P.aff_sorted[COMP * g.n + p];
#pragma unroll
      for (int o = 0; o < 3; o++) {  // node at offset o - 1 from the cell on each axis
        ax[o] = (double)ca.x * ((ci + o - 1 + (hx ? 0.5 : 0.0)) * g.h - (double)ps.x);
        ay[o] = (double)ca.y * ((cj + o - 1 + (hy ? 0.5 : 0.0)) * g.h - (double)ps.y);
        az[o] = (double)ca.z * ((ck + o - 1 + (hz ? 0.5 : 0.0)) * g.h - (double)ps.z);
      }
    }
#pragma unroll
    for (int ox = 0; ox < 3; ox++) {
      if (!hx && ox == 0) continue;
#pragma unroll
      for (int oy = 0; oy < 3; oy++) {
        if (!hy && oy == 0) continue;
#pragma unroll
        for (int oz = 0; oz < 3; oz++) {
          if (!hz && oz == 0) continue;
          const int q = ox * 9 + oy * 3 + oz;
          const double w = wx[ox] * wy[oy] * wz[oz];
          sw[q] += w;
          if (COMP < 3) swv[q] += w * (APIC ? v + ax[ox] + ay[oy] + az[oz] : v);
        }
      }
    }
  }
  const size_t nc = (size_t)g.nc;
#pragma unroll
  for (int q = 0; q < 27; q++) {
    const int ox = q / 9, oy = (q / 3) % 3, oz = q % 3;
    if ((!hx && ox == 0) || (!hy && oy == 0) || (!hz && oz == 0)) continue;
    if (COMP < 3)
      P.m_vel[((size_t)COMP * 27 + q) * nc + c] = make_float2((float)sw[q], (float)swv[q]);
    else
      P.m_den[(size_t)q * nc + c] = (float)sw[q];
  }
}

// The face pass's brick map (cleared by k_bin_count): occupied cell c marks its own brick and, where
// it lies on a brick face, the bricks across that face (edges and corners included), so that the brick
// of every cell within one cell of c, per axis, is marked.
__device__ __forceinline__ void mark_bricks(const Geo& g, const DevPtrs& P, int c) {
  const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
  const int bi = i / BRICK_W, bj = j / BRICK_W, bk = k / BRICK_W;
  const int bnx = (g.nx + BRICK_W - 1) / BRICK_W, bny = (g.ny + BRICK_W - 1) / BRICK_W;
  const int bnz = (g.nz + BRICK_W - 1) / BRICK_W;
  auto lo = [](int x, int b) { return x % BRICK_W == 0 && b > 0 ? -1 : 0; };
  auto hi = [](int x, int b, int nb) { return x % BRICK_W == BRICK_W - 1 && b + 1 < nb ? 1 : 0; };
  const int i0 = lo(i, bi), i1 = hi(i, bi, bnx), j0 = lo(j, bj), j1 = hi(j, bj, bny);
  const int k0 = lo(k, bk), k1 = hi(k, bk, bnz);
  for (int dk = k0; dk <= k1; dk++)
    for (int dj = j0; dj <= j1; dj++)
      for (int di = i0; di <= i1; di++) P.brick_occ[(bi + di) + bnx * ((bj + dj) + bny * (bk + dk))] = 1;
}

// One thread per (occupied cell, component); blockIdx.y is the component (3 = density). The occupied
// cells are the liquid list's (every non-solid cell with parcels) and the solid cells with parcels, so
// the grid strides over that compact range (its size is known on the device only) instead of the whole
// grid. Each cell's partials depend on that cell alone, so the order of the cells is free. One
// instantiation per transfer, chosen on the host, so the FLIP/PIC kernel is not held to the APIC
// kernel's register count.
template <bool APIC>
__global__ void __launch_bounds__(P2G_CELL_THREADS) k_p2g_cells(Geo g, DevPtrs P) {
  const SimScalars* sc = P.sc;
  if (!sc->active) return;
  const int m = sc->m, total = m + sc->n_occ_solid;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int c = t < m ? P.list[t] : P.occ_solid[t - m];
    const int p0 = P.start[c], p1 = P.start[c + 1];
    if (blockIdx.y == 0) mark_bricks(g, P, c);
    switch (blockIdx.y) {
      case 0: cell_moments<0, APIC>(g, P, c, p0, p1); break;
      case 1: cell_moments<1, APIC>(g, P, c, p0, p1); break;
      case 2: cell_moments<2, APIC>(g, P, c, p0, p1); break;
      default: cell_moments<3, APIC>(g, P, c, p0, p1); break;
    }
  }
}

// Whether a source cell of face (comp, i, j, k) in face_sums may hold parcels. The source cells are
// within one cell of cell (i, j, k) per axis (offsets {-1, 0} on the face axis, {-1, 0, +1} on the
// others), so one of them holding parcels marks the brick of (i, j, k) (mark_bricks); the last face
// of an axis (i = nx, ...) reads the brick of the cell before it. A face that no parcel reaches sums
// nothing: its weights and weighted velocities are 0.
__device__ __forceinline__ bool face_reached(const Geo& g, const DevPtrs& P, int i, int j, int k) {
  return P.brick_occ[brick_of(g, min(i, g.nx - 1), min(j, g.ny - 1), min(k, g.nz - 1))] != 0;
}

// Weighted sums at face (i, j, k) of component COMP: the partials of the source cells at offsets
// o = node - cell (face axis {0, 1}, others {-1, 0, 1}), interior cells only, in a fixed order. The
// 18 occupancy loads are issued together, then the partials of the occupied cells as predicated
// loads, so the loads overlap instead of waiting on one another.
template <int COMP>
__device__ __forceinline__ void face_sums(const Geo& g, const DevPtrs& P, int i, int j, int k, double* sw,
                                          double* swv) {
  constexpr int NX = COMP == 0 ? 2 : 3, NY = COMP == 1 ? 2 : 3, NZ = COMP == 2 ? 2 : 3;
  constexpr int NS = NX * NY * NZ;
  const size_t nc = (size_t)g.nc;
  float2 m[NS];
  bool use[NS];
  size_t idx[NS];
#pragma unroll
  for (int z = 0; z < NZ; z++) {
    const int oz = 1 - z;
    const int cz = k - oz;
    const bool inz = cz >= 1 && cz <= g.nz - 2;
    const int czc = min(max(cz, 1), g.nz - 2);
#pragma unroll
    for (int y = 0; y < NY; y++) {
      const int oy = 1 - y;
      const int cy = j - oy;
      const bool iny = cy >= 1 && cy <= g.ny - 2;
      const int cyc = min(max(cy, 1), g.ny - 2);
#pragma unroll
      for (int x = 0; x < NX; x++) {
        const int ox = 1 - x;
        const int cx = i - ox;
        const bool inx = cx >= 1 && cx <= g.nx - 2;
        const int cxc = min(max(cx, 1), g.nx - 2);
        const int c = cxc + g.nx * (cyc + g.ny * czc);
        const int q = (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1);
        const int e = (z * NY + y) * NX + x;
        use[e] = inx && iny && inz && P.occ[c] != 0;
        idx[e] = ((size_t)COMP * 27 + q) * nc + c;
      }
    }
  }
  // predicated loads: only occupied cells' partials are read (the others were never written)
#pragma unroll
  for (int e = 0; e < NS; e++) m[e] = use[e] ? P.m_vel[idx[e]] : make_float2(0.f, 0.f);
  double a = 0.0, b = 0.0;
#pragma unroll
  for (int e = 0; e < NS; e++) {
    a += use[e] ? (double)m[e].x : 0.0;
    b += use[e] ? (double)m[e].y : 0.0;
  }
  *sw = a;
  *swv = b;
}

// One thread per face: weighted average of the parcel velocities, gravity, wall velocity and valid
// mask (solver3d.ts:410-471, 545-562).
__global__ void k_p2g(Geo g, DevPtrs P) {
  const SimScalars* sc = P.sc;
  if (!sc->active) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nf) return;
  Face F = decode_face(g, f);
  double sw = 0.0, swv = 0.0;
  if (!face_reached(g, P, F.i, F.j, F.k))
    ;
  else if (F.comp == 0)
    face_sums<0>(g, P, F.i, F.j, F.k, &sw, &swv);
  else if (F.comp == 1)
    face_sums<1>(g, P, F.i, F.j, F.k, &sw, &swv);
  else
    face_sums<2>(g, P, F.i, F.j, F.k, &sw, &swv);
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

// |divergence| of liquid cell (i, j, k) after projection (divergenceRhs on the projected faces,
// solver3d.ts:473-493, 542): the six face velocities with the gradient applied.
__device__ __forceinline__ double projected_div(const Geo& g, const DevPtrs& P, int i, int j, int k) {
  const int ux = g.nx + 1, vy = g.ny + 1;
  const double d = (projected(g, P, 0, i + 1, j, k, ux, g.ny) - projected(g, P, 0, i, j, k, ux, g.ny)) +
                   (projected(g, P, 1, i, j + 1, k, g.nx, vy) - projected(g, P, 1, i, j, k, g.nx, vy)) +
                   (projected(g, P, 2, i, j, k + 1, g.nx, g.ny) - projected(g, P, 2, i, j, k, g.nx, g.ny));
  return fabs(d);
}

__device__ __forceinline__ void grad_ext1_face(const Geo& g, const DevPtrs& P, int f, const Face& F) {
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

// Gradient update and first extrapolation layer per face; the u-face threads whose +x cell is liquid
// also measure that cell's divergence after projection (max over cells, one atomic per warp).
__global__ void k_grad_ext1(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long bits = 0ull;
  if (f < g.nf) {
    const Face F = decode_face(g, f);
    if (F.comp == 0 && F.i < g.nx && P.cell[F.i + g.nx * (F.j + g.ny * F.k)] == FLUID)
      bits = (unsigned long long)__double_as_longlong(projected_div(g, P, F.i, F.j, F.k));
    grad_ext1_face(g, P, f, F);
    // the correction velocity of every face, once (applyGradient into zeroed uc, vc, wc:
    // solver3d.ts:629-631, 674); advection samples it like the velocity field
    if (g.kappa > 0 && sc->corr_any) P.uc[f] = grad_term(g, P, P.qc, F.comp, F.i, F.j, F.k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = ob > bits ? ob : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(&sc->max_div_bits, bits);
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
  const int nxy = g.nx * g.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    int c = P.list[t];
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / nxy;
    // density: trilinear weights of the parcels of the 27 neighbouring cells (solver3d.ts:633-642),
    // summed from the node partials of those cells in a fixed order (occupancy loads together, then
    // predicated loads of the occupied cells' partials)
    float dv[27];
    bool du[27];
    size_t di[27];
#pragma unroll
    for (int z = 0; z < 3; z++) {
      const int oz = 1 - z, cz = k - oz;
      const bool inz = cz >= 1 && cz <= g.nz - 2;
      const int czc = min(max(cz, 1), g.nz - 2);
#pragma unroll
      for (int y = 0; y < 3; y++) {
        const int oy = 1 - y, cy = j - oy;
        const bool iny = cy >= 1 && cy <= g.ny - 2;
        const int cyc = min(max(cy, 1), g.ny - 2);
#pragma unroll
        for (int x = 0; x < 3; x++) {
          const int ox = 1 - x, cx = i - ox;
          const bool inx = cx >= 1 && cx <= g.nx - 2;
          const int cxc = min(max(cx, 1), g.nx - 2);
          const int cc = cxc + g.nx * (cyc + g.ny * czc);
          const int e = (z * 3 + y) * 3 + x;
          du[e] = inx && iny && inz && P.occ[cc] != 0;
          di[e] = (size_t)((ox + 1) * 9 + (oy + 1) * 3 + (oz + 1)) * g.nc + cc;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 27; e++) dv[e] = du[e] ? P.m_den[di[e]] : 0.f;
    double dens = 0;
#pragma unroll
    for (int e = 0; e < 27; e++) dens += du[e] ? (double)dv[e] : 0.0;
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
  }
  // deterministic per-block partial sums (fixed shuffle tree, then warps in order); the flag is folded
  // per warp so that one atomic per warp reaches the scalar block
  for (int o = 16; o > 0; o >>= 1) {
    isum += __shfl_down_sync(0xffffffffu, isum, o);
    icnt += __shfl_down_sync(0xffffffffu, icnt, o);
  }
  any = __any_sync(0xffffffffu, any != 0) ? 1 : 0;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_sum[warp] = isum;
    s_cnt[warp] = icnt;
    if (any) atomicOr(&sc->corr_any, 1);
  }
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

// 128-thread blocks, five resident per SM (at most 102 registers a thread), so that the parcels of a
// 4 mm pour (88,856) fit in one wave of the 148 SMs.
constexpr int ADVECT_THREADS = 128;

struct Sten {
  int base, sx, sxy;
  double fx, fy, fz;
};

// solver3d.ts:339-362 for component comp (0/1/2 = u/v/w faces), from the point's coordinates already
// divided by h (qx = x / h, ...): the component's offset is subtracted after the division, as the
// reference does, so the three components and every field sampled at one point share the divisions.
__device__ __forceinline__ Sten face_stencil_q(const Geo& g, int comp, double qx, double qy, double qz) {
  double ox = comp == 0 ? 0.0 : 0.5, oy = comp == 1 ? 0.0 : 0.5, oz = comp == 2 ? 0.0 : 0.5;
  int sx = g.nx + (comp == 0), sy = g.ny + (comp == 1), sz = g.nz + (comp == 2);
  double gx = qx - ox, gy = qy - oy, gz = qz - oz;
  // clamp(floor(g), 0, s - 2); a NaN coordinate clamps to 0, so no index is ever formed from a NaN
  // (its weights stay NaN and the sample is NaN, as the reference's is)
  auto clampi = [](double f, int hi) { return f >= 0.0 ? (f <= (double)hi ? f : (double)hi) : 0.0; };
  double i = clampi(floor(gx), sx - 2);
  double j = clampi(floor(gy), sy - 2);
  double k = clampi(floor(gz), sz - 2);
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

// sample() without a valid mask (solver3d.ts:386-408) at a point given divided by h.
__device__ __forceinline__ double sample_q(const Geo& g, const float* field, int comp, double qx, double qy,
                                           double qz) {
  Sten s = face_stencil_q(g, comp, qx, qy, qz);
  double all = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) all += corner_w(s, c) * (double)field[corner(s, c)];
  return all;
}

// Gradient of the trilinear interpolant of one component from its 8 corner values u (corner order of
// corner()) over stencil s, unmasked (the 3D form of C = sum_i u_i grad w_ip, src/sim/solver.ts:958-964):
// per axis the corner differences along it, weighted by the other two axes' weights, over h.
__device__ __forceinline__ float4 interp_gradient(const Geo& g, const Sten& s, const double u[8]) {
  const double fx = s.fx, fy = s.fy, fz = s.fz;
  const double gx = ((1 - fy) * (1 - fz) * (u[1] - u[0]) + fy * (1 - fz) * (u[3] - u[2]) +
                     (1 - fy) * fz * (u[5] - u[4]) + fy * fz * (u[7] - u[6])) / g.h;
  const double gy = ((1 - fx) * (1 - fz) * (u[2] - u[0]) + fx * (1 - fz) * (u[3] - u[1]) +
                     (1 - fx) * fz * (u[6] - u[4]) + fx * fz * (u[7] - u[5])) / g.h;
  const double gz = ((1 - fx) * (1 - fy) * (u[4] - u[0]) + fx * (1 - fy) * (u[5] - u[1]) +
                     (1 - fx) * fy * (u[6] - u[2]) + fx * fy * (u[7] - u[3])) / g.h;
  return make_float4((float)gx, (float)gy, (float)gz, 0.f);
}

__device__ __forceinline__ void set_status(SimScalars* sc, int from, int to) {  // solver3d.ts:790-794
  atomicSub(&sc->counts[from], 1);
  atomicAdd(&sc->counts[to], 1);
}

// One parcel's grid-to-particle update and advection; returns the FP64 bits of its |v|^2 when it
// stays in the pot (the stableDt input of the next substep), else 0. APIC is the transfer
// (g.apic), fixed per instantiation so that the FLIP kernel does not carry the affine state.
template <bool APIC>
__device__ __forceinline__ unsigned long long advect_one(const Geo& g, const DevPtrs& P, SimScalars* sc, int p) {
  float4 pos = P.pos_sorted[p];
  float4 vel = P.vel_sorted[p];
  int meta = __float_as_int(vel.w);
  int st = meta & 0xff;
  const double dt = sc->dt;
  if (st != IN_POT && APIC)  // a removed parcel keeps its own affine state (the slot is re-used every substep)
#pragma unroll
    for (int a = 0; a < 3; a++) P.aff_home[a * g.n + p] = P.aff_sorted[a * g.n + p];
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
    return 0ull;
  }
  if (st != IN_POT) {
    P.pos_home[p] = pos;
    P.vel_home[p] = vel;
    return 0ull;
  }
  const double x0 = pos.x, y0 = pos.y, z0 = pos.z;
  double vx = vel.x, vy = vel.y, vz = vel.z;
  // Every field sampled at the parcel's position, with one stencil per face component: gridToParticles
  // (solver3d.ts:607-624: the FLIP/PIC blend of valid-masked samples of u and uprev; APIC: the masked
  // sample of u and the gradient of each component's interpolant, src/sim/solver.ts:956-986 in 3D), the
  // unmasked sample of u that starts the midpoint step and the correction velocity (solver3d.ts:704-727).
  const bool corr = g.kappa > 0 && sc->corr_any;
  const double qx0 = x0 / g.h, qy0 = y0 / g.h, qz0 = z0 / g.h;
  double u1[3], cs[3], vg[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const Sten s = face_stencil_q(g, a, qx0, qy0, qz0);
    double fu[8];
    double all = 0, acc = 0, ws = 0, allp = 0, accp = 0, call = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int idx = corner(s, c);
      const double w = corner_w(s, c);
      fu[c] = (double)P.u[idx];
      const bool ok = P.valid[idx] != 0;
      all += w * fu[c];
      if (ok) {
        acc += w * fu[c];
        ws += w;
      }
      if (!APIC) {
        const double fp = (double)P.uprev[idx];
        allp += w * fp;
        if (ok) accp += w * fp;
      }
      if (corr) call += w * P.uc[idx];
    }
    u1[a] = all;
    cs[a] = call;
    const double un = ws > 1e-9 ? acc / ws : all;
    if (APIC) {
      vg[a] = un;
      P.aff_home[a * g.n + p] = interp_gradient(g, s, fu);
    } else {
      const double uo = ws > 1e-9 ? accp / ws : allp;
      const double v = a == 0 ? vx : a == 1 ? vy : vz;
      vg[a] = (1 - g.flip) * un + g.flip * (v + un - uo);
    }
  }
  vx = vg[0];
  vy = vg[1];
  vz = vg[2];
  // advect (solver3d.ts:704-787)
  double loc0[3], loc1[3], out[3];
  to_local(g, sc->c0, sc->s0, x0, y0, z0, loc0);
  const double xm = x0 + 0.5 * dt * u1[0], ym = y0 + 0.5 * dt * u1[1], zm = z0 + 0.5 * dt * u1[2];
  const double qxm = xm / g.h, qym = ym / g.h, qzm = zm / g.h;
  double x1 = x0 + dt * sample_q(g, P.u, 0, qxm, qym, qzm);
  double y1 = y0 + dt * sample_q(g, P.u, 1, qxm, qym, qzm);
  double z1 = z0 + dt * sample_q(g, P.u, 2, qxm, qym, qzm);
  if (corr) {
    x1 += dt * cs[0];
    y1 += dt * cs[1];
    z1 += dt * cs[2];
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
  if (!g.full && z1 < g.h) {  // symmetry plane (half domain only)
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
    return 0ull;
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
                   z1 >= (g.nz - 1) * g.h || (g.full && z1 <= lo);
    if ((!inside_body && !near_spout) || at_edge) new_st = SPILLED;
  }
  if (new_st != IN_POT) {
    set_status(sc, IN_POT, new_st);
    if (new_st == DISCHARGED) atomicAdd(&sc->by_origin[(meta >> 8) & 0xff], 1);
    vel.w = __int_as_float((meta & ~0xff) | new_st);
  } else {
    // stableDt (solver3d.ts:269-274) of the next substep, from the velocity as stored: a state saved
    // now and restored (pl_set_state recounts it the same way) continues with the same dt
    const double fx = vel.x, fy = vel.y, fz = vel.z;
    const double sp = DADD(DADD(DMUL(fx, fx), DMUL(fy, fy)), DMUL(fz, fz));
    P.pos_home[p] = pos;
    P.vel_home[p] = vel;
    return (unsigned long long)__double_as_longlong(sp);
  }
  P.pos_home[p] = pos;
  P.vel_home[p] = vel;
  return 0ull;
}

// The maximum speed is folded per warp (bit patterns of non-negative doubles order like the values),
// so one atomic per warp reaches the scalar block instead of one per parcel.
template <bool APIC>
__global__ void __launch_bounds__(ADVECT_THREADS, 5) k_advect(Geo g, DevPtrs P) {
  SimScalars* sc = P.sc;
  if (!sc->active) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long bits = p < g.n ? advect_one<APIC>(g, P, sc, p) : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = ob > bits ? ob : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(&sc->max_speed_bits, bits);
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
  P.render[3 * id] = x;
  P.render[3 * id + 1] = y;
  P.render[3 * id + 2] = z;
  if (g.full) return;  // both halves are simulated: no mirror image
  int m = id + g.n;
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
  k_bin_count<<<blocks(max(max(max(g.n, g.nc), SCAN_MAX_TILES), g.tiled ? g.ntx * g.nty * g.nz : 0), 256), 256, 0,
                st>>>(g, P);
  k_scan_classify<<<blocks(g.nbins, SCAN_TILE), SCAN_THREADS, 0, st>>>(g, P);
  k_bin_place<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
  k_bin_permute<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
}

// The cells' node partials, then the faces (k_p2g, this stream) and the density stage (k_density,
// the second stream) side by side: both only read the partials, and they write disjoint arrays.
void launch_p2g_cells(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  const dim3 grid(min(blocks(g.nc, P2G_CELL_THREADS), P2G_CELL_BLOCKS), 4);
  if (g.apic)
    k_p2g_cells<true><<<grid, P2G_CELL_THREADS, 0, st>>>(g, P);
  else
    k_p2g_cells<false><<<grid, P2G_CELL_THREADS, 0, st>>>(g, P);
}
void launch_p2g_faces(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_p2g<<<blocks(g.nf, 128), 128, 0, st>>>(g, P);  // 128: 0.2810 -> 0.2801 ms per 4 mm substep
}

void launch_stage_extrap(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_grad_ext1<<<blocks(g.nf, 256), 256, 0, st>>>(g, P);
  k_ext2<<<blocks(g.nf, 256), 256, 0, st>>>(g, P);
}

void launch_stage_density(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_density<<<DENSITY_BLOCKS, 128, 0, st>>>(g, P);  // 128 (one liquid cell a thread at 4 mm): -0.5 us
}

void launch_stage_advect(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  if (g.apic)
    k_advect<true><<<blocks(g.n, ADVECT_THREADS), ADVECT_THREADS, 0, st>>>(g, P);
  else
    k_advect<false><<<blocks(g.n, ADVECT_THREADS), ADVECT_THREADS, 0, st>>>(g, P);
}

void launch_render(const Geo& g, const DevPtrs& P, cudaStream_t st) {
  k_render<<<blocks(g.n, 256), 256, 0, st>>>(g, P);
}

void launch_export_correction(const Geo& g, const DevPtrs& P, float* out, cudaStream_t st) {
  k_export_correction<<<blocks(g.nf, 256), 256, 0, st>>>(g, P, out);
}

// ---------------------------------------------------------------- recording frames

// Every stride-th parcel (in id order) quantised as the recording format stores it (format.ts:60):
// max(0, min(65535, Math.round(f / quantum))) of the FP32 position, the division in FP64 and
// Math.round's halves toward +infinity; out[3 k + c] for the parcel with id = k * stride.
__global__ void k_quantize(DevPtrs P, int n, int stride, double quantum, uint16_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = P.pos_home[i];
  const int id = __float_as_int(p.w);
  if (id < 0 || id >= n || id % stride) return;
  const int k = id / stride;
  const float c[3] = {p.x, p.y, p.z};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double t = double(c[a]) / quantum;
    double r = floor(t);
    if (t - r >= 0.5) r += 1.0;
    r = fmin(fmax(r, 0.0), 65535.0);
    out[3 * k + a] = uint16_t(r);
  }
}

void launch_quantize(const DevPtrs& P, int n, int stride, double quantum, uint16_t* out, cudaStream_t st) {
  k_quantize<<<(n + 255) / 256, 256, 0, st>>>(P, n, stride, quantum, out);
}

}  // namespace pl
