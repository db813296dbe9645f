// Shared definitions of the pour-substep engine: the constant geometry record, the device-resident
// scalar state of a simulation, the frame transforms and the teapot signed-distance function.
//
// Layout in device memory (one simulation):
//   parcels   pos float4[N] (x, y, z, id bits), vel float4[N] (vx, vy, vz, status | origin << 8),
//             frac float4[N] (cell fractions fx, fy, fz computed in FP64, bin key bits);
//             two copies: "home" (order of the last substep) and "sorted" (this substep's bins).
//   bins      cnt/start int32[nbins+1] with nbins = cells + REMOVED_BINS; counting sort by cell.
//   cells     cell u8[C], lidx int32[C] (position in the liquid list or -1), q f64[C].
//   faces     u, uprev float[F] (u then v then w), valid u8[F], extrapolation ping-pong float[F].
//   liquid    list int32[C] of FLUID cells in index order + per-solve vectors (solver scratch).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pourlab.h"

#define PL_HD __host__ __device__ __forceinline__

namespace pl {

constexpr uint8_t AIR = 0, FLUID = 1, SOLID = 2;
constexpr uint32_t IN_POT = 0, DISCHARGED = 1, SPILLED = 2, LOST = 3;
constexpr double PI = 3.141592653589793;
constexpr double DEG = PI / 180;
// Parcels that left the pot are binned behind the cells, spread over this many bins by id so that
// every bin stays short (the within-bin order is made canonical by id).
constexpr int REMOVED_BINS = 1024;
// Bounded device-side waits: iterations before a spin gives up and sets an error flag.
constexpr int SPIN_LIMIT = 1 << 22;
// Bins one substep's scan can cover (SCAN_MAX_TILES tiles of 2048 bins; see kernels.h).
constexpr int SCAN_MAX_BINS = 4096 * 2048;

// Error flags (SimScalars::errors).
constexpr int ERR_SCAN_TIMEOUT = 1;
constexpr int ERR_SOLVER_SIZE = 2;
constexpr int ERR_SOLVER_TIMEOUT = 4;  // a cluster solve's bounded wait for a neighbour gave up

// Column tiles of the cluster solver's cell order: the liquid cells sorted by (8 x 8 column tile,
// k, j, i), so that contiguous ranges of that order are compact blocks. One 64-bit mask per
// (tile, plane) marks the liquid cells; grids with more tile planes than TILE_PLANES_MAX keep the
// list order.
constexpr int TILE_W = 8;
constexpr int TILE_PLANES_MAX = 8192;

// Constant per simulation: grid, physics, pot geometry (vessel3d.ts:34-59, solver3d.ts:116-182).
struct Geo {
  int nx, ny, nz, n;
  int nc, nu, nv, nw, nf;
  // 1 / sx and 1 / (sx * sy) of each face component's extents (sx = nx + (comp == 0), ...), for
  // decode_face's quotients (geo_face_reciprocals fills them)
  float inv_sx[3], inv_sxy[3];
  int nbins;
  double h;
  double pwx, pwy;    // pivotWorld
  double pivx, pivy;  // pivot (local)
  double gravity, flip, kappa, cfl, max_substep, duration;
  double tol;
  int max_iter;
  int precond;
  int precision;
  int solve_cluster;  // launch shape of the cluster solves (set by the tuner)
  int solve_threads;
  int ntx, nty;  // column tiles along x and y
  int tiled;     // the cluster solver orders its cells by column tile (ntx * nty * nz <= TILE_PLANES_MAX)
  int apic;      // affine particle-grid transfer (PL_TRANSFER_APIC)
  int full;      // both halves of the pot, no symmetry plane (PL_DOMAIN_FULL)
  int box_solve;      // grid-scale pressure solves (PL_PRECOND_BOX_MG / PL_PRECOND_LEARNED)
  int bx, by, bz;     // their power-of-two box (>= the grid, every side >= 8)
  double zoff;   // world z of the pot-local plane z = 0 (h for the half domain)
  double vol_factor;  // parcels' volume scale in the accounting: 2 (the half stands for the pot), 1 (full)
  double parcel_volume;
  double R;  // Math.hypot(nx, ny) * h  (solver3d.ts:275)
  // teapot
  double radius, height, wall, bore, ax, ay, dx, dy, spout_length, tipx, tipy;
};

// PourController fields (motion.ts:21-38) as stored on the device.
struct DevController {
  int phase, pour;
  double angle, phase_start, start_angle, start_rate, last_rate, flow_rate, last_discharged, target,
      manual_rate;
};

// Device-resident scalar state of one simulation. Written by the controller kernel at the start of
// each substep, by the kernels of that substep, and read by the host after it synchronises.
struct SimScalars {
  // persistent state
  double time;
  long long steps;
  double phi, omega;
  DevController ctl;
  pl_motion motion;
  double end_time;  // advance() target: substeps run while time < end_time - 1e-12
  int force_step;   // run the next substep regardless of end_time (step(dt) semantics)
  int scan_tile;    // dynamic tile counter of the bin scan
  double forced_dt; // > 0: dt of the forced substep; else the stable dt
  // this substep
  int active;
  int spin_limit;  // polls before the bin scan's bounded look-back wait gives up (0: SPIN_LIMIT)
  double dt, phi1;
  double c0, s0, c1, s1;
  // counters (integer: order-independent, deterministic)
  int counts[4];
  int by_origin[3];
  int failures;
  int last_iters;
  int corr_iters;
  int m;         // liquid cells of this substep
  int errors;    // ERR_* bits
  int outliers;  // in-pot parcels outside the interior cells (clamped into it)
  int corr_any;  // density rhs has a non-zero entry
  int mg_status;  // 1: the cluster multigrid solve ran; 0: the wavefront solver must run
  int n_occ_solid;  // SOLID cells holding in-pot parcels this substep (entries of DevPtrs::occ_solid)
  unsigned long long max_speed_bits;  // max |v|^2 (FP64 bits) of in-pot parcels after advect
  unsigned long long max_div_bits;    // max |div| (FP64 bits) after projection
  double interior;                    // mean interior density ratio
  int interior_count;
  int pad1;
  double last_residual;
  double corr_residual;
  // globaltimer stamps (ns) of a two-system cluster solve: start, start of the correction system,
  // end (the host splits the solve stage's event time into pressure and correction with them)
  unsigned long long t_solve[3];
  // bits of the pose whose cosine and sine c1, s1 hold (the next substep reuses them as c0, s0); a
  // NaN pattern when the host has set the pose, so that they are formed anew
  unsigned long long phi_trig_bits;
};

// ---------------------------------------------------------------- frames (solver3d.ts:232-260)
// The products and sums are written with explicit round-to-nearest intrinsics on the device so
// that nvcc does not contract them into FMAs: these feed the cell classification, which must
// agree with the FP64 reference bit for bit.
#ifdef __CUDA_ARCH__
#define DMUL(a, b) __dmul_rn((a), (b))
#define DADD(a, b) __dadd_rn((a), (b))
#define DSUB(a, b) __dsub_rn((a), (b))
#else
#define DMUL(a, b) ((a) * (b))
#define DADD(a, b) ((a) + (b))
#define DSUB(a, b) ((a) - (b))
#endif

PL_HD void to_local(const Geo& g, double c, double s, double wx, double wy, double wz, double* out) {
  double rx = DSUB(wx, g.pwx);
  double ry = DSUB(wy, g.pwy);
  out[0] = DADD(DADD(DMUL(c, rx), DMUL(s, ry)), g.pivx);
  out[1] = DADD(DADD(DMUL(-s, rx), DMUL(c, ry)), g.pivy);
  out[2] = DSUB(wz, g.zoff);
}

PL_HD void to_world(const Geo& g, double c, double s, double lx, double ly, double lz, double* out) {
  double rx = DSUB(lx, g.pivx);
  double ry = DSUB(ly, g.pivy);
  out[0] = DADD(DSUB(DMUL(c, rx), DMUL(s, ry)), g.pwx);
  out[1] = DADD(DADD(DMUL(s, rx), DMUL(c, ry)), g.pwy);
  out[2] = DADD(lz, g.zoff);
}

PL_HD double dmax(double a, double b) { return a > b ? a : b; }
PL_HD double dmin(double a, double b) { return a < b ? a : b; }

// Signed distance to the pot walls, negative inside the solid (vessel3d.ts:62-95), FP64 and with
// the reference's operation order.
PL_HD double teapot_sdf(const Geo& g, double x, double y, double z) {
  double hw = g.wall / 2;
  double r = sqrt(DADD(DMUL(x, x), DMUL(z, z)));
  double ring = DSUB(fabs(DSUB(r, DADD(g.radius, hw))), hw);
  double yIn = dmax(-DADD(y, g.wall), DSUB(y, g.height));
  double side = dmax(ring, yIn);
  double floorD = dmax(DSUB(fabs(DADD(y, hw)), hw), DSUB(r, DADD(g.radius, g.wall)));
  double solid = dmin(side, floorD);
  // spout axis (vessel3d.ts:62-71)
  double px = DSUB(x, g.ax);
  double py = DSUB(y, g.ay);
  double s = DADD(DMUL(px, g.dx), DMUL(py, g.dy));
  double L = g.spout_length;
  double sc = s < 0 ? 0 : s > L ? L : s;
  double qx = DSUB(px, DMUL(sc, g.dx));
  double qy = DSUB(py, DMUL(sc, g.dy));
  double dist = sqrt(DADD(DADD(DMUL(qx, qx), DMUL(qy, qy)), DMUL(z, z)));
  double along = dmax(-s, DSUB(s, L));
  double tube = dmax(DSUB(fabs(DSUB(dist, DADD(g.bore, hw))), hw), along);
  solid = dmin(solid, dmax(tube, DSUB(g.radius, r)));
  double bore = dmax(dmax(DSUB(dist, g.bore), DSUB(-s, g.wall)), DSUB(s, L));
  return dmax(solid, -bore);
}

// Math.hypot as the JavaScript engine evaluates it: normalise by the largest magnitude and
// Kahan-sum the squares (so results agree with the reference in the last bit).
template <int N>
PL_HD double js_hypot(const double* v) {
  double a[N];
  double mx = 0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    a[i] = fabs(v[i]);
    if (a[i] > mx) mx = a[i];
  }
  if (mx == 0 || mx != mx) return mx;
  double sum = 0, comp = 0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    double q = a[i] / mx;
    double summand = DSUB(DMUL(q, q), comp);
    double prelim = DADD(sum, summand);
    comp = DSUB(DSUB(prelim, sum), summand);
    sum = prelim;
  }
  return DMUL(sqrt(sum), mx);
}
PL_HD double js_hypot3(double a, double b, double c) {
  double v[3] = {a, b, c};
  return js_hypot<3>(v);
}
PL_HD double js_hypot2(double a, double b) {
  double v[2] = {a, b};
  return js_hypot<2>(v);
}

// Face-index decoding: faces are stored u (nx+1,ny,nz), then v (nx,ny+1,nz), then w (nx,ny,nz+1).
struct Face {
  int comp, i, j, k, sx, sy, sz, local;
};
// floor(n / d) for 0 <= n < 2^24 and 1 <= d with the quotient below 2^20, from the float reciprocal
// inv = 1/d: the product's relative error is below 2^-22, so the truncated estimate is off by at most
// one, which the exact integer remainder corrects.
PL_HD int quot_small(int n, int d, float inv) {
  int q = int(float(n) * inv);
  const int r = n - q * d;
  if (r < 0) q--;
  else if (r >= d) q++;
  return q;
}

PL_HD void geo_face_reciprocals(Geo& g) {
  for (int c = 0; c < 3; c++) {
    const int sx = g.nx + (c == 0), sy = g.ny + (c == 1);
    g.inv_sx[c] = 1.0f / float(sx);
    g.inv_sxy[c] = 1.0f / float(sx * sy);
  }
}

PL_HD Face decode_face(const Geo& g, int f) {
  Face r;
  int rem = f;
  r.comp = 0;
  if (rem >= g.nu) {
    rem -= g.nu;
    r.comp = 1;
    if (rem >= g.nv) {
      rem -= g.nv;
      r.comp = 2;
    }
  }
  r.sx = g.nx + (r.comp == 0);
  r.sy = g.ny + (r.comp == 1);
  r.sz = g.nz + (r.comp == 2);
  r.local = rem;
  const int sxy = r.sx * r.sy;
  r.k = quot_small(rem, sxy, g.inv_sxy[r.comp]);
  const int in_plane = rem - r.k * sxy;
  r.j = quot_small(in_plane, r.sx, g.inv_sx[r.comp]);
  r.i = in_plane - r.j * r.sx;
  return r;
}
PL_HD int comp_base(const Geo& g, int comp) { return comp == 0 ? 0 : comp == 1 ? g.nu : g.nu + g.nv; }

// Bricks of BRICK_W^3 cells: a coarse occupancy map lets the face pass skip the neighbourhood gathers
// of faces that no parcel can reach.
constexpr int BRICK_W = 4;
PL_HD int brick_count(const Geo& g) {
  return ((g.nx + BRICK_W - 1) / BRICK_W) * ((g.ny + BRICK_W - 1) / BRICK_W) * ((g.nz + BRICK_W - 1) / BRICK_W);
}
PL_HD int brick_of(const Geo& g, int i, int j, int k) {
  const int bnx = (g.nx + BRICK_W - 1) / BRICK_W, bny = (g.ny + BRICK_W - 1) / BRICK_W;
  return i / BRICK_W + bnx * (j / BRICK_W + bny * (k / BRICK_W));
}

// Cell type with the solid border outside the grid (solver3d.ts:453-469).
__device__ __forceinline__ uint8_t cell_at(const Geo& g, const uint8_t* cell, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return SOLID;
  return cell[i + g.nx * (j + g.ny * k)];
}

// Per-simulation device pointers.
struct DevPtrs {
  // parcels
  float4 *pos_home, *vel_home, *pos_sorted, *vel_sorted, *frac_sorted, *frac_tmp;
  // APIC: per parcel the gradients of u, v and w (xyz of three float4, aff[comp * n + p]), in both orders
  float4 *aff_home, *aff_sorted;
  int *key, *rank;
  int2* placed;  // (id, home slot) in bin order before the in-bin sort
  // bins and cells
  int *cnt, *start;
  uint8_t* cell;
  int* lidx;
  int* list;
  double* q;   // pressure (valid on liquid cells)
  double* qc;  // density-correction potential
  // faces
  float *u, *uprev, *uext;
  uint8_t *valid, *vext;
  double* uc;  // density-correction face velocity -grad qc of this substep (valid when sc->corr_any)
  // liquid-cell work (solver), indexed by position in the liquid list
  double* rhs;      // density-correction rhs
  double* density;  // particle density
  double* interior_part;  // per-block partial sums of the interior ratio
  int* interior_cnt_part;
  // scan
  unsigned long long* scan_state;  // decoupled look-back descriptors
  // solver scratch (list-indexed)
  void* solver_ws;
  size_t solver_ws_bytes;
  void* mg_ws;  // multigrid hierarchy
  // cluster solver order (positions in the column-tile order of the liquid cells)
  unsigned long long* tile_mask;  // ntx * nty * nz masks of liquid cells, bit (j % 8) * 8 + i % 8
  int* tnb;    // 6 * nc: tile-order position of the -x,+x,-y,+y,-z,+z liquid neighbour or -1
  int* tperm;  // nc: liquid-list index of the cell at each tile-order position
  // particle-to-grid node partials of this substep (cell-indexed, valid where occ[c] != 0):
  // m_vel[(comp * 27 + slot) * nc + c] = (sum w, sum w v) of cell c's parcels for the comp-face node
  // at offset slot = (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1) from the cell; m_den[slot * nc + c] =
  // sum w for the cell-centred node at that offset (density)
  uint8_t* occ;  // cell holds in-pot parcels
  // per 4 x 4 x 4 brick of cells (brick_of): some cell of the brick holds in-pot parcels (written by
  // the cell-partials pass, read by the face pass)
  uint8_t* brick_occ;
  // the SOLID cells that hold in-pot parcels (n_occ_solid of them, in no fixed order); with the liquid
  // list they are every occupied cell
  int* occ_solid;
  float2* m_vel;
  float* m_den;
  // grid-scale solves: the liquid system embedded in the box (cell types, rhs), the box solution and
  // the solve's outcome (iterations, converged, max-norm residual)
  uint8_t* box_cell;
  float* box_b;
  double* box_x;
  double* box_out;
  float* box_b2;  // the density-correction solve's rhs, solution and outcome (it runs beside the pressure)
  double* box_x2;
  double* box_out2;
  // render
  float* render;
  SimScalars* sc;
};

}  // namespace pl
