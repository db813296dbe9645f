// Host-side construction of a simulation (new Simulation3D(cfg), solver3d.ts:116-228): domain sweep
// over the tilt range, grid sizes, 2x2x2 jittered seeding with mulberry32 (src/sim/rng.ts:5-14),
// the parcel volume and the origin layers. Runs in FP64 on the host with the reference's operation
// order (compiled without FMA contraction) so that the seeded state, and with it the origin tags,
// match the reference bit for bit. The parcels then move to the device in FP32.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "setup.h"

namespace pl {

namespace {

struct Mulberry32 {  // rng.ts:5-14
  uint32_t a;
  double next() {
    a = a + 0x6d2b79f5u;
    uint32_t t = a;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return double(t ^ (t >> 14)) / 4294967296.0;
  }
};

bool in_cavity(const Geo& g, double x, double y, double z) {  // vessel3d.ts:98-103
  if (y >= 0 && y <= g.height && x * x + z * z <= g.radius * g.radius) return true;
  double px = x - g.ax, py = y - g.ay;
  double s = px * g.dx + py * g.dy;
  double L = g.spout_length;
  double sc = s < 0 ? 0 : s > L ? L : s;
  double qx = px - sc * g.dx, qy = py - sc * g.dy;
  double dist = std::sqrt(qx * qx + qy * qy + z * z);
  return s >= 0 && s <= L && dist <= g.bore;
}

}  // namespace

int host_construct(const pl_config& cfg, HostInit* out, char* err, size_t errlen) {
  const pl_teapot& t = cfg.teapot;
  if (!(cfg.h > 0) || !(t.radius > 0) || !(cfg.initial_volume > 0) || !(cfg.duration >= 0)) {
    snprintf(err, errlen, "pl_create: invalid config (h, radius, initial_volume and duration must be positive)");
    return PL_E_ARG;
  }
  Geo& g = out->geo;
  g = Geo{};
  const double h = cfg.h;
  g.h = h;
  g.zoff = h;  // world z of the pot's symmetry plane (toLocal, solver3d.ts:232-240)
  // buildTeapot3D (vessel3d.ts:46-59)
  double a = (t.spout_angle_deg * PI) / 180;
  g.radius = t.radius;
  g.height = t.height;
  g.wall = t.wall;
  g.bore = t.bore_radius;
  g.spout_length = t.spout_length;
  g.ax = t.radius - t.wall;
  g.ay = t.inlet_height;
  g.dx = std::cos(a);
  g.dy = std::sin(a);
  g.tipx = g.ax + std::cos(a) * t.spout_length;
  g.tipy = g.ay + std::sin(a) * t.spout_length;
  out->fill_height = cfg.initial_volume / (PI * t.radius * t.radius);
  // domain sweep (solver3d.ts:125-157)
  const double pts[6][2] = {
      {-t.radius - t.wall, -t.wall},      {-t.radius - t.wall, t.height + 0.02},
      {t.radius + t.wall, -t.wall},       {t.radius + t.wall, t.height + 0.02},
      {g.tipx + 0.02, g.tipy + 0.02},     {g.tipx + 0.02, g.tipy - 0.03},
  };
  double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
  double maxA = std::max(cfg.motion.max_angle_deg, cfg.motion.hold_angle_deg);
  for (double ang = 0; ang <= maxA; ang += 2) {
    double ph = (-ang * PI) / 180;
    double c = std::cos(ph), s = std::sin(ph);
    for (const auto& p : pts) {
      double rx = p[0] - cfg.pivot[0], ry = p[1] - cfg.pivot[1];
      double wx = c * rx - s * ry, wy = s * rx + c * ry;
      x0 = std::min(x0, wx);
      x1 = std::max(x1, wx);
      y0 = std::min(y0, wy);
      y1 = std::max(y1, wy);
    }
  }
  double m3 = 3 * h;
  g.pwx = -x0 + m3;
  g.pwy = -y0 + m3;
  g.pivx = cfg.pivot[0];
  g.pivy = cfg.pivot[1];
  double fnx = std::ceil((x1 - x0 + 2 * m3) / h);
  double fny = std::ceil((y1 - y0 + 2 * m3) / h);
  double fnz = std::ceil((t.radius + t.wall + 2 * h) / h) + 1;
  if (!(fnx >= 4 && fny >= 4 && fnz >= 4) || fnx * fny * fnz > 6.0e7 || fnx + fny + fnz > 2048) {
    snprintf(err, errlen, "pl_create: grid %gx%gx%g out of range", fnx, fny, fnz);
    return PL_E_ARG;
  }
  g.nx = int(fnx);
  g.ny = int(fny);
  g.nz = int(fnz);  // the half domain's z extent; the full domain is resized after seeding
  const int nz_half = g.nz;
  const bool full = cfg.domain == PL_DOMAIN_FULL;
  if (full && 2.0 * fnx * fny * fnz > 6.0e7) {
    snprintf(err, errlen, "pl_create: full-domain grid %gx%gx%g out of range", fnx, fny, 2 * fnz - 2);
    return PL_E_ARG;
  }
  g.nc = g.nx * g.ny * g.nz;
  g.nu = (g.nx + 1) * g.ny * g.nz;
  g.nv = g.nx * (g.ny + 1) * g.nz;
  g.nw = g.nx * g.ny * (g.nz + 1);
  g.nf = g.nu + g.nv + g.nw;
  geo_face_reciprocals(g);
  g.nbins = g.nc + REMOVED_BINS;
  if (g.nbins > SCAN_MAX_BINS) {
    snprintf(err, errlen, "pl_create: %d cells exceed the bin scan capacity", g.nc);
    return PL_E_ARG;
  }
  // seeding (solver3d.ts:184-200); toLocal at phi = 0 is exact: cos 0 = 1, sin 0 = 0
  Mulberry32 rng{cfg.seed};
  const double s = h / 2;
  std::vector<double> xs;
  xs.reserve(size_t(g.nc) * 3);
  for (int k = 0; k < g.nz * 2; k++)
    for (int j = 0; j < g.ny * 2; j++)
      for (int i = 0; i < g.nx * 2; i++) {
        double wx = (i + 0.5 + (rng.next() - 0.5) * 0.5) * s;
        double wy = (j + 0.5 + (rng.next() - 0.5) * 0.5) * s;
        double wz = (k + 0.5 + (rng.next() - 0.5) * 0.5) * s;
        double loc[3];
        to_local(g, 1.0, 0.0, wx, wy, wz, loc);
        if (loc[2] < 0 || loc[1] < 0 || loc[1] > out->fill_height) continue;
        if (!in_cavity(g, loc[0], loc[1], loc[2])) continue;
        if (teapot_sdf(g, loc[0], loc[1], loc[2]) < 0.4 * h) continue;
        xs.push_back(wx);
        xs.push_back(wy);
        xs.push_back(wz);
      }
  const int n = int(xs.size() / 3);
  if (n == 0) {
    snprintf(err, errlen, "pl_create: no parcels seeded");
    return PL_E_ARG;
  }
  g.n = n;
  g.parcel_volume = cfg.initial_volume / (2 * double(n));
  out->x.resize(n);
  out->y.resize(n);
  out->z.resize(n);
  std::vector<float> y0f(n);
  for (int p = 0; p < n; p++) {
    out->x[p] = xs[3 * p];
    out->y[p] = xs[3 * p + 1];
    out->z[p] = xs[3 * p + 2];
    double loc[3];
    to_local(g, 1.0, 0.0, out->x[p], out->y[p], out->z[p], loc);
    y0f[p] = float(loc[1]);
  }
  // equal-volume bands by Float32 y0 with the index as tiebreak (solver3d.ts:220-226)
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return y0f[i] < y0f[j]; });
  out->origin.assign(n, 0);
  out->band_counts[0] = out->band_counts[1] = out->band_counts[2] = 0;
  for (int r = 0; r < n; r++) {
    int k = std::min(2, int(std::floor((double(r) * 3) / n)));
    out->origin[order[r]] = uint8_t(k);
    out->band_counts[k]++;
  }
  g.vol_factor = 2;
  if (full) {
    // Full domain: both halves. The z grid mirrors the interior cells about the pot's symmetry plane,
    // which becomes a cell face at world z = zoff; every seeded parcel gets its mirror image (ids
    // n..2n-1, same origin layer), so the seeded half is the reference's, and the pot holds both.
    g.nz = 2 * nz_half - 2;
    g.zoff = (nz_half - 1) * h;
    out->x.resize(2 * size_t(n));
    out->y.resize(2 * size_t(n));
    out->z.resize(2 * size_t(n));
    out->origin.resize(2 * size_t(n));
    for (int p = 0; p < n; p++) {
      const double lz = out->z[p] - h;  // pot-local z of the seeded parcel (half-domain frame)
      out->z[p] = lz + g.zoff;
      out->x[n + p] = out->x[p];
      out->y[n + p] = out->y[p];
      out->z[n + p] = -lz + g.zoff;
      out->origin[n + p] = out->origin[p];
    }
    for (int k = 0; k < 3; k++) out->band_counts[k] *= 2;
    g.n = 2 * n;
    g.vol_factor = 1;
    g.nc = g.nx * g.ny * g.nz;
    g.nu = (g.nx + 1) * g.ny * g.nz;
    g.nv = g.nx * (g.ny + 1) * g.nz;
    g.nw = g.nx * g.ny * (g.nz + 1);
    g.nf = g.nu + g.nv + g.nw;
  geo_face_reciprocals(g);
    g.nbins = g.nc + REMOVED_BINS;
    if (g.nbins > SCAN_MAX_BINS) {
      snprintf(err, errlen, "pl_create: %d cells exceed the bin scan capacity", g.nc);
      return PL_E_ARG;
    }
  }
  g.full = full ? 1 : 0;
  // physics
  g.gravity = cfg.gravity;
  g.flip = cfg.flip_ratio;
  g.kappa = cfg.density_correction;
  g.cfl = cfg.cfl;
  g.max_substep = cfg.max_substep;
  g.duration = cfg.duration;
  g.tol = cfg.pressure_tolerance;
  g.max_iter = cfg.pressure_max_iterations;
  g.precond = cfg.preconditioner;
  g.precision = cfg.solve_precision;
  g.ntx = (g.nx + TILE_W - 1) / TILE_W;
  g.nty = (g.ny + TILE_W - 1) / TILE_W;
  g.tiled = g.ntx * g.nty * g.nz <= TILE_PLANES_MAX ? 1 : 0;
  if (cfg.transfer != PL_TRANSFER_FLIP && cfg.transfer != PL_TRANSFER_APIC) {
    snprintf(err, errlen, "pl_create: unknown transfer %d", cfg.transfer);
    return PL_E_ARG;
  }
  if (cfg.domain != PL_DOMAIN_HALF && cfg.domain != PL_DOMAIN_FULL) {
    snprintf(err, errlen, "pl_create: unknown domain %d", cfg.domain);
    return PL_E_ARG;
  }
  g.apic = cfg.transfer == PL_TRANSFER_APIC ? 1 : 0;
  if (cfg.preconditioner < PL_PRECOND_MIC0 || cfg.preconditioner > PL_PRECOND_LEARNED) {
    snprintf(err, errlen, "pl_create: unknown preconditioner %d", cfg.preconditioner);
    return PL_E_ARG;
  }
  if (cfg.solve_precision != PL_SOLVE_F64 && cfg.solve_precision != PL_SOLVE_MIXED) {
    snprintf(err, errlen, "pl_create: unknown solve precision %d", cfg.solve_precision);
    return PL_E_ARG;
  }
  if (cfg.preconditioner == PL_PRECOND_LEARNED && cfg.solve_precision != PL_SOLVE_MIXED) {
    snprintf(err, errlen, "pl_create: the learned preconditioner runs with FP32 vectors (PL_SOLVE_MIXED)");
    return PL_E_ARG;
  }
  g.box_solve = (cfg.preconditioner == PL_PRECOND_BOX_MG || cfg.preconditioner == PL_PRECOND_LEARNED) ? 1 : 0;
  {
    auto p2 = [](int v) {
      int b = 8;
      while (b < v) b *= 2;
      return b;
    };
    g.bx = p2(g.nx), g.by = p2(g.ny), g.bz = p2(g.nz);
  }
  g.solve_cluster = cfg.solve_cluster > 0 ? cfg.solve_cluster : 16;
  g.solve_threads = cfg.solve_threads > 0 ? cfg.solve_threads : 512;
  if (g.solve_cluster > 16 || g.solve_threads < 32 || g.solve_threads > 1024 || g.solve_threads % 32) {
    snprintf(err, errlen, "pl_create: solve shape %d x %d out of range", g.solve_cluster, g.solve_threads);
    return PL_E_ARG;
  }
  {
    double v[2] = {double(g.nx), double(g.ny)};
    g.R = js_hypot<2>(v) * h;  // solver3d.ts:275
  }
  return PL_OK;
}

}  // namespace pl
