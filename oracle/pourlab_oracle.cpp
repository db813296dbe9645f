// TEST INFRASTRUCTURE ONLY — the CPU oracle of the pour-substep engine.
//
// A sequential FP64 restatement of PourLab's 3D reference solver, statement by statement and in
// the reference's operation order, so that its results can be pinned bit-for-bit against the
// reference's committed goldens. Each function names the reference lines it follows
// (paths inside marcelpetrick/teapotFluidSimulation). Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load this library; the CUDA engine never does.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off: no fused multiply-add, so every product
// and sum rounds as JavaScript's IEEE doubles do).
//
// JavaScript math that the restatement reproduces:
//   - Math.hypot: V8 normalises by the largest magnitude and Kahan-sums the squares
//     (js_hypot below); sqrt(x*x+y*y) would differ in the last bit.
//   - x ** 2 is x * x (the pow special case for an exponent of 2); s ** 3 uses pow().
//   - Math.cos/sin/pow: glibc's (like V8's they are within an ulp). One controller angle in the
//     reference's recording differs in its last bit at t = 1.0 s for that reason; the chaotic flow
//     amplifies it after about 2 s, so later recorded frames are compared statistically.

#include "pourlab_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

constexpr uint8_t AIR = 0, FLUID = 1, SOLID = 2;
constexpr uint8_t IN_POT = 0, DISCHARGED = 1, SPILLED = 2, LOST = 3;
constexpr double PI = 3.141592653589793;  // Math.PI
constexpr double DEG = PI / 180;          // motion.ts:13

// JavaScript Math.min / Math.max on two numbers (NaN propagates; -0 < +0).
inline double js_max(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  if (a == 0 && b == 0) return std::signbit(a) ? b : a;
  return a > b ? a : b;
}
inline double js_min(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  if (a == 0 && b == 0) return std::signbit(a) ? a : b;
  return a < b ? a : b;
}

// Math.hypot(...values) as V8 evaluates it.
double js_hypot(const double* v, int n) {
  double mx = 0;
  bool nan = false;
  double absv[4];
  for (int i = 0; i < n; i++) {
    if (std::isnan(v[i])) {
      nan = true;
      absv[i] = 0;
    } else {
      absv[i] = std::fabs(v[i]);
      if (absv[i] > mx) mx = absv[i];
    }
  }
  if (mx == INFINITY) return INFINITY;
  if (nan) return NAN;
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (int i = 0; i < n; i++) {
    double q = absv[i] / mx;
    double summand = q * q - comp;
    double prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return std::sqrt(sum) * mx;
}
inline double hypot2(double a, double b) {
  double v[2] = {a, b};
  return js_hypot(v, 2);
}
inline double hypot3(double a, double b, double c) {
  double v[3] = {a, b, c};
  return js_hypot(v, 3);
}

// ---------------------------------------------------------------- rng.ts:5-14 (mulberry32)
struct Rng {
  uint32_t a;
  explicit Rng(uint32_t seed) : a(seed) {}
  double next() {
    a = a + 0x6d2b79f5u;
    uint32_t t = a;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return double(t ^ (t >> 14)) / 4294967296.0;
  }
};

// ---------------------------------------------------------------- vessel3d.ts:34-103
struct Teapot {
  pl_teapot c;
  double ax, ay, dx, dy, tipX, tipY;
};

Teapot build_teapot(const pl_teapot& cfg) {  // vessel3d.ts:46-59
  Teapot t;
  t.c = cfg;
  double a = (cfg.spout_angle_deg * PI) / 180;
  t.ax = cfg.radius - cfg.wall;
  t.ay = cfg.inlet_height;
  t.dx = std::cos(a);
  t.dy = std::sin(a);
  t.tipX = t.ax + std::cos(a) * cfg.spout_length;
  t.tipY = t.ay + std::sin(a) * cfg.spout_length;
  return t;
}

// vessel3d.ts:62-71: distance to the spout axis segment and the axial parameter.
inline void spout_axis(const Teapot& t, double x, double y, double z, double* dist, double* s) {
  double px = x - t.ax;
  double py = y - t.ay;
  double sv = px * t.dx + py * t.dy;
  double L = t.c.spout_length;
  double sc = sv < 0 ? 0 : sv > L ? L : sv;
  double qx = px - sc * t.dx;
  double qy = py - sc * t.dy;
  *dist = std::sqrt(qx * qx + qy * qy + z * z);
  *s = sv;
}

double teapot_sdf(const Teapot& t, double x, double y, double z) {  // vessel3d.ts:74-95
  const pl_teapot& c = t.c;
  double hw = c.wall / 2;
  double r = std::sqrt(x * x + z * z);
  double ring = std::fabs(r - (c.radius + hw)) - hw;
  double yIn = js_max(-(y + c.wall), y - c.height);
  double side = js_max(ring, yIn);
  double floorD = js_max(std::fabs(y + hw) - hw, r - (c.radius + c.wall));
  double solid = js_min(side, floorD);
  double dist, s;
  spout_axis(t, x, y, z, &dist, &s);
  double L = c.spout_length;
  double along = js_max(-s, s - L);
  double tube = js_max(std::fabs(dist - (c.bore_radius + hw)) - hw, along);
  solid = js_min(solid, js_max(tube, c.radius - r));
  double bore = js_max(js_max(dist - c.bore_radius, -s - c.wall), s - L);
  return js_max(solid, -bore);
}

bool in_cavity(const Teapot& t, double x, double y, double z) {  // vessel3d.ts:98-103
  const pl_teapot& c = t.c;
  if (y >= 0 && y <= c.height && x * x + z * z <= c.radius * c.radius) return true;
  double dist, s;
  spout_axis(t, x, y, z, &dist, &s);
  return s >= 0 && s <= c.spout_length && dist <= c.bore_radius;
}

// ---------------------------------------------------------------- motion.ts:21-159
struct Controller {
  pl_motion cfg;
  int phase = PL_PHASE_WAIT;
  double angle = 0;
  double phaseStart = 0, startAngle = 0, startRate = 0, lastRate = 0;
  int pour = 0;
  double flowRate = 0, lastDischarged = 0;
  double target = 0, manualRate = 0;
  int events = 0;

  explicit Controller(const pl_motion& c) : cfg(c) {  // motion.ts:46-50
    if (c.kind == PL_MOTION_STILL) phase = PL_PHASE_DONE;
    if (c.kind == PL_MOTION_MANUAL) phase = PL_PHASE_MANUAL;
  }
  void setTarget(double angleDeg, double) {  // motion.ts:40-44
    double a = js_max(0, js_min(cfg.max_angle_deg, angleDeg));
    target = a * DEG;
  }
  double pourTarget() const {  // motion.ts:53-56
    int reps = std::max(1, cfg.repeats);
    return (cfg.target_volume * (pour + 1)) / reps;
  }
  void enter(int ph, double t) {  // motion.ts:62-68
    phase = ph;
    phaseStart = t;
    startAngle = angle;
    startRate = lastRate;
    events++;
  }
  bool shouldReturn(double t, double discharged) const {  // motion.ts:145-154
    if (cfg.kind == PL_MOTION_TILT) return phase == PL_PHASE_HOLD && t - phaseStart >= cfg.hold_time;
    if (phase == PL_PHASE_HOLD && t - phaseStart >= cfg.max_hold) return true;
    if (cfg.target_volume <= 0) return false;
    double inTransit = js_max(0, flowRate) * cfg.anticipation * cfg.return_duration;
    return discharged + inTransit >= pourTarget();
  }
  double advance(double t, double dt, double discharged) {  // motion.ts:74-143
    const pl_motion& c = cfg;
    if (dt > 0) {
      double inst = (discharged - lastDischarged) / dt;
      double k = js_min(1, dt / 0.25);
      flowRate += (inst - flowRate) * k;
    }
    lastDischarged = discharged;
    double prev = angle;
    if (phase == PL_PHASE_MANUAL) {
      if (dt > 0) {
        double desired = js_max(-90 * DEG, js_min(90 * DEG, (target - angle) / 0.15));
        double maxChange = 600 * DEG * dt;
        manualRate += js_max(-maxChange, js_min(maxChange, desired - manualRate));
        angle += manualRate * dt;
        lastRate = (angle - prev) / dt;
      }
      return angle;
    }
    double hold = c.hold_angle_deg * DEG;
    double maxA = c.max_angle_deg * DEG;
    int reps = std::max(1, c.repeats);
    for (int guard = 0; guard < 4; guard++) {
      double el = t - phaseStart;
      if (phase == PL_PHASE_WAIT && t >= c.start_delay) {
        enter(PL_PHASE_TILT_IN, c.start_delay);
      } else if ((phase == PL_PHASE_TILT_IN || phase == PL_PHASE_HOLD) && shouldReturn(t, discharged)) {
        enter(PL_PHASE_RETURN, t);
      } else if (phase == PL_PHASE_TILT_IN && el >= c.tilt_duration) {
        angle = hold;
        enter(PL_PHASE_HOLD, phaseStart + c.tilt_duration);
      } else if (phase == PL_PHASE_RETURN && el >= c.return_duration) {
        angle = 0;
        pour++;
        enter(PL_PHASE_REST, phaseStart + c.return_duration);
      } else if (phase == PL_PHASE_REST && pour < reps && el >= c.repeat_gap) {
        enter(PL_PHASE_TILT_IN, phaseStart + c.repeat_gap);
      } else if (phase == PL_PHASE_REST && pour >= reps) {
        enter(PL_PHASE_DONE, t);
      } else {
        break;
      }
    }
    double el = t - phaseStart;
    switch (phase) {
      case PL_PHASE_TILT_IN: {
        double s = js_min(1, el / c.tilt_duration);
        angle = startAngle + (hold - startAngle) * 0.5 * (1 - std::cos(PI * s));
        break;
      }
      case PL_PHASE_HOLD:
        angle = js_min(maxA, startAngle + c.hold_tilt_rate * DEG * el);
        break;
      case PL_PHASE_RETURN: {
        double T = c.return_duration;
        double s = js_min(1, el / T);
        double h00 = 2 * std::pow(s, 3) - 3 * (s * s) + 1;
        double h10 = std::pow(s, 3) - 2 * (s * s) + s;
        angle = h00 * startAngle + h10 * T * startRate;
        break;
      }
      default:
        angle = 0;
    }
    if (dt > 0) lastRate = (angle - prev) / dt;
    return angle;
  }
};

// ---------------------------------------------------------------- Pcg3D, solver3d.ts:827-974
struct SolveResult {
  int iterations;
  bool converged;
  double residual;
};

struct Pcg3D {
  int nx, ny;
  std::vector<double> adiag, ai, aj, ak, pc, r, z, s, as;
  std::vector<int32_t> list;
  int m = 0;

  Pcg3D(int nx_, int ny_, int nz) : nx(nx_), ny(ny_) {  // solver3d.ts:840-856
    size_t n = size_t(nx) * ny * nz;
    adiag.assign(n, 0);
    ai.assign(n, 0);
    aj.assign(n, 0);
    ak.assign(n, 0);
    pc.assign(n, 0);
    r.assign(n, 0);
    z.assign(n, 0);
    s.assign(n, 0);
    as.assign(n, 0);
    list.assign(n, 0);
  }

  // pin (may be null): cells whose diagonal gets +1, the gauge fix of src/sim/pressure.ts:265
  SolveResult solve(const uint8_t* cell, size_t ncell, const double* b, double* q, double tol,
                    int maxIter, const uint8_t* pin = nullptr) {  // solver3d.ts:858-937
    const int nxy = nx * ny;
    std::fill(adiag.begin(), adiag.end(), 0);
    std::fill(ai.begin(), ai.end(), 0);
    std::fill(aj.begin(), aj.end(), 0);
    std::fill(ak.begin(), ak.end(), 0);
    std::fill(pc.begin(), pc.end(), 0);
    std::fill(q, q + ncell, 0.0);
    int mm = 0;
    for (size_t c = 0; c < ncell; c++)
      if (cell[c] == FLUID) list[mm++] = int32_t(c);
    m = mm;
    double bnorm = 0;
    const int offs[6] = {-1, 1, -nx, nx, -nxy, nxy};
    for (int t = 0; t < m; t++) {
      int c = list[t];
      double d = 0;
      for (int o : offs)
        if (cell[c + o] != SOLID) d++;
      if (pin && pin[c]) d++;
      adiag[c] = d;
      ai[c] = cell[c + 1] == FLUID ? -1 : 0;
      aj[c] = cell[c + nx] == FLUID ? -1 : 0;
      ak[c] = cell[c + nxy] == FLUID ? -1 : 0;
      bnorm = js_max(bnorm, std::fabs(b[c]));
    }
    if (m == 0 || bnorm < 1e-14) return {0, true, bnorm};
    const double tau = 0.97;
    for (int t = 0; t < m; t++) {
      int c = list[t];
      double pi = pc[c - 1], pj = pc[c - nx], pk = pc[c - nxy];
      double e1 = ai[c - 1] * pi, e2 = aj[c - nx] * pj, e3 = ak[c - nxy] * pk;
      double e = adiag[c] - e1 * e1 - e2 * e2 - e3 * e3 -
                 tau * (ai[c - 1] * (aj[c - 1] + ak[c - 1]) * pi * pi +
                        aj[c - nx] * (ai[c - nx] + ak[c - nx]) * pj * pj +
                        ak[c - nxy] * (ai[c - nxy] + aj[c - nxy]) * pk * pk);
      if (e < 0.25 * adiag[c]) e = adiag[c];
      pc[c] = e > 0 ? 1 / std::sqrt(e) : 0;
    }
    for (int t = 0; t < m; t++) r[list[t]] = b[list[t]];
    precondition(r.data(), z.data());
    double sigma = 0;
    for (int t = 0; t < m; t++) {
      int c = list[t];
      s[c] = z[c];
      sigma += z[c] * r[c];
    }
    double target = js_max(tol * bnorm, 1e-14);
    double res = bnorm;
    for (int it = 1; it <= maxIter; it++) {
      applyA(s.data(), as.data());
      double sas = 0;
      for (int t = 0; t < m; t++) sas += s[list[t]] * as[list[t]];
      if (!(sas > 0)) break;
      double alpha = sigma / sas;
      res = 0;
      for (int t = 0; t < m; t++) {
        int c = list[t];
        q[c] += alpha * s[c];
        r[c] -= alpha * as[c];
        res = js_max(res, std::fabs(r[c]));
      }
      if (res <= target) return {it, true, res};
      precondition(r.data(), z.data());
      double sn = 0;
      for (int t = 0; t < m; t++) sn += z[list[t]] * r[list[t]];
      double beta = sn / sigma;
      for (int t = 0; t < m; t++) {
        int c = list[t];
        s[c] = z[c] + beta * s[c];
      }
      sigma = sn;
    }
    return {maxIter, res <= target, res};
  }

  void applyA(const double* x, double* y) const {  // solver3d.ts:939-953
    const int nxy = nx * ny;
    for (int t = 0; t < m; t++) {
      int c = list[t];
      y[c] = adiag[c] * x[c] + ai[c] * x[c + 1] + ai[c - 1] * x[c - 1] + aj[c] * x[c + nx] +
             aj[c - nx] * x[c - nx] + ak[c] * x[c + nxy] + ak[c - nxy] * x[c - nxy];
    }
  }

  void precondition(const double* rr, double* zz) {  // solver3d.ts:955-973
    const int nxy = nx * ny;
    double* qv = as.data();
    for (int t = 0; t < m; t++) {
      int c = list[t];
      double v = rr[c] - ai[c - 1] * pc[c - 1] * qv[c - 1] - aj[c - nx] * pc[c - nx] * qv[c - nx] -
                 ak[c - nxy] * pc[c - nxy] * qv[c - nxy];
      qv[c] = v * pc[c];
    }
    for (int t = m - 1; t >= 0; t--) {
      int c = list[t];
      double v = qv[c] - ai[c] * pc[c] * zz[c + 1] - aj[c] * pc[c] * zz[c + nx] -
                 ak[c] * pc[c] * zz[c + nxy];
      zz[c] = v * pc[c];
    }
  }
};

}  // namespace

// ---------------------------------------------------------------- Simulation3D, solver3d.ts:62-824
struct plo_sim {
  pl_config cfg;
  Teapot pot;
  Controller controller;
  int nx, ny, nz;
  double h, fillHeight;
  double pivotWorld[2];
  int n;
  double parcelVolume;
  double zoff = 0;       // world z of the pot-local plane z = 0 (h for the half domain)
  double volFactor = 2;  // the half stands for the pot (2); both halves simulated (1)
  std::vector<double> x, y, z, vx, vy, vz;
  std::vector<double> aff[3][3];  // APIC: gradient of velocity component a along axis b, per parcel
  std::vector<uint8_t> origin, status;
  std::vector<float> y0;
  int bandCounts[3] = {0, 0, 0};
  std::vector<int32_t> dischargeOrder;
  double time = 0;
  int64_t steps = 0;
  double phi = 0, omega = 0;
  std::vector<uint8_t> cell;
  std::vector<double> u, v, w, uPrev, vPrev, wPrev, uw, vw, ww;
  std::vector<uint8_t> uValid, vValid, wValid;
  std::vector<double> rhs, q, density, uc, vc, wc;
  Pcg3D* pcg = nullptr;
  int lastIterations = 0, lastCorrIterations = 0, failures = 0;
  double maxDiv = 0, interior = 1;
  int counts[4] = {0, 0, 0, 0};
  double st[3] = {0, 0, 0};

  explicit plo_sim(const pl_config& c) : cfg(c), pot(build_teapot(c.teapot)), controller(c.motion) {}
  ~plo_sim() { delete pcg; }

  // solver3d.ts:116-228
  void construct() {
    h = cfg.h;
    zoff = h;  // the half domain's plane; the full domain moves it after seeding
    const pl_teapot& t = cfg.teapot;
    fillHeight = cfg.initial_volume / (PI * t.radius * t.radius);
    const double pts[6][2] = {
        {-t.radius - t.wall, -t.wall},
        {-t.radius - t.wall, t.height + 0.02},
        {t.radius + t.wall, -t.wall},
        {t.radius + t.wall, t.height + 0.02},
        {pot.tipX + 0.02, pot.tipY + 0.02},
        {pot.tipX + 0.02, pot.tipY - 0.03},
    };
    double x0 = INFINITY, x1 = -INFINITY, y0v = INFINITY, y1 = -INFINITY;
    double maxA = js_max(cfg.motion.max_angle_deg, cfg.motion.hold_angle_deg);
    for (double a = 0; a <= maxA; a += 2) {
      double ph = (-a * PI) / 180;
      double c = std::cos(ph), s = std::sin(ph);
      for (const auto& p : pts) {
        double rx = p[0] - cfg.pivot[0];
        double ry = p[1] - cfg.pivot[1];
        double wx = c * rx - s * ry;
        double wy = s * rx + c * ry;
        x0 = js_min(x0, wx);
        x1 = js_max(x1, wx);
        y0v = js_min(y0v, wy);
        y1 = js_max(y1, wy);
      }
    }
    double m = 3 * h;
    pivotWorld[0] = -x0 + m;
    pivotWorld[1] = -y0v + m;
    nx = int(std::ceil((x1 - x0 + 2 * m) / h));
    ny = int(std::ceil((y1 - y0v + 2 * m) / h));
    nz = int(std::ceil((t.radius + t.wall + 2 * h) / h)) + 1;

    Rng rng(cfg.seed);
    double s = h / 2;
    std::vector<double> xs;
    double loc[3];
    for (int k = 0; k < nz * 2; k++)
      for (int j = 0; j < ny * 2; j++)
        for (int i = 0; i < nx * 2; i++) {
          double wx = (i + 0.5 + (rng.next() - 0.5) * 0.5) * s;
          double wy = (j + 0.5 + (rng.next() - 0.5) * 0.5) * s;
          double wz = (k + 0.5 + (rng.next() - 0.5) * 0.5) * s;
          toLocal(wx, wy, wz, loc);
          if (loc[2] < 0 || loc[1] < 0 || loc[1] > fillHeight) continue;
          if (!in_cavity(pot, loc[0], loc[1], loc[2])) continue;
          if (teapot_sdf(pot, loc[0], loc[1], loc[2]) < 0.4 * h) continue;
          xs.push_back(wx);
          xs.push_back(wy);
          xs.push_back(wz);
        }
    n = int(xs.size() / 3);
    parcelVolume = cfg.initial_volume / (2 * double(n));
    x.resize(n);
    y.resize(n);
    z.resize(n);
    vx.assign(n, 0);
    vy.assign(n, 0);
    vz.assign(n, 0);
    for (auto& row : aff)
      for (auto& c : row) c.assign(n, 0);
    origin.assign(n, 0);
    status.assign(n, 0);
    y0.resize(n);
    for (int p = 0; p < n; p++) {
      x[p] = xs[3 * p];
      y[p] = xs[3 * p + 1];
      z[p] = xs[3 * p + 2];
      toLocal(x[p], y[p], z[p], loc);
      y0[p] = float(loc[1]);
    }
    // solver3d.ts:221-226: order by Float32 y0, index breaks ties.
    std::vector<int32_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
      if (y0[a] != y0[b]) return y0[a] < y0[b];
      return a < b;
    });
    for (int r = 0; r < n; r++) {
      int k = std::min(2, int(std::floor((double(r) * 3) / n)));
      origin[order[r]] = uint8_t(k);
      bandCounts[k]++;
    }
    volFactor = 2;
    if (cfg.domain == PL_DOMAIN_FULL) {
      // Full domain (no counterpart in the reference): both halves, the symmetry plane a cell face at
      // world z = zoff, every seeded parcel plus its mirror image (ids n..2n-1, same origin layer).
      const int nzHalf = nz;
      nz = 2 * nzHalf - 2;
      zoff = (nzHalf - 1) * h;
      const int nh = n;
      n = 2 * nh;
      x.resize(n), y.resize(n), z.resize(n), vx.assign(n, 0), vy.assign(n, 0), vz.assign(n, 0);
      origin.resize(n), status.assign(n, 0), y0.resize(n);
      for (auto& row : aff)
        for (auto& c : row) c.assign(n, 0);
      for (int p = 0; p < nh; p++) {
        const double lz = z[p] - h;
        z[p] = lz + zoff;
        x[nh + p] = x[p];
        y[nh + p] = y[p];
        z[nh + p] = -lz + zoff;
        origin[nh + p] = origin[p];
        y0[nh + p] = y0[p];
      }
      for (int k = 0; k < 3; k++) bandCounts[k] *= 2;
      volFactor = 1;
    }
    size_t nc = size_t(nx) * ny * nz;
    cell.assign(nc, 0);
    size_t nu = size_t(nx + 1) * ny * nz, nv = size_t(nx) * (ny + 1) * nz, nw = size_t(nx) * ny * (nz + 1);
    u.assign(nu, 0);
    uPrev.assign(nu, 0);
    uw.assign(nu, 0);
    uValid.assign(nu, 0);
    uc.assign(nu, 0);
    v.assign(nv, 0);
    vPrev.assign(nv, 0);
    vw.assign(nv, 0);
    vValid.assign(nv, 0);
    vc.assign(nv, 0);
    w.assign(nw, 0);
    wPrev.assign(nw, 0);
    ww.assign(nw, 0);
    wValid.assign(nw, 0);
    wc.assign(nw, 0);
    rhs.assign(nc, 0);
    q.assign(nc, 0);
    density.assign(nc, 0);
    pcg = new Pcg3D(nx, ny, nz);
    counts[0] = n;
    counts[1] = counts[2] = counts[3] = 0;
  }

  // solver3d.ts:232-260
  void toLocal(double wx, double wy, double wz, double* out) const { toLocalAt(phi, wx, wy, wz, out); }
  void toLocalAt(double ph, double wx, double wy, double wz, double* out) const {
    double c = std::cos(ph), s = std::sin(ph);
    double rx = wx - pivotWorld[0];
    double ry = wy - pivotWorld[1];
    out[0] = c * rx + s * ry + cfg.pivot[0];
    out[1] = -s * rx + c * ry + cfg.pivot[1];
    out[2] = wz - zoff;
  }
  void toWorldAt(double ph, double lx, double ly, double lz, double* out) const {
    double c = std::cos(ph), s = std::sin(ph);
    double rx = lx - cfg.pivot[0];
    double ry = ly - cfg.pivot[1];
    out[0] = c * rx - s * ry + pivotWorld[0];
    out[1] = s * rx + c * ry + pivotWorld[1];
    out[2] = lz + zoff;
  }

  bool finished() const { return time >= cfg.duration - 1e-9; }  // solver3d.ts:264-266

  double stableDt() const {  // solver3d.ts:268-278
    double m = 0;
    for (int p = 0; p < n; p++) {
      if (status[p] != IN_POT) continue;
      double s = vx[p] * vx[p] + vy[p] * vy[p] + vz[p] * vz[p];
      if (s > m) m = s;
    }
    double R = hypot2(nx, ny) * h;
    double speed = std::sqrt(m) + std::sqrt(5 * h * cfg.gravity) + std::fabs(omega) * R;
    return js_min(cfg.max_substep, (cfg.cfl * h) / speed);
  }

  void advance(double duration) {  // solver3d.ts:281-286
    double end = time + duration;
    while (time < end - 1e-12 && !finished()) step(js_min(stableDt(), cfg.duration - time));
  }

  void step(double dt) {  // solver3d.ts:288-309
    double discharged = counts[DISCHARGED] * parcelVolume * volFactor;
    double tilt1 = controller.advance(time + dt, dt, discharged);
    double phi1 = -tilt1;
    omega = (phi1 - phi) / dt;
    classify();
    particlesToGrid();
    uPrev = u;
    vPrev = v;
    wPrev = w;
    applyGravity(dt);
    setSolidFaces();
    project();
    markValid();
    extrapolate();
    gridToParticles();
    densityCorrection(dt);
    advect(dt, phi1);
    phi = phi1;
    time += dt;
    steps++;
  }

  void classify() {  // solver3d.ts:313-336
    double loc[3];
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t c = i + size_t(nx) * (j + size_t(ny) * k);
          if (i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1) {
            cell[c] = SOLID;
            continue;
          }
          toLocal((i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h, loc);
          cell[c] = teapot_sdf(pot, loc[0], loc[1], loc[2]) < 0 ? SOLID : AIR;
        }
    for (int p = 0; p < n; p++) {
      if (status[p] != IN_POT) continue;
      double fi = std::floor(x[p] / h), fj = std::floor(y[p] / h), fk = std::floor(z[p] / h);
      if (std::isnan(fi + fj + fk)) continue;  // cell[NaN] reads undefined in JavaScript: no-op
      if (fi < 1 || fj < 1 || fk < 1 || fi >= nx - 1 || fj >= ny - 1 || fk >= nz - 1) continue;
      size_t c = size_t(fi) + size_t(nx) * (size_t(fj) + size_t(ny) * size_t(fk));
      if (cell[c] == AIR) cell[c] = FLUID;
    }
  }

  // A stencil of a NaN position: every corner index is NaN in the reference, and a typed array indexed
  // with NaN reads undefined (NaN in arithmetic, falsy as a mask) and ignores writes.
  static constexpr size_t NAN_INDEX = ~size_t(0);

  // solver3d.ts:339-362 (NAN_INDEX when a coordinate is NaN)
  size_t stencil(double px, double py, double pz, double ox, double oy, double oz, int sx, int sy, int sz,
                 double* out) const {
    double gx = px / h - ox, gy = py / h - oy, gz = pz / h - oz;
    double i = js_max(0, js_min(sx - 2, std::floor(gx)));
    double j = js_max(0, js_min(sy - 2, std::floor(gy)));
    double k = js_max(0, js_min(sz - 2, std::floor(gz)));
    out[0] = js_max(0, js_min(1, gx - i));
    out[1] = js_max(0, js_min(1, gy - j));
    out[2] = js_max(0, js_min(1, gz - k));
    if (std::isnan(i + j + k)) return NAN_INDEX;
    return size_t(i) + size_t(sx) * (size_t(j) + size_t(sy) * size_t(k));
  }

  // solver3d.ts:366-377: corner indices and weights in the reference's order.
  template <class F>
  void forEachCorner(size_t base, int sx, int sy, F cb) const {
    double fx = st[0], fy = st[1], fz = st[2];
    size_t sxy = size_t(sx) * sy;
    cb(base, (1 - fx) * (1 - fy) * (1 - fz));
    cb(base + 1, fx * (1 - fy) * (1 - fz));
    cb(base + sx, (1 - fx) * fy * (1 - fz));
    cb(base + sx + 1, fx * fy * (1 - fz));
    cb(base + sxy, (1 - fx) * (1 - fy) * fz);
    cb(base + sxy + 1, fx * (1 - fy) * fz);
    cb(base + sxy + sx, (1 - fx) * fy * fz);
    cb(base + sxy + sx + 1, fx * fy * fz);
  }

  void dims(int comp, double* o, int* sz) const {  // solver3d.ts:379-384
    if (comp == 0) {
      o[0] = 0, o[1] = 0.5, o[2] = 0.5, sz[0] = nx + 1, sz[1] = ny, sz[2] = nz;
    } else if (comp == 1) {
      o[0] = 0.5, o[1] = 0, o[2] = 0.5, sz[0] = nx, sz[1] = ny + 1, sz[2] = nz;
    } else {
      o[0] = 0.5, o[1] = 0.5, o[2] = 0, sz[0] = nx, sz[1] = ny, sz[2] = nz + 1;
    }
  }

  // solver3d.ts:386-408
  double sample(const std::vector<double>& field, int comp, double px, double py, double pz,
                const std::vector<uint8_t>* valid) {
    double o[3];
    int sz[3];
    dims(comp, o, sz);
    size_t base = stencil(px, py, pz, o[0], o[1], o[2], sz[0], sz[1], sz[2], st);
    if (base == NAN_INDEX) return NAN;  // all = NaN, ws = 0
    double acc = 0, ws = 0, all = 0;
    forEachCorner(base, sz[0], sz[1], [&](size_t idx, double wgt) {
      all += wgt * field[idx];
      if (!valid || (*valid)[idx]) {
        acc += wgt * field[idx];
        ws += wgt;
      }
    });
    if (!valid) return all;
    return ws > 1e-9 ? acc / ws : all;
  }

  void particlesToGrid() {  // solver3d.ts:410-431
    std::vector<double>* fields[3][3] = {{&u, &uw, &vx}, {&v, &vw, &vy}, {&w, &ww, &vz}};
    for (int comp = 0; comp < 3; comp++) {
      std::vector<double>& f = *fields[comp][0];
      std::vector<double>& wt = *fields[comp][1];
      const std::vector<double>& vel = *fields[comp][2];
      std::fill(f.begin(), f.end(), 0);
      std::fill(wt.begin(), wt.end(), 0);
      double o[3];
      int sz[3];
      dims(comp, o, sz);
      const bool apic = cfg.transfer == PL_TRANSFER_APIC;
      for (int p = 0; p < n; p++) {
        if (status[p] != IN_POT) continue;
        size_t base = stencil(x[p], y[p], z[p], o[0], o[1], o[2], sz[0], sz[1], sz[2], st);
        if (base == NAN_INDEX) continue;  // writes to NaN indices are ignored
        double vp = vel[p];
        if (apic) {  // affine field at each corner face (src/sim/solver.ts:553-587 in 3D)
          const size_t sxy = size_t(sz[0]) * sz[1];
          const double fi = double(base % sz[0]), fj = double((base / sz[0]) % sz[1]), fk = double(base / sxy);
          const double cx = aff[comp][0][p], cy = aff[comp][1][p], cz = aff[comp][2][p];
          const double d0x = (fi + o[0]) * h - x[p], d0y = (fj + o[1]) * h - y[p], d0z = (fk + o[2]) * h - z[p];
          forEachCorner(base, sz[0], sz[1], [&](size_t idx, double wgt) {
            const size_t rel = idx - base;
            const int di = int(rel % sz[0]), dj = int((rel / sz[0]) % sz[1]), dk = int(rel / sxy);
            const double a = vp + cx * (d0x + di * h) + cy * (d0y + dj * h) + cz * (d0z + dk * h);
            f[idx] += wgt * a;
            wt[idx] += wgt;
          });
          continue;
        }
        forEachCorner(base, sz[0], sz[1], [&](size_t idx, double wgt) {
          f[idx] += wgt * vp;
          wt[idx] += wgt;
        });
      }
      for (size_t i = 0; i < f.size(); i++) f[i] = wt[i] > 1e-9 ? f[i] / wt[i] : 0;
    }
  }

  void applyGravity(double dt) {  // solver3d.ts:433-443
    double g = cfg.gravity * dt;
    for (int k = 0; k < nz; k++)
      for (int j = 1; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          uint8_t below = cell[i + size_t(nx) * (j - 1 + size_t(ny) * k)];
          uint8_t above = cell[i + size_t(nx) * (j + size_t(ny) * k)];
          if (below == FLUID || above == FLUID) v[i + size_t(nx) * (j + size_t(ny + 1) * k)] -= g;
        }
  }

  void setSolidFaces() {  // solver3d.ts:446-471
    double om = omega;
    double pwx = pivotWorld[0], pwy = pivotWorld[1];
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i <= nx; i++) {
          uint8_t a = i > 0 ? cell[i - 1 + size_t(nx) * (j + size_t(ny) * k)] : SOLID;
          uint8_t b = i < nx ? cell[i + size_t(nx) * (j + size_t(ny) * k)] : SOLID;
          if (a == SOLID || b == SOLID) u[i + size_t(nx + 1) * (j + size_t(ny) * k)] = -om * ((j + 0.5) * h - pwy);
        }
    for (int k = 0; k < nz; k++)
      for (int j = 0; j <= ny; j++)
        for (int i = 0; i < nx; i++) {
          uint8_t a = j > 0 ? cell[i + size_t(nx) * (j - 1 + size_t(ny) * k)] : SOLID;
          uint8_t b = j < ny ? cell[i + size_t(nx) * (j + size_t(ny) * k)] : SOLID;
          if (a == SOLID || b == SOLID) v[i + size_t(nx) * (j + size_t(ny + 1) * k)] = om * ((i + 0.5) * h - pwx);
        }
    for (int k = 0; k <= nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          uint8_t a = k > 0 ? cell[i + size_t(nx) * (j + size_t(ny) * (k - 1))] : SOLID;
          uint8_t b = k < nz ? cell[i + size_t(nx) * (j + size_t(ny) * k)] : SOLID;
          if (a == SOLID || b == SOLID) w[i + size_t(nx) * (j + size_t(ny) * k)] = 0;
        }
  }

  double divergenceRhs() {  // solver3d.ts:473-493
    std::fill(rhs.begin(), rhs.end(), 0);
    double m = 0;
    for (int k = 1; k < nz - 1; k++)
      for (int j = 1; j < ny - 1; j++)
        for (int i = 1; i < nx - 1; i++) {
          size_t c = i + size_t(nx) * (j + size_t(ny) * k);
          if (cell[c] != FLUID) continue;
          double d = u[i + 1 + size_t(nx + 1) * (j + size_t(ny) * k)] - u[i + size_t(nx + 1) * (j + size_t(ny) * k)] +
                     v[i + size_t(nx) * (j + 1 + size_t(ny + 1) * k)] - v[i + size_t(nx) * (j + size_t(ny + 1) * k)] +
                     w[i + size_t(nx) * (j + size_t(ny) * (k + 1))] - w[i + size_t(nx) * (j + size_t(ny) * k)];
          rhs[c] = -d;
          if (std::fabs(d) > m) m = std::fabs(d);
        }
    return m / h;
  }

  // solver3d.ts:496-528
  void applyGradient(const std::vector<double>& qq, std::vector<double>& fu, std::vector<double>& fv,
                     std::vector<double>& fw, double sign) {
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 1; i < nx; i++) {
          size_t a = i - 1 + size_t(nx) * (j + size_t(ny) * k);
          size_t b = a + 1;
          if (cell[a] == SOLID || cell[b] == SOLID || (cell[a] != FLUID && cell[b] != FLUID)) continue;
          fu[i + size_t(nx + 1) * (j + size_t(ny) * k)] += sign * (qq[b] - qq[a]);
        }
    for (int k = 0; k < nz; k++)
      for (int j = 1; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t a = i + size_t(nx) * (j - 1 + size_t(ny) * k);
          size_t b = a + nx;
          if (cell[a] == SOLID || cell[b] == SOLID || (cell[a] != FLUID && cell[b] != FLUID)) continue;
          fv[i + size_t(nx) * (j + size_t(ny + 1) * k)] += sign * (qq[b] - qq[a]);
        }
    for (int k = 1; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t a = i + size_t(nx) * (j + size_t(ny) * (k - 1));
          size_t b = a + size_t(nx) * ny;
          if (cell[a] == SOLID || cell[b] == SOLID || (cell[a] != FLUID && cell[b] != FLUID)) continue;
          fw[i + size_t(nx) * (j + size_t(ny) * k)] += sign * (qq[b] - qq[a]);
        }
  }

  void project() {  // solver3d.ts:530-543
    divergenceRhs();
    SolveResult res = pcg->solve(cell.data(), cell.size(), rhs.data(), q.data(), cfg.pressure_tolerance,
                                 cfg.pressure_max_iterations);
    lastIterations = res.iterations;
    if (!res.converged) failures++;
    applyGradient(q, u, v, w, -1);
    maxDiv = divergenceRhs();
  }

  void markValid() {  // solver3d.ts:545-562
    auto mark = [&](std::vector<uint8_t>& valid, int sx, int sy, int sz, int comp) {
      for (int k = 0; k < sz; k++)
        for (int j = 0; j < sy; j++)
          for (int i = 0; i < sx; i++) {
            int ia = comp == 0 ? i - 1 : i;
            int ja = comp == 1 ? j - 1 : j;
            int ka = comp == 2 ? k - 1 : k;
            uint8_t a = ia >= 0 && ja >= 0 && ka >= 0 ? cell[ia + size_t(nx) * (ja + size_t(ny) * ka)] : SOLID;
            uint8_t b = i < nx && j < ny && k < nz ? cell[i + size_t(nx) * (j + size_t(ny) * k)] : SOLID;
            valid[i + size_t(sx) * (j + size_t(sy) * k)] =
                a == SOLID || b == SOLID || a == FLUID || b == FLUID ? 1 : 0;
          }
    };
    mark(uValid, nx + 1, ny, nz, 0);
    mark(vValid, nx, ny + 1, nz, 1);
    mark(wValid, nx, ny, nz + 1, 2);
  }

  void extrapolate() {  // solver3d.ts:565-605
    auto ex = [&](std::vector<double>& f, const std::vector<uint8_t>& valid, int sx, int sy, int sz) {
      std::vector<uint8_t> vm = valid;
      std::vector<size_t> add;
      std::vector<double> vals;
      size_t sxy = size_t(sx) * sy;
      for (int layer = 0; layer < 2; layer++) {
        add.clear();
        vals.clear();
        for (int k = 0; k < sz; k++)
          for (int j = 0; j < sy; j++)
            for (int i = 0; i < sx; i++) {
              size_t c = i + size_t(sx) * (j + size_t(sy) * k);
              if (vm[c]) continue;
              double s = 0;
              int cnt = 0;
              auto nb = [&](size_t d, bool ok) {
                if (ok && vm[d]) {
                  s += f[d];
                  cnt++;
                }
              };
              nb(c - 1, i > 0);
              nb(c + 1, i < sx - 1);
              nb(c - sx, j > 0);
              nb(c + sx, j < sy - 1);
              nb(c - sxy, k > 0);
              nb(c + sxy, k < sz - 1);
              if (cnt > 0) {
                add.push_back(c);
                vals.push_back(s / cnt);
              }
            }
        for (size_t t = 0; t < add.size(); t++) {
          f[add[t]] = vals[t];
          vm[add[t]] = 1;
        }
      }
    };
    ex(u, uValid, nx + 1, ny, nz);
    ex(v, vValid, nx, ny + 1, nz);
    ex(w, wValid, nx, ny, nz + 1);
  }

  // Gradient of component comp's trilinear interpolant at (px, py, pz) from the unmasked corners (the
  // 3D form of src/sim/solver.ts:958-964).
  void interpGradient(const std::vector<double>& field, int comp, double px, double py, double pz, double* g3) {
    double o[3];
    int sz[3];
    dims(comp, o, sz);
    size_t base = stencil(px, py, pz, o[0], o[1], o[2], sz[0], sz[1], sz[2], st);
    if (base == NAN_INDEX) {
      g3[0] = g3[1] = g3[2] = NAN;
      return;
    }
    const size_t sx = size_t(sz[0]), sxy = size_t(sz[0]) * sz[1];
    double u[8];
    for (int c = 0; c < 8; c++) u[c] = field[base + (c & 1) + ((c & 2) ? sx : 0) + ((c & 4) ? sxy : 0)];
    const double fx = st[0], fy = st[1], fz = st[2];
    g3[0] = ((1 - fy) * (1 - fz) * (u[1] - u[0]) + fy * (1 - fz) * (u[3] - u[2]) + (1 - fy) * fz * (u[5] - u[4]) +
             fy * fz * (u[7] - u[6])) / h;
    g3[1] = ((1 - fx) * (1 - fz) * (u[2] - u[0]) + fx * (1 - fz) * (u[3] - u[1]) + (1 - fx) * fz * (u[6] - u[4]) +
             fx * fz * (u[7] - u[5])) / h;
    g3[2] = ((1 - fx) * (1 - fy) * (u[4] - u[0]) + fx * (1 - fy) * (u[5] - u[1]) + (1 - fx) * fy * (u[6] - u[2]) +
             fx * fy * (u[7] - u[3])) / h;
  }

  void gridToParticles() {  // solver3d.ts:607-624
    double a = cfg.flip_ratio;
    if (cfg.transfer == PL_TRANSFER_APIC) {  // src/sim/solver.ts:956-986 in 3D: PIC sample + gradient
      const std::vector<double>* f[3] = {&u, &v, &w};
      const std::vector<uint8_t>* va[3] = {&uValid, &vValid, &wValid};
      std::vector<double>* vel[3] = {&vx, &vy, &vz};
      for (int p = 0; p < n; p++) {
        if (status[p] != IN_POT) continue;
        for (int comp = 0; comp < 3; comp++) {
          (*vel[comp])[p] = sample(*f[comp], comp, x[p], y[p], z[p], va[comp]);
          double g3[3];
          interpGradient(*f[comp], comp, x[p], y[p], z[p], g3);
          for (int b = 0; b < 3; b++) aff[comp][b][p] = g3[b];
        }
      }
      return;
    }
    for (int p = 0; p < n; p++) {
      if (status[p] != IN_POT) continue;
      double px = x[p], py = y[p], pz = z[p];
      double un = sample(u, 0, px, py, pz, &uValid);
      double vn = sample(v, 1, px, py, pz, &vValid);
      double wn = sample(w, 2, px, py, pz, &wValid);
      double uo = sample(uPrev, 0, px, py, pz, &uValid);
      double vo = sample(vPrev, 1, px, py, pz, &vValid);
      double wo = sample(wPrev, 2, px, py, pz, &wValid);
      vx[p] = (1 - a) * un + a * (vx[p] + un - uo);
      vy[p] = (1 - a) * vn + a * (vy[p] + vn - vo);
      vz[p] = (1 - a) * wn + a * (vz[p] + wn - wo);
    }
  }

  void densityCorrection(double dt) {  // solver3d.ts:627-675
    double kappa = cfg.density_correction;
    std::fill(uc.begin(), uc.end(), 0);
    std::fill(vc.begin(), vc.end(), 0);
    std::fill(wc.begin(), wc.end(), 0);
    std::fill(density.begin(), density.end(), 0);
    double ds[3];
    for (int p = 0; p < n; p++) {
      if (status[p] != IN_POT) continue;
      size_t base = stencil(x[p], y[p], z[p], 0.5, 0.5, 0.5, nx, ny, nz, ds);
      if (base == NAN_INDEX) continue;
      st[0] = ds[0], st[1] = ds[1], st[2] = ds[2];
      forEachCorner(base, nx, ny, [&](size_t idx, double wgt) { density[idx] += wgt; });
    }
    std::fill(rhs.begin(), rhs.end(), 0);
    int interiorCount = 0;
    double sum = 0;
    bool any = false;
    size_t nxy = size_t(nx) * ny;
    for (int k = 1; k < nz - 1; k++)
      for (int j = 1; j < ny - 1; j++)
        for (int i = 1; i < nx - 1; i++) {
          size_t c = i + size_t(nx) * (j + size_t(ny) * k);
          if (cell[c] != FLUID) continue;
          double ratio = density[c] / 8;
          bool isInterior = cell[c - 1] != AIR && cell[c + 1] != AIR && cell[c - nx] != AIR &&
                            cell[c + nx] != AIR && cell[c - nxy] != AIR && cell[c + nxy] != AIR;
          if (isInterior) {
            interiorCount++;
            sum += ratio;
          }
          if (kappa > 0 && (ratio > 1 || isInterior)) {
            rhs[c] = (kappa * (ratio - 1) * h) / dt;
            any = true;
          }
        }
    interior = interiorCount > 0 ? sum / interiorCount : 1;
    lastCorrIterations = 0;
    if (!any) return;
    std::vector<double> qc(cell.size(), 0.0);
    SolveResult r = pcg->solve(cell.data(), cell.size(), rhs.data(), qc.data(), 1e-4, 80);
    lastCorrIterations = r.iterations;
    applyGradient(qc, uc, vc, wc, -1);
  }

  void setStatus(int p, uint8_t s) {  // solver3d.ts:790-794
    counts[status[p]]--;
    counts[s]++;
    status[p] = s;
  }

  void advect(double dt, double phi1) {  // solver3d.ts:677-788
    double out[3], loc0[3], loc1[3];
    bool corr = cfg.density_correction > 0;
    const double eps = 1e-4;
    double margin = 0.1 * h;
    const pl_teapot& pc = pot.c;
    double lo = h * 1.01;
    double hiX = (nx - 1) * h, hiY = (ny - 1) * h, hiZ = (nz - 1) * h;
    double g = cfg.gravity;
    for (int p = 0; p < n; p++) {
      uint8_t stp = status[p];
      if (stp == DISCHARGED || stp == SPILLED) {
        if (y[p] > -1) {
          vy[p] -= g * dt;
          x[p] += vx[p] * dt;
          y[p] += vy[p] * dt;
          z[p] += vz[p] * dt;
        }
        continue;
      }
      if (stp != IN_POT) continue;
      double x0 = x[p], yy0 = y[p], z0 = z[p];
      toLocal(x0, yy0, z0, loc0);
      double u1 = sample(u, 0, x0, yy0, z0, nullptr);
      double v1 = sample(v, 1, x0, yy0, z0, nullptr);
      double w1 = sample(w, 2, x0, yy0, z0, nullptr);
      double xm = x0 + 0.5 * dt * u1;
      double ym = yy0 + 0.5 * dt * v1;
      double zm = z0 + 0.5 * dt * w1;
      double x1 = x0 + dt * sample(u, 0, xm, ym, zm, nullptr);
      double y1 = yy0 + dt * sample(v, 1, xm, ym, zm, nullptr);
      double z1 = z0 + dt * sample(w, 2, xm, ym, zm, nullptr);
      if (corr) {
        x1 += dt * sample(uc, 0, x0, yy0, z0, nullptr);
        y1 += dt * sample(vc, 1, x0, yy0, z0, nullptr);
        z1 += dt * sample(wc, 2, x0, yy0, z0, nullptr);
      }
      toLocalAt(phi1, x1, y1, z1, loc1);
      double d = teapot_sdf(pot, loc1[0], loc1[1], loc1[2]);
      if (d < margin) {
        double gx = teapot_sdf(pot, loc1[0] + eps, loc1[1], loc1[2]) - teapot_sdf(pot, loc1[0] - eps, loc1[1], loc1[2]);
        double gy = teapot_sdf(pot, loc1[0], loc1[1] + eps, loc1[2]) - teapot_sdf(pot, loc1[0], loc1[1] - eps, loc1[2]);
        double gz = teapot_sdf(pot, loc1[0], loc1[1], loc1[2] + eps) - teapot_sdf(pot, loc1[0], loc1[1], loc1[2] - eps);
        double gl = hypot3(gx, gy, gz);
        if (gl == 0 || std::isnan(gl)) gl = 1;  // `|| 1`: 0 and NaN are falsy
        double push = margin - d;
        loc1[0] += (gx / gl) * push;
        loc1[1] += (gy / gl) * push;
        loc1[2] += (gz / gl) * push;
        toWorldAt(phi1, loc1[0], loc1[1], loc1[2], out);
        x1 = out[0];
        y1 = out[1];
        z1 = out[2];
        double c = std::cos(phi1), s = std::sin(phi1);
        double nwx = (c * gx - s * gy) / gl;
        double nwy = (s * gx + c * gy) / gl;
        double nwz = gz / gl;
        double wvx = -omega * (y1 - pivotWorld[1]);
        double wvy = omega * (x1 - pivotWorld[0]);
        double rn = (vx[p] - wvx) * nwx + (vy[p] - wvy) * nwy + vz[p] * nwz;
        if (rn < 0) {
          vx[p] -= rn * nwx;
          vy[p] -= rn * nwy;
          vz[p] -= rn * nwz;
        }
      }
      if (cfg.domain != PL_DOMAIN_FULL && z1 < h) {  // symmetry plane (half domain)
        z1 = 2 * h - z1;
        vz[p] = std::fabs(vz[p]);
      }
      if (!std::isfinite(x1 + y1 + z1)) {
        setStatus(p, LOST);
        continue;
      }
      x[p] = x1;
      y[p] = y1;
      z[p] = z1;
      toLocalAt(phi1, x1, y1, z1, loc1);
      double s0 = (loc0[0] - pot.tipX) * pot.dx + (loc0[1] - pot.tipY) * pot.dy;
      double s1 = (loc1[0] - pot.tipX) * pot.dx + (loc1[1] - pot.tipY) * pot.dy;
      if (s0 < 0 && s1 >= 0) {
        double rx = loc1[0] - pot.tipX - s1 * pot.dx;
        double ry = loc1[1] - pot.tipY - s1 * pot.dy;
        if (hypot3(rx, ry, loc1[2]) < pc.bore_radius + 3 * pc.wall) {
          setStatus(p, DISCHARGED);
          dischargeOrder.push_back(p);
          continue;
        }
      }
      double r = hypot2(loc1[0], loc1[2]);
      bool insideBody = r < pc.radius + 2 * pc.wall && loc1[1] > -2 * pc.wall;
      bool nearSpout = loc1[0] > 0 && loc1[0] < pot.tipX + 0.03;
      bool atEdge = x1 <= lo || y1 <= lo || x1 >= hiX || y1 >= hiY || z1 >= hiZ ||
                    (cfg.domain == PL_DOMAIN_FULL && z1 <= lo);
      if ((!insideBody && !nearSpout) || atEdge) setStatus(p, SPILLED);
    }
  }

  void diagnostics(pl_diagnostics* d) const {  // solver3d.ts:796-814
    double vml = parcelVolume * volFactor * 1e6;
    d->time = time;
    d->steps = steps;
    d->angle_deg = controller.angle / DEG;
    d->phase = controller.phase;
    d->particles = n;
    d->grid[0] = nx, d->grid[1] = ny, d->grid[2] = nz;
    d->pressure_iterations = lastIterations;
    d->pressure_failures = failures;
    d->correction_iterations = lastCorrIterations;
    d->discharged_ml = counts[DISCHARGED] * vml;
    d->spilled_ml = counts[SPILLED] * vml;
    d->lost_ml = counts[LOST] * vml;
    d->in_pot_ml = counts[IN_POT] * vml;
    d->max_divergence = maxDiv;
    d->interior_density = interior;
  }
};

// ---------------------------------------------------------------- C ABI

extern "C" {

int plo_create(const pl_config* cfg, plo_sim** out) {
  if (!cfg || !out || !(cfg->h > 0)) return PL_E_ARG;
  plo_sim* s = new plo_sim(*cfg);
  s->construct();
  *out = s;
  return PL_OK;
}

void plo_destroy(plo_sim* s) { delete s; }

int plo_get_sizes(const plo_sim* s, pl_sizes* o) {
  o->n = s->n;
  o->nx = s->nx, o->ny = s->ny, o->nz = s->nz;
  o->h = s->h;
  o->parcel_volume = s->parcelVolume;
  o->pivot_world[0] = s->pivotWorld[0], o->pivot_world[1] = s->pivotWorld[1];
  o->fill_height = s->fillHeight;
  for (int k = 0; k < 3; k++) o->band_counts[k] = s->bandCounts[k];
  o->step_copy_bytes = 0;  // no device scalar block on the CPU
  return PL_OK;
}

double plo_stable_dt(plo_sim* s) { return s->stableDt(); }
int plo_finished(const plo_sim* s) { return s->finished() ? 1 : 0; }

int plo_step(plo_sim* s, double dt) {
  if (!(dt > 0)) dt = js_min(s->stableDt(), s->cfg.duration - s->time);
  s->step(dt);
  return PL_OK;
}

int plo_advance(plo_sim* s, double duration, pl_diagnostics* out) {
  s->advance(duration);
  if (out) s->diagnostics(out);
  return PL_OK;
}

int plo_set_tilt_target(plo_sim* s, double angle_deg, double time) {
  s->controller.setTarget(angle_deg, time);
  return PL_OK;
}

int plo_diagnostics(const plo_sim* s, pl_diagnostics* out) {
  s->diagnostics(out);
  return PL_OK;
}

int plo_discharged_fractions(const plo_sim* s, double out[3]) {  // solver3d.ts:817-823
  size_t n = s->dischargeOrder.size();
  if (n == 0) return PL_NONE;
  double c[3] = {0, 0, 0};
  for (int32_t p : s->dischargeOrder) c[s->origin[p]]++;
  for (int k = 0; k < 3; k++) out[k] = c[k] / double(n);
  return PL_OK;
}

int plo_read_particles(const plo_sim* s, double* x, double* y, double* z, double* vx, double* vy,
                       double* vz, uint8_t* status) {
  size_t n = size_t(s->n);
  if (x) std::memcpy(x, s->x.data(), n * 8);
  if (y) std::memcpy(y, s->y.data(), n * 8);
  if (z) std::memcpy(z, s->z.data(), n * 8);
  if (vx) std::memcpy(vx, s->vx.data(), n * 8);
  if (vy) std::memcpy(vy, s->vy.data(), n * 8);
  if (vz) std::memcpy(vz, s->vz.data(), n * 8);
  if (status) std::memcpy(status, s->status.data(), n);
  return PL_OK;
}

int plo_read_origin(const plo_sim* s, uint8_t* origin) {
  std::memcpy(origin, s->origin.data(), size_t(s->n));
  return PL_OK;
}

int plo_read_y0(const plo_sim* s, float* y0) {
  std::memcpy(y0, s->y0.data(), size_t(s->n) * 4);
  return PL_OK;
}

int plo_discharge_order(const plo_sim* s, int32_t* out, int32_t cap) {
  int32_t n = int32_t(s->dischargeOrder.size());
  for (int32_t i = 0; i < n && i < cap; i++) out[i] = s->dischargeOrder[i];
  return n;
}

int plo_get_state(const plo_sim* s, pl_sim_state* st) {
  std::memset(st, 0, sizeof(*st));
  st->time = s->time;
  st->steps = s->steps;
  st->phi = s->phi;
  st->omega = s->omega;
  for (int k = 0; k < 4; k++) st->counts[k] = s->counts[k];
  int byOrigin[3] = {0, 0, 0};
  for (int32_t p : s->dischargeOrder) byOrigin[s->origin[p]]++;
  for (int k = 0; k < 3; k++) st->discharged_by_origin[k] = byOrigin[k];
  st->last_iterations = s->lastIterations;
  st->failures = s->failures;
  st->max_div = s->maxDiv;
  st->interior = s->interior;
  const Controller& c = s->controller;
  st->controller.phase = c.phase;
  st->controller.pour = c.pour;
  st->controller.angle = c.angle;
  st->controller.phase_start = c.phaseStart;
  st->controller.start_angle = c.startAngle;
  st->controller.start_rate = c.startRate;
  st->controller.last_rate = c.lastRate;
  st->controller.flow_rate = c.flowRate;
  st->controller.last_discharged = c.lastDischarged;
  st->controller.target = c.target;
  st->controller.manual_rate = c.manualRate;
  return PL_OK;
}

int plo_set_state(plo_sim* s, const pl_sim_state* st, const double* x, const double* y,
                  const double* z, const double* vx, const double* vy, const double* vz,
                  const uint8_t* status) {
  size_t n = size_t(s->n);
  if (x) std::memcpy(s->x.data(), x, n * 8);
  if (y) std::memcpy(s->y.data(), y, n * 8);
  if (z) std::memcpy(s->z.data(), z, n * 8);
  if (vx) std::memcpy(s->vx.data(), vx, n * 8);
  if (vy) std::memcpy(s->vy.data(), vy, n * 8);
  if (vz) std::memcpy(s->vz.data(), vz, n * 8);
  if (x && y && z && status)  // new parcels: the APIC affine parts restart at zero (as in the engine)
    for (auto& row : s->aff)
      for (auto& c : row) std::fill(c.begin(), c.end(), 0.0);
  if (status) {
    std::memcpy(s->status.data(), status, n);
    for (int k = 0; k < 4; k++) s->counts[k] = 0;
    for (size_t p = 0; p < n; p++) s->counts[s->status[p]]++;
    // Discharge order is only used through its per-origin counts; rebuild it in id order.
    s->dischargeOrder.clear();
    for (size_t p = 0; p < n; p++)
      if (s->status[p] == DISCHARGED) s->dischargeOrder.push_back(int32_t(p));
  }
  if (st) {
    s->time = st->time;
    s->steps = st->steps;
    s->phi = st->phi;
    s->omega = st->omega;
    s->lastIterations = st->last_iterations;
    s->failures = st->failures;
    s->maxDiv = st->max_div;
    s->interior = st->interior;
    Controller& c = s->controller;
    c.phase = st->controller.phase;
    c.pour = st->controller.pour;
    c.angle = st->controller.angle;
    c.phaseStart = st->controller.phase_start;
    c.startAngle = st->controller.start_angle;
    c.startRate = st->controller.start_rate;
    c.lastRate = st->controller.last_rate;
    c.flowRate = st->controller.flow_rate;
    c.lastDischarged = st->controller.last_discharged;
    c.target = st->controller.target;
    c.manualRate = st->controller.manual_rate;
  }
  return PL_OK;
}

int plo_get_field(const plo_sim* s, int32_t field, void* out, size_t count) {
  auto faces = [&](const std::vector<double>& a, const std::vector<double>& b, const std::vector<double>& c) {
    size_t need = a.size() + b.size() + c.size();
    if (count < need) return PL_E_ARG;
    double* o = static_cast<double*>(out);
    std::memcpy(o, a.data(), a.size() * 8);
    std::memcpy(o + a.size(), b.data(), b.size() * 8);
    std::memcpy(o + a.size() + b.size(), c.data(), c.size() * 8);
    return PL_OK;
  };
  auto cells = [&](const std::vector<double>& a) {
    if (count < a.size()) return PL_E_ARG;
    std::memcpy(out, a.data(), a.size() * 8);
    return PL_OK;
  };
  switch (field) {
    case PL_FIELD_CELL:
      if (count < s->cell.size()) return PL_E_ARG;
      std::memcpy(out, s->cell.data(), s->cell.size());
      return PL_OK;
    case PL_FIELD_VELOCITY:
      return faces(s->u, s->v, s->w);
    case PL_FIELD_VELOCITY_PREV:
      return faces(s->uPrev, s->vPrev, s->wPrev);
    case PL_FIELD_PRESSURE:
      return cells(s->q);
    case PL_FIELD_CORRECTION:
      return faces(s->uc, s->vc, s->wc);
    case PL_FIELD_VALID: {
      size_t need = s->uValid.size() + s->vValid.size() + s->wValid.size();
      if (count < need) return PL_E_ARG;
      uint8_t* o = static_cast<uint8_t*>(out);
      std::memcpy(o, s->uValid.data(), s->uValid.size());
      std::memcpy(o + s->uValid.size(), s->vValid.data(), s->vValid.size());
      std::memcpy(o + s->uValid.size() + s->vValid.size(), s->wValid.data(), s->wValid.size());
      return PL_OK;
    }
    case PL_FIELD_DENSITY:
      return cells(s->density);
    case PL_FIELD_RHS:
      return cells(s->rhs);
    default:
      return PL_E_ARG;
  }
}

int plo_pcg_solve(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny, int32_t nz,
                  double tol, int32_t max_iter, int32_t* converged, double* residual) {
  Pcg3D pcg(nx, ny, nz);
  SolveResult r = pcg.solve(cell, size_t(nx) * ny * nz, b, q, tol, max_iter);
  if (converged) *converged = r.converged ? 1 : 0;
  if (residual) *residual = r.residual;
  return r.iterations;
}

// One snapshot of the Poisson batch: cells may carry PL_POISSON_PIN on FLUID cells (diagonal + 1);
// FLUID cells on the grid border are not unknowns. FP64 Pcg3D.solve with MIC(0).
int plo_poisson_solve_box(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny, int32_t nz,
                          double tol, int32_t max_iter, int32_t* converged, double* residual) {
  const size_t nc = size_t(nx) * ny * nz;
  std::vector<uint8_t> base(nc), pin(nc);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const size_t c = (size_t(k) * ny + j) * nx + i;
        uint8_t t = cell[c] & 3;
        const bool border = i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1;
        if (border && t == FLUID) t = AIR;  // a border FLUID cell is not an unknown: Dirichlet, like AIR
        base[c] = t;
        pin[c] = (t == FLUID && (cell[c] & 4)) ? 1 : 0;
      }
  Pcg3D pcg(nx, ny, nz);
  SolveResult r = pcg.solve(base.data(), nc, b, q, tol, max_iter, pin.data());
  if (converged) *converged = r.converged ? 1 : 0;
  if (residual) *residual = r.residual;
  return r.iterations;
}

int plo_poisson_solve(const uint8_t* cell, const double* b, double* q, int32_t n, double tol, int32_t max_iter,
                      int32_t* converged, double* residual) {
  return plo_poisson_solve_box(cell, b, q, n, n, n, tol, max_iter, converged, residual);
}

void plo_get_affine(const plo_sim* s, double* c9) {
  for (int p = 0; p < s->n; p++)
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) c9[9 * p + 3 * a + b] = s->aff[a][b][p];
}

void plo_set_affine(plo_sim* s, const double* c9) {
  for (int p = 0; p < s->n; p++)
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) s->aff[a][b][p] = c9[9 * p + 3 * a + b];
}

double plo_teapot_sdf(const pl_teapot* t, double x, double y, double z) {
  Teapot tp = build_teapot(*t);
  return teapot_sdf(tp, x, y, z);
}

int plo_in_cavity(const pl_teapot* t, double x, double y, double z) {
  Teapot tp = build_teapot(*t);
  return in_cavity(tp, x, y, z) ? 1 : 0;
}

void plo_rng(uint32_t seed, int32_t n, double* out) {
  Rng r(seed);
  for (int32_t i = 0; i < n; i++) out[i] = r.next();
}

double plo_js_hypot3(double a, double b, double c) { return hypot3(a, b, c); }

}  // extern "C"
