// C ABI of the pour engine (include/pourlab.h): construction, the substep graph, stepping and the
// read-back of parcels, fields and diagnostics.
//
// A substep is a fixed sequence of kernels (kernels.cu, solver.cu) captured once into a CUDA graph.
// All per-substep decisions (stable dt, controller, liquid-cell count, solver convergence) are made
// on the device, so advance() launches the graph back to back and synchronises only to learn when
// the requested duration has elapsed; substeps launched past the end return immediately.
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "cheb.h"
#include "kernels.h"
#include "poisson.h"
#include "unet.h"
#include "mg.h"
#include "setup.h"

using namespace pl;

namespace {

thread_local std::string g_err;
thread_local int g_fail_allocs = 0;  // pl_inject_fault(PL_FAULT_ALLOC, n): pl_create allocations left to fail

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return fail(PL_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

// A NaN bit pattern no pose takes: SimScalars.phi_trig_bits when the pose's cosine and sine must be
// formed anew (a new simulation, or a state set from the host).
constexpr unsigned long long kPoseTrigUnset = 0x7ff8dead00000001ull;

}  // namespace

struct pl_sim {
  Geo g{};
  DevPtrs P{};
  int device = 0;
  cudaStream_t st = nullptr;
  cudaGraphExec_t exec = nullptr;
  void* mem = nullptr;
  size_t mem_bytes = 0;
  SimScalars hs{};  // host mirror, current after every synchronising call
  double fill_height = 0;
  int band_counts[3] = {0, 0, 0};
  std::vector<uint8_t> origin;
  pl_config cfg{};
  float* export_buf = nullptr;  // F floats for exported face fields
  SimScalars* pinned = nullptr; // page-locked staging of the scalar block
  int timing = 0;
  int pending = 0;  // substeps queued by pl_enqueue_substeps since the last pull
  int free_running = 0;  // the device's control fields already say "run until finished" (no copy needed)
  cudaEvent_t ev[PL_STAGES + 3] = {};  // stage boundaries on st (0-7) and the density branch on st2 (8-9)
  pl::PoissonImpl* box = nullptr;  // grid-scale solver (PL_PRECOND_BOX_MG / PL_PRECOND_LEARNED)
  pl::PoissonImpl* box2 = nullptr; // ... and the density correction's (multigrid), run beside it
  cudaStream_t st2 = nullptr;      // the second stream of the substep capture
  cudaEvent_t fork = nullptr, join = nullptr;    // the grid-scale correction solve's branch
  cudaEvent_t fork0 = nullptr, join0 = nullptr;  // the density stage's branch
  pl::UNetImpl* net = nullptr;     // its network (PL_PRECOND_LEARNED), owned by the caller
};

namespace {
int pull_scalars(pl_sim* s);

// Bring the host mirror up to date before a call reads it or writes it back to the device.
int settle(pl_sim* s) { return s->pending ? pull_scalars(s) : PL_OK; }

int pull_scalars(pl_sim* s) {
  CK(cudaMemcpyAsync(s->pinned, s->P.sc, sizeof(SimScalars), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  std::memcpy(&s->hs, s->pinned, sizeof(SimScalars));
  s->pending = 0;
  if (s->hs.errors) {
    int e = s->hs.errors;
    return fail(PL_E_TIMEOUT, "device error flags 0x%x (%s%s%s)", e,
                (e & ERR_SCAN_TIMEOUT) ? "bin scan wait gave up " : "",
                (e & ERR_SOLVER_SIZE) ? "solver wavefronts exceed capacity " : "",
                (e & ERR_SOLVER_TIMEOUT) ? "cluster solve wait gave up" : "");
  }
  return PL_OK;
}

int push_scalars(pl_sim* s) {
  s->free_running = 0;
  std::memcpy(s->pinned, &s->hs, sizeof(SimScalars));
  CK(cudaMemcpyAsync(s->P.sc, s->pinned, sizeof(SimScalars), cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return PL_OK;
}

// One substep, stage by stage; with timing on, an event is recorded at every stage boundary (event
// record nodes inside the graph).
int record_substep(pl_sim* s) {
  const Geo& g = s->g;
  const DevPtrs& P = s->P;
  cudaStream_t st = s->st;
  auto mark_on = [&](int i, cudaStream_t on) {  // external: becomes an event-record node of the captured graph
    if (s->timing) cudaEventRecordWithFlags(s->ev[i], on, cudaEventRecordExternal);
  };
  auto mark = [&](int i) { mark_on(i, st); };
  // execution order: bin, p2g, density, pressure, correction, extrapolation, advect (the density
  // stage needs only the parcels and cell types, so it runs before the solves)
  mark(0);
  launch_stage_bin(g, P, st);
  mark(1);
  // P2G: the cells' node partials, then the faces here and the density stage on the second stream
  // (both only read the partials); the density stage's event marks the wait for it
  launch_p2g_cells(g, P, st);
  cudaEventRecord(s->fork0, st);
  cudaStreamWaitEvent(s->st2, s->fork0, 0);
  mark_on(8, s->st2);
  launch_stage_density(g, P, s->st2);
  mark_on(9, s->st2);
  cudaEventRecord(s->join0, s->st2);
  launch_p2g_faces(g, P, st);
  mark(2);
  cudaStreamWaitEvent(st, s->join0, 0);
  mark(3);
  char err[256] = "";
  if (g.box_solve) {  // both solves side by side in the pressure stage
    if (launch_box_solves(g, P, s->box, s->box2, st, s->st2, s->fork, s->join, err, sizeof err))
      return fail(PL_E_CUDA, "%s", err);
  } else {
    launch_pressure_solve(g, P, st);
  }
  mark(4);
  if (!g.box_solve) launch_correction_solve(g, P, st);
  mark(5);
  launch_stage_extrap(g, P, st);
  mark(6);
  launch_stage_advect(g, P, st);
  mark(7);
  return PL_OK;
}

// Event interval [first, second] of each stage (enum pl_stage order) in the execution order above. P2G
// ends when both its face pass and the density branch beside it are done; the density stage is its
// own branch's interval on the second stream, which overlaps P2G. The six other stages tile the
// substep.
const int kStageEvents[PL_STAGES][2] = {{0, 1}, {1, 3}, {3, 4}, {5, 6}, {8, 9}, {4, 5}, {6, 7}};

int build_graph(pl_sim* s) {
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  if (s->g.box_solve && s->cfg.preconditioner == PL_PRECOND_LEARNED && !s->net) return PL_OK;  // pl_set_unet
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
  const int rc = record_substep(s);
  const cudaError_t ce = cudaStreamEndCapture(s->st, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return fail(PL_E_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ce));
  cudaError_t e = cudaGraphInstantiate(&s->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(PL_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  return PL_OK;
}

double host_stable_dt(const pl_sim* s) {  // solver3d.ts:268-278 on the device's max speed
  const Geo& g = s->g;
  double m;
  std::memcpy(&m, &s->hs.max_speed_bits, 8);
  double speed = std::sqrt(m) + std::sqrt(5 * g.h * g.gravity) + std::fabs(s->hs.omega) * g.R;
  return std::min(g.max_substep, (g.cfl * g.h) / speed);
}

bool host_finished(const pl_sim* s) { return s->hs.time >= s->g.duration - 1e-9; }

// Parcels in id order -> home layout (slot = id).
int upload_parcels(pl_sim* s, const double* x, const double* y, const double* z, const double* vx, const double* vy,
                   const double* vz, const uint8_t* status) {
  const int n = s->g.n;
  std::vector<float4> pos(n), vel(n);
  for (int p = 0; p < n; p++) {
    int st = status ? status[p] : 0;
    pos[p] = make_float4((float)x[p], (float)y[p], (float)z[p], 0.f);
    std::memcpy(&pos[p].w, &p, 4);
    vel[p] = make_float4(vx ? (float)vx[p] : 0.f, vy ? (float)vy[p] : 0.f, vz ? (float)vz[p] : 0.f, 0.f);
    int meta = st | (int(s->origin[p]) << 8);
    std::memcpy(&vel[p].w, &meta, 4);
  }
  CK(cudaMemcpyAsync(s->P.pos_home, pos.data(), size_t(n) * 16, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->P.vel_home, vel.data(), size_t(n) * 16, cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return PL_OK;
}

// Home layout -> id order.
int download_parcels(pl_sim* s, std::vector<float4>& pos, std::vector<float4>& vel) {
  const int n = s->g.n;
  std::vector<float4> hp(n), hv(n);
  CK(cudaMemcpyAsync(hp.data(), s->P.pos_home, size_t(n) * 16, cudaMemcpyDeviceToHost, s->st));
  CK(cudaMemcpyAsync(hv.data(), s->P.vel_home, size_t(n) * 16, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  pos.resize(n);
  vel.resize(n);
  for (int i = 0; i < n; i++) {
    int id;
    std::memcpy(&id, &hp[i].w, 4);
    if (id < 0 || id >= n) return fail(PL_E_STATE, "parcel layout corrupt (id %d at slot %d)", id, i);
    pos[id] = hp[i];
    vel[id] = hv[i];
  }
  return PL_OK;
}

}  // namespace

extern "C" {

const char* pl_last_error(void) { return g_err.c_str(); }

void pl_default_teapot(pl_teapot* t) {
  *t = pl_teapot{0.065, 0.15, 0.008, 0.035, 0.01, 45.0, 0.14};
}

void pl_default_motion(pl_motion* m) {
  std::memset(m, 0, sizeof *m);
  m->kind = PL_MOTION_POUR;
  m->start_delay = 0.5;
  m->tilt_duration = 2;
  m->hold_angle_deg = 22;
  m->hold_tilt_rate = 3;
  m->max_angle_deg = 80;
  m->return_duration = 1.2;
  m->max_hold = 20;  // gentlePour3D overrides the default 12 (presets3d.ts:17)
  m->hold_time = 1.5;
  m->target_volume = 400 * 1e-6;  // 400 * ML, evaluated as the reference does
  m->anticipation = 0.254;
  m->repeats = 1;
  m->repeat_gap = 1.5;
  m->settle_time = 2;
}

void pl_gentle_pour(double cell_mm, double seconds, pl_config* c) {
  std::memset(c, 0, sizeof *c);
  pl_default_teapot(&c->teapot);
  c->h = cell_mm / 1000;
  c->initial_volume = 1500 * 1e-6;
  pl_default_motion(&c->motion);
  c->pivot[0] = 0;
  c->pivot[1] = 0.06;
  c->gravity = 9.81;
  c->flip_ratio = 0.95;
  c->density_correction = 0.3;
  c->cfl = 0.8;
  c->max_substep = 1.0 / 200;
  c->pressure_tolerance = 1e-6;
  c->pressure_max_iterations = 400;
  c->seed = 1;
  c->duration = seconds;
  c->preconditioner = PL_PRECOND_MIC0;
  c->solve_precision = PL_SOLVE_F64;
  c->device = -1;
}

int pl_create(const pl_config* cfg, pl_sim** out) {
  if (!cfg || !out) return fail(PL_E_ARG, "pl_create: null argument");
  *out = nullptr;
  char err[256] = "";
  HostInit init;
  int rc = host_construct(*cfg, &init, err, sizeof err);
  if (rc) return fail(rc, "%s", err);
  pl_sim* s = new pl_sim();
  s->cfg = *cfg;
  s->g = init.geo;
  s->fill_height = init.fill_height;
  for (int k = 0; k < 3; k++) s->band_counts[k] = init.band_counts[k];
  s->origin = init.origin;
  const Geo& g = s->g;
  cudaError_t e = cudaSuccess;
  if (cfg->device >= 0)
    e = cudaSetDevice(cfg->device);
  else
    e = cudaGetDevice(&s->device);
  if (cfg->device >= 0) s->device = cfg->device;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->fork0, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->join0, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->pinned, sizeof(SimScalars), cudaHostAllocDefault);
  for (int i = 0; i < PL_STAGES + 3 && e == cudaSuccess; i++) e = cudaEventCreate(&s->ev[i]);
  if (e != cudaSuccess) {
    pl_destroy(s);
    return fail(PL_E_CUDA, "pl_create: stream, events or pinned staging: %s", cudaGetErrorString(e));
  }
  // one allocation for everything
  const size_t N = g.n, C = g.nc, F = g.nf, B = g.nbins + 1, NB = size_t(g.bx) * g.by * g.bz;
  size_t sizes[] = {
      N * 16, N * 16, N * 16, N * 16, N * 16, N * 16,  // pos/vel home, pos/vel sorted, frac sorted/tmp
      N * 4,  N * 4,  N * 8,                           // key, rank, placed
      B * 4,  B * 4,                                   // cnt, start
      C,      C * 4,  C * 4,                           // cell, lidx, list
      C * 8,  C * 8,                                   // q, qc
      F * 4,  F * 4,  F * 4, F, F, F * 8,              // u, uprev, uext, valid, vext, uc
      C * 8,  C * 8,                                   // rhs, density
      DENSITY_BLOCKS * 8, DENSITY_BLOCKS * 4,          // interior partials
      SCAN_MAX_TILES * 8,                              // scan descriptors
      solver_ws_bytes(int(C)),                         // solver
      N * 6 * 4,                                       // render
      sizeof(SimScalars), F * 4,                       // scalars, export
      mg_ws_bytes(g, nullptr),                         // multigrid hierarchy
      size_t(g.ntx) * g.nty * g.nz * 8,                // column-tile masks
      C * 6 * 4, C * 4,                                // tile-order neighbours, permutation
      C, C * 3 * 27 * 8, C * 27 * 4,                   // occupancy, node partials (velocity, density)
      g.apic ? N * 48 : 16, g.apic ? N * 48 : 16,      // APIC affine vectors (home, sorted)
      g.box_solve ? NB : 16, g.box_solve ? NB * 4 : 16,  // grid-scale solves: box cells, rhs
      g.box_solve ? NB * 8 : 16, 32,                     // box solution, outcome
      g.box_solve ? NB * 4 : 16, g.box_solve ? NB * 8 : 16, 32,  // the correction's rhs, solution, outcome
      size_t(brick_count(g)), C * 4,                     // brick occupancy, occupied solid cells
  };
  size_t total = 0;
  for (size_t b : sizes) total += al256(b);
  if (g_fail_allocs > 0) {  // injected: the allocation fails as cudaMalloc reports running out of memory
    g_fail_allocs--;
    e = cudaErrorMemoryAllocation;
  } else {
    e = cudaMalloc(&s->mem, total);
  }
  if (e != cudaSuccess) {
    pl_destroy(s);
    return fail(PL_E_NOMEM, "cudaMalloc(%zu): %s", total, cudaGetErrorString(e));
  }
  s->mem_bytes = total;
  cudaMemsetAsync(s->mem, 0, total, s->st);
  char* p = static_cast<char*>(s->mem);
  int idx = 0;
  auto take = [&]() {
    char* r = p;
    p += al256(sizes[idx++]);
    return (void*)r;
  };
  DevPtrs& P = s->P;
  P.pos_home = (float4*)take();
  P.vel_home = (float4*)take();
  P.pos_sorted = (float4*)take();
  P.vel_sorted = (float4*)take();
  P.frac_sorted = (float4*)take();
  P.frac_tmp = (float4*)take();
  P.key = (int*)take();
  P.rank = (int*)take();
  P.placed = (int2*)take();
  P.cnt = (int*)take();
  P.start = (int*)take();
  P.cell = (uint8_t*)take();
  P.lidx = (int*)take();
  P.list = (int*)take();
  P.q = (double*)take();
  P.qc = (double*)take();
  P.u = (float*)take();
  P.uprev = (float*)take();
  P.uext = (float*)take();
  P.valid = (uint8_t*)take();
  P.vext = (uint8_t*)take();
  P.uc = (double*)take();
  P.rhs = (double*)take();
  P.density = (double*)take();
  P.interior_part = (double*)take();
  P.interior_cnt_part = (int*)take();
  P.scan_state = (unsigned long long*)take();
  P.solver_ws = take();
  P.solver_ws_bytes = solver_ws_bytes(int(C));
  P.render = (float*)take();
  P.sc = (SimScalars*)take();
  s->export_buf = (float*)take();
  P.mg_ws = take();
  P.tile_mask = (unsigned long long*)take();
  P.tnb = (int*)take();
  P.tperm = (int*)take();
  P.occ = (uint8_t*)take();
  P.m_vel = (float2*)take();
  P.m_den = (float*)take();
  P.aff_home = (float4*)take();
  P.aff_sorted = (float4*)take();
  P.box_cell = (uint8_t*)take();
  P.box_b = (float*)take();
  P.box_x = (double*)take();
  P.box_out = (double*)take();
  P.box_b2 = (float*)take();
  P.box_x2 = (double*)take();
  P.box_out2 = (double*)take();
  P.brick_occ = (uint8_t*)take();
  P.occ_solid = (int*)take();
  if (g.box_solve) {
    int brc = 0;
    char berr[256] = "";
    s->box = pl::poisson_create(g.bx, g.by, g.bz, 1,
                                cfg->preconditioner == PL_PRECOND_LEARNED ? PL_POISSON_LEARNED : PL_POISSON_MG,
                                g.precision, berr, sizeof berr, &brc);
    if (s->box)  // the correction's own solver: it runs at the same time as the pressure's
      s->box2 = pl::poisson_create(g.bx, g.by, g.bz, 1, PL_POISSON_MG, g.precision, berr, sizeof berr, &brc);
    cudaError_t ce = cudaSuccess;
    if (s->box2) ce = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming);
    if (s->box2 && ce == cudaSuccess) ce = cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming);
    if (!s->box || !s->box2 || ce != cudaSuccess) {
      pl_destroy(s);
      return fail(brc ? brc : PL_E_CUDA, "pl_create: grid-scale solver: %s", berr);
    }
  }
  mg_configure();
  cheb_configure();
  int nn = g.n;
  cudaMemcpyAsync(P.start + g.nbins, &nn, 4, cudaMemcpyHostToDevice, s->st);
  // initial scalars
  SimScalars& hs = s->hs;
  std::memset(&hs, 0, sizeof hs);
  hs.motion = cfg->motion;
  hs.ctl.phase = cfg->motion.kind == PL_MOTION_STILL    ? PL_PHASE_DONE
                 : cfg->motion.kind == PL_MOTION_MANUAL ? PL_PHASE_MANUAL
                                                        : PL_PHASE_WAIT;
  hs.counts[0] = g.n;
  hs.interior = 1;
  hs.phi_trig_bits = kPoseTrigUnset;
  rc = push_scalars(s);
  if (!rc) {
    std::vector<double> zero;
    rc = upload_parcels(s, init.x.data(), init.y.data(), init.z.data(), nullptr, nullptr, nullptr, nullptr);
  }
  if (!rc) rc = build_graph(s);
  if (rc) {
    std::string msg = g_err;
    pl_destroy(s);
    g_err = msg;
    return rc;
  }
  *out = s;
  return PL_OK;
}

int pl_plan(const pl_config* cfg, pl_sizes* o, double* x, double* y, double* z, uint8_t* origin) {
  if (!cfg || !o) return fail(PL_E_ARG, "pl_plan: null argument");
  char err[256] = "";
  HostInit init;
  int rc = host_construct(*cfg, &init, err, sizeof err);
  if (rc) return fail(rc, "%s", err);
  const Geo& g = init.geo;
  std::memset(o, 0, sizeof *o);
  o->n = g.n;
  o->nx = g.nx;
  o->ny = g.ny;
  o->nz = g.nz;
  o->h = g.h;
  o->parcel_volume = g.parcel_volume;
  o->pivot_world[0] = g.pwx;
  o->pivot_world[1] = g.pwy;
  o->fill_height = init.fill_height;
  for (int k = 0; k < 3; k++) o->band_counts[k] = init.band_counts[k];
  o->step_copy_bytes = int32_t(sizeof(SimScalars));
  const size_t n = size_t(g.n);
  if (x) std::memcpy(x, init.x.data(), n * 8);
  if (y) std::memcpy(y, init.y.data(), n * 8);
  if (z) std::memcpy(z, init.z.data(), n * 8);
  if (origin) std::memcpy(origin, init.origin.data(), n);
  return PL_OK;
}

void pl_destroy(pl_sim* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->box) pl::poisson_destroy(s->box);
  if (s->box2) pl::poisson_destroy(s->box2);
  if (s->fork) cudaEventDestroy(s->fork);
  if (s->join) cudaEventDestroy(s->join);
  if (s->fork0) cudaEventDestroy(s->fork0);
  if (s->join0) cudaEventDestroy(s->join0);
  if (s->st2) cudaStreamDestroy(s->st2);
  if (s->mem) cudaFree(s->mem);
  for (int i = 0; i < PL_STAGES + 3; i++)
    if (s->ev[i]) cudaEventDestroy(s->ev[i]);
  if (s->pinned) cudaFreeHost(s->pinned);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

int pl_enqueue_substeps(pl_sim* s, int32_t count) {
  if (!s || count < 0) return fail(PL_E_ARG, "pl_enqueue_substeps: bad argument");
  if (!s->exec) return fail(PL_E_STATE, "pl_enqueue_substeps: the learned preconditioner needs a network (pl_set_unet)");
  cudaSetDevice(s->device);
  s->hs.end_time = INFINITY;  // run until finished
  s->hs.force_step = 0;
  if (!s->free_running) {
    // only the control fields change: copy end_time .. forced_dt (once; the substeps leave them as
    // they are, so later calls launch the graph alone until a call pushes the scalar block again)
    std::memcpy(s->pinned, &s->hs, sizeof(SimScalars));
    const size_t off = offsetof(SimScalars, end_time);
    const size_t len = offsetof(SimScalars, active) - off;
    CK(cudaMemcpyAsync((char*)s->P.sc + off, (char*)s->pinned + off, len, cudaMemcpyHostToDevice, s->st));
    s->free_running = 1;
  }
  for (int i = 0; i < count; i++) CK(cudaGraphLaunch(s->exec, s->st));
  s->pending = 1;
  return PL_OK;
}

void* pl_stream(const pl_sim* s) { return s ? (void*)s->st : nullptr; }

int pl_autotune_solver(const pl_config* cfg, int32_t substeps, int32_t* best_cluster, int32_t* best_threads,
                       float* best_ms) {
  if (!cfg || substeps < 1 || !best_cluster || !best_threads) return fail(PL_E_ARG, "pl_autotune_solver: bad argument");
  pl_config c = *cfg;
  c.preconditioner = PL_PRECOND_CHEB;
  const int clusters[] = {16, 12, 8, 4};
  const int threads[] = {512, 1024, 256};
  float best = INFINITY;
  int bc = 0, bt = 0;
  for (int ci : clusters)
    for (int ti : threads) {
      c.solve_cluster = ci;
      c.solve_threads = ti;
      pl_sim* s = nullptr;
      if (pl_create(&c, &s) != PL_OK) {
        cudaGetLastError();
        continue;
      }
      int rc = pl_enable_stage_timing(s, 1);
      float tot = 0;
      for (int k = 0; k < substeps + 1 && rc == PL_OK; k++) {
        rc = pl_step(s, -1.0);
        float ms[PL_STAGES];
        if (rc == PL_OK) rc = pl_stage_times(s, ms);
        if (rc == PL_OK && k > 0) tot += ms[PL_STAGE_PRESSURE] + ms[PL_STAGE_CORRECTION];  // first one warms up
      }
      const bool ran = rc == PL_OK && s->hs.mg_status == 1;  // the cluster solve (not the fallback) ran
      pl_destroy(s);
      cudaGetLastError();
      if (!ran) continue;
      tot /= substeps;
      if (tot < best) {
        best = tot;
        bc = ci;
        bt = ti;
      }
    }
  if (bc == 0) return fail(PL_E_STATE, "pl_autotune_solver: no launch shape ran");
  *best_cluster = bc;
  *best_threads = bt;
  if (best_ms) *best_ms = best;
  return PL_OK;
}

int pl_inject_fault(int32_t kind, int32_t count) {
  if (kind != PL_FAULT_ALLOC || count < 0) return fail(PL_E_ARG, "pl_inject_fault: unknown fault %d or count %d", kind, count);
  g_fail_allocs = count;
  return PL_OK;
}

int pl_set_wait_limit(pl_sim* s, int32_t polls) {
  if (!s || polls < 0) return fail(PL_E_ARG, "pl_set_wait_limit: bad argument");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  s->hs.spin_limit = polls;
  return push_scalars(s);
}

int pl_enable_stage_timing(pl_sim* s, int32_t on) {
  if (!s) return fail(PL_E_ARG, "pl_enable_stage_timing: null handle");
  cudaSetDevice(s->device);
  CK(cudaStreamSynchronize(s->st));
  s->timing = on ? 1 : 0;
  return build_graph(s);
}

int pl_stage_times(pl_sim* s, float ms[PL_STAGES]) {
  if (!s || !ms) return fail(PL_E_ARG, "pl_stage_times: null argument");
  if (!s->timing) return fail(PL_E_STATE, "pl_stage_times: stage timing is off");
  CK(cudaStreamSynchronize(s->st));
  for (int i = 0; i < PL_STAGES; i++)
    CK(cudaEventElapsedTime(&ms[i], s->ev[kStageEvents[i][0]], s->ev[kStageEvents[i][1]]));
  if (s->g.precond == PL_PRECOND_CHEB) {
    // both systems ran in the pressure stage's cluster launch: move the correction system's device
    // time (kernel timestamps) from the pressure stage to the correction stage
    unsigned long long t[3];
    CK(cudaMemcpy(t, &s->P.sc->t_solve[0], sizeof t, cudaMemcpyDeviceToHost));
    if (t[2] >= t[1] && t[1] >= t[0]) {
      const float corr = float(double(t[2] - t[1]) * 1e-6);
      const float moved = std::min(corr, ms[PL_STAGE_PRESSURE]);
      ms[PL_STAGE_PRESSURE] -= moved;
      ms[PL_STAGE_CORRECTION] += moved;
    }
  }
  return PL_OK;
}

int pl_get_sizes(const pl_sim* s, pl_sizes* o) {
  if (!s || !o) return fail(PL_E_ARG, "pl_get_sizes: null argument");
  std::memset(o, 0, sizeof *o);
  o->n = s->g.n;
  o->nx = s->g.nx;
  o->ny = s->g.ny;
  o->nz = s->g.nz;
  o->h = s->g.h;
  o->parcel_volume = s->g.parcel_volume;
  o->pivot_world[0] = s->g.pwx;
  o->pivot_world[1] = s->g.pwy;
  o->fill_height = s->fill_height;
  for (int k = 0; k < 3; k++) o->band_counts[k] = s->band_counts[k];
  o->step_copy_bytes = int32_t(sizeof(SimScalars));
  return PL_OK;
}

int pl_stable_dt(pl_sim* s, double* out) {
  if (!s || !out) return fail(PL_E_ARG, "pl_stable_dt: null argument");
  int rc = settle(s);
  if (rc) return rc;
  *out = host_stable_dt(s);
  return PL_OK;
}

int pl_finished(const pl_sim* s) { return s && host_finished(s) ? 1 : 0; }

int pl_step(pl_sim* s, double dt) {
  if (!s) return fail(PL_E_ARG, "pl_step: null handle");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  s->hs.force_step = 1;
  s->hs.forced_dt = dt > 0 ? dt : 0;
  if (!s->exec) return fail(PL_E_STATE, "pl_step: the learned preconditioner needs a network (pl_set_unet)");
  rc = push_scalars(s);
  if (rc) return rc;
  CK(cudaGraphLaunch(s->exec, s->st));
  return pull_scalars(s);
}

int pl_advance(pl_sim* s, double duration, pl_diagnostics* out) {
  if (!s) return fail(PL_E_ARG, "pl_advance: null handle");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  if (!s->exec) return fail(PL_E_STATE, "pl_advance: the learned preconditioner needs a network (pl_set_unet)");
  const double end = s->hs.time + duration;  // solver3d.ts:282
  s->hs.end_time = end;
  s->hs.force_step = 0;
  rc = push_scalars(s);
  if (rc) return rc;
  for (int guard = 0; guard < 1000000; guard++) {
    if (!(s->hs.time < end - 1e-12 && !host_finished(s))) break;
    double remaining = std::min(end, s->g.duration) - s->hs.time;
    double dt = host_stable_dt(s);
    long k = (long)std::ceil(remaining / dt * 1.05) + 1;
    k = std::max(1L, std::min(k, 4096L));
    for (long i = 0; i < k; i++) CK(cudaGraphLaunch(s->exec, s->st));
    rc = pull_scalars(s);
    if (rc) return rc;
  }
  return out ? pl_get_diagnostics(s, out) : PL_OK;
}

int pl_sync(pl_sim* s) {
  if (!s) return fail(PL_E_ARG, "pl_sync: null handle");
  cudaSetDevice(s->device);
  return pull_scalars(s);
}

int pl_set_tilt_target(pl_sim* s, double angle_deg, double time) {  // motion.ts:40-44
  if (!s) return fail(PL_E_ARG, "pl_set_tilt_target: null handle");
  (void)time;
  int rc = settle(s);
  if (rc) return rc;
  double a = std::max(0.0, std::min(s->hs.motion.max_angle_deg, angle_deg));
  s->hs.ctl.target = a * DEG;
  return push_scalars(s);
}

int pl_controller(const pl_sim* s, double* angle_deg, int32_t* phase) {
  if (!s) return fail(PL_E_ARG, "pl_controller: null handle");
  if (angle_deg) *angle_deg = s->hs.ctl.angle / DEG;
  if (phase) *phase = s->hs.ctl.phase;
  return PL_OK;
}

int pl_get_diagnostics(pl_sim* s, pl_diagnostics* d) {  // solver3d.ts:796-814
  if (!s || !d) return fail(PL_E_ARG, "pl_get_diagnostics: null argument");
  int rc = settle(s);
  if (rc) return rc;
  const SimScalars& h = s->hs;
  const double v = s->g.parcel_volume * s->g.vol_factor * 1e6;
  std::memset(d, 0, sizeof *d);
  d->time = h.time;
  d->steps = h.steps;
  d->angle_deg = h.ctl.angle / DEG;
  d->phase = h.ctl.phase;
  d->particles = s->g.n;
  d->grid[0] = s->g.nx;
  d->grid[1] = s->g.ny;
  d->grid[2] = s->g.nz;
  d->pressure_iterations = h.last_iters;
  d->pressure_failures = h.failures;
  d->correction_iterations = h.corr_iters;
  d->discharged_ml = h.counts[1] * v;
  d->spilled_ml = h.counts[2] * v;
  d->lost_ml = h.counts[3] * v;
  d->in_pot_ml = h.counts[0] * v;
  double md;
  std::memcpy(&md, &h.max_div_bits, 8);
  d->max_divergence = md / s->g.h;
  d->interior_density = h.interior;
  d->liquid_cells = h.m;
  return PL_OK;
}

int pl_discharged_fractions(pl_sim* s, double out[3]) {  // solver3d.ts:817-823
  if (!s || !out) return fail(PL_E_ARG, "pl_discharged_fractions: null argument");
  int rc = settle(s);
  if (rc) return rc;
  const int* c = s->hs.by_origin;
  int n = c[0] + c[1] + c[2];
  if (n == 0) return PL_NONE;
  for (int k = 0; k < 3; k++) out[k] = double(c[k]) / double(n);
  return PL_OK;
}

int pl_read_particles(pl_sim* s, float* pos4, float* vel4, uint32_t* status) {
  if (!s) return fail(PL_E_ARG, "pl_read_particles: null handle");
  std::vector<float4> pos, vel;
  int rc = download_parcels(s, pos, vel);
  if (rc) return rc;
  for (int p = 0; p < s->g.n; p++) {
    if (pos4) {
      pos4[4 * p] = pos[p].x;
      pos4[4 * p + 1] = pos[p].y;
      pos4[4 * p + 2] = pos[p].z;
      pos4[4 * p + 3] = 0.f;
    }
    if (vel4) {
      vel4[4 * p] = vel[p].x;
      vel4[4 * p + 1] = vel[p].y;
      vel4[4 * p + 2] = vel[p].z;
      vel4[4 * p + 3] = 0.f;
    }
    if (status) {
      int meta;
      std::memcpy(&meta, &vel[p].w, 4);
      status[p] = uint32_t(meta & 0xff);
    }
  }
  return PL_OK;
}

// Slot of every parcel id in the home layout.
static int home_slots(pl_sim* s, std::vector<int>& slot) {
  const int n = s->g.n;
  std::vector<float4> hp(n);
  CK(cudaMemcpyAsync(hp.data(), s->P.pos_home, size_t(n) * 16, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  slot.assign(n, -1);
  for (int i = 0; i < n; i++) {
    int id;
    std::memcpy(&id, &hp[i].w, 4);
    if (id < 0 || id >= n) return fail(PL_E_STATE, "parcel layout corrupt (id %d at slot %d)", id, i);
    slot[id] = i;
  }
  return PL_OK;
}

int pl_get_affine(pl_sim* s, float* c9) {
  if (!s || !c9) return fail(PL_E_ARG, "pl_get_affine: null argument");
  if (!s->g.apic) return fail(PL_E_STATE, "pl_get_affine: the simulation does not use APIC");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  std::vector<int> slot;
  if ((rc = home_slots(s, slot))) return rc;
  const int n = s->g.n;
  std::vector<float4> a(size_t(3) * n);
  CK(cudaMemcpyAsync(a.data(), s->P.aff_home, size_t(n) * 48, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  for (int id = 0; id < n; id++)
    for (int comp = 0; comp < 3; comp++) {
      const float4 v = a[size_t(comp) * n + slot[id]];
      c9[9 * id + 3 * comp] = v.x;
      c9[9 * id + 3 * comp + 1] = v.y;
      c9[9 * id + 3 * comp + 2] = v.z;
    }
  return PL_OK;
}

int pl_set_affine(pl_sim* s, const float* c9) {
  if (!s || !c9) return fail(PL_E_ARG, "pl_set_affine: null argument");
  if (!s->g.apic) return fail(PL_E_STATE, "pl_set_affine: the simulation does not use APIC");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  std::vector<int> slot;
  if ((rc = home_slots(s, slot))) return rc;
  const int n = s->g.n;
  std::vector<float4> a(size_t(3) * n);
  for (int id = 0; id < n; id++)
    for (int comp = 0; comp < 3; comp++)
      a[size_t(comp) * n + slot[id]] =
          make_float4(c9[9 * id + 3 * comp], c9[9 * id + 3 * comp + 1], c9[9 * id + 3 * comp + 2], 0.f);
  CK(cudaMemcpyAsync(s->P.aff_home, a.data(), size_t(n) * 48, cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return PL_OK;
}

int pl_read_particles_f64(pl_sim* s, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                          uint8_t* status) {
  if (!s) return fail(PL_E_ARG, "pl_read_particles_f64: null handle");
  std::vector<float4> pos, vel;
  int rc = download_parcels(s, pos, vel);
  if (rc) return rc;
  for (int p = 0; p < s->g.n; p++) {
    if (x) x[p] = pos[p].x;
    if (y) y[p] = pos[p].y;
    if (z) z[p] = pos[p].z;
    if (vx) vx[p] = vel[p].x;
    if (vy) vy[p] = vel[p].y;
    if (vz) vz[p] = vel[p].z;
    if (status) {
      int meta;
      std::memcpy(&meta, &vel[p].w, 4);
      status[p] = uint8_t(meta & 0xff);
    }
  }
  return PL_OK;
}

int pl_read_origin(const pl_sim* s, uint8_t* origin) {
  if (!s || !origin) return fail(PL_E_ARG, "pl_read_origin: null argument");
  std::memcpy(origin, s->origin.data(), s->origin.size());
  return PL_OK;
}

int pl_read_quantized_positions(pl_sim* s, int32_t stride, double quantum, uint16_t* xyz3) {
  if (!s || !xyz3 || stride < 1 || !(quantum > 0))
    return fail(PL_E_ARG, "pl_read_quantized_positions: bad argument");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  const int n = s->g.n;
  const int kept = (n + stride - 1) / stride;
  uint16_t* dev = reinterpret_cast<uint16_t*>(s->P.render);  // scratch: 6 bytes per kept parcel <= 12 n
  pl::launch_quantize(s->P, n, stride, quantum, dev, s->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(xyz3, dev, size_t(kept) * 6, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  return PL_OK;
}

int pl_read_render_positions(pl_sim* s, float* xyz6n) {
  if (!s || !xyz6n) return fail(PL_E_ARG, "pl_read_render_positions: null argument");
  cudaSetDevice(s->device);
  launch_render(s->g, s->P, s->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(xyz6n, s->P.render, size_t(s->g.n) * (s->g.full ? 3 : 6) * 4, cudaMemcpyDeviceToHost,
                     s->st));
  CK(cudaStreamSynchronize(s->st));
  return PL_OK;
}

int pl_get_state(pl_sim* s, pl_sim_state* st) {
  if (!s || !st) return fail(PL_E_ARG, "pl_get_state: null argument");
  int rc = settle(s);
  if (rc) return rc;
  const SimScalars& h = s->hs;
  std::memset(st, 0, sizeof *st);
  st->time = h.time;
  st->steps = h.steps;
  st->phi = h.phi;
  st->omega = h.omega;
  for (int k = 0; k < 4; k++) st->counts[k] = h.counts[k];
  for (int k = 0; k < 3; k++) st->discharged_by_origin[k] = h.by_origin[k];
  st->last_iterations = h.last_iters;
  st->failures = h.failures;
  double md;
  std::memcpy(&md, &h.max_div_bits, 8);
  st->max_div = md / s->g.h;
  st->interior = h.interior;
  const DevController& c = h.ctl;
  st->controller = pl_controller_state{c.phase,     c.pour,      c.angle,     c.phase_start,     c.start_angle, c.start_rate,
                                       c.last_rate, c.flow_rate, c.last_discharged, c.target, c.manual_rate};
  return PL_OK;
}

int pl_set_state(pl_sim* s, const pl_sim_state* st, const double* x, const double* y, const double* z,
                 const double* vx, const double* vy, const double* vz, const uint8_t* status) {
  if (!s) return fail(PL_E_ARG, "pl_set_state: null handle");
  cudaSetDevice(s->device);
  int rc0 = settle(s);
  if (rc0) return rc0;
  SimScalars& h = s->hs;
  const int n = s->g.n;
  if (x && y && z && status) {
    int rc = upload_parcels(s, x, y, z, vx, vy, vz, status);
    if (rc) return rc;
    if (s->g.apic) CK(cudaMemsetAsync(s->P.aff_home, 0, size_t(n) * 48, s->st));  // affine parts restart at 0
    for (int k = 0; k < 4; k++) h.counts[k] = 0;
    for (int k = 0; k < 3; k++) h.by_origin[k] = 0;
    double m = 0;
    for (int p = 0; p < n; p++) {
      if (status[p] > 3) return fail(PL_E_ARG, "pl_set_state: status %d of parcel %d", status[p], p);
      h.counts[status[p]]++;
      if (status[p] == PL_DISCHARGED) h.by_origin[s->origin[p]]++;
      if (status[p] == PL_IN_POT && vx && vy && vz) {
        double a = (float)vx[p], b = (float)vy[p], c = (float)vz[p];
        double sp = a * a + b * b + c * c;  // as k_advect forms it (no contraction: -ffp-contract=off)
        if (sp > m) m = sp;
      }
    }
    std::memcpy(&h.max_speed_bits, &m, 8);
  } else if (x || y || z || status) {
    return fail(PL_E_ARG, "pl_set_state: x, y, z and status go together");
  }
  if (st) {
    h.time = st->time;
    h.steps = st->steps;
    h.phi = st->phi;
    h.phi_trig_bits = kPoseTrigUnset;  // the pose's cosine and sine are formed anew
    h.omega = st->omega;
    h.last_iters = st->last_iterations;
    h.failures = st->failures;
    h.interior = st->interior;
    double md = st->max_div * s->g.h;
    std::memcpy(&h.max_div_bits, &md, 8);
    const pl_controller_state& c = st->controller;
    h.ctl = DevController{c.phase,     c.pour,      c.angle,           c.phase_start, c.start_angle, c.start_rate,
                          c.last_rate, c.flow_rate, c.last_discharged, c.target,      c.manual_rate};
  }
  return push_scalars(s);
}

int pl_get_field(pl_sim* s, int32_t field, void* out, size_t count) {
  if (!s || !out) return fail(PL_E_ARG, "pl_get_field: null argument");
  cudaSetDevice(s->device);
  const Geo& g = s->g;
  const size_t C = g.nc, F = g.nf;
  auto faces = [&](const float* src) -> int {
    if (count < F) return fail(PL_E_ARG, "pl_get_field: buffer holds %zu of %zu", count, F);
    std::vector<float> tmp(F);
    CK(cudaMemcpyAsync(tmp.data(), src, F * 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    double* o = static_cast<double*>(out);
    for (size_t i = 0; i < F; i++) o[i] = tmp[i];
    return PL_OK;
  };
  auto listed = [&](const double* src) -> int {  // list-indexed -> grid, zero off the list
    if (count < C) return fail(PL_E_ARG, "pl_get_field: buffer holds %zu of %zu", count, C);
    int m = s->hs.m;
    std::vector<int> list(std::max(m, 1));
    std::vector<double> v(std::max(m, 1));
    if (m > 0) {
      CK(cudaMemcpyAsync(list.data(), s->P.list, size_t(m) * 4, cudaMemcpyDeviceToHost, s->st));
      CK(cudaMemcpyAsync(v.data(), src, size_t(m) * 8, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
    }
    double* o = static_cast<double*>(out);
    std::fill(o, o + C, 0.0);
    for (int t = 0; t < m; t++) o[list[t]] = v[t];
    return PL_OK;
  };
  switch (field) {
    case PL_FIELD_CELL:
      if (count < C) return fail(PL_E_ARG, "pl_get_field: buffer holds %zu of %zu", count, C);
      CK(cudaMemcpyAsync(out, s->P.cell, C, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      return PL_OK;
    case PL_FIELD_VELOCITY:
      return faces(s->P.u);
    case PL_FIELD_VELOCITY_PREV:
      return faces(s->P.uprev);
    case PL_FIELD_PRESSURE:
      return listed(s->P.q);
    case PL_FIELD_CORRECTION:
      launch_export_correction(g, s->P, s->export_buf, s->st);
      CK(cudaGetLastError());
      return faces(s->export_buf);
    case PL_FIELD_VALID:
      if (count < F) return fail(PL_E_ARG, "pl_get_field: buffer holds %zu of %zu", count, F);
      CK(cudaMemcpyAsync(out, s->P.valid, F, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      return PL_OK;
    case PL_FIELD_DENSITY:
      return listed(s->P.density);
    case PL_FIELD_RHS:
      return listed(s->P.rhs);
    default:
      return fail(PL_E_ARG, "pl_get_field: unknown field %d", field);
  }
}

int pl_pcg_solve_device(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny, int32_t nz,
                        double tol, int32_t max_iter, int32_t preconditioner, int32_t precision, void* stream,
                        int32_t* iterations, int32_t* converged, double* residual) {
  if (!cell || !b || !q) return fail(PL_E_ARG, "pl_pcg_solve_device: null buffer");
  char err[256] = "";
  int rc = standalone_pcg(cell, b, q, nx, ny, nz, tol, max_iter, preconditioner, precision, (cudaStream_t)stream,
                          iterations, converged, residual, err, sizeof err);
  if (rc) return fail(rc, "%s", err);
  return PL_OK;
}

int pl_pcg_solve_device_noalloc(const uint8_t* cell, const double* b, double* q, int32_t nx, int32_t ny,
                                int32_t nz, double tol, int32_t max_iter, void* stream, int32_t* iterations,
                                int32_t* converged, double* residual) {
  if (!cell || !b || !q) return fail(PL_E_ARG, "pl_pcg_solve_device_noalloc: null buffer");
  char err[256] = "";
  int rc = standalone_pcg_noalloc(cell, b, q, nx, ny, nz, tol, max_iter, (cudaStream_t)stream, iterations,
                                  converged, residual, err, sizeof err);
  if (rc) return fail(rc, "%s", err);
  return PL_OK;
}

// ------------------------------------------------------------------ Poisson batch

struct pl_unet {
  pl::UNetImpl* impl;
  int device;
};

struct pl_poisson {
  pl::PoissonImpl* impl;
  int n, count, device;
};

int pl_poisson_generate(int32_t n, int32_t first, int32_t count, uint8_t* cell, float* b, int32_t threads) {
  if (!cell) return fail(PL_E_ARG, "pl_poisson_generate: null buffer");
  if (n < 8 || n > 512 || (n & (n - 1)) || count < 1 || first < 0)
    return fail(PL_E_ARG, "pl_poisson_generate: n must be a power of two in [8, 512] and count >= 1 (n=%d count=%d)",
                n, count);
  return pl::poisson_generate(n, first, count, cell, b, threads);
}

int pl_poisson_gauge_fix(int32_t n, int32_t count, uint8_t* cell, float* b, int32_t* enclosed) {
  if (!cell || !b) return fail(PL_E_ARG, "pl_poisson_gauge_fix: null buffer");
  if (n < 3 || count < 1) return fail(PL_E_ARG, "pl_poisson_gauge_fix: bad size n=%d count=%d", n, count);
  const size_t nc = size_t(n) * n * n;
  for (int s = 0; s < count; s++) {
    const int e = pl::gauge_fix_one(n, cell + s * nc, b + s * nc);
    if (enclosed) enclosed[s] = e;
  }
  return PL_OK;
}

int pl_poisson_create_box(int32_t nx, int32_t ny, int32_t nz, int32_t count, int32_t method, int32_t precision,
                          pl_poisson** out) {
  if (!out) return fail(PL_E_ARG, "pl_poisson_create: null argument");
  *out = nullptr;
  auto pow2 = [](int v) { return v >= 8 && v <= 512 && (v & (v - 1)) == 0; };
  if (!pow2(nx) || !pow2(ny) || !pow2(nz) || count < 1)
    return fail(PL_E_ARG, "pl_poisson_create: box extents must be powers of two in [8, 512] and count >= 1 "
                "(%dx%dx%d, count=%d)", nx, ny, nz, count);
  if (method != PL_POISSON_MIC0 && method != PL_POISSON_MG && method != PL_POISSON_LEARNED)
    return fail(PL_E_ARG, "pl_poisson_create: unknown method %d", method);
  if (precision != PL_SOLVE_F64 && precision != PL_SOLVE_MIXED)
    return fail(PL_E_ARG, "pl_poisson_create: unknown precision %d", precision);
  if ((long long)nx * ny * nz * count > (1ll << 31) - 1)
    return fail(PL_E_ARG, "pl_poisson_create: %d boxes of %dx%dx%d cells exceed 2^31 cells", count, nx, ny, nz);
  char err[256] = "";
  int rc = 0;
  pl::PoissonImpl* impl = pl::poisson_create(nx, ny, nz, count, method, precision, err, sizeof err, &rc);
  if (!impl) return fail(rc ? rc : PL_E_CUDA, "%s", err);
  pl_poisson* h = new pl_poisson{impl, nx, count, 0};
  cudaGetDevice(&h->device);
  *out = h;
  return PL_OK;
}

int pl_poisson_create(int32_t n, int32_t count, int32_t method, int32_t precision, pl_poisson** out) {
  return pl_poisson_create_box(n, n, n, count, method, precision, out);
}

int pl_poisson_solve(pl_poisson* h, const uint8_t* cell, const float* b, double* x, double tol, int32_t max_iter,
                     void* stream, int32_t* iterations, double* residual, int32_t* converged) {
  if (!h || !cell || !b || !x) return fail(PL_E_ARG, "pl_poisson_solve: null argument");
  if (!(tol >= 0) || max_iter < 1) return fail(PL_E_ARG, "pl_poisson_solve: bad tolerance or iteration cap");
  cudaSetDevice(h->device);
  char err[256] = "";
  int rc = pl::poisson_solve(h->impl, cell, b, x, tol, max_iter, (cudaStream_t)stream, iterations, residual, converged,
                             err, sizeof err);
  if (rc) return fail(rc, "%s", err);
  return PL_OK;
}

int pl_set_unet(pl_sim* s, pl_unet* u) {
  if (!s || !u) return fail(PL_E_ARG, "pl_set_unet: null argument");
  if (s->cfg.preconditioner != PL_PRECOND_LEARNED)
    return fail(PL_E_STATE, "pl_set_unet: the simulation was not created with PL_PRECOND_LEARNED");
  cudaSetDevice(s->device);
  int rc = settle(s);
  if (rc) return rc;
  char err[256] = "";
  rc = pl::unet_prepare(u->impl, s->g.bx, s->g.by, s->g.bz, 1, err, sizeof err);  // workspace before the capture
  if (rc) return fail(rc, "%s", err);
  s->net = u->impl;
  pl::poisson_set_unet(s->box, u->impl);
  return build_graph(s);
}

int pl_poisson_set_unet(pl_poisson* h, pl_unet* u) {
  if (!h || !u) return fail(PL_E_ARG, "pl_poisson_set_unet: null argument");
  pl::poisson_set_unet(h->impl, u->impl);
  return PL_OK;
}

size_t pl_poisson_device_bytes(const pl_poisson* h) { return h ? pl::poisson_bytes(h->impl) : 0; }

int pl_poisson_history(const pl_poisson* h, int32_t snapshot, double* max_residual, int32_t capacity,
                       int32_t* recorded, int32_t* learned_iterations) {
  if (!h || (capacity > 0 && !max_residual)) return fail(PL_E_ARG, "pl_poisson_history: null argument");
  if (pl::poisson_history(h->impl, snapshot, max_residual, capacity, recorded, learned_iterations))
    return fail(PL_E_ARG, "pl_poisson_history: snapshot %d out of range or no solve yet", snapshot);
  return PL_OK;
}

void pl_poisson_destroy(pl_poisson* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  pl::poisson_destroy(h->impl);
  delete h;
}

// ------------------------------------------------------------------ learned preconditioner


int pl_unet_create(uint32_t seed, pl_unet** out) {
  if (!out) return fail(PL_E_ARG, "pl_unet_create: null argument");
  *out = nullptr;
  char err[256] = "";
  int rc = 0;
  pl::UNetImpl* impl = pl::unet_create(seed, err, sizeof err, &rc);
  if (!impl) return fail(rc ? rc : PL_E_CUDA, "%s", err);
  pl_unet* u = new pl_unet{impl, 0};
  cudaGetDevice(&u->device);
  *out = u;
  return PL_OK;
}

int pl_unet_set_loss(pl_unet* u, int32_t kind) {
  if (!u) return fail(PL_E_ARG, "pl_unet_set_loss: null argument");
  if (kind != PL_UNET_LOSS_L2 && kind != PL_UNET_LOSS_ENERGY) return fail(PL_E_ARG, "pl_unet_set_loss: kind %d", kind);
  pl::unet_set_loss(u->impl, kind);
  return PL_OK;
}

int pl_unet_set_conv_kernel(pl_unet* u, int32_t kind) {
  if (!u) return fail(PL_E_ARG, "pl_unet_set_conv_kernel: null argument");
  if (pl::unet_set_conv_kernel(u->impl, kind)) return fail(PL_E_ARG, "pl_unet_set_conv_kernel: kind %d", kind);
  return PL_OK;
}

int pl_unet_error(pl_unet* u) {
  if (!u) return fail(PL_E_ARG, "pl_unet_error: null argument");
  cudaSetDevice(u->device);
  return pl::unet_error(u->impl);
}

int32_t pl_unet_num_params(const pl_unet* u) { return u ? pl::unet_nparams(u->impl) : 0; }

int pl_unet_get_params(pl_unet* u, float* host) {
  if (!u || !host) return fail(PL_E_ARG, "pl_unet_get_params: null argument");
  cudaSetDevice(u->device);
  int rc = pl::unet_get_params(u->impl, host);
  return rc ? fail(rc, "pl_unet_get_params: %s", cudaGetErrorString(cudaGetLastError())) : PL_OK;
}

int pl_unet_set_params(pl_unet* u, const float* host) {
  if (!u || !host) return fail(PL_E_ARG, "pl_unet_set_params: null argument");
  cudaSetDevice(u->device);
  int rc = pl::unet_set_params(u->impl, host);
  return rc ? fail(rc, "pl_unet_set_params: %s", cudaGetErrorString(cudaGetLastError())) : PL_OK;
}

int pl_unet_apply(pl_unet* u, const uint8_t* cell, const float* r, float* z, int32_t nx, int32_t ny, int32_t nz,
                  int32_t count, void* stream) {
  if (!u || !cell || !r || !z) return fail(PL_E_ARG, "pl_unet_apply: null argument");
  cudaSetDevice(u->device);
  char err[256] = "";
  int rc = pl::unet_apply(u->impl, cell, r, z, nx, ny, nz, count, (cudaStream_t)stream, err, sizeof err);
  return rc ? fail(rc, "%s", err) : PL_OK;
}

int pl_unet_train_step(pl_unet* u, const uint8_t* cell, const float* r, const float* e, int32_t nx, int32_t ny,
                       int32_t nz, int32_t count, float lr, float* loss, void* stream) {
  if (!u || !cell || !r || !e || !loss) return fail(PL_E_ARG, "pl_unet_train_step: null argument");
  cudaSetDevice(u->device);
  char err[256] = "";
  int rc = pl::unet_gradient(u->impl, cell, r, e, nx, ny, nz, count, lr, 1, loss, nullptr, (cudaStream_t)stream, err,
                             sizeof err);
  return rc ? fail(rc, "%s", err) : PL_OK;
}

int pl_unet_gradient(pl_unet* u, const uint8_t* cell, const float* r, const float* e, int32_t nx, int32_t ny,
                     int32_t nz, int32_t count, float* loss, float* grad, void* stream) {
  if (!u || !cell || !r || !e || !loss || !grad) return fail(PL_E_ARG, "pl_unet_gradient: null argument");
  cudaSetDevice(u->device);
  char err[256] = "";
  int rc = pl::unet_gradient(u->impl, cell, r, e, nx, ny, nz, count, 0.f, 0, loss, grad, (cudaStream_t)stream, err,
                             sizeof err);
  return rc ? fail(rc, "%s", err) : PL_OK;
}

void pl_unet_destroy(pl_unet* u) {
  if (!u) return;
  cudaSetDevice(u->device);
  pl::unet_destroy(u->impl);
  delete u;
}

// ------------------------------------------------------------------ ensembles

int pl_ensemble_configs(uint32_t seed, int32_t count, double cell_mm, double seconds, pl_config* out) {
  if (!out || count < 1 || !(cell_mm > 0) || !(seconds > 0)) return fail(PL_E_ARG, "pl_ensemble_configs: bad argument");
  uint32_t a = seed;
  auto next = [&]() {  // mulberry32 (src/sim/rng.ts:5-14)
    a += 0x6d2b79f5u;
    uint32_t t = a;
    t = (t ^ (t >> 15)) * (t | 1u);
    t ^= t + (t ^ (t >> 7)) * (t | 61u);
    return double(t ^ (t >> 14)) / 4294967296.0;
  };
  for (int i = 0; i < count; i++) {
    pl_config& c = out[i];
    pl_gentle_pour(cell_mm, seconds, &c);
    c.initial_volume = (0.6 + 0.4 * next()) * 1e-3;  // fill U[0.6, 1.0] L
    c.motion.max_angle_deg = 60 + 50 * next();      // peak tilt U[60, 110] degrees
    c.motion.tilt_duration = 4 + 8 * next();        // tilt-in ramp U[4, 12] s
    c.seed = seed + 1 + uint32_t(i);
  }
  return PL_OK;
}

struct pl_ensemble {
  std::vector<pl_sim*> sims;
};

void pl_ensemble_destroy(pl_ensemble* e) {
  if (!e) return;
  for (pl_sim* s : e->sims) pl_destroy(s);
  delete e;
}

int pl_ensemble_create(const pl_config* cfgs, int32_t count, pl_ensemble** out) {
  if (!cfgs || count < 1 || !out) return fail(PL_E_ARG, "pl_ensemble_create: bad argument");
  *out = nullptr;
  pl_ensemble* e = new pl_ensemble();
  for (int i = 0; i < count; i++) {
    pl_sim* s = nullptr;
    const int rc = pl_create(&cfgs[i], &s);
    if (rc) {
      const std::string msg = g_err;
      pl_ensemble_destroy(e);
      return fail(rc, "pl_ensemble_create: pour %d: %s", i, msg.c_str());
    }
    e->sims.push_back(s);
  }
  *out = e;
  return PL_OK;
}

int32_t pl_ensemble_size(const pl_ensemble* e) { return e ? int32_t(e->sims.size()) : 0; }

pl_sim* pl_ensemble_member(pl_ensemble* e, int32_t i) {
  return e && i >= 0 && i < int32_t(e->sims.size()) ? e->sims[i] : nullptr;
}

int pl_ensemble_enqueue(pl_ensemble* e, int32_t substeps) {
  if (!e || substeps < 0) return fail(PL_E_ARG, "pl_ensemble_enqueue: bad argument");
  for (pl_sim* s : e->sims) {  // control fields as pl_enqueue_substeps sets them
    if (!s->exec) return fail(PL_E_STATE, "pl_ensemble_enqueue: a pour has no substep graph");
    cudaSetDevice(s->device);
    int rc = settle(s);
    if (rc) return rc;
    s->hs.end_time = INFINITY;
    s->hs.force_step = 0;
    std::memcpy(s->pinned, &s->hs, sizeof(SimScalars));
    const size_t off = offsetof(SimScalars, end_time);
    const size_t len = offsetof(SimScalars, active) - off;
    CK(cudaMemcpyAsync((char*)s->P.sc + off, (char*)s->pinned + off, len, cudaMemcpyHostToDevice, s->st));
  }
  for (int k = 0; k < substeps; k++)  // interleaved: every pour's next substep before anyone's following one
    for (pl_sim* s : e->sims) CK(cudaGraphLaunch(s->exec, s->st));
  for (pl_sim* s : e->sims) {
    const int rc = pull_scalars(s);
    if (rc) return rc;
  }
  return PL_OK;
}

int pl_ensemble_advance(pl_ensemble* e, double duration) {
  if (!e || !(duration >= 0)) return fail(PL_E_ARG, "pl_ensemble_advance: bad argument");
  std::vector<double> end(e->sims.size());
  for (size_t i = 0; i < e->sims.size(); i++) {
    pl_sim* s = e->sims[i];
    if (!s->exec) return fail(PL_E_STATE, "pl_ensemble_advance: a pour has no substep graph");
    cudaSetDevice(s->device);
    int rc = settle(s);
    if (rc) return rc;
    end[i] = s->hs.time + duration;  // solver3d.ts:282, per pour
    s->hs.end_time = end[i];
    s->hs.force_step = 0;
    rc = push_scalars(s);
    if (rc) return rc;
  }
  for (int guard = 0; guard < 1000000; guard++) {
    std::vector<long> k(e->sims.size(), 0);
    long kmax = 0;
    for (size_t i = 0; i < e->sims.size(); i++) {
      const pl_sim* s = e->sims[i];
      if (!(s->hs.time < end[i] - 1e-12 && !host_finished(s))) continue;
      const double remaining = std::min(end[i], s->g.duration) - s->hs.time;
      k[i] = std::max(1L, std::min((long)std::ceil(remaining / host_stable_dt(s) * 1.05) + 1, 256L));
      kmax = std::max(kmax, k[i]);
    }
    if (kmax == 0) break;
    for (long q = 0; q < kmax; q++)  // interleaved launches on the pours' own streams
      for (size_t i = 0; i < e->sims.size(); i++)
        if (q < k[i]) CK(cudaGraphLaunch(e->sims[i]->exec, e->sims[i]->st));
    for (size_t i = 0; i < e->sims.size(); i++)
      if (k[i]) {
        const int rc = pull_scalars(e->sims[i]);
        if (rc) return rc;
      }
  }
  return PL_OK;
}

}  // extern "C"
