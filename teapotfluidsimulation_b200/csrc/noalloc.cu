// pl_pcg_solve_device_noalloc: the standalone MIC(0) FP64 solve (pl_pcg_solve_device) with its
// scratch in a fixed static device array instead of cudaMalloc.
//
// Who needs it: hosts that own all device memory themselves (a pool or arena they hand out, a
// budget that forbids allocations outside it, a runtime that must not block on the allocator) and
// so cannot let a library call cudaMalloc/cudaFree on their behalf. The caller still passes the
// cell types, the rhs and the solution buffer.
//
// The array lives in this translation unit's own device module. With the CUDA runtime's lazy module
// loading (the default), a process that never calls this entry point never loads the module and
// never holds the array; a process that calls it holds it on that device until exit.
#include <cstdio>

#include "pcg_block.cuh"

namespace pl {

namespace {

// The scratch covers grids of up to PL_NOALLOC_MAX_CELLS cells: the solver workspace, the cell-to-
// list map, the liquid list, the list-ordered rhs and solution and the result slots (~30 MB).
// Nothing in it has to start at zero: every word a kernel reads was written earlier in the same
// call (the prep kernel writes the whole cell-to-list map and the liquid count, the set-up kernel
// every list-indexed entry the solve reads). One copy exists per device, so calls that overlap on
// one device (two host threads, or a second call while the first is still running) overwrite each
// other's scratch.
constexpr size_t al256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t NOALLOC_WS_BYTES = 8 * al256((size_t)PL_NOALLOC_MAX_CELLS * 8) +
                                    al256((size_t)PL_NOALLOC_MAX_CELLS * 24) +
                                    2 * al256((size_t)PL_NOALLOC_MAX_CELLS * 4) +
                                    al256((MAX_LEVELS + 1) * 4) + al256(16);
constexpr size_t NOALLOC_BYTES = NOALLOC_WS_BYTES + (size_t)PL_NOALLOC_MAX_CELLS * (4 * 2 + 8 * 2) + 256;
__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of the scratch in the current context. In host code the array's name is only a
// handle for this lookup, never an address a kernel may be given. The lookup runs on every call:
// the address belongs to the context that loaded the module, so a cached address would be stale
// after a device reset or in another context on the same device. It allocates nothing; the first
// lookup in a context loads the module (and with it the array), so that first call should come
// before any stream capture on the device.
int noalloc_scratch(void** base, char* err, size_t errlen) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    int dev = -1;
    cudaGetDevice(&dev);
    snprintf(err, errlen, "pl_pcg_solve_device_noalloc: cudaGetSymbolAddress on device %d: %s", dev,
             e != cudaSuccess ? cudaGetErrorString(e) : "null address");
    return PL_E_CUDA;
  }
  *base = p;
  return PL_OK;
}

}  // namespace

int standalone_pcg_noalloc(const uint8_t* cell, const double* b, double* q, int nx, int ny, int nz, double tol,
                           int max_iter, cudaStream_t st, int* iterations, int* converged, double* residual,
                           char* err, size_t errlen) {
  if (nx < 3 || ny < 3 || nz < 3 || nx + ny + nz > MAX_LEVELS) {
    snprintf(err, errlen, "pl_pcg_solve_device_noalloc: grid %dx%dx%d out of range", nx, ny, nz);
    return PL_E_ARG;
  }
  const long long ncl = (long long)nx * ny * nz;
  if (ncl > PL_NOALLOC_MAX_CELLS) {
    snprintf(err, errlen,
             "pl_pcg_solve_device_noalloc: grid %dx%dx%d has %lld cells, more than the fixed scratch holds "
             "(PL_NOALLOC_MAX_CELLS = %d); use pl_pcg_solve_device",
             nx, ny, nz, ncl, PL_NOALLOC_MAX_CELLS);
    return PL_E_ARG;
  }
  const int nc = (int)ncl;
  const size_t wsb = solver_ws_bytes(nc);
  if (wsb + (size_t)nc * (4 * 2 + 8 * 2) + 256 > NOALLOC_BYTES) {  // cannot happen for nc <= the maximum
    snprintf(err, errlen, "pl_pcg_solve_device_noalloc: scratch layout exceeds %zu bytes", NOALLOC_BYTES);
    return PL_E_ARG;
  }
  // An error left pending by the caller's own earlier launches is reported as such and left in
  // place, so that the check after this call's launches sees only this call's launch errors.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "pl_pcg_solve_device_noalloc: a CUDA error was already pending before the call: %s",
             cudaGetErrorString(e));
    return PL_E_CUDA;
  }
  void* mem = nullptr;
  int rc = noalloc_scratch(&mem, err, errlen);
  if (rc) return rc;
  SolverWs W = solver_ws_carve(mem, nc);
  char* p = static_cast<char*>(mem) + wsb;
  int* lidx = (int*)p;
  int* list = lidx + nc;
  double* bl = (double*)(list + nc);  // 2 * nc ints from a 256-byte boundary: 8-byte aligned
  double* ql = bl + nc;
  int* small = (int*)(ql + nc);  // [0] m, [1..2] result
  double* resd = (double*)(small + 4);
  k_standalone_prep<<<1, 1024, 0, st>>>(cell, nx, ny, nz, lidx, list, small);
  k_standalone_setup<<<DENSITY_BLOCKS, 256, 0, st>>>(cell, b, nx, ny, lidx, list, small, W, bl);
  k_standalone_pcg<<<1, SOLVER_THREADS, 0, st>>>(W, small, bl, ql, tol, max_iter, small + 1, resd);
  k_standalone_scatter<<<(nc + 255) / 256, 256, 0, st>>>(lidx, ql, q, nc);
  int hres[3];
  double hr = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hres, small, 12, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hr, resd, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "pl_pcg_solve_device_noalloc: %s", cudaGetErrorString(e));
    return PL_E_CUDA;
  }
  if (iterations) *iterations = hres[1];
  if (converged) *converged = hres[2];
  if (residual) *residual = hr;
  return PL_OK;
}

}  // namespace pl
