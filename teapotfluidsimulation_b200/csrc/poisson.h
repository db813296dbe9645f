// Batched dense-grid pressure-Poisson solves (poisson.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace pl {

struct PoissonImpl;
struct UNetImpl;

int poisson_generate(int n, int first, int count, uint8_t* cell, float* b, int threads);
int gauge_fix_one(int n, uint8_t* cell, float* b);
PoissonImpl* poisson_create(int nx, int ny, int nz, int count, int method, int precision, char* err, size_t errlen,
                            int* rc);
int poisson_solve(PoissonImpl* h, const uint8_t* cell, const float* b, double* x, double tol, int max_iter,
                  cudaStream_t st, int* iters, double* res, int* conv, char* err, size_t errlen);
void poisson_destroy(PoissonImpl* h);
// Device-driven use inside a stream capture (the pour engine's grid-scale solves): the levels of a
// box's cell types, then solves on them, each a graph while-loop; the last solve's outcome
// (iterations, converged, max-norm residual) written to device memory. MG or LEARNED, one box.
int poisson_capture_setup(PoissonImpl* h, const uint8_t* cell, cudaStream_t st, char* err, size_t errlen);
int poisson_capture_solve(PoissonImpl* h, const float* b, double* x, double tol, int max_iter, cudaStream_t st,
                          char* err, size_t errlen);
void poisson_capture_result(PoissonImpl* h, double* out3, cudaStream_t st);
void poisson_set_unet(PoissonImpl* h, UNetImpl* u);
size_t poisson_bytes(const PoissonImpl* h);
int poisson_history(const PoissonImpl* h, int snapshot, double* out, int capacity, int* recorded, int* learned_it);

}  // namespace pl
