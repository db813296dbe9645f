// Chebyshev-preconditioned CG on one thread-block cluster (see cheb.cu).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace pl {

constexpr int CHEB_CLUSTER = 16;       // largest cluster (non-portable size, one CTA per SM)
constexpr int CHEB_MAX_THREADS = 1024;  // largest CTA
constexpr int CHEB_SMEM = 220 * 1024;   // dynamic shared memory per CTA
constexpr int CHEB_DEGREE = 12;        // polynomial degree (stencil applications per CG iteration)
constexpr double CHEB_LO = 0.01;        // lower end of the D^-1 A interval the polynomial targets (the
                                        // spectrum starts near 1e-3 on 4 mm pour systems; 0.01 takes
                                        // ~10% fewer CG iterations than 0.03 at degree 12)
constexpr int CHEB_KMAX = 4;           // most cells per thread (their state stays in registers)

struct ChebArgs {
  const double* b;  // list-indexed rhs
  double* q;        // list-indexed solution
  double tol;
  int max_iter;
  int is_correction;
  int mixed;
  int degree;
  double cheb_lo;
  int cluster;     // CTAs in the cluster (launch shape, chosen by the tuner)
  int threads;     // threads per CTA (at most 1024 / cells per thread)
  int smem_bytes;  // dynamic shared memory per CTA
  int m_bound;     // liquid cells the launch is sized for (cells per thread from it)
  int gate;        // run only if the solve before it could not take the system (mg_status == 0)
  // a second system on the same liquid cells, solved after the first in the same launch (jobs = 2):
  // the density correction after the pressure
  int jobs;
  const double* b2;
  double* q2;
  double tol2;
  int max_iter2;
  // jobs = 2 on two clusters of one launch at once (cluster j solves system j) instead of one after
  // the other: the two systems are independent, so the launch takes the longer of the two
  int parallel;
};

void cheb_configure();
void launch_cheb_solve(const Geo& g, const DevPtrs& P, const SolverWs& W, const ChebArgs& a, cudaStream_t st);

}  // namespace pl
