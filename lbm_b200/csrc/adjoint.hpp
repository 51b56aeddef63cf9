// adjoint.hpp -- launchers of the adjoint kernels (adjoint_fp64.cu) for the
// adjoint-run driver (adjoint_run.cu).  All launches go to stream st with the
// box's plane-tile launch shape L; populations are q-major (a[q*n + cell]).
#pragma once

#include <cuda_runtime.h>

#include "lbm_solver.cuh"

namespace lbm {
namespace adj {

// Scratch doubles per cell the collide backward needs.
constexpr int kCollideScratch = 19;
// Partial-sum blocks of sum() and of a Poisson check.
constexpr int kSumBlocks = 296;

// Collide backward (first: the run's first collision).  lfin, lgin, lkf may
// be null.  Writes lphi..lw (overwritten, not added).
void collide_backward(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, bool first,
                      const double* phi, const double* rho, const double* u, const double* v, const double* w,
                      const double* lf, const double* lg, const double* ldux, const double* ldvy,
                      const double* ldwz, double* lfin, double* lgin, double* lphi, double* lrho, double* lu,
                      double* lv, double* lw, double* scratch, double* lkf);
// Moments backward, added to lf and lg.
void moments_backward_add(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, const double* phi,
                          const double* lphi, const double* lrho, const double* lu, const double* lv,
                          const double* lw, double* lf, double* lg);
// Correction backward, added to lp and lrho.
void correct_backward_add(cudaStream_t st, const Launch& L, const Geom& g, const double* p, const double* rho,
                          const double* lu, const double* lv, const double* lw, double* lp, double* lrho);
// Poisson adjoint: y = lp on every q; one transposed sweep (check: also the
// relative-change partials, 2 x L.nblocks doubles); the final multiplier's
// dJ/ds (ls) and dJ/drho (added to lrho).
void poisson_init(cudaStream_t st, const Launch& L, const Geom& g, const double* lp, double* y);
// pi = sum_q y_q (the first check's reference for a given starting iterate).
void poisson_pi(cudaStream_t st, const Launch& L, const Geom& g, const double* y, double* pi);
void poisson_sweep(cudaStream_t st, const Launch& L, const Geom& g, bool check, const double* yin, double* yout,
                   const double* rho, const double* lp, double* pi_prev, double* part);
void poisson_final(cudaStream_t st, const Launch& L, const Geom& g, const double* y, const double* h,
                   const double* rho, double* ls, double* lrho);
void prep_backward(cudaStream_t st, const Launch& L, const Geom& g, const double* ls, double mean_ls,
                   double* ldux, double* ldvy, double* ldwz);
// Block partials (kSumBlocks) of a[0..n); the host adds them in order.
void sum_partials(cudaStream_t st, const double* a, long long n, double* part);
void add_const(cudaStream_t st, double* a, long long n, double alpha);

}  // namespace adj
}  // namespace lbm
