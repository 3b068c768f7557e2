// Mixed-precision solve: shared declarations of k_mixed.cu and mixed.cpp.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nppb {

constexpr int kMixedMaxN = 4096;
constexpr int kMixedRows = 32;  // rows of A per CTA in the equilibration and residual kernels

enum : int { kRefineActive = 0, kRefineConverged = 1, kRefineStalled = 2 };

// Per-system refinement state (device).
struct RefineState {
  double anorm;  // ||A||_inf
  double bnorm;  // max |B|
  double eta;    // last normwise backward error
  double prev;   // eta of the previous iteration
  int status;    // kRefine*
  int iters;     // corrections applied
  // running maxima of non-negative doubles, as their bit patterns (atomicMax);
  // zero at the start of every residual pass
  unsigned long long rmax_bits;  // max |R|
  unsigned long long xmax_bits;  // max |X|
};

// st and cmax (count * n doubles of column maxima) must be zero on entry.
cudaError_t mixed_equilibrate(const double* A, int count, int n, int equil, float* A32, double* rs,
                              double* cs, double* cmax, RefineState* st, cudaStream_t s);
// The row pass of mixed_equilibrate alone: row scales rs, ||A||_inf into st,
// column maxima of diag(rs)|A| into cmax (no FP32 copy of A).
cudaError_t mixed_equil_scan(const double* A, int count, int n, int equil, double* rs, double* cmax,
                             RefineState* st, cudaStream_t s);
cudaError_t mixed_scale_rhs(const double* B, int count, int n, int nrhs, const double* rs, float* B32,
                            RefineState* st, cudaStream_t s);
cudaError_t mixed_apply(double* X, const float* Y, const double* cs, int count, int n, int nrhs,
                        const RefineState* st, int init, cudaStream_t s);
// decide = 1: update status / iters and count the still-active systems into *active
// (a system is stalled when its contraction cannot reach tol in max_iter - iter corrections).
// R32 (optional): r * R in FP32, row i stored at row rpos[i] (the pivoted order) when rpos is given.
// R64 (optional): r * R in FP64, natural row order.
cudaError_t mixed_residual(const double* A, const double* B, const double* X, int count, int n, int nrhs,
                           const double* rs, float* R32, const int32_t* rpos, RefineState* st, double tol,
                           int iter, int max_iter, int decide, int* active, cudaStream_t s,
                           double* R64 = nullptr);
// R64 = -diag(rs) A X in FP64 for the systems still refining (no state update).
cudaError_t mixed_matvec(const double* A, const double* X, int count, int n, int nrhs, const double* rs,
                         double* R64, RefineState* st, cudaStream_t s);
// rpos[s*n + i] = position of row i after the swaps of ipiv (s*n .. s*n+n-1).
cudaError_t mixed_row_positions(const int32_t* ipiv, int count, int n, int32_t* rpos, cudaStream_t s);
cudaError_t mixed_ferr(const double* X, const double* Xt, int count, int n, int nrhs, double* ferr,
                       cudaStream_t s);
cudaError_t mixed_mark_fp32_failures(const int32_t* info32, RefineState* st, int count, cudaStream_t s);

}  // namespace nppb
