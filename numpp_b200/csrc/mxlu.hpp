// Randomised blocked LU in FP32 on the tcgen05 tensor cores: the
// factorisation of the mixed-precision solve. Shared declarations of
// k_mxlu.cu and mixed.cpp.
//
// No counterpart in the reference (NumPP factors in double with partial
// pivoting only, src/linalg/linalg.cpp:48-71). The FP32 factors here are a
// preconditioner for FP64 iterative refinement, so their pivoting is free to
// differ: the equilibrated matrix is mixed by a depth-2 recursive butterfly
// transform on both sides (Parker; Baboulin, Dongarra, Herrmann and Tomov,
// ACM TOMS 39(2), 2013), M = U^T (Dr A Dc) V, and M is factored in 128-column
// blocks with partial pivoting over a window of 256 rows: the diagonal
// block's and the next block's (the multipliers stay below 2 in practice where
// pivoting within the block alone let them reach 1e2 and more).
// Per block k (K = 128 k):
//   diag   the 256 x 128 window panel factored with partial pivoting in one
//          CTA per system: the packed L11 U11 of the 128 rows chosen, the other
//          rows' multipliers (their L21), L11^-1 and U11^-1 (blocked
//          inversion), and the window's row order;
//   perm   that order applied to the rest of the window's rows, left and right
//          of the block (as LAPACK's row interchanges), and the new panel row
//          transposed;
//   trsmL  L21 = A21 U11^-1 below the window  (tcgen05 GEMM, K = 128)
//   trsmU  U12^T = A12^T L11^-T               (tcgen05 GEMM on the transposed panel row)
//   trail  A22 -= L21 U12                     (tcgen05 GEMM, K = 128).
// The composed row order P goes to the right-hand sides: M = P^T L U.
// The GEMM operands come in by TMA (non-multicast, this GPU's own memory)
// in 128-byte-swizzled tiles; products are error-compensated TF32
// (hi*hi + hi*lo + lo*hi) with FP32 accumulators in TMEM.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "mixed.hpp"

namespace nppb {

constexpr int kMxNB = 128;  // block width: the K of every GEMM and the TMEM accumulator's rows

// Padded order of the factorisation: a multiple of the block width (the pad is
// an identity block, the right-hand sides' pad rows are zero).
inline int mx_padded(int n) { return (n + kMxNB - 1) / kMxNB * kMxNB; }

struct MxBufs {
  int count = 0, n = 0, N = 0;
  float* M = nullptr;      // count x N x N: the transformed matrix, then L (unit, below) and U
  float* T = nullptr;      // 2 x count x N x 128: transposed panel rows (A12^T, then U12^T), two buffers
  float* Linv = nullptr;   // count x N x 128: L_kk^-1 P_kk of block k at rows 128k .. 128k+127
  float* Uinv = nullptr;   // count x N x 128: U_kk^-1
  float* UinvT = nullptr;  // count x N x 128: U_kk^-T
  int32_t* info = nullptr; // count: 0, or 1 + first column whose pivot was zero / not finite
  double* rbt = nullptr;   // 12 x N/2: the butterflies' random diagonals (computed by mx_build)
  int32_t* perm = nullptr;   // count x N/128 x 256: each block's window order (window row of each position)
  int32_t* rowpos = nullptr; // count x N: final position of every row of M
  int split3 = 1;          // error-compensated TF32 (1) or plain TF32 (0) products
};

// Device bytes of the factorisation's buffers for a batch (M, T, Linv, Uinv, UinvT, info, rbt, perm, rowpos).
size_t mx_workspace_bytes(int count, int n);
// Carve the buffers out of one allocation of mx_workspace_bytes (256-byte aligned).
void mx_carve(MxBufs& b, void* base, int count, int n);

// M = U^T (diag(rs) A diag(cs)) V with cs = power-of-two scales of cmax (1
// without equilibration), padded; writes cs and initialises the refinement
// state (eta, prev = inf, active, no corrections).
cudaError_t mx_build(const double* A, const double* rs, const double* cmax, int equil, double* cs,
                     RefineState* st, const MxBufs& b, cudaStream_t s);
// Blocked factorisation of M (every system).
cudaError_t mx_factor(const MxBufs& b, cudaStream_t s);
// Y (count x N x nrhs) = U^T pad(R) for R (count x n x nrhs, FP32, already
// row-scaled); only systems still refining when only_active.
cudaError_t mx_rhs_in(const float* R, float* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b,
                      cudaStream_t s);
// Y <- (P L U)^-1 Y in place (forward then back substitution by blocks).
cudaError_t mx_solve(float* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b, cudaStream_t s);
// X (count x n x nrhs, FP64) = cs * (V Y)[0:n] (init) or X += that (systems still refining).
cudaError_t mx_apply(const float* Y, double* X, const double* cs, int nrhs, const RefineState* st, int init,
                     const MxBufs& b, cudaStream_t s);
// The same three steps on FP64 vectors (FP32 factors, FP64 accumulation): the
// preconditioner of the GMRES refinement. R is already row-scaled; chunks of
// up to 4 right-hand sides per substitution.
cudaError_t mx_rhs_in64(const double* R, double* Y, int nrhs, const RefineState* st, int only_active,
                        const MxBufs& b, cudaStream_t s);
cudaError_t mx_solve64(double* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b,
                       cudaStream_t s);
cudaError_t mx_apply64(const double* Y, double* X, const double* cs, int nrhs, const RefineState* st, int init,
                       const MxBufs& b, cudaStream_t s);
// Bounded waits of the GEMM kernel that ran out since the last call (each
// such CTA skipped its stores); the counter is reset. -1: unreadable.
int mx_timeouts_take();
// One-time kernel attribute setup (dynamic shared memory opt-in).
cudaError_t mx_prepare();

}  // namespace nppb
