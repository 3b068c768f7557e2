// Step-wise batched LU (orders > 32): shared types of k_step.cu and plan.cpp.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "nppb_internal.hpp"

namespace nppb {

constexpr int kStepNB = 32;     // panel width
constexpr int kStepMaxN = 4096;  // largest order: a cluster of 8 CTAs x 512 threads, one panel row each
constexpr int kStepNBO = 128;   // outer block of the two-level (blocked) factorisation: 4 panels

// Per-system state carried from one step to the next (one slot per system,
// SysDesc::pad_ is the slot index). T is the factor precision.
template <class T>
struct StepScratchT {
  T linv[kStepNB * kStepNB];       // L11^-1 of the current panel, row-major
  int top_src[kStepNB];            // panel-relative source row of each top position
  int disp_dst[kStepNB];           // displaced old top rows: their new positions
  int disp_src[kStepNB];           //   ... and their old positions
  int ndisp;
  int info;                        // 0, or first zero pivot + 1 (later launches skip)
  int nswap;
  int pad_;
  double det, logabs, sign;        // running det / log|det| / sign
};
using StepScratch = StepScratchT<double>;

// Row moves and L11^-1 of the panels of one outer block (two-level
// factorisation): the trailing columns get them after the block.
template <class T>
struct StepHistT {
  T linv[kStepNBO / kStepNB][kStepNB * kStepNB];
  int top_src[kStepNBO / kStepNB][kStepNB];
  int disp_dst[kStepNBO / kStepNB][kStepNB];
  int disp_src[kStepNBO / kStepNB][kStepNB];
  int ndisp[kStepNBO / kStepNB];
};

using StepHist = StepHistT<double>;

// Smallest order that takes the two-level factorisation of uniform batches:
// NPPB_BLOCKED_MIN_N (read once per process); 0, the default, keeps the
// one-level schedule with look-ahead.
int blocked_min_n();

// Strip kinds.
enum : int16_t { kSegMatrix = 0, kSegRhs = 1, kSegInv = 2, kSegLeft = 3 };

// One CTA of k_update / k_back / k_forward: a 64-column strip of one system.
struct StepItem {
  int32_t sys;    // index into desc
  int16_t kind;
  int16_t width;  // columns in this strip (<= 64)
  int32_t c0;     // first column
  int32_t pad_;
};

template <class T>
struct StepArgsT {
  const SysDesc* desc;
  StepScratchT<T>* scratch;
  const T* A;        // step-0 source of the matrices (nullptr: factor LU in place)
  T* LU;
  int32_t* ipiv;
  const T* B;
  T* X;
  T* inv;
  double* det;
  double* sign;
  double* logabs;
  int32_t* info;
  int solve_only;    // getrs from stored factors: no factorisation state to consult
  // Uniform batch (desc == nullptr): system s has order un, unrhs right-hand
  // sides, A / LU / inverse at s*un*un, B / X at s*un*unrhs, ipiv at s*un,
  // scratch slot s; an inverse for every system when uinv != 0.
  int un, unrhs, uinv;
  int uleft;         // uniform batch keeps its factors: carry row moves left of each panel
  int unopiv;        // no row exchanges: pivot on the diagonal, a pivot <= 0 stops the system
  int umode;         // FP32 factors: trailing product in FP32 FMA (0), TF32 (1), BF16 (2), 3xTF32 (3) on mma.sync,
                     // or TF32 (4) / 3xTF32 (5) on tcgen05 with TMEM accumulators
  // Two-level factorisation of a uniform batch (ubend > 0): the panels of the
  // outer block [ubbeg, ubend) update only the block's columns (and the
  // right-hand sides / inverse); row moves reach the columns left of the
  // panel inside the block. utrail: the items are the matrix strips right of
  // the block (the trailing pass after it), whose row moves and L11^-1 come
  // from hist[sys] slot hslot; urow_end > 0 stops k_update at that row. The
  // panel records its row moves and L11^-1 in slot hslot when hist is set.
  //
  // The trailing pass first applies the block's row moves (umoves = 1: moves
  // only, panel by panel), then the triangular solves and in-block updates
  // (umoves = 2: U12 of rows already in place), as LAPACK's blocked getrf
  // orders laswp before trsm.
  StepHistT<T>* hist;
  int hslot;
  int ubbeg, ubend;
  int utrail;
  int umoves;
  int urow_end;
};
using StepArgs = StepArgsT<double>;

// Work items of a uniform batch at step k0 (k_update) and of its back
// substitution, per system; grids are count times these.
__host__ __device__ inline int uniform_update_strips(int n, int nrhs, int inv, int k0, int left = 0) {
  const int trail = n - k0 - kStepNB;
  return (trail > 0 ? (trail + 63) / 64 : 0) + (nrhs + 63) / 64 + (inv ? (n + 63) / 64 : 0) +
         (left ? (k0 + 63) / 64 : 0);
}
// The same inside an outer block [bbeg, bend) of the two-level factorisation:
// matrix strips [k0+32, bend), right-hand sides, inverse, and the moves-only
// strips left of the panel from column left ? 0 : bbeg.
__host__ __device__ inline int blocked_update_strips(int n, int nrhs, int inv, int k0, int left, int bbeg,
                                                     int bend) {
  const int mat = bend - k0 - kStepNB;
  const int lo = left ? 0 : bbeg;
  return (mat > 0 ? (mat + 63) / 64 : 0) + (nrhs + 63) / 64 + (inv ? (n + 63) / 64 : 0) +
         (k0 > lo ? (k0 - lo + 63) / 64 : 0);
}
// Matrix strips right of an outer block: the trailing pass after it.
__host__ __device__ inline int trailing_strips(int n, int bend) { return bend < n ? (n - bend + 63) / 64 : 0; }
__host__ __device__ inline int uniform_back_strips(int n, int nrhs, int inv) {
  return (nrhs + 63) / 64 + (inv ? (n + 63) / 64 : 0);
}

cudaError_t step_prepare();
// Bounded waits of the tensor-core update that ran out since the last call
// (each such CTA skipped its stores); the counter is reset. -1: unreadable.
int tc_timeouts_take();
// Panel of every listed system at column k0; mmax = largest n - k0 among them.
// list == nullptr: systems 0..nsys-1 of a uniform batch. Likewise items ==
// nullptr below means the uniform-batch items, derived from the block index.
// T = double (FP64 DMMA updates) or float (FP32 factors for the mixed path).
template <class T>
cudaError_t launch_panel(const StepArgsT<T>& sa, const int32_t* list, int nsys, int mmax, int k0,
                         cudaStream_t st);
// Row moves + U12 + trailing update for each strip item of step k0 (nmax >= n of any item).
// launch_update = launch_rows, then launch_trailing with part 0. A uniform
// batch (items == nullptr) can split the trailing update for look-ahead:
// part 1 launches only the first matrix strip of every system (nitems =
// systems), part 2 every other strip (nitems = all strips).
template <class T>
cudaError_t launch_rows(const StepArgsT<T>& sa, const StepItem* items, int nitems, int k0, cudaStream_t st);
template <class T>
cudaError_t launch_trailing(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int k0, int part,
                            cudaStream_t st);
template <class T>
cudaError_t launch_update(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int k0,
                          cudaStream_t st);
// Two-level factorisation of a uniform batch: after the panels of the outer
// block [bbeg, bend), C -= L U on rows [bend, n) x columns [cbeg, cend) of
// every system (FP64 factors; DMMA tiles).
template <class T>
cudaError_t launch_block_gemm(const StepArgsT<T>& sa, int count, int bbeg, int bend, int cbeg, int cend,
                              cudaStream_t st);
// The block's row moves, U12 and block-row updates on every strip right of it.
template <class T>
cudaError_t launch_block_rows(const StepArgsT<T>& sa, int count, int bbeg, int bend, cudaStream_t st);
// Back substitution of each strip item (nmax >= n of any item, wmax >= the
// width of any item: strips of at most 8 columns take the narrow kernels).
template <class T>
cudaError_t launch_back(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int wmax,
                        cudaStream_t st);
// getrs from stored factors: launch_forward gathers X = P B (unless permute
// is false: X already holds the permuted right-hand sides) and runs the
// forward substitution; the caller then runs launch_back.
template <class T>
cudaError_t launch_forward(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int wmax,
                           cudaStream_t st, bool permute = true);

}  // namespace nppb
