// LU-preconditioned restarted GMRES for the correction equation of the mixed
// solve (GMRES-based iterative refinement: Carson and Higham, SIAM J. Sci.
// Comput. 40(2), 2018). Shared declarations of k_gmres.cu and mixed.cpp.
//
// Each outer step of the refinement solves M^-1 A d = M^-1 r, r = b - A x in
// FP64, with left-preconditioned GMRES: M^-1 is the FP32 factorisation (the
// butterflies, the scales and the blocked LU) applied to FP64 vectors with
// FP64 accumulation, so the preconditioned operator is a fixed linear map
// applied at working precision, and the Krylov vectors, the Arnoldi
// orthogonalisation (classical Gram-Schmidt, twice) and the Givens rotations
// are FP64. No counterpart in the reference (NumPP's solve is one FP64 LU).
// Instances: one per (system, right-hand-side column), all advanced in
// lockstep; an instance whose estimated residual reached tau * beta, or that
// broke down, stops and waits for the others.
#pragma once

#include <cuda_runtime.h>

#include "mixed.hpp"

namespace nppb {

constexpr int kGmM = 30;  // Krylov dimension of one outer step (no restarts inside it)

struct GmState {
  double beta;                // ||z0||_2
  double g[kGmM + 1];         // the rotated right-hand side of the small least-squares problem
  double R[kGmM][kGmM + 1];   // column k: the Hessenberg column after the rotations
  double c[kGmM], sn[kGmM];   // the rotations
  int k;                      // Arnoldi steps taken
  int done;                   // finished (converged, broke down, or not refining)
};

// V (kGmM + 1 planes of count x n x nrhs) gets V_0 = Z / ||Z||; the state is reset.
cudaError_t gm_start(const double* Z, double* V, GmState* gs, const RefineState* st, int count, int n, int nrhs,
                     cudaStream_t s);
// W = -M^-1 A V_k (the preconditioned product, negated as mixed_matvec leaves
// it): V_{k+1}, column k of H, its rotation; instances still iterating are
// counted into *active.
cudaError_t gm_arnoldi(const double* W, double* V, GmState* gs, const RefineState* st, int count, int n,
                       int nrhs, int k, double tau, int* active, cudaStream_t s);
// X += V_0..V_{k-1} y, R y = g (each instance's own k) for the systems still refining.
cudaError_t gm_update(const double* V, double* X, const GmState* gs, const RefineState* st, int count, int n,
                      int nrhs, cudaStream_t s);

}  // namespace nppb
