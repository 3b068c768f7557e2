// Internal declarations shared by the kernels (.cu) and the C++20 host runtime.
// Nothing here is part of the C ABI (include/numpp_b200.h is).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nppb {

// One linear system of a packed (possibly uneven) batch. All offsets are in
// elements of the matching base pointer of Batch. Row-major storage.
struct SysDesc {
  int32_t n;        // order
  int32_t nrhs;     // right-hand-side columns (0 = none)
  int32_t idx;      // slot in the per-system outputs (info, det, sign, logabs)
  int32_t pad_;
  int64_t a_off;    // A (n x n)
  int64_t lu_off;   // LU workspace / factor output (n x n)
  int64_t b_off;    // B and X (n x nrhs)
  int64_t inv_off;  // inverse output (n x n), < 0 = none
  int64_t piv_off;  // ipiv (n int32)
};

// What a launch produces for each system.
enum : int {
  kWantLU = 1,        // keep LU + ipiv (getrf); otherwise LU is scratch
  kWantSolve = 2,     // X = A^-1 B
  kWantDet = 4,       // det
  kWantSlogdet = 8,   // sign, logabsdet
  kWantInv = 16,      // inverse (only systems with inv_off >= 0 in grouped mode)
  kInPlace = 32,      // A == LU: factor in place, skip the copy
  kSolveOnly = 64,    // getrs from existing LU + ipiv (no factorisation)
  kNoPivot = 128,     // no row exchanges: the pivot is the diagonal, and a pivot <= 0
                      // stops the system (the LU behind the Cholesky factor)
};

// A batch of systems. With desc == nullptr the batch is uniform: system s has
// order n, nrhs columns, A at s*n*n, B/X at s*n*nrhs, LU and inv at s*n*n,
// ipiv at s*n.
struct Batch {
  const double* A;
  double* LU;
  int32_t* ipiv;
  const double* B;
  double* X;
  double* inv;
  double* det;
  double* sign;
  double* logabs;
  int32_t* info;
  const SysDesc* desc;
  int32_t n, nrhs;
  int flags;
};

// Per-system view resolved on the device.
struct SysView {
  int n, nrhs, idx;
  const double* A;
  double* LU;
  int32_t* ipiv;
  const double* B;
  double* X;
  double* inv;  // nullptr = no inverse for this system
};

#ifdef __CUDACC__
__device__ __forceinline__ SysView sys_view(const Batch& bt, int s) {
  SysView v;
  if (bt.desc) {
    const SysDesc d = bt.desc[s];
    v.n = d.n; v.nrhs = d.nrhs; v.idx = d.idx;
    v.A = bt.A + d.a_off;
    v.LU = bt.LU + d.lu_off;
    v.ipiv = bt.ipiv + d.piv_off;
    v.B = bt.B ? bt.B + d.b_off : nullptr;
    v.X = bt.X ? bt.X + d.b_off : nullptr;
    v.inv = (bt.inv && d.inv_off >= 0) ? bt.inv + d.inv_off : nullptr;
  } else {
    const int64_t n = bt.n, nn = n * n;
    v.n = bt.n; v.nrhs = bt.nrhs; v.idx = s;
    v.A = bt.A + s * nn;
    v.LU = bt.LU ? bt.LU + s * nn : nullptr;
    v.ipiv = bt.ipiv ? bt.ipiv + s * n : nullptr;
    v.B = bt.B ? bt.B + s * n * bt.nrhs : nullptr;
    v.X = bt.X ? bt.X + s * n * bt.nrhs : nullptr;
    v.inv = bt.inv ? bt.inv + s * nn : nullptr;
  }
  return v;
}
#endif

// ---- kernel launchers (each .cu file defines its own) ----

// Order <= 32: one warp per system, rows in registers. `order` lists the
// systems to run (nullptr = 0..nsys-1). np = padded order class (8/16/32).
cudaError_t launch_lu_warp(const Batch& bt, const int32_t* order, int nsys, int np,
                           cudaStream_t st);

// Row-major C[m,n] = A[m,k] B[k,n] in FP64 on DMMA (device pointers).
cudaError_t launch_gemm_f64(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                            const double* B, int64_t ldb, double* C, int64_t ldc,
                            cudaStream_t st);

// `batch` contiguous row-major FP64 GEMMs: C[z] = A[z] B[z] (m x k, k x n, m x n).
cudaError_t launch_gemm_f64_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* A,
                                    const double* B, double* C, cudaStream_t st);
// Row-major FP32 GEMM (SIMT), used for the gemm slot's float32 form.
cudaError_t launch_gemm_f32(int64_t m, int64_t n, int64_t k, const float* A, const float* B,
                            float* C, cudaStream_t st);

}  // namespace nppb
