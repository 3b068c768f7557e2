// Batched Cholesky factor of (count, n, n) FP64 stacks. C++20.
//
// The reference factors one matrix at a time, column by column, reading only
// the lower triangle and stopping with "Matrix is not positive definite" at a
// diagonal <= 0 (src/linalg/linalg.cpp:117-136; stacks batched.cpp:77). Here
// the whole stack runs on the LU kernels: the matrix is made symmetric from its
// lower triangle, factored as A = L_u U without row exchanges (a pivot <= 0
// stops the system: for a symmetric matrix the pivots are the squares of the
// Cholesky diagonal), and L = L_u diag(sqrt(u_jj)). Orders <= 32 take the
// warp-per-system kernel, larger ones the step-wise kernels. Twice the flops
// of a dedicated Cholesky, on kernels that are already tuned.
#include <cuda_runtime.h>

#include <new>

#include "../../include/numpp_b200.h"
#include "nppb_internal.hpp"
#include "nppb_step.hpp"
#include "runtime.hpp"

using namespace nppb;

namespace {

#define NPPB_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)

template <class F>
int guarded(F&& f) {
  try {
    clear_error();
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return NPPB_E_NOMEM;
  }
}

// W = the symmetric matrix whose lower triangle is A's.
__global__ void k_sym_lower(const double* __restrict__ A, double* __restrict__ W, int64_t count, int64_t n) {
  const int64_t total = count * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = i / (n * n), e = i - s * n * n, r = e / n, c = e - r * n;
    W[i] = r >= c ? A[i] : A[s * n * n + c * n + r];
  }
}

// L = L_u diag(sqrt(u_jj)) from the unpivoted LU factors in W (unit-lower L_u
// below the diagonal, U on and above it); zero above the diagonal.
__global__ void k_chol_form(const double* __restrict__ W, double* __restrict__ L, int64_t count, int64_t n) {
  const int64_t total = count * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = i / (n * n), e = i - s * n * n, r = e / n, c = e - r * n;
    const double d = sqrt(W[s * n * n + c * n + c]);
    L[i] = r > c ? W[i] * d : (r == c ? d : 0.0);
  }
}

int cholesky_device(int64_t count, int32_t n, const double* dA, double* dL, int32_t* dinfo, cudaStream_t st) {
  const size_t nn = (size_t)n * n, c = (size_t)count;
  DevMem w_m, sc_m, piv_m;
  NPPB_CUDA(w_m.alloc(sizeof(double) * c * nn, st), "workspace");
  double* W = w_m.as<double>();
  const unsigned grid = 148 * 8;
  k_sym_lower<<<grid, 256, 0, st>>>(dA, W, count, n);
  NPPB_CUDA(cudaGetLastError(), "symmetrise");
  if (n <= 32) {
    NPPB_CUDA(piv_m.alloc(sizeof(int32_t) * c * n, st), "workspace");
    Batch bt{};
    bt.A = W;
    bt.LU = W;
    bt.ipiv = piv_m.as<int32_t>();
    bt.info = dinfo;
    bt.n = n;
    bt.nrhs = 0;
    bt.flags = kWantLU | kInPlace | kNoPivot;
    NPPB_CUDA(launch_lu_warp(bt, nullptr, (int)count, n <= 8 ? 8 : (n <= 16 ? 16 : 32), st), "factorisation");
  } else {
    NPPB_CUDA(sc_m.alloc(sizeof(StepScratch) * c, st), "workspace");
    StepArgs sa{};
    sa.scratch = sc_m.as<StepScratch>();
    sa.A = nullptr;  // in place on the symmetric copy
    sa.LU = W;
    sa.info = dinfo;
    sa.un = n;
    sa.unopiv = 1;
    NPPB_CUDA(run_step_uniform(sa, (int)count, st), "factorisation");
  }
  k_chol_form<<<grid, 256, 0, st>>>(W, dL, count, n);
  NPPB_CUDA(cudaGetLastError(), "factor");
  // the workspaces are freed in stream order when w_m / sc_m / piv_m go out of scope
  return NPPB_OK;
}

int check_args(int64_t count, int32_t n) {
  if (count < 0 || n < 0) {
    set_error("negative count or order");
    return NPPB_E_ARG;
  }
  if (count > INT32_MAX) {
    set_error("batch count above 2^31-1");
    return NPPB_E_RANGE;
  }
  if (n > kStepMaxN) {
    set_error("order above 4096 is not served by the batched path");
    return NPPB_E_RANGE;
  }
  return NPPB_OK;
}

}  // namespace

extern "C" {

int nppb_d_cholesky_batched(int64_t count, int32_t n, const double* dA, double* dL, int32_t* dinfo,
                            void* stream) {
  return guarded([&]() -> int {
    const int rc = check_args(count, n);
    if (rc != NPPB_OK) return rc;
    if (!count || !n) return NPPB_OK;
    if (!dA || !dL || !dinfo) {
      set_error("cholesky needs A, L and info");
      return NPPB_E_ARG;
    }
    if (!device()) return NPPB_E_NODEV;
    return cholesky_device(count, n, dA, dL, dinfo, static_cast<cudaStream_t>(stream));
  });
}

int nppb_cholesky_batched(int64_t count, int32_t n, const double* A, double* L, int32_t* info) {
  return guarded([&]() -> int {
    const int rc = check_args(count, n);
    if (rc != NPPB_OK) return rc;
    if (!count || !n) return NPPB_OK;
    if (!A || !L || !info) {
      set_error("cholesky needs A, L and info");
      return NPPB_E_ARG;
    }
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t nn = (size_t)count * n * n;
    DevMem dA, dL, dI;
    NPPB_CUDA(dA.alloc(sizeof(double) * nn, st), "allocation");
    NPPB_CUDA(dL.alloc(sizeof(double) * nn, st), "allocation");
    NPPB_CUDA(dI.alloc(sizeof(int32_t) * count, st), "allocation");
    NPPB_CUDA(cudaMemcpyAsync(dA.as<double>(), A, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "copy");
    const int r = cholesky_device(count, n, dA.as<double>(), dL.as<double>(), dI.as<int32_t>(), st);
    if (r != NPPB_OK) return r;
    NPPB_CUDA(cudaMemcpyAsync(L, dL.as<double>(), sizeof(double) * nn, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaMemcpyAsync(info, dI.as<int32_t>(), sizeof(int32_t) * count, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    NPPB_CUDA(cudaGetLastError(), "kernel");
    return NPPB_OK;
  });
}

}  // extern "C"
