// Stacked matmul and matrix_power on the batched FP64 kernels. C++20.
//
// The reference's matmul is 2-D only (src/backend/backend.cpp:121-177 rejects
// ndim > 2) and its stacked matrix_power maps the 2-D routine over the stack
// (src/linalg/batched.cpp:83-84 -> linalg.cpp:440-454: binary exponentiation
// with matmul, inv first for negative powers). Here both run on the device
// over a whole stack at once: the batched DMMA GEMM (one launch per product
// for every matrix of the stack) and the batched inverse.
#include <cuda_runtime.h>

#include <new>
#include <string>
#include <utility>

#include "../../include/numpp_b200.h"
#include "nppb_internal.hpp"
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

__global__ void k_identity_batched(double* R, int64_t count, int64_t n) {
  const int64_t total = count * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i % (n * n);
    R[i] = (e / n == e % n) ? 1.0 : 0.0;
  }
}

// R = A^p for a (count, n, n) stack on the device; singular A with p < 0 -> info.
int matrix_power_device(int64_t count, int32_t n, int64_t p, const double* dA, double* dR, int32_t* dinfo,
                        cudaStream_t st) {
  const size_t nn = (size_t)n * n, c = (size_t)count;
  DevMem base, tmp;
  NPPB_CUDA(base.alloc(sizeof(double) * c * nn, st), "workspace");
  NPPB_CUDA(tmp.alloc(sizeof(double) * c * nn, st), "workspace");
  if (p < 0) {
    const int rc = nppb_d_linalg_batched(count, n, 0, NPPB_WANT_INV, dA, nullptr, nullptr, base.as<double>(),
                                         nullptr, nullptr, nullptr, nullptr, nullptr, dinfo, st);
    if (rc != NPPB_OK) return rc;
  } else {
    NPPB_CUDA(cudaMemcpyAsync(base.as<double>(), dA, sizeof(double) * c * nn, cudaMemcpyDeviceToDevice, st), "copy");
    if (dinfo) NPPB_CUDA(cudaMemsetAsync(dinfo, 0, sizeof(int32_t) * c, st), "memset");
  }
  uint64_t e = p < 0 ? (uint64_t)(-(p + 1)) + 1 : (uint64_t)p;
  // result starts at the identity; binary exponentiation as the reference does
  k_identity_batched<<<148 * 4, 256, 0, st>>>(dR, count, n);
  NPPB_CUDA(cudaGetLastError(), "identity");
  double* b = base.as<double>();
  double* t = tmp.as<double>();
  while (e > 0) {
    if (e & 1) {
      NPPB_CUDA(launch_gemm_f64_batched(count, n, n, n, dR, b, t, st), "matmul");
      NPPB_CUDA(cudaMemcpyAsync(dR, t, sizeof(double) * c * nn, cudaMemcpyDeviceToDevice, st), "copy");
    }
    e >>= 1;
    if (e) {
      NPPB_CUDA(launch_gemm_f64_batched(count, n, n, n, b, b, t, st), "matmul");
      std::swap(b, t);
    }
  }
  // b / t may have swapped: keep both buffers alive until the stream is done
  NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
  return NPPB_OK;
}

}  // namespace

extern "C" {

int nppb_d_gemm_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* dA, const double* dB,
                        double* dC, void* stream) {
  return guarded([&]() -> int {
    if (batch < 0 || m < 0 || n < 0 || k < 0) {
      set_error("negative batch or GEMM extent");
      return NPPB_E_ARG;
    }
    if (!batch || !m || !n) return NPPB_OK;
    if ((k && (!dA || !dB)) || !dC) {
      set_error("null GEMM operand");
      return NPPB_E_ARG;
    }
    if (!device()) return NPPB_E_NODEV;
    NPPB_CUDA(launch_gemm_f64_batched(batch, m, n, k, dA, dB, dC, static_cast<cudaStream_t>(stream)),
              "batched gemm");
    return NPPB_OK;
  });
}

int nppb_gemm_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* A, const double* B, double* C) {
  return guarded([&]() -> int {
    if (batch < 0 || m < 0 || n < 0 || k < 0) {
      set_error("negative batch or GEMM extent");
      return NPPB_E_ARG;
    }
    if (!batch || !m || !n) return NPPB_OK;
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t a = (size_t)batch * m * k, b = (size_t)batch * k * n, c = (size_t)batch * m * n;
    DevMem dA, dB, dC;
    NPPB_CUDA(dA.alloc(sizeof(double) * (a ? a : 1), st), "allocation");
    NPPB_CUDA(dB.alloc(sizeof(double) * (b ? b : 1), st), "allocation");
    NPPB_CUDA(dC.alloc(sizeof(double) * c, st), "allocation");
    if (a) NPPB_CUDA(cudaMemcpyAsync(dA.as<double>(), A, sizeof(double) * a, cudaMemcpyHostToDevice, st), "copy");
    if (b) NPPB_CUDA(cudaMemcpyAsync(dB.as<double>(), B, sizeof(double) * b, cudaMemcpyHostToDevice, st), "copy");
    NPPB_CUDA(launch_gemm_f64_batched(batch, m, n, k, dA.as<double>(), dB.as<double>(), dC.as<double>(), st),
              "batched gemm");
    NPPB_CUDA(cudaMemcpyAsync(C, dC.as<double>(), sizeof(double) * c, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    return NPPB_OK;
  });
}

int nppb_matrix_power_batched(int64_t count, int32_t n, int64_t p, const double* A, double* R, int32_t* info) {
  return guarded([&]() -> int {
    if (count < 0 || n < 0) {
      set_error("negative count or order");
      return NPPB_E_ARG;
    }
    if (!count || !n) return NPPB_OK;
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t nn = (size_t)count * n * n;
    DevMem dA, dR, dI;
    NPPB_CUDA(dA.alloc(sizeof(double) * nn, st), "allocation");
    NPPB_CUDA(dR.alloc(sizeof(double) * nn, st), "allocation");
    NPPB_CUDA(dI.alloc(sizeof(int32_t) * count, st), "allocation");
    NPPB_CUDA(cudaMemcpyAsync(dA.as<double>(), A, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "copy");
    const int rc = matrix_power_device(count, n, p, dA.as<double>(), dR.as<double>(), dI.as<int32_t>(), st);
    if (rc != NPPB_OK) return rc;
    NPPB_CUDA(cudaMemcpyAsync(R, dR.as<double>(), sizeof(double) * nn, cudaMemcpyDeviceToHost, st), "copy");
    if (info)
      NPPB_CUDA(cudaMemcpyAsync(info, dI.as<int32_t>(), sizeof(int32_t) * count, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    return NPPB_OK;
  });
}

}  // extern "C"
