// C entry points over the reference's own CUDA backend (NumPP's
// src/backend/cuda_backend.cu, compiled unmodified from its source tree into
// oracle/_ref/refcuda/): its GpuVTable gemm slot, for the a10 head-to-head.
// Test and measurement infrastructure only.
#include <cstdint>

#include "numpp/backend/gpu_vtable.hpp"

extern "C" {

// 1 when the reference's backend sees a device (its gpu_vtable() is non-null).
int ref_cuda_available() { return numpp::gpu_vtable() != nullptr ? 1 : 0; }

// C[m x n] = A[m x k] B[k x n], row-major host buffers, through the
// reference's own call (copies in, its tiled kernel, copies out);
// dtype 0 = float64, 1 = float32. 1 on success, 0 when the slot declines.
int ref_cuda_gemm(int dtype, int64_t m, int64_t n, int64_t k, const void* A, const void* B, void* C) {
  const numpp::GpuVTable* vt = numpp::gpu_vtable();
  if (!vt || !vt->gemm) return 0;
  return vt->gemm(dtype == 1 ? numpp::DTypeId::Float32 : numpp::DTypeId::Float64, m, n, k, A, B, C) ? 1 : 0;
}
}
