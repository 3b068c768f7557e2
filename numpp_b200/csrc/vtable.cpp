// The B200 backend translation unit for NumPP's weak GPU vtable: compiled in
// place of src/backend/gpu_null.cpp / cuda_backend.cu (selected by NumPP's
// src/CMakeLists.txt:78-101), it defines numpp::gpu_vtable() over the C ABI.
// Null when no compute-capability 10.x device is present, like the CUDA
// backend's probe (src/backend/cuda_backend.cu:120-123,320), so NumPP's CPU
// path is then unchanged. C++20.
#include "../../include/numpp/backend/gpu_vtable.hpp"

#include <limits>

#include "../../include/numpp_b200.h"

namespace numpp {
namespace {

bool f64(DTypeId dt) { return dt == DTypeId::Float64; }

bool fits(int64_t count, int64_t n, int64_t nrhs) {
  return count >= 0 && n >= 0 && nrhs >= 0 && count <= std::numeric_limits<int32_t>::max() &&
         n <= nppb_max_order() && nrhs <= std::numeric_limits<int32_t>::max();
}

bool ew_binary(int op, DTypeId dt, int64_t n, const void* a, const void* b, void* out) {
  return nppb_elementwise_binary(op, (int)dt, n, a, b, out) == NPPB_OK;
}
bool ew_unary(int op, DTypeId dt, int64_t n, const void* a, void* out) {
  return nppb_elementwise_unary(op, (int)dt, n, a, out) == NPPB_OK;
}
bool reduce_slot(int op, DTypeId dt, int64_t n, const void* a, void* out) {
  return nppb_reduce(op, (int)dt, n, a, out) == NPPB_OK;
}
bool gemm_slot(DTypeId dt, int64_t m, int64_t n, int64_t k, const void* A, const void* B, void* C) {
  return nppb_gemm((int)dt, m, n, k, A, B, C) == NPPB_OK;
}
bool getrf_slot(DTypeId dt, int64_t count, int64_t n, void* A, int32_t* ipiv, int32_t* info) {
  return f64(dt) && fits(count, n, 0) &&
         nppb_getrf_batched(count, (int32_t)n, (double*)A, ipiv, info) == NPPB_OK;
}
bool getrs_slot(DTypeId dt, int64_t count, int64_t n, int64_t nrhs, const void* LU,
                const int32_t* ipiv, void* B) {
  return f64(dt) && fits(count, n, nrhs) &&
         nppb_getrs_batched(count, (int32_t)n, (int32_t)nrhs, (const double*)LU, ipiv, (double*)B) ==
             NPPB_OK;
}
bool solve_slot(DTypeId dt, int64_t count, int64_t n, int64_t nrhs, const void* A, const void* B,
                void* X, int32_t* info) {
  return f64(dt) && fits(count, n, nrhs) &&
         nppb_solve_batched(count, (int32_t)n, (int32_t)nrhs, (const double*)A, (const double*)B,
                            (double*)X, info) == NPPB_OK;
}
bool inv_slot(DTypeId dt, int64_t count, int64_t n, const void* A, void* Ainv, int32_t* info) {
  return f64(dt) && fits(count, n, 0) &&
         nppb_inv_batched(count, (int32_t)n, (const double*)A, (double*)Ainv, info) == NPPB_OK;
}
bool det_slot(DTypeId dt, int64_t count, int64_t n, const void* A, void* det) {
  return f64(dt) && fits(count, n, 0) &&
         nppb_det_batched(count, (int32_t)n, (const double*)A, (double*)det) == NPPB_OK;
}
bool slogdet_slot(DTypeId dt, int64_t count, int64_t n, const void* A, void* sign, void* logabs) {
  return f64(dt) && fits(count, n, 0) &&
         nppb_slogdet_batched(count, (int32_t)n, (const double*)A, (double*)sign, (double*)logabs) ==
             NPPB_OK;
}

const GpuVTable g_table{
    "b200",      &ew_binary,  &ew_unary, &reduce_slot, &gemm_slot,   nullptr,
    nullptr,     nullptr,     &getrf_slot, &getrs_slot, &solve_slot, &inv_slot,
    &det_slot,   &slogdet_slot,
};

}  // namespace

const GpuVTable* gpu_vtable() { return nppb_device_available() ? &g_table : nullptr; }

}  // namespace numpp

// C-level handle on the table for hosts that cannot name the C++ symbol.
extern "C" const void* nppb_gpu_vtable(void) { return numpp::gpu_vtable(); }
