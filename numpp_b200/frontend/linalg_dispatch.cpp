// NumPP front-end dispatch for the B200 backend. C++20.
//
// Compiled into libnumpp (NumPP's tree, its headers) together with:
//  * numpp_b200/csrc/vtable.cpp in place of src/backend/gpu_null.cpp (the GPU
//    backend translation unit NumPP's src/CMakeLists.txt:78-101 selects), and
//  * NumPP's unmodified src/linalg/linalg.cpp and src/linalg/batched.cpp
//    built with the token renames
//      -Dsolve=ref_solve -Dinv=ref_inv -Ddet=ref_det -Dslogdet=ref_slogdet
//      -Dmatrix_power=ref_matrix_power
//    so that their definitions of these five functions (2-D and stacked)
//    become numpp::linalg::ref_* / numpp::linalg::batched::ref_*.
//
// This file then defines the public numpp::linalg::{solve, inv, det,
// slogdet, matrix_power} (linalg.hpp:29-33) and their batched:: forms
// (batched.hpp:17-21). Each serves a real square input on the device through
// the GpuVTable batched slots (2-D inputs as a stack of one, so the 2-D route
// of linalg.cpp:368-439 reaches the device too), with the reference's
// semantics: the dtype policy of la_kind (linalg.cpp:20-26: float32 in ->
// float32 out, every other real dtype -> float64, computed in double), the
// NumPy-1 vector right-hand-side rule (linalg.cpp:368-385, batched.cpp:92),
// linalg_error("Singular matrix") for solve / inv, det 0 and slogdet (0, -inf)
// for singular matrices (linalg.cpp:393-439), and last_backend() = Cuda.
// Everything else (no device, complex input, empty or non-square shapes,
// mismatched right-hand sides, a slot that declines) goes to the reference's
// own code, which raises its own errors.
#include <cstdint>
#include <limits>
#include <vector>

#include "numpp/backend/backend.hpp"
#include "numpp/backend/gpu_vtable.hpp"
#include "numpp/core/error.hpp"
#include "numpp/linalg/batched.hpp"
#include "numpp/linalg/linalg.hpp"
#include "numpp_b200.h"

namespace numpp {
namespace linalg {

// The reference's definitions, compiled under these names.
ndarray ref_solve(const ndarray& a, const ndarray& b);
ndarray ref_inv(const ndarray& a);
ndarray ref_det(const ndarray& a);
SignLogDet ref_slogdet(const ndarray& a);
ndarray ref_matrix_power(const ndarray& a, int64_t n);
namespace batched {
ndarray ref_solve(const ndarray& a, const ndarray& b);
ndarray ref_inv(const ndarray& a);
ndarray ref_det(const ndarray& a);
SignLogDet ref_slogdet(const ndarray& a);
ndarray ref_matrix_power(const ndarray& a, int64_t n);
}  // namespace batched

namespace {

// A real square stack (2-D or more) the device can take: count matrices of order n.
struct Stack {
  Shape lead;
  int64_t count = 1, n = 0;
  DType out;  // la_kind's output dtype
};

bool device_stack(const ndarray& a, DType rt, Stack& s) {
  const int64_t nd = a.ndim();
  if (nd < 2 || rt.is_complex()) return false;
  s.n = a.shape()[nd - 1];
  if (a.shape()[nd - 2] != s.n || s.n == 0) return false;
  s.lead.assign(a.shape().begin(), a.shape().end() - 2);
  s.count = 1;
  for (int64_t d : s.lead) s.count *= d;
  if (s.count == 0 || s.n > std::numeric_limits<int32_t>::max()) return false;
  s.out = rt == kFloat32 ? kFloat32 : kFloat64;
  return true;
}

ndarray f64c(const ndarray& a) { return a.astype(kFloat64).ascontiguousarray(); }

void singular_check(const std::vector<int32_t>& info) {
  for (int32_t v : info)
    if (v) throw linalg_error("Singular matrix");
}

bool dev_solve(const ndarray& a, const ndarray& b, ndarray& out) {
  const GpuVTable* vt = gpu_vtable();
  Stack s;
  if (!vt || !vt->solve_batched || !device_stack(a, result_type(a.dtype(), b.dtype()), s)) return false;
  const int64_t nd = a.ndim();
  const bool bvec = nd == 2 ? b.ndim() == 1 : b.ndim() == nd - 1;
  // b is lead + (n) or lead + (n, k); anything else is the reference's to reject
  if (b.ndim() != (bvec ? nd - 1 : nd)) return false;
  for (int64_t d = 0; d < nd - 2; ++d)
    if (b.shape()[d] != a.shape()[d]) return false;
  if (b.shape()[nd - 2] != s.n) return false;
  const int64_t k = bvec ? 1 : b.shape()[nd - 1];
  if (k <= 0) return false;
  ndarray A = f64c(a), B = f64c(b);
  ndarray X(b.shape(), kFloat64, Order::C);
  std::vector<int32_t> info(static_cast<size_t>(s.count));
  if (!vt->solve_batched(DTypeId::Float64, s.count, s.n, k, A.bytes(), B.bytes(), X.bytes(), info.data()))
    return false;
  singular_check(info);
  set_last_backend(Backend::Cuda);
  out = X.astype(s.out);
  return true;
}

bool dev_inv(const ndarray& a, ndarray& out) {
  const GpuVTable* vt = gpu_vtable();
  Stack s;
  if (!vt || !vt->inv_batched || !device_stack(a, a.dtype(), s)) return false;
  ndarray A = f64c(a);
  ndarray R(a.shape(), kFloat64, Order::C);
  std::vector<int32_t> info(static_cast<size_t>(s.count));
  if (!vt->inv_batched(DTypeId::Float64, s.count, s.n, A.bytes(), R.bytes(), info.data())) return false;
  singular_check(info);
  set_last_backend(Backend::Cuda);
  out = R.astype(s.out);
  return true;
}

bool dev_det(const ndarray& a, ndarray& out) {
  const GpuVTable* vt = gpu_vtable();
  Stack s;
  if (!vt || !vt->det_batched || !device_stack(a, a.dtype(), s)) return false;
  ndarray A = f64c(a);
  ndarray D(s.lead, kFloat64, Order::C);  // shape () for a 2-D input
  if (!vt->det_batched(DTypeId::Float64, s.count, s.n, A.bytes(), D.bytes())) return false;
  set_last_backend(Backend::Cuda);
  out = D.astype(s.out);
  return true;
}

bool dev_slogdet(const ndarray& a, SignLogDet& out) {
  const GpuVTable* vt = gpu_vtable();
  Stack s;
  if (!vt || !vt->slogdet_batched || !device_stack(a, a.dtype(), s)) return false;
  ndarray A = f64c(a);
  ndarray S(s.lead, kFloat64, Order::C), L(s.lead, kFloat64, Order::C);
  if (!vt->slogdet_batched(DTypeId::Float64, s.count, s.n, A.bytes(), S.bytes(), L.bytes())) return false;
  set_last_backend(Backend::Cuda);
  out.sign = S.astype(s.out);
  out.logabsdet = L.astype(s.out);
  return true;
}

// matrix_power (linalg.cpp:440-454): binary exponentiation on the device's
// batched GEMM, the batched inverse first for p < 0 (C ABI; the vtable has no
// slot for it).
bool dev_matrix_power(const ndarray& a, int64_t p, ndarray& out) {
  Stack s;
  if (!gpu_vtable() || !device_stack(a, a.dtype(), s)) return false;
  ndarray A = f64c(a);
  ndarray R(a.shape(), kFloat64, Order::C);
  std::vector<int32_t> info(static_cast<size_t>(s.count));
  if (nppb_matrix_power_batched(s.count, static_cast<int32_t>(s.n), p, reinterpret_cast<const double*>(A.bytes()),
                                reinterpret_cast<double*>(R.bytes()), info.data()) != NPPB_OK)
    return false;
  singular_check(info);
  set_last_backend(Backend::Cuda);
  out = R.astype(s.out);
  return true;
}

}  // namespace

ndarray solve(const ndarray& a, const ndarray& b) {
  ndarray r;
  return dev_solve(a, b, r) ? r : ref_solve(a, b);
}
ndarray inv(const ndarray& a) {
  ndarray r;
  return dev_inv(a, r) ? r : ref_inv(a);
}
ndarray det(const ndarray& a) {
  ndarray r;
  return dev_det(a, r) ? r : ref_det(a);
}
SignLogDet slogdet(const ndarray& a) {
  SignLogDet r;
  return dev_slogdet(a, r) ? r : ref_slogdet(a);
}
ndarray matrix_power(const ndarray& a, int64_t n) {
  ndarray r;
  return dev_matrix_power(a, n, r) ? r : ref_matrix_power(a, n);
}

namespace batched {
ndarray solve(const ndarray& a, const ndarray& b) {
  ndarray r;
  return dev_solve(a, b, r) ? r : ref_solve(a, b);
}
ndarray inv(const ndarray& a) {
  ndarray r;
  return dev_inv(a, r) ? r : ref_inv(a);
}
ndarray det(const ndarray& a) {
  ndarray r;
  return dev_det(a, r) ? r : ref_det(a);
}
SignLogDet slogdet(const ndarray& a) {
  SignLogDet r;
  return dev_slogdet(a, r) ? r : ref_slogdet(a);
}
ndarray matrix_power(const ndarray& a, int64_t n) {
  ndarray r;
  return dev_matrix_power(a, n, r) ? r : ref_matrix_power(a, n);
}
}  // namespace batched

}  // namespace linalg
}  // namespace numpp
