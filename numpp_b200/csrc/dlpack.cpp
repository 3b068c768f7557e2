// DLPack device handoff: the batched entry points on DLTensor descriptors of
// device-resident stacks (no host copy). C++20.
//
// NumPP's interop layer (src/interop/interop.cpp:28-129) exchanges host
// tensors only; this is the device side of the same exchange. Each tensor is
// checked (device, dtype, shape, compact strides, alignment), reduced to a
// pointer, and the call forwarded to nppb_d_linalg_batched /
// nppb_d_gemm_batched on the caller's stream.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/numpp_b200.h"
#include "../../include/numpp_b200_dlpack.h"
#include "runtime.hpp"

using namespace nppb;

namespace {

struct View {
  char* ptr = nullptr;
  std::vector<int64_t> shape;
  int64_t size = 1;
};

enum class Kind { F64, I32 };

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

// Checks one tensor and fills v. NPPB_DECLINED for a host tensor or another
// float width (the CPU path keeps those), NPPB_E_ARG for everything else.
int view_of(const DLTensor* t, Kind kind, const char* name, View& v) {
  const std::string nm(name);
  if (!t) return fail(NPPB_E_ARG, nm + ": null tensor");
  if (t->device.device_type != kDLCUDA)
    return fail(NPPB_DECLINED, nm + ": not a CUDA tensor (the host entry points serve host memory)");
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return fail(NPPB_E_CUDA, "cudaGetDevice failed");
  if (t->device.device_id != cur)
    return fail(NPPB_E_ARG, nm + ": on device " + std::to_string(t->device.device_id) + ", current device is " +
                                std::to_string(cur));
  const DLDataType d = t->dtype;
  if (d.lanes != 1) return fail(NPPB_E_ARG, nm + ": vector lanes are not supported");
  int64_t esize = 0;
  if (kind == Kind::F64) {
    if (d.code == kDLFloat && d.bits != 64)
      return fail(NPPB_DECLINED, nm + ": float" + std::to_string(d.bits) + " is served by the CPU path");
    if (d.code != kDLFloat) return fail(NPPB_DECLINED, nm + ": only float64 is served by the batched path");
    esize = 8;
  } else {
    if (d.code != kDLInt || d.bits != 32) return fail(NPPB_E_ARG, nm + ": info must be int32");
    esize = 4;
  }
  if (t->ndim < 0) return fail(NPPB_E_ARG, nm + ": negative ndim");
  if (t->ndim > 0 && !t->shape) return fail(NPPB_E_ARG, nm + ": null shape");
  v.shape.assign(t->shape, t->shape + t->ndim);
  v.size = 1;
  for (int64_t s : v.shape) {
    if (s < 0) return fail(NPPB_E_ARG, nm + ": negative extent");
    v.size *= s;
  }
  if (t->strides && v.size > 0) {
    int64_t want = 1;
    for (int i = t->ndim - 1; i >= 0; --i) {
      if (v.shape[i] != 1 && t->strides[i] != want)
        return fail(NPPB_E_ARG, nm + ": not C-contiguous (make it contiguous first)");
      want *= v.shape[i];
    }
  }
  v.ptr = static_cast<char*>(t->data) + t->byte_offset;
  if (v.size > 0 && !t->data) return fail(NPPB_E_ARG, nm + ": null data");
  if (reinterpret_cast<uintptr_t>(v.ptr) % static_cast<uintptr_t>(esize))
    return fail(NPPB_E_ARG, nm + ": data + byte_offset is not aligned to its element size");
  return NPPB_OK;
}

bool same(const std::vector<int64_t>& a, const std::vector<int64_t>& b) { return a == b; }

std::string shape_str(const std::vector<int64_t>& s) {
  std::string r = "(";
  for (size_t i = 0; i < s.size(); ++i) r += (i ? ", " : "") + std::to_string(s[i]);
  return r + (s.size() == 1 ? ",)" : ")");
}

#define NPPB_RC(expr)               \
  do {                              \
    int rc_ = (expr);               \
    if (rc_ != NPPB_OK) return rc_; \
  } while (0)

int dl_linalg(int flags, const DLTensor* a, const DLTensor* b, DLTensor* x, DLTensor* inv, DLTensor* det,
              DLTensor* sign, DLTensor* logabs, DLTensor* info, cudaStream_t st) {
  if (flags & NPPB_WANT_LU) return fail(NPPB_E_ARG, "NPPB_WANT_LU: factors are kept through nppb_d_linalg_batched");
  if (flags & ~(NPPB_WANT_SOLVE | NPPB_WANT_DET | NPPB_WANT_SLOGDET | NPPB_WANT_INV))
    return fail(NPPB_E_ARG, "unknown flag bits");
  View A;
  NPPB_RC(view_of(a, Kind::F64, "a", A));
  const int nd = static_cast<int>(A.shape.size());
  if (nd < 2 || A.shape[nd - 1] != A.shape[nd - 2])
    return fail(NPPB_E_ARG, "a: last 2 dimensions of the array must be square, got " + shape_str(A.shape));
  const std::vector<int64_t> lead(A.shape.begin(), A.shape.end() - 2);
  const int64_t n = A.shape[nd - 1];
  int64_t count = 1;
  for (int64_t s : lead) count *= s;
  if (n > INT32_MAX) return fail(NPPB_E_RANGE, "order above 2^31-1");

  double *pB = nullptr, *pX = nullptr, *pInv = nullptr, *pDet = nullptr, *pSign = nullptr, *pLog = nullptr;
  int32_t* pInfo = nullptr;
  int64_t nrhs = 0;
  if (flags & NPPB_WANT_SOLVE) {
    View B, X;
    NPPB_RC(view_of(b, Kind::F64, "b", B));
    NPPB_RC(view_of(x, Kind::F64, "x", X));
    std::vector<int64_t> vec_shape(A.shape.begin(), A.shape.end() - 1);
    if (B.shape.size() == static_cast<size_t>(nd - 1)) {  // stack of vectors (NumPy-1 rule)
      if (!same(B.shape, vec_shape))
        return fail(NPPB_E_ARG, "b: expected " + shape_str(vec_shape) + ", got " + shape_str(B.shape));
      nrhs = 1;
    } else if (B.shape.size() == static_cast<size_t>(nd)) {
      std::vector<int64_t> want = vec_shape;
      want.push_back(B.shape[nd - 1]);
      if (!same(B.shape, want))
        return fail(NPPB_E_ARG, "b: expected " + shape_str(vec_shape) + " + (k,), got " + shape_str(B.shape));
      nrhs = B.shape[nd - 1];
    } else {
      return fail(NPPB_E_ARG, "b: ndim must be a.ndim - 1 or a.ndim");
    }
    if (!same(X.shape, B.shape)) return fail(NPPB_E_ARG, "x: must have b's shape " + shape_str(B.shape));
    if (nrhs > INT32_MAX) return fail(NPPB_E_RANGE, "nrhs above 2^31-1");
    pB = reinterpret_cast<double*>(B.ptr);
    pX = reinterpret_cast<double*>(X.ptr);
  }
  if (flags & NPPB_WANT_INV) {
    View I;
    NPPB_RC(view_of(inv, Kind::F64, "inv", I));
    if (!same(I.shape, A.shape)) return fail(NPPB_E_ARG, "inv: must have a's shape " + shape_str(A.shape));
    pInv = reinterpret_cast<double*>(I.ptr);
  }
  auto per_system = [&](DLTensor* t, Kind k, const char* name, char** out) -> int {
    View V;
    NPPB_RC(view_of(t, k, name, V));
    if (!same(V.shape, lead)) return fail(NPPB_E_ARG, std::string(name) + ": must have shape " + shape_str(lead));
    *out = V.ptr;
    return NPPB_OK;
  };
  char* p = nullptr;
  if (flags & NPPB_WANT_DET) {
    NPPB_RC(per_system(det, Kind::F64, "det", &p));
    pDet = reinterpret_cast<double*>(p);
  }
  if (flags & NPPB_WANT_SLOGDET) {
    NPPB_RC(per_system(sign, Kind::F64, "sign", &p));
    pSign = reinterpret_cast<double*>(p);
    NPPB_RC(per_system(logabs, Kind::F64, "logabs", &p));
    pLog = reinterpret_cast<double*>(p);
  }
  if (info) {
    NPPB_RC(per_system(info, Kind::I32, "info", &p));
    pInfo = reinterpret_cast<int32_t*>(p);
  }
  return nppb_d_linalg_batched(count, static_cast<int32_t>(n), static_cast<int32_t>(nrhs), flags,
                               reinterpret_cast<const double*>(A.ptr), pB, pX, pInv, pDet, pSign, pLog, nullptr,
                               nullptr, pInfo, st);
}

int dl_matmul(const DLTensor* a, const DLTensor* b, DLTensor* c, cudaStream_t st) {
  View A, B, Cv;
  NPPB_RC(view_of(a, Kind::F64, "a", A));
  NPPB_RC(view_of(b, Kind::F64, "b", B));
  NPPB_RC(view_of(c, Kind::F64, "c", Cv));
  const size_t nd = A.shape.size();
  if (nd < 2 || B.shape.size() != nd || Cv.shape.size() != nd)
    return fail(NPPB_E_ARG, "matmul: a, b and c need the same ndim >= 2");
  const std::vector<int64_t> lead(A.shape.begin(), A.shape.end() - 2);
  const int64_t m = A.shape[nd - 2], k = A.shape[nd - 1], n = B.shape[nd - 1];
  std::vector<int64_t> wb = lead, wc = lead;
  wb.push_back(k);
  wb.push_back(n);
  wc.push_back(m);
  wc.push_back(n);
  if (!same(B.shape, wb)) return fail(NPPB_E_ARG, "matmul: shape mismatch, b must be " + shape_str(wb));
  if (!same(Cv.shape, wc)) return fail(NPPB_E_ARG, "matmul: c must be " + shape_str(wc));
  int64_t batch = 1;
  for (int64_t s : lead) batch *= s;
  return nppb_d_gemm_batched(batch, m, n, k, reinterpret_cast<const double*>(A.ptr),
                             reinterpret_cast<const double*>(B.ptr), reinterpret_cast<double*>(Cv.ptr), st);
}

int dl_cholesky(const DLTensor* a, DLTensor* l, DLTensor* info, cudaStream_t st) {
  View A, Lv, I;
  NPPB_RC(view_of(a, Kind::F64, "a", A));
  const int nd = static_cast<int>(A.shape.size());
  if (nd < 2 || A.shape[nd - 1] != A.shape[nd - 2])
    return fail(NPPB_E_ARG, "a: last 2 dimensions of the array must be square, got " + shape_str(A.shape));
  NPPB_RC(view_of(l, Kind::F64, "l", Lv));
  if (!same(Lv.shape, A.shape)) return fail(NPPB_E_ARG, "l: must have a's shape " + shape_str(A.shape));
  NPPB_RC(view_of(info, Kind::I32, "info", I));
  const std::vector<int64_t> lead(A.shape.begin(), A.shape.end() - 2);
  if (!same(I.shape, lead)) return fail(NPPB_E_ARG, "info: must have shape " + shape_str(lead));
  const int64_t n = A.shape[nd - 1];
  int64_t count = 1;
  for (int64_t s : lead) count *= s;
  if (n > INT32_MAX) return fail(NPPB_E_RANGE, "order above 2^31-1");
  return nppb_d_cholesky_batched(count, static_cast<int32_t>(n), reinterpret_cast<const double*>(A.ptr),
                                 reinterpret_cast<double*>(Lv.ptr), reinterpret_cast<int32_t*>(I.ptr), st);
}

}  // namespace

extern "C" {

int nppb_dl_cholesky(const DLTensor* a, DLTensor* l, DLTensor* info, void* stream) {
  try {
    clear_error();
    return dl_cholesky(a, l, info, static_cast<cudaStream_t>(stream));
  } catch (const std::exception& e) {
    set_error(e.what());
    return NPPB_E_NOMEM;
  }
}


int nppb_dl_linalg(int flags, const DLTensor* a, const DLTensor* b, DLTensor* x, DLTensor* inv, DLTensor* det,
                   DLTensor* sign, DLTensor* logabs, DLTensor* info, void* stream) {
  try {
    clear_error();
    return dl_linalg(flags, a, b, x, inv, det, sign, logabs, info, static_cast<cudaStream_t>(stream));
  } catch (const std::exception& e) {
    set_error(e.what());
    return NPPB_E_NOMEM;
  }
}

int nppb_dl_matmul(const DLTensor* a, const DLTensor* b, DLTensor* c, void* stream) {
  try {
    clear_error();
    return dl_matmul(a, b, c, static_cast<cudaStream_t>(stream));
  } catch (const std::exception& e) {
    set_error(e.what());
    return NPPB_E_NOMEM;
  }
}

}  // extern "C"
