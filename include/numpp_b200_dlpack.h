/* numpp_b200 DLPack device handoff: the batched solve path on device-resident
 * stacks described by DLPack tensors, with no host copy.
 *
 * NumPP's interop layer exchanges host tensors only
 * (src/interop/interop.cpp:28-66 to_dlpack writes kDLCPU at :35; :68-129
 * from_dlpack adopts the buffer as host memory and never reads the device),
 * and its vendored DLPack header already
 * names kDLCUDA (include/numpp/interop/dlpack.h:9). These entry points are the
 * device side of that exchange: a framework that holds a stack on the GPU
 * (PyTorch, CuPy, JAX, another NumPP build) hands its DLTensor over and the
 * results land in DLTensors it allocated, enqueued on the caller's stream.
 *
 * Every tensor must be: kDLCUDA on the current device, C-contiguous (strides
 * NULL or the compact row-major strides; size-1 axes may carry any stride),
 * data + byte_offset aligned to its element size. Float64 for matrices and
 * results, int32 for info. A float tensor of another width, or a tensor that
 * is not on a CUDA device, is declined (NPPB_DECLINED: NumPP's CPU path keeps
 * it); a wrong shape, stride or device id is NPPB_E_ARG. Nothing is retained:
 * the caller keeps ownership of every tensor (no deleter is called).
 */
#pragma once

#include <stdint.h>

#include "numpp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The DLPack C ABI (DLTensor v0.x: data, device, ndim, dtype, shape, strides,
 * byte_offset). Define NPPB_DLPACK_EXTERNAL after including another copy of
 * dlpack.h (NumPP's include/numpp/interop/dlpack.h or dmlc's) to use that one. */
#if !defined(NPPB_DLPACK_EXTERNAL) && !defined(DLPACK_DLPACK_H_)
typedef enum { kDLCPU = 1, kDLCUDA = 2, kDLCUDAHost = 3, kDLOpenCL = 4 } DLDeviceType;
typedef struct {
  DLDeviceType device_type;
  int32_t device_id;
} DLDevice;
typedef enum { kDLInt = 0, kDLUInt = 1, kDLFloat = 2, kDLBfloat = 4, kDLComplex = 5, kDLBool = 6 } DLDataTypeCode;
typedef struct {
  uint8_t code;
  uint8_t bits;
  uint16_t lanes;
} DLDataType;
typedef struct {
  void* data;
  DLDevice device;
  int32_t ndim;
  DLDataType dtype;
  int64_t* shape;
  int64_t* strides; /* elements; NULL = C-contiguous */
  uint64_t byte_offset;
} DLTensor;
#endif

/* solve / inv / det / slogdet of a (..., n, n) stack (src/linalg/linalg.cpp:366-439,
 * stacks src/linalg/batched.cpp:75-108). `flags`: NPPB_WANT_SOLVE | _DET |
 * _SLOGDET | _INV (NPPB_WANT_LU is refused). Shapes, with lead = a.shape[:-2]:
 *   b, x    lead + (n,) (a stack of vectors: b.ndim == a.ndim - 1, NumPP's rule
 *           at batched.cpp:92) or lead + (n, k); x has b's shape (x may be b)
 *   inv     a's shape
 *   det, sign, logabs, info   lead (info int32: 0 ok, k > 0 zero pivot at k)
 * Tensors for outputs not asked for may be NULL; info may be NULL. */
int nppb_dl_linalg(int flags, const DLTensor* a, const DLTensor* b, DLTensor* x, DLTensor* inv, DLTensor* det,
                   DLTensor* sign, DLTensor* logabs, DLTensor* info, void* stream);

/* cholesky of a (..., n, n) stack (src/linalg/linalg.cpp:117-136): l gets
 * a's shape, info the lead shape (int32; > 0: not positive definite). Only
 * the lower triangle of a is read. info is required. */
int nppb_dl_cholesky(const DLTensor* a, DLTensor* l, DLTensor* info, void* stream);

/* c = a @ b over a stack: a lead + (m, k), b lead + (k, n), c lead + (m, n),
 * the same lead on all three (src/backend/backend.cpp:121-177 for one matrix). */
int nppb_dl_matmul(const DLTensor* a, const DLTensor* b, DLTensor* c, void* stream);

#ifdef __cplusplus
}
#endif
