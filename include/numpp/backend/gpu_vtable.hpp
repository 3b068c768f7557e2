#pragma once
// NumPP's GPU weak vtable, extended with batched dense linear-algebra slots.
//
// Drop-in for NumPP's include/numpp/backend/gpu_vtable.hpp:10-56. The op enums
// and the first eight members (name .. separable_corr1d) keep the reference's
// names, signatures and order, so existing aggregate initialisers of the table
// stay valid; the batched slots are appended after them and value-initialise to
// null in any table that does not set them. Slot conventions are the
// reference's: contiguous native-dtype host buffers, the caller allocates every
// output, `false` means "not served, use the portable CPU kernel".
//
// Inside NumPP's tree DTypeId comes from numpp/core/dtype.hpp; built on its own
// (this repository) the same enumeration is declared here with the reference's
// values (dtype.hpp:16-22), which the slots rely on (Float32 = 10, Float64 = 11).

#include <cstdint>

#if __has_include("numpp/core/dtype.hpp")
#include "numpp/core/dtype.hpp"
#else
namespace numpp {
enum class DTypeId : uint8_t {
  Bool = 0,
  Int8, Int16, Int32, Int64,
  UInt8, UInt16, UInt32, UInt64,
  Float16, Float32, Float64,
  Complex64, Complex128,
  String, Bytes, Datetime64, Timedelta64, Struct,
};
}  // namespace numpp
#endif

namespace numpp {

enum GpuBinOp { kGAdd = 0, kGSub, kGMul, kGDiv };
enum GpuUnOp { kGNeg = 0, kGSqrt, kGExp };
enum GpuRedOp { kGSum = 0, kGProd };

struct GpuVTable {
  const char* name;
  bool (*elementwise_binary)(int op, DTypeId dt, int64_t n, const void* a, const void* b, void* out);
  bool (*elementwise_unary)(int op, DTypeId dt, int64_t n, const void* a, void* out);
  bool (*reduce)(int op, DTypeId dt, int64_t n, const void* a, void* out);
  // Row-major C[m,n] = A[m,k] * B[k,n] (float32 / float64).
  bool (*gemm)(DTypeId dt, int64_t m, int64_t n, int64_t k, const void* A, const void* B, void* C);
  bool (*csr_spmv)(DTypeId dt, int64_t rows, int64_t cols, int64_t nnz, const int64_t* indptr,
                   const int64_t* indices, const void* data, const void* x, void* y);
  bool (*pairwise_sqdist)(DTypeId dt, int64_t m, int64_t n, int64_t dim, const void* A,
                          const void* B, void* D);
  bool (*separable_corr1d)(DTypeId dt, int64_t lines, int64_t len, const void* in,
                           const void* weights, int64_t klen, int64_t origin, int mode,
                           double cval, void* out);

  // ---- appended: batched dense linear algebra on (count, n, n) stacks ----
  // float64 only (NumPP computes linalg in double: linalg.cpp:20-26); any other
  // dtype returns false. info[i] = k+1 for the first exactly-zero pivot k of
  // matrix i, else 0 (the front-end raises linalg_error("Singular matrix") for
  // solve / inv, and returns det 0 / slogdet (0, -inf), linalg.cpp:393-439).
  // ipiv: LAPACK-style 0-based swap list per matrix.
  bool (*getrf_batched)(DTypeId dt, int64_t count, int64_t n, void* A, int32_t* ipiv,
                        int32_t* info);
  bool (*getrs_batched)(DTypeId dt, int64_t count, int64_t n, int64_t nrhs, const void* LU,
                        const int32_t* ipiv, void* B);
  bool (*solve_batched)(DTypeId dt, int64_t count, int64_t n, int64_t nrhs, const void* A,
                        const void* B, void* X, int32_t* info);
  bool (*inv_batched)(DTypeId dt, int64_t count, int64_t n, const void* A, void* Ainv,
                      int32_t* info);
  bool (*det_batched)(DTypeId dt, int64_t count, int64_t n, const void* A, void* det);
  bool (*slogdet_batched)(DTypeId dt, int64_t count, int64_t n, const void* A, void* sign,
                          void* logabsdet);
};

// Null unless a GPU backend translation unit provides a real one (and, for the
// B200 backend, a compute-capability 10.x device is present).
const GpuVTable* gpu_vtable();

}  // namespace numpp
