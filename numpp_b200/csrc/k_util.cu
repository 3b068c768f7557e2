// Small device fills used by the host runtime.
#include "runtime.hpp"

namespace nppb {
namespace {
template <class T>
__global__ void k_fill(T* p, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}
template <class T>
cudaError_t fill(T* p, int64_t n, T v, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + 255) / 256;
  k_fill<T><<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(p, n, v);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_fill_f64(double* p, int64_t n, double v, cudaStream_t st) { return fill(p, n, v, st); }
cudaError_t launch_fill_i32(int32_t* p, int64_t n, int32_t v, cudaStream_t st) { return fill(p, n, v, st); }

}  // namespace nppb
