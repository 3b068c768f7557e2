// Host runtime shared by the C ABI entry points: device probe, per-thread
// streams and error text, stream-ordered device allocations. C++20.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "nppb_internal.hpp"
#include "nppb_step.hpp"

namespace nppb {

struct Device {
  int id = -1;
  int sms = 0;
  int cc_major = 0, cc_minor = 0;
};

// The current CUDA device if it is compute capability 10.x, else nullptr
// (message in last_error()). Probed once per device, thread-safe.
const Device* device();

void set_error(std::string msg);
const char* last_error();
void clear_error();

// Maps a CUDA failure to a status code and records the message.
int cuda_status(cudaError_t e, const char* what);

// A non-blocking stream owned by the calling thread (host-buffer entry points).
cudaStream_t thread_stream();

// Stream-ordered device allocation, freed on the same stream on destruction.
class DevMem {
 public:
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { release(); }
  cudaError_t alloc(size_t bytes, cudaStream_t st);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p_); }
  bool empty() const { return p_ == nullptr; }

 private:
  void* p_ = nullptr;
  cudaStream_t st_ = nullptr;
};

// Fills on the device (k_util.cu).
cudaError_t launch_fill_f64(double* p, int64_t n, double v, cudaStream_t st);
cudaError_t launch_fill_i32(int32_t* p, int64_t n, int32_t v, cudaStream_t st);

// Uniform batch of order n <= 32 on the warp-per-system kernel.
cudaError_t run_warp_uniform(const Batch& bt, int64_t count, int n, cudaStream_t st);

// Uniform batch of orders 33..4096 on the step-wise kernels (descriptors and
// work items derived from block indices, no plan). sa carries the pointers,
// the LU workspace, the per-system scratch and un / unrhs / uinv.
template <class T>
cudaError_t run_step_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st);
// getrs on a uniform batch from factors (LU, ipiv) a uleft=1 factorisation left: B -> X;
// prepermuted: X already holds P B (B is not read).
template <class T>
cudaError_t run_step_solve_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st, bool prepermuted = false);

// One-time kernel attribute setup (dynamic shared memory opt-in), done before
// any stream capture.
cudaError_t prepare_kernels();

}  // namespace nppb
