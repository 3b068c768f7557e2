// Host runtime: device probe, errors, per-thread streams, allocations, and the
// order -> kernel choice for uniform batches. C++20.
#include "runtime.hpp"

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/numpp_b200.h"
#include "nppb_step.hpp"

namespace nppb {
namespace {

thread_local std::string t_error;

struct DeviceTable {
  std::mutex mu;
  std::vector<Device> devs;      // by ordinal; id == -1 until probed
  std::vector<int> probed;       // 0 unprobed, 1 ok, -1 not sm_100
};
DeviceTable& table() {
  static DeviceTable t;
  return t;
}

}  // namespace

void set_error(std::string msg) { t_error = std::move(msg); }
const char* last_error() { return t_error.c_str(); }
void clear_error() { t_error.clear(); }

int cuda_status(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? NPPB_E_NOMEM : NPPB_E_CUDA;
}

const Device* device() {
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) {
    cudaGetLastError();
    set_error("no CUDA device");
    return nullptr;
  }
  DeviceTable& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  if ((int)t.devs.size() <= cur) {
    t.devs.resize(cur + 1);
    t.probed.resize(cur + 1, 0);
  }
  if (t.probed[cur] == 0) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, cur) != cudaSuccess) {
      cudaGetLastError();
      t.probed[cur] = -1;
    } else if (p.major != 10) {
      t.probed[cur] = -1;
    } else {
      Device& d = t.devs[cur];
      d.id = cur;
      d.sms = p.multiProcessorCount;
      d.cc_major = p.major;
      d.cc_minor = p.minor;
      t.probed[cur] = prepare_kernels() == cudaSuccess ? 1 : -1;
      // workspaces come from this process's default stream-ordered pool: keep
      // freed blocks in the pool instead of returning them at every synchronise
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, cur) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      cudaGetLastError();
    }
  }
  if (t.probed[cur] != 1) {
    set_error("device is not an sm_100 (B200-class) GPU or kernel setup failed");
    return nullptr;
  }
  return &t.devs[cur];
}

cudaStream_t thread_stream() {
  struct Holder {
    cudaStream_t s = nullptr;
    int dev = -1;
    ~Holder() {
      if (s) cudaStreamDestroy(s);
    }
  };
  thread_local Holder h;
  int cur = 0;
  cudaGetDevice(&cur);
  if (!h.s || h.dev != cur) {
    if (h.s) cudaStreamDestroy(h.s);
    cudaStreamCreateWithFlags(&h.s, cudaStreamNonBlocking);
    h.dev = cur;
  }
  return h.s;
}

cudaError_t DevMem::alloc(size_t bytes, cudaStream_t st) {
  release();
  st_ = st;
  if (bytes == 0) return cudaSuccess;
  return cudaMallocAsync(&p_, bytes, st);
}

void DevMem::release() {
  if (p_) cudaFreeAsync(p_, st_);
  p_ = nullptr;
}

cudaError_t prepare_kernels() { return step_prepare(); }

template <class T>
cudaError_t run_step_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st) {
  const int n = sa.un;
  if (n <= 32 || n > kStepMaxN || count <= 0) return cudaErrorInvalidValue;
  for (int k0 = 0; k0 < n; k0 += kStepNB) {
    cudaError_t e = launch_panel(sa, nullptr, count, n - k0, k0, st);
    if (e != cudaSuccess) return e;
    const int64_t items = (int64_t)count * uniform_update_strips(n, sa.unrhs, sa.uinv, k0, sa.uleft);
    if (items > INT32_MAX) return cudaErrorInvalidValue;
    e = launch_update(sa, nullptr, (int)items, n, k0, st);
    if (e != cudaSuccess) return e;
  }
  const int64_t back = (int64_t)count * uniform_back_strips(n, sa.unrhs, sa.uinv);
  if (back > INT32_MAX) return cudaErrorInvalidValue;
  return launch_back(sa, nullptr, (int)back, sa.un, sa.uinv ? 64 : std::min(64, sa.unrhs), st);
}
template cudaError_t run_step_uniform<double>(const StepArgsT<double>&, int, cudaStream_t);
template cudaError_t run_step_uniform<float>(const StepArgsT<float>&, int, cudaStream_t);

template <class T>
cudaError_t run_step_solve_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st, bool prepermuted) {
  const int64_t items = (int64_t)count * uniform_back_strips(sa.un, sa.unrhs, 0);
  if (sa.un <= 32 || items > INT32_MAX || count <= 0) return cudaErrorInvalidValue;
  StepArgsT<T> s2 = sa;
  s2.solve_only = 1;
  s2.uinv = 0;
  cudaError_t e = launch_forward(s2, nullptr, (int)items, sa.un, std::min(64, sa.unrhs), st, !prepermuted);
  if (e != cudaSuccess) return e;
  return launch_back(s2, nullptr, (int)items, s2.un, std::min(64, s2.unrhs), st);
}
template cudaError_t run_step_solve_uniform<double>(const StepArgsT<double>&, int, cudaStream_t, bool);
template cudaError_t run_step_solve_uniform<float>(const StepArgsT<float>&, int, cudaStream_t, bool);

cudaError_t run_warp_uniform(const Batch& bt, int64_t count, int n, cudaStream_t st) {
  if (n > 32) return cudaErrorInvalidValue;
  return launch_lu_warp(bt, nullptr, static_cast<int>(count), n <= 8 ? 8 : (n <= 16 ? 16 : 32), st);
}

}  // namespace nppb
