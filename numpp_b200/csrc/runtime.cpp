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

namespace {

// A side stream and two events per device for the look-ahead of the current
// thread's uniform factorisations (created on first use, kept for the thread).
struct Lookahead {
  cudaStream_t side = nullptr;   // the rest of the trailing update
  cudaStream_t panel = nullptr;  // the next panel, at the highest stream priority: its
                                 // clusters take SMs ahead of the update's CTAs
  cudaEvent_t first = nullptr, rest = nullptr, next = nullptr;
};

Lookahead* lookahead_for_device() {
  struct Holder {
    std::vector<Lookahead> per_dev;
    ~Holder() {
      for (auto& l : per_dev) {
        for (cudaStream_t t : {l.side, l.panel})
          if (t) cudaStreamDestroy(t);
        for (cudaEvent_t e : {l.first, l.rest, l.next})
          if (e) cudaEventDestroy(e);
      }
    }
  };
  thread_local Holder h;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  if ((int)h.per_dev.size() <= dev) h.per_dev.resize(dev + 1);
  Lookahead& l = h.per_dev[dev];
  if (!l.side) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithFlags(&l.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&l.panel, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.first, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.rest, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.next, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  return &l;
}

}  // namespace

// Uniform factorisation with look-ahead: after the row moves of step k, the
// strip that holds the next panel's columns is updated first; the next panel
// then runs on a high-priority stream while the other strips update on a side
// stream, and the next step's row moves (on `st`) wait for both. Every element sees the same
// operations in the same order as without look-ahead. Step 0 keeps the plain
// order: its out-of-place update reads the panel's row-move lists, which the
// next panel overwrites.
template <class T>
cudaError_t run_step_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st) {
  const int n = sa.un;
  if (n <= 32 || n > kStepMaxN || count <= 0) return cudaErrorInvalidValue;
  Lookahead* la = lookahead_for_device();
  cudaError_t e = launch_panel(sa, nullptr, count, n, 0, st);
  for (int k0 = 0; k0 < n && e == cudaSuccess; k0 += kStepNB) {
    const int64_t items = (int64_t)count * uniform_update_strips(n, sa.unrhs, sa.uinv, k0, sa.uleft);
    if (items > INT32_MAX) return cudaErrorInvalidValue;
    const bool next = k0 + kStepNB < n;
    e = launch_rows(sa, nullptr, (int)items, k0, st);
    if (e != cudaSuccess) break;
    if (!next) break;  // last panel: nothing below it
    if (k0 == 0 || !la) {
      e = launch_trailing(sa, nullptr, (int)items, n, k0, 0, st);
      if (e == cudaSuccess) e = launch_panel(sa, nullptr, count, n - k0 - kStepNB, k0 + kStepNB, st);
      continue;
    }
    e = launch_trailing(sa, nullptr, count, n, k0, 1, st);
    if (e == cudaSuccess) e = cudaEventRecord(la->first, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(la->panel, la->first, 0);
    if (e == cudaSuccess) e = launch_panel(sa, nullptr, count, n - k0 - kStepNB, k0 + kStepNB, la->panel);
    if (e == cudaSuccess) e = cudaEventRecord(la->next, la->panel);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(la->side, la->first, 0);
    if (e == cudaSuccess) e = launch_trailing(sa, nullptr, (int)items, n, k0, 2, la->side);
    if (e == cudaSuccess) e = cudaEventRecord(la->rest, la->side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, la->next, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, la->rest, 0);
  }
  if (e != cudaSuccess) return e;
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
