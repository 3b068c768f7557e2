// Host runtime: device probe, errors, per-thread streams, allocations, and the
// order -> kernel choice for uniform batches. C++20.
#include "runtime.hpp"

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/numpp_b200.h"
#include "mxlu.hpp"
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

cudaError_t prepare_kernels() {
  cudaError_t e = step_prepare();
  return e == cudaSuccess ? mx_prepare() : e;
}

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
cudaError_t run_step_blocked(const StepArgsT<T>& sa0, int count, cudaStream_t st);

int blocked_min_n() {
  static const int v = [] {
    const char* s = std::getenv("NPPB_BLOCKED_MIN_N");
    return s ? std::atoi(s) : 0;  // off unless asked for: not yet faster than look-ahead at 1024..4096
  }();
  return v;
}

template <class T>
cudaError_t run_step_uniform(const StepArgsT<T>& sa, int count, cudaStream_t st) {
  const int n = sa.un;
  if (n <= 32 || n > kStepMaxN || count <= 0) return cudaErrorInvalidValue;
  if (sa.hist) return run_step_blocked(sa, count, st);
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
// Two-level factorisation (sa.hist set): outer blocks of kStepNBO columns.
// The panels of a block update only the block's columns (all rows below),
// the right-hand sides and the inverse, and carry their row moves left of the
// panel inside the block; each records its row moves and L11^-1. Then every
// strip right of the block gets the recorded row moves, U12 and the block
// rows' updates (k_block_rows), and one DMMA GEMM with K = kStepNBO updates
// everything below and right of the block: the trailing matrix is read and
// written once per block instead of once per panel.
//
// Look-ahead across blocks: the GEMM's first kStepNBO columns (the next
// block) run first; the next block's panels then go on a high-priority
// stream while the rest of the GEMM runs on a side stream, and the next
// trailing pass waits for it. Every element sees the same operations in the
// same order either way.
template <class T>
cudaError_t run_step_blocked(const StepArgsT<T>& sa0, int count, cudaStream_t st) {
  StepArgsT<T> sa = sa0;
  const int n = sa.un;
  cudaError_t e = cudaSuccess;
  if (sa.A && sa.A != sa.LU) {  // in place from the start: the trailing pass reads the factor matrix
    e = cudaMemcpyAsync(sa.LU, sa.A, sizeof(T) * (size_t)count * n * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  sa.A = nullptr;
  sa.utrail = 0;
  sa.urow_end = 0;
  // (not when factors are kept: their row moves reach the L columns the GEMM remainder reads)
  Lookahead* la = sa.uleft ? nullptr : lookahead_for_device();
  cudaStream_t cs = st;  // the chain of panels and block updates
  if (la) {
    e = cudaEventRecord(la->first, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(la->panel, la->first, 0);
    if (e != cudaSuccess) return e;
    cs = la->panel;
  }
  bool rest_pending = false;  // a GEMM remainder on the side stream
  for (int K0 = 0; K0 < n && e == cudaSuccess; K0 += kStepNBO) {
    const int bend = std::min(n, K0 + kStepNBO);
    sa.ubbeg = K0;
    sa.ubend = bend;
    for (int k0 = K0; k0 < bend && e == cudaSuccess; k0 += kStepNB) {
      sa.hslot = (k0 - K0) / kStepNB;
      e = launch_panel(sa, nullptr, count, n - k0, k0, cs);
      if (e != cudaSuccess) break;
      const int64_t items =
          (int64_t)count * blocked_update_strips(n, sa.unrhs, sa.uinv, k0, sa.uleft, K0, bend);
      if (items > INT32_MAX) return cudaErrorInvalidValue;
      if (items > 0) {
        e = launch_rows(sa, nullptr, (int)items, k0, cs);
        if (e == cudaSuccess && k0 + kStepNB < n) e = launch_trailing(sa, nullptr, (int)items, n, k0, 0, cs);
      }
    }
    if (e != cudaSuccess || bend >= n) break;
    if (rest_pending) {  // the previous block's GEMM remainder covers these columns
      e = cudaStreamWaitEvent(cs, la->rest, 0);
      rest_pending = false;
      if (e != cudaSuccess) break;
    }
    e = launch_block_rows(sa, count, K0, bend, cs);
    if (e != cudaSuccess) break;
    const int split = std::min(n, bend + kStepNBO);
    if (la && split < n) {
      e = cudaEventRecord(la->next, cs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(la->side, la->next, 0);
      if (e == cudaSuccess) e = launch_block_gemm(sa, count, K0, bend, split, n, la->side);
      if (e == cudaSuccess) e = cudaEventRecord(la->rest, la->side);
      rest_pending = true;
      if (e == cudaSuccess) e = launch_block_gemm(sa, count, K0, bend, bend, split, cs);
    } else {
      e = launch_block_gemm(sa, count, K0, bend, bend, n, cs);
    }
  }
  if (rest_pending && e == cudaSuccess) e = cudaStreamWaitEvent(cs, la->rest, 0);
  if (e != cudaSuccess) return e;
  sa.ubbeg = sa.ubend = 0;
  const int64_t back = (int64_t)count * uniform_back_strips(n, sa.unrhs, sa.uinv);
  if (back > INT32_MAX) return cudaErrorInvalidValue;
  e = launch_back(sa, nullptr, (int)back, sa.un, sa.uinv ? 64 : std::min(64, sa.unrhs), cs);
  if (e == cudaSuccess && cs != st) {
    e = cudaEventRecord(la->first, cs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, la->first, 0);
  }
  return e;
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
