// Uneven batches: size-class packing, one persistent launch per class, the
// classes replayed together as one CUDA graph. C++20.
//
// The reference loops the 2-D routine over every matrix of a stack
// (src/linalg/batched.cpp:51-108); systems of different orders are separate
// calls there. Here a plan sorts the systems into classes by order
// (<=8, <=16, <=32 on the warp kernel; <=64, <=128, <=256, <=512 on the CTA
// kernel), longest first inside a class so the persistent CTAs finish
// together, uploads the descriptors once, and on execute launches every class
// on its own stream branch of a captured graph so classes share the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/numpp_b200.h"
#include "runtime.hpp"

using namespace nppb;

struct nppb_plan {
  struct Class {
    bool warp;      // warp kernel (np) or CTA kernel (nmax)
    int bound;      // np or nmax
    int64_t first;  // slice of h_order
    int64_t num;
    int grid;       // CTA kernel only
    double flops;   // algorithmic (LAPACK counts) of the outputs asked for
    double bytes;   // algorithmic minimum traffic
  };
  int dev = -1;
  int64_t count = 0;
  int flags = 0;
  int64_t a_elems = 0, b_elems = 0, inv_elems = 0, lu_elems = 0, piv_elems = 0;
  std::vector<Class> classes;
  SysDesc* d_desc = nullptr;
  int32_t* d_order = nullptr;
  double* d_lu = nullptr;
  int32_t* d_piv = nullptr;

  std::mutex mu;
  bool use_graph = true;
  std::array<const void*, 8> key{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;
  std::vector<cudaStream_t> side;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;

  // device staging for execute_host, allocated on first use
  double *hA = nullptr, *hB = nullptr, *hX = nullptr, *hInv = nullptr, *hDet = nullptr,
         *hSign = nullptr, *hLog = nullptr;
  int32_t* hInfo = nullptr;

  ~nppb_plan();
};

nppb_plan::~nppb_plan() {
  int prev = -1;
  cudaGetDevice(&prev);
  if (dev >= 0) cudaSetDevice(dev);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (auto s : side) cudaStreamDestroy(s);
  for (auto e : join) cudaEventDestroy(e);
  if (fork) cudaEventDestroy(fork);
  if (cap) cudaStreamDestroy(cap);
  for (void* p : {(void*)d_desc, (void*)d_order, (void*)d_lu, (void*)d_piv, (void*)hA, (void*)hB,
                  (void*)hX, (void*)hInv, (void*)hDet, (void*)hSign, (void*)hLog, (void*)hInfo})
    if (p) cudaFree(p);
  if (prev >= 0) cudaSetDevice(prev);
}

namespace {

// p: A, B, X, Inv, Det, Sign, Logabs, info
Batch plan_batch(const nppb_plan& pl, const void* const* p) {
  Batch bt{};
  bt.A = (const double*)p[0];
  bt.B = (const double*)p[1];
  bt.X = (double*)p[2];
  bt.inv = (pl.flags & NPPB_WANT_INV) ? (double*)p[3] : nullptr;
  bt.det = (double*)p[4];
  bt.sign = (double*)p[5];
  bt.logabs = (double*)p[6];
  bt.info = (int32_t*)p[7];
  bt.LU = pl.d_lu;
  bt.ipiv = pl.d_piv;
  bt.desc = pl.d_desc;
  bt.flags = pl.flags & ~NPPB_WANT_LU;
  return bt;
}

cudaError_t launch_class(const nppb_plan& pl, const nppb_plan::Class& c, const Batch& bt,
                         cudaStream_t st) {
  const int32_t* order = pl.d_order + c.first;
  if (c.warp) return launch_lu_warp(bt, order, (int)c.num, c.bound, st);
  return launch_lu_cta(bt, order, (int)c.num, c.bound, c.grid, st);
}

#define NPPB_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)

int arg_error(const std::string& m) {
  set_error(m);
  return NPPB_E_ARG;
}

int build(nppb_plan& pl, int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
          const int64_t* b_off, const int64_t* inv_off, int flags) {
  if (count < 0 || count > INT32_MAX) return arg_error("bad system count");
  if (flags & ~(NPPB_WANT_LU | NPPB_WANT_SOLVE | NPPB_WANT_DET | NPPB_WANT_SLOGDET | NPPB_WANT_INV))
    return arg_error("unknown flag bits");
  if (count && (!n || !a_off)) return arg_error("n and a_off are required");
  const bool solve = flags & NPPB_WANT_SOLVE, inv = flags & NPPB_WANT_INV;
  if (solve && count && (!nrhs || !b_off)) return arg_error("solve needs nrhs and b_off");
  if (inv && count && !inv_off) return arg_error("inverse needs inv_off");
  const Device* d = device();
  if (!d) return NPPB_E_NODEV;
  pl.dev = d->id;
  pl.count = count;
  pl.flags = flags;
  if (const char* e = std::getenv("NPPB_NO_GRAPH")) pl.use_graph = !(e[0] == '1');

  std::vector<SysDesc> desc(count);
  // class index: 0..2 warp (8/16/32), 3..6 CTA (64/128/256/512)
  static constexpr int kBounds[7] = {8, 16, 32, 64, 128, 256, 512};
  std::vector<std::vector<int32_t>> members(7);
  int64_t lu = 0, piv = 0;
  for (int64_t i = 0; i < count; ++i) {
    const int ni = n[i];
    const int ki = solve ? nrhs[i] : 0;
    if (ni < 0 || ni > kCtaMaxN) {
      set_error("system " + std::to_string(i) + ": order " + std::to_string(ni) + " outside [0, " +
                std::to_string(kCtaMaxN) + "]");
      return ni < 0 ? NPPB_E_ARG : NPPB_E_RANGE;
    }
    if (ki < 0) return arg_error("negative nrhs");
    if (a_off[i] < 0 || (solve && b_off[i] < 0)) return arg_error("negative offset");
    SysDesc& s = desc[i];
    s.n = ni;
    s.nrhs = ki;
    s.idx = (int32_t)i;
    s.pad_ = 0;
    s.a_off = a_off[i];
    s.lu_off = lu;
    s.b_off = solve ? b_off[i] : 0;
    s.inv_off = (inv && inv_off[i] >= 0) ? inv_off[i] : -1;
    s.piv_off = piv;
    lu += (int64_t)ni * ni;
    piv += ni;
    pl.a_elems = std::max(pl.a_elems, a_off[i] + (int64_t)ni * ni);
    if (solve) pl.b_elems = std::max(pl.b_elems, b_off[i] + (int64_t)ni * ki);
    if (s.inv_off >= 0) pl.inv_elems = std::max(pl.inv_elems, s.inv_off + (int64_t)ni * ni);
    int c = 0;
    while (ni > kBounds[c]) ++c;
    members[c].push_back((int32_t)i);
  }
  pl.lu_elems = lu;
  pl.piv_elems = piv;
  std::vector<int32_t> order;
  order.reserve(count);
  for (int c = 0; c < 7; ++c) {
    auto& m = members[c];
    if (m.empty()) continue;
    std::stable_sort(m.begin(), m.end(), [&](int32_t x, int32_t y) {
      if (desc[x].n != desc[y].n) return desc[x].n > desc[y].n;
      return desc[x].nrhs > desc[y].nrhs;
    });
    nppb_plan::Class cl;
    cl.flops = 0.0;
    cl.bytes = 0.0;
    for (int32_t i : m) {
      const double nd = desc[i].n, kd = desc[i].nrhs;
      cl.flops += 2.0 / 3.0 * nd * nd * nd - 0.5 * nd * nd + 5.0 / 6.0 * nd;  // getrf
      cl.bytes += 8.0 * nd * nd + 4.0 * 5;                                       // A, per-system outputs
      if (solve) {
        cl.flops += 2.0 * nd * nd * kd - nd * kd;                                // getrs
        cl.bytes += 16.0 * nd * kd;                                              // B in, X out
      }
      if (desc[i].inv_off >= 0) {
        cl.flops += 4.0 / 3.0 * nd * nd * nd;                                    // getri-equivalent
        cl.bytes += 8.0 * nd * nd;
      }
    }
    cl.warp = c < 3;
    cl.bound = kBounds[c];
    cl.first = (int64_t)order.size();
    cl.num = (int64_t)m.size();
    cl.grid = cl.warp ? 0 : lu_cta_grid((int)cl.num, cl.bound, d->sms);
    pl.classes.push_back(cl);
    order.insert(order.end(), m.begin(), m.end());
  }
  if (count) {
    NPPB_CUDA(cudaMalloc(&pl.d_desc, sizeof(SysDesc) * count), "plan descriptors");
    NPPB_CUDA(cudaMalloc(&pl.d_order, sizeof(int32_t) * count), "plan order");
    NPPB_CUDA(cudaMemcpy(pl.d_desc, desc.data(), sizeof(SysDesc) * count, cudaMemcpyHostToDevice),
              "plan upload");
    NPPB_CUDA(cudaMemcpy(pl.d_order, order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice),
              "plan upload");
  }
  if (lu) NPPB_CUDA(cudaMalloc(&pl.d_lu, sizeof(double) * lu), "plan LU workspace");
  if (piv) NPPB_CUDA(cudaMalloc(&pl.d_piv, sizeof(int32_t) * piv), "plan pivot workspace");
  return NPPB_OK;
}

int execute(nppb_plan& pl, const void* const* ptrs, cudaStream_t st) {
  if (pl.classes.empty()) return NPPB_OK;
  if (pl.a_elems && !ptrs[0]) return arg_error("A is null");
  if ((pl.flags & NPPB_WANT_SOLVE) && pl.b_elems && (!ptrs[1] || !ptrs[2]))
    return arg_error("solve needs B and X");
  if ((pl.flags & NPPB_WANT_INV) && pl.inv_elems && !ptrs[3]) return arg_error("inverse needs Inv");
  if ((pl.flags & NPPB_WANT_DET) && !ptrs[4]) return arg_error("det needs Det");
  if ((pl.flags & NPPB_WANT_SLOGDET) && (!ptrs[5] || !ptrs[6])) return arg_error("slogdet needs Sign, Logabs");
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != pl.dev) return arg_error("plan used on a different device than it was created on");
  const Batch bt = plan_batch(pl, ptrs);
  std::lock_guard<std::mutex> lk(pl.mu);
  if (!pl.use_graph) {
    for (const auto& c : pl.classes) NPPB_CUDA(launch_class(pl, c, bt, st), "class launch");
    return NPPB_OK;
  }
  std::array<const void*, 8> key;
  std::copy(ptrs, ptrs + 8, key.begin());
  if (!pl.exec || key != pl.key) {
    if (!pl.cap) {
      NPPB_CUDA(cudaStreamCreateWithFlags(&pl.cap, cudaStreamNonBlocking), "stream");
      NPPB_CUDA(cudaEventCreateWithFlags(&pl.fork, cudaEventDisableTiming), "event");
      for (size_t i = 0; i < pl.classes.size(); ++i) {
        cudaStream_t s;
        cudaEvent_t e;
        NPPB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        NPPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        pl.side.push_back(s);
        pl.join.push_back(e);
      }
    }
    if (pl.exec) { cudaGraphExecDestroy(pl.exec); pl.exec = nullptr; }
    if (pl.graph) { cudaGraphDestroy(pl.graph); pl.graph = nullptr; }
    NPPB_CUDA(cudaStreamBeginCapture(pl.cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaEventRecord(pl.fork, pl.cap);
    for (size_t i = 0; i < pl.classes.size() && err == cudaSuccess; ++i) {
      err = cudaStreamWaitEvent(pl.side[i], pl.fork, 0);
      if (err == cudaSuccess) err = launch_class(pl, pl.classes[i], bt, pl.side[i]);
      if (err == cudaSuccess) err = cudaEventRecord(pl.join[i], pl.side[i]);
      if (err == cudaSuccess) err = cudaStreamWaitEvent(pl.cap, pl.join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(pl.cap, &g);
    if (err == cudaSuccess) err = end;
    if (err != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return cuda_status(err, "graph capture");
    }
    pl.graph = g;
    NPPB_CUDA(cudaGraphInstantiate(&pl.exec, pl.graph, 0), "graph instantiate");
    pl.key = key;
  }
  NPPB_CUDA(cudaGraphLaunch(pl.exec, st), "graph launch");
  return NPPB_OK;
}

template <class F>
int guarded(F&& f) {
  try {
    clear_error();
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return NPPB_E_NOMEM;
  }
}

int ensure(void** p, size_t bytes) {
  if (*p || bytes == 0) return NPPB_OK;
  NPPB_CUDA(cudaMalloc(p, bytes), "plan staging");
  return NPPB_OK;
}

}  // namespace

extern "C" {

int nppb_plan_create(nppb_plan** plan, int64_t count, const int32_t* n, const int32_t* nrhs,
                     const int64_t* a_off, const int64_t* b_off, const int64_t* inv_off, int flags) {
  return guarded([&]() -> int {
    if (!plan) return arg_error("plan is null");
    *plan = nullptr;
    auto* pl = new nppb_plan();
    const int rc = build(*pl, count, n, nrhs, a_off, b_off, inv_off, flags);
    if (rc != NPPB_OK) {
      delete pl;
      return rc;
    }
    *plan = pl;
    return NPPB_OK;
  });
}

int nppb_plan_sizes(const nppb_plan* plan, int64_t* a_elems, int64_t* b_elems, int64_t* inv_elems) {
  if (!plan) return arg_error("plan is null");
  if (a_elems) *a_elems = plan->a_elems;
  if (b_elems) *b_elems = plan->b_elems;
  if (inv_elems) *inv_elems = plan->inv_elems;
  return NPPB_OK;
}

int nppb_plan_execute(nppb_plan* plan, const double* dA, const double* dB, double* dX, double* dInv,
                      double* dDet, double* dSign, double* dLogabs, int32_t* dinfo, void* stream) {
  return guarded([&]() -> int {
    if (!plan) return arg_error("plan is null");
    const void* ptrs[8] = {dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo};
    return execute(*plan, ptrs, static_cast<cudaStream_t>(stream));
  });
}

int nppb_plan_execute_host(nppb_plan* plan, const double* A, const double* B, double* X, double* Inv,
                           double* Det, double* Sign, double* Logabs, int32_t* info) {
  return guarded([&]() -> int {
    if (!plan) return arg_error("plan is null");
    nppb_plan& pl = *plan;
    const int f = pl.flags;
    const size_t c = (size_t)pl.count;
    int rc = ensure((void**)&pl.hA, sizeof(double) * pl.a_elems);
    if (rc == NPPB_OK && (f & NPPB_WANT_SOLVE)) rc = ensure((void**)&pl.hB, sizeof(double) * pl.b_elems);
    if (rc == NPPB_OK && (f & NPPB_WANT_SOLVE)) rc = ensure((void**)&pl.hX, sizeof(double) * pl.b_elems);
    if (rc == NPPB_OK && (f & NPPB_WANT_INV)) rc = ensure((void**)&pl.hInv, sizeof(double) * pl.inv_elems);
    if (rc == NPPB_OK && (f & NPPB_WANT_DET)) rc = ensure((void**)&pl.hDet, sizeof(double) * c);
    if (rc == NPPB_OK && (f & NPPB_WANT_SLOGDET)) rc = ensure((void**)&pl.hSign, sizeof(double) * c);
    if (rc == NPPB_OK && (f & NPPB_WANT_SLOGDET)) rc = ensure((void**)&pl.hLog, sizeof(double) * c);
    if (rc == NPPB_OK) rc = ensure((void**)&pl.hInfo, sizeof(int32_t) * c);
    if (rc != NPPB_OK) return rc;
    cudaStream_t st = thread_stream();
    auto h2d = [&](void* d, const void* h, size_t bytes) {
      return bytes ? cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    auto d2h = [&](void* h, const void* d, size_t bytes) {
      return (bytes && h) ? cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
    };
    if (pl.a_elems && !A) return arg_error("A is null");
    NPPB_CUDA(h2d(pl.hA, A, sizeof(double) * pl.a_elems), "host to device copy");
    if (f & NPPB_WANT_SOLVE) {
      if (pl.b_elems && (!B || !X)) return arg_error("solve needs B and X");
      NPPB_CUDA(h2d(pl.hB, B, sizeof(double) * pl.b_elems), "host to device copy");
    }
    const void* ptrs[8] = {pl.hA, pl.hB, pl.hX, pl.hInv, pl.hDet, pl.hSign, pl.hLog, pl.hInfo};
    rc = execute(pl, ptrs, st);
    if (rc != NPPB_OK) return rc;
    if (f & NPPB_WANT_SOLVE) NPPB_CUDA(d2h(X, pl.hX, sizeof(double) * pl.b_elems), "device to host copy");
    if (f & NPPB_WANT_INV) NPPB_CUDA(d2h(Inv, pl.hInv, sizeof(double) * pl.inv_elems), "device to host copy");
    if (f & NPPB_WANT_DET) NPPB_CUDA(d2h(Det, pl.hDet, sizeof(double) * c), "device to host copy");
    if (f & NPPB_WANT_SLOGDET) {
      NPPB_CUDA(d2h(Sign, pl.hSign, sizeof(double) * c), "device to host copy");
      NPPB_CUDA(d2h(Logabs, pl.hLog, sizeof(double) * c), "device to host copy");
    }
    NPPB_CUDA(d2h(info, pl.hInfo, sizeof(int32_t) * c), "device to host copy");
    NPPB_CUDA(cudaStreamSynchronize(st), "stream synchronize");
    return NPPB_OK;
  });
}

int nppb_plan_num_classes(const nppb_plan* plan) {
  return plan ? (int)plan->classes.size() : 0;
}

int nppb_plan_class_info(const nppb_plan* plan, int c, int* is_warp, int* bound, int64_t* systems,
                         double* flops, double* bytes) {
  if (!plan || c < 0 || c >= (int)plan->classes.size()) return arg_error("bad plan or class index");
  const auto& cl = plan->classes[c];
  if (is_warp) *is_warp = cl.warp ? 1 : 0;
  if (bound) *bound = cl.bound;
  if (systems) *systems = cl.num;
  if (flops) *flops = cl.flops;
  if (bytes) *bytes = cl.bytes;
  return NPPB_OK;
}

int nppb_plan_time_classes(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                           double* dInv, double* dDet, double* dSign, double* dLogabs,
                           int32_t* dinfo, void* stream, int reps, float* ms_out) {
  return guarded([&]() -> int {
    if (!plan || reps < 1 || !ms_out) return arg_error("bad plan, reps or ms_out");
    const void* ptrs[8] = {dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo};
    const Batch bt = plan_batch(*plan, ptrs);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    NPPB_CUDA(cudaEventCreate(&e0), "event");
    NPPB_CUDA(cudaEventCreate(&e1), "event");
    int rc = NPPB_OK;
    for (size_t c = 0; c < plan->classes.size() && rc == NPPB_OK; ++c) {
      cudaError_t e = cudaEventRecord(e0, st);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = launch_class(*plan, plan->classes[c], bt, st);
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) rc = cuda_status(e, "class timing");
      ms_out[c] = ms / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
  });
}

int nppb_plan_destroy(nppb_plan* plan) {
  delete plan;
  return NPPB_OK;
}

int nppb_solve_grouped(int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                       const int64_t* b_off, const int64_t* inv_off, int flags, const double* A,
                       const double* B, double* X, double* Inv, double* Det, double* Sign,
                       double* Logabs, int32_t* info) {
  nppb_plan* pl = nullptr;
  int rc = nppb_plan_create(&pl, count, n, nrhs, a_off, b_off, inv_off, flags);
  if (rc != NPPB_OK) return rc;
  pl->use_graph = false;  // a one-shot call gains nothing from capture
  rc = nppb_plan_execute_host(pl, A, B, X, Inv, Det, Sign, Logabs, info);
  nppb_plan_destroy(pl);
  return rc;
}

}  // extern "C"
