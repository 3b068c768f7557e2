// Batched execution plans: size classes, step schedules, CUDA graphs. C++20.
//
// The reference loops the 2-D routine over every matrix of a stack
// (src/linalg/batched.cpp:51-108); systems of different orders are separate
// calls there. A plan takes a whole (possibly uneven) batch at once:
//  * orders <= 32 go to the warp-per-system kernel, one launch per padded order
//    class (8 / 16 / 32);
//  * orders 33..4096 go to the step-wise path: systems sorted by order, step s
//    (columns 32s..32s+31) is one panel launch per panel-height class plus one
//    update launch over every (system, 64-column strip) still active, then one
//    back-substitution launch.
// Descriptors, work lists and workspaces are built and uploaded once; execute
// replays everything as one CUDA graph whose branches (warp classes, step
// chain) overlap on the GPU.
#include "plan.hpp"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <cerrno>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>

#include <sys/stat.h>

#include "../../include/numpp_b200.h"

namespace nppb {
namespace {

int arg_error(const std::string& m) {
  set_error(m);
  return NPPB_E_ARG;
}

#define NPPB_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return nppb::cuda_status(e_, what); \
  } while (0)

// Device allocation of a plan: plain, or stream-ordered on `ord` (no device
// synchronisation; used by plans built and dropped per batch).
cudaError_t plan_alloc(void** p, size_t bytes, cudaStream_t ord) {
  return ord ? cudaMallocAsync(p, bytes, ord) : cudaMalloc(p, bytes);
}

template <class T>
int upload(T** d, const std::vector<T>& h, cudaStream_t ord) {
  if (h.empty()) return NPPB_OK;
  NPPB_CUDA(plan_alloc(reinterpret_cast<void**>(d), sizeof(T) * h.size(), ord), "plan allocation");
  // from pageable memory: the call returns once the source has been staged
  if (ord) NPPB_CUDA(cudaMemcpyAsync(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, ord), "plan upload");
  else NPPB_CUDA(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice), "plan upload");
  return NPPB_OK;
}

// one class per k_panel configuration (CTA size, rows per thread, cluster size)
int panel_class(int m) {
  return m <= 64 ? 0 : m <= 128 ? 1 : m <= 256 ? 2 : m <= 512 ? 3 : m <= 1024 ? 4 : m <= 2048 ? 5 : 6;
}

void add_strips(std::vector<StepItem>& out, int32_t sys, int16_t kind, int c0, int c1) {
  for (int c = c0; c < c1; c += 64) {
    StepItem it{};
    it.sys = sys;
    it.kind = kind;
    it.width = (int16_t)std::min(64, c1 - c);
    it.c0 = c;
    out.push_back(it);
  }
}

}  // namespace

Plan::~Plan() {
  int prev = -1;
  cudaGetDevice(&prev);
  if (dev >= 0) cudaSetDevice(dev);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (auto s : side) cudaStreamDestroy(s);
  for (auto s : la_side) cudaStreamDestroy(s);
  for (auto e : la_first) cudaEventDestroy(e);
  for (auto e : la_rest) cudaEventDestroy(e);
  for (auto e : join) cudaEventDestroy(e);
  if (fork) cudaEventDestroy(fork);
  if (done) cudaEventDestroy(done);
  if (cap) cudaStreamDestroy(cap);
  for (void* p : {(void*)d_desc, (void*)d_order, (void*)d_lu, (void*)d_piv, (void*)d_scratch,
                  (void*)d_step_list, (void*)d_items, (void*)d_back})
    if (p) {
      if (alloc_stream) cudaFreeAsync(p, alloc_stream);
      else cudaFree(p);
    }
  for (void* p : {(void*)hA, (void*)hB, (void*)hX, (void*)hInv, (void*)hDet, (void*)hSign, (void*)hLog, (void*)hInfo})
    if (p) cudaFree(p);
  if (prev >= 0) cudaSetDevice(prev);
}

int Plan::build(int64_t cnt, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                const int64_t* b_off, const int64_t* inv_off, int fl, bool solve_only_, bool own_lu,
                const int64_t* lu_off_ext, const int64_t* piv_off_ext) {
  if ((lu_off_ext == nullptr) != (piv_off_ext == nullptr)) return arg_error("factor offsets come in pairs");
  ext_factors = lu_off_ext != nullptr;
  if (ext_factors) own_lu = false;
  if (cnt < 0 || cnt > INT32_MAX) return arg_error("bad system count");
  if (fl & ~(NPPB_WANT_LU | NPPB_WANT_SOLVE | NPPB_WANT_DET | NPPB_WANT_SLOGDET | NPPB_WANT_INV))
    return arg_error("unknown flag bits");
  if (cnt && (!n || !a_off)) return arg_error("n and a_off are required");
  const bool solve = fl & NPPB_WANT_SOLVE, want_inv = fl & NPPB_WANT_INV;
  if (solve && cnt && (!nrhs || !b_off)) return arg_error("solve needs nrhs and b_off");
  if (want_inv && cnt && !inv_off) return arg_error("inverse needs inv_off");
  const Device* d = device();
  if (!d) return NPPB_E_NODEV;
  dev = d->id;
  count = cnt;
  flags = fl;
  solve_only = solve_only_;
  if (const char* e = std::getenv("NPPB_NO_GRAPH")) use_graph = !(e[0] == '1');

  std::vector<SysDesc> desc(cnt);
  static constexpr int kWarpBounds[3] = {8, 16, 32};
  std::vector<std::vector<int32_t>> warp_members(3);
  std::vector<int32_t> step_members;
  int64_t lu = 0, piv = 0;
  for (int64_t i = 0; i < cnt; ++i) {
    const int ni = n[i];
    const int ki = solve ? nrhs[i] : 0;
    if (ni < 0 || ni > kStepMaxN) {
      set_error("system " + std::to_string(i) + ": order " + std::to_string(ni) + " outside [0, " +
                std::to_string(kStepMaxN) + "]");
      return ni < 0 ? NPPB_E_ARG : NPPB_E_RANGE;
    }
    if (ki < 0) return arg_error("negative nrhs");
    if (a_off[i] < 0 || (solve && b_off[i] < 0)) return arg_error("negative offset");
    SysDesc& s = desc[i];
    s.n = ni;
    s.nrhs = ki;
    s.idx = (int32_t)i;
    s.pad_ = -1;
    s.a_off = a_off[i];
    s.lu_off = ext_factors ? lu_off_ext[i] : own_lu ? lu : a_off[i];
    s.b_off = solve ? b_off[i] : 0;
    s.inv_off = (want_inv && inv_off[i] >= 0) ? inv_off[i] : -1;
    s.piv_off = ext_factors ? piv_off_ext[i] : piv;
    lu += (int64_t)ni * ni;
    piv += ni;
    a_elems = std::max(a_elems, a_off[i] + (int64_t)ni * ni);
    if (solve) b_elems = std::max(b_elems, b_off[i] + (int64_t)ni * ki);
    if (s.inv_off >= 0) inv_elems = std::max(inv_elems, s.inv_off + (int64_t)ni * ni);
    if (ni <= 32) {
      int c = 0;
      while (ni > kWarpBounds[c]) ++c;
      warp_members[c].push_back((int32_t)i);
    } else {
      step_members.push_back((int32_t)i);
    }
  }
  lu_elems = own_lu ? lu : 0;
  piv_elems = ext_factors ? 0 : piv;

  // warp classes: longest first
  std::vector<int32_t> order;
  order.reserve(cnt);
  for (int c = 0; c < 3; ++c) {
    auto& mb = warp_members[c];
    if (mb.empty()) continue;
    std::stable_sort(mb.begin(), mb.end(), [&](int32_t x, int32_t y) {
      if (desc[x].n != desc[y].n) return desc[x].n > desc[y].n;
      return desc[x].nrhs > desc[y].nrhs;
    });
    WarpClass wc;
    wc.bound = kWarpBounds[c];
    wc.first = (int64_t)order.size();
    wc.num = (int64_t)mb.size();
    wc.flops = wc.bytes = 0.0;
    for (int32_t i : mb) add_cost(desc[i], wc.flops, wc.bytes);
    kind_flops[kKindWarp] += wc.flops;
    warp_classes.push_back(wc);
    order.insert(order.end(), mb.begin(), mb.end());
  }

  // step-wise set: descending order, slot = rank
  std::stable_sort(step_members.begin(), step_members.end(),
                   [&](int32_t x, int32_t y) { return desc[x].n > desc[y].n; });
  for (size_t r = 0; r < step_members.size(); ++r) desc[step_members[r]].pad_ = (int32_t)r;
  nstep_sys = (int64_t)step_members.size();
  std::vector<StepItem> items, back;
  step_flops = step_bytes = 0.0;
  for (int32_t i : step_members) add_cost(desc[i], step_flops, step_bytes);
  if (nstep_sys) {
    step_nmax = desc[step_members[0]].n;
    const int G = (int)std::min<int64_t>(nchains, nstep_sys);
    // chain g takes every G-th system of the sorted list: similar order mixes
    std::vector<int32_t> list;
    list.reserve(nstep_sys);
    std::vector<int64_t> chain_first(G);
    for (int g = 0; g < G; ++g) {
      chain_first[g] = (int64_t)list.size();
      for (int64_t r = g; r < nstep_sys; r += G) list.push_back(step_members[r]);
    }
    for (int g = 0; g < G; ++g) {
      const int64_t first = chain_first[g];
      const int64_t num = (g + 1 < G ? chain_first[g + 1] : (int64_t)list.size()) - first;
      Chain ch;
      ch.nmax = desc[list[first]].n;
      if (!solve_only) {
        for (int k0 = 0; k0 < ch.nmax; k0 += kStepNB) {
          Step st;
          st.k0 = k0;
          int64_t act = 0;
          while (act < num && desc[list[first + act]].n > k0) ++act;
          // panel launches: contiguous runs with the same panel-height class
          int64_t b = 0;
          while (b < act) {
            const int pc = panel_class(desc[list[first + b]].n - k0);
            int64_t e = b;
            while (e < act && panel_class(desc[list[first + e]].n - k0) == pc) ++e;
            st.panels.push_back({first + b, e - b, desc[list[first + b]].n - k0});
            b = e;
          }
          st.item_first = (int64_t)items.size();
          st.nmax = ch.nmax;
          // the first matrix strip of every system (it holds the next panel's
          // columns) ahead of the other strips, for look-ahead
          std::vector<StepItem> rest;
          for (int64_t r = 0; r < act; ++r) {
            const int32_t si = list[first + r];
            const SysDesc& s = desc[si];
            {
              const double m = s.n - k0, kb = std::min(32.0, m);
              const double w = (s.n - k0 - kb) + (solve ? s.nrhs : 0) + (s.inv_off >= 0 ? s.n : 0);
              for (int j = 0; j < (int)kb; ++j) kind_flops[kKindPanel] += (m - j - 1) * (1.0 + 2.0 * (kb - j - 1));
              kind_flops[kKindUpdate] += kb * kb * w + 2.0 * (m - kb) * kb * w;
            }
            std::vector<StepItem> mat;
            add_strips(mat, si, kSegMatrix, k0 + kStepNB, s.n);
            if (!mat.empty()) {
              items.push_back(mat[0]);
              rest.insert(rest.end(), mat.begin() + 1, mat.end());
            }
            if (solve && s.nrhs) add_strips(rest, si, kSegRhs, 0, s.nrhs);
            if (s.inv_off >= 0) add_strips(rest, si, kSegInv, 0, s.n);
            if ((fl & NPPB_WANT_LU) && k0 > 0) add_strips(rest, si, kSegLeft, 0, k0);
          }
          st.nfirst = (int64_t)items.size() - st.item_first;
          items.insert(items.end(), rest.begin(), rest.end());
          st.item_count = (int64_t)items.size() - st.item_first;
          ch.steps.push_back(st);
        }
      }
      // substitution strips, narrow (<= 8 columns of an order above 512) and
      // the others in separate launch sequences: each strip's arithmetic
      // depends on its own width and its system's order only
      std::vector<StepItem> cb;
      for (int64_t r = 0; r < num; ++r) {
        const int32_t si = list[first + r];
        const SysDesc& s = desc[si];
        const double cols = (solve ? s.nrhs : 0) + ((s.inv_off >= 0 && !solve_only) ? s.n : 0);
        kind_flops[kKindBack] += (double)s.n * s.n * cols * (solve_only ? 2.0 : 1.0);
        if (solve && s.nrhs) add_strips(cb, si, kSegRhs, 0, s.nrhs);
        if (s.inv_off >= 0 && !solve_only) add_strips(cb, si, kSegInv, 0, s.n);
      }
      auto narrow = [&](const StepItem& it) { return it.width <= 8 && desc[it.sys].n > 512; };
      std::stable_partition(cb.begin(), cb.end(), narrow);
      ch.back_first = (int64_t)back.size();
      int narrow_nmax = 0;
      for (const StepItem& it : cb) {
        if (narrow(it)) {
          ++ch.narrow_count;
          narrow_nmax = std::max(narrow_nmax, desc[it.sys].n);
        }
        back.push_back(it);
      }
      ch.narrow_nmax = narrow_nmax;
      ch.back_count = (int64_t)back.size() - ch.back_first;
      chains.push_back(ch);
    }
    step_members.swap(list);
  }
  // look-ahead pays when panels are long (orders above 512); many small
  // systems already fill the GPU in every launch
  if (lookahead_mode < 0) lookahead = step_nmax > 512;
  else lookahead = lookahead_mode != 0;
  nback = (int64_t)back.size();

  int rc = upload(&d_desc, desc, alloc_stream);
  if (rc == NPPB_OK) rc = upload(&d_order, order, alloc_stream);
  if (rc == NPPB_OK) rc = upload(&d_step_list, step_members, alloc_stream);
  if (rc == NPPB_OK) rc = upload(&d_items, items, alloc_stream);
  if (rc == NPPB_OK) rc = upload(&d_back, back, alloc_stream);
  if (rc != NPPB_OK) return rc;
  if (nstep_sys)
    NPPB_CUDA(plan_alloc(reinterpret_cast<void**>(&d_scratch), sizeof(StepScratch) * nstep_sys, alloc_stream),
              "plan scratch");
  if (lu_elems)
    NPPB_CUDA(plan_alloc(reinterpret_cast<void**>(&d_lu), sizeof(double) * lu_elems, alloc_stream),
              "plan LU workspace");
  if (piv_elems)
    NPPB_CUDA(plan_alloc(reinterpret_cast<void**>(&d_piv), sizeof(int32_t) * piv_elems, alloc_stream),
              "plan pivot workspace");
  return NPPB_OK;
}

void Plan::add_cost(const SysDesc& s, double& fl, double& by) const {
  const double nd = s.n, kd = s.nrhs;
  if (!solve_only) {
    fl += 2.0 / 3.0 * nd * nd * nd - 0.5 * nd * nd + 5.0 / 6.0 * nd;  // getrf
    by += 8.0 * nd * nd + 20.0;                                        // A, per-system outputs
  } else {
    by += 8.0 * nd * nd;                                               // reads L and U
  }
  if (flags & NPPB_WANT_SOLVE) {
    fl += 2.0 * nd * nd * kd - nd * kd;                                // getrs
    by += 16.0 * nd * kd;
  }
  if (s.inv_off >= 0) {
    fl += 4.0 / 3.0 * nd * nd * nd;                                    // getri-equivalent
    by += 8.0 * nd * nd;
  }
}

Batch Plan::warp_batch(const Ptrs& p) const {
  Batch bt{};
  bt.A = p.A ? p.A : p.LU;
  bt.B = p.B;
  bt.X = p.X;
  bt.inv = (flags & NPPB_WANT_INV) ? p.Inv : nullptr;
  bt.det = p.Det;
  bt.sign = p.Sign;
  bt.logabs = p.Logabs;
  bt.info = p.info;
  bt.LU = p.LU;
  bt.ipiv = p.ipiv;
  bt.desc = d_desc;
  bt.flags = flags | (solve_only ? (kSolveOnly | kWantSolve) : 0) | (p.A ? 0 : kInPlace);
  return bt;
}

StepArgs Plan::step_args(const Ptrs& p) const {
  StepArgs sa{};
  sa.desc = d_desc;
  sa.scratch = d_scratch;
  sa.A = p.A;
  sa.LU = p.LU;
  sa.ipiv = p.ipiv;
  sa.B = p.B;
  sa.X = p.X;
  sa.inv = (flags & NPPB_WANT_INV) ? p.Inv : nullptr;
  sa.det = p.Det;
  sa.sign = p.Sign;
  sa.logabs = p.Logabs;
  sa.info = p.info;
  sa.solve_only = solve_only ? 1 : 0;
  return sa;
}

cudaError_t Plan::launch_warp(const Ptrs& p, int cls, cudaStream_t st) const {
  const WarpClass& c = warp_classes[cls];
  return launch_lu_warp(warp_batch(p), d_order + c.first, (int)c.num, c.bound, st);
}

cudaError_t Plan::launch_chain(const Ptrs& p, int c, cudaStream_t st) const {
  const StepArgs sa = step_args(p);
  const Chain& ch = chains[c];
  if (solve_only) {
    cudaError_t e = substitute(sa, ch, st, true);
    if (e != cudaSuccess) return e;
    return substitute(sa, ch, st, false);
  }
  // Look-ahead (from step 1 on: step 0's out-of-place update reads the row-move
  // lists the next panel overwrites): after the row moves of step s, the first
  // strip of every system is updated, the panels of step s+1 run on `st`
  // while the other strips update on the chain's side stream, and step s+1's
  // row moves wait for both. Same operations per element, in the same order.
  const bool la = c < (int)la_side.size() && la_side[c];
  auto panels = [&](const Step& s) -> cudaError_t {
    for (const auto& pr : s.panels) {
      cudaError_t e = launch_panel(sa, d_step_list + pr.first, (int)pr.num, pr.mmax, s.k0, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  if (!ch.steps.empty()) {
    cudaError_t e = panels(ch.steps[0]);
    if (e != cudaSuccess) return e;
  }
  for (size_t k = 0; k < ch.steps.size(); ++k) {
    const Step& s = ch.steps[k];
    const StepItem* items = d_items + s.item_first;
    cudaError_t e = launch_rows(sa, items, (int)s.item_count, s.k0, st);
    if (e != cudaSuccess) return e;
    const bool next = k + 1 < ch.steps.size();
    if (!la || k == 0 || !next || s.nfirst == 0) {
      e = launch_trailing(sa, items, (int)s.item_count, s.nmax, s.k0, 0, st);
      if (e == cudaSuccess && next) e = panels(ch.steps[k + 1]);
      if (e != cudaSuccess) return e;
      continue;
    }
    e = launch_trailing(sa, items, (int)s.nfirst, s.nmax, s.k0, 1, st);
    if (e == cudaSuccess) e = cudaEventRecord(la_first[c], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(la_side[c], la_first[c], 0);
    if (e == cudaSuccess)
      e = launch_trailing(sa, items + s.nfirst, (int)(s.item_count - s.nfirst), s.nmax, s.k0, 0, la_side[c]);
    if (e == cudaSuccess) e = cudaEventRecord(la_rest[c], la_side[c]);
    if (e == cudaSuccess) e = panels(ch.steps[k + 1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, la_rest[c], 0);
    if (e != cudaSuccess) return e;
  }
  return substitute(sa, ch, st, false);
}

cudaError_t Plan::ensure_lookahead() {
  if (solve_only || !lookahead) return cudaSuccess;
  while (la_side.size() < chains.size()) {
    cudaStream_t s;
    cudaEvent_t a, b;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    la_side.push_back(s);
    if ((e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming)) != cudaSuccess) return e;
    la_first.push_back(a);
    if ((e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming)) != cudaSuccess) return e;
    la_rest.push_back(b);
  }
  return cudaSuccess;
}

cudaError_t Plan::substitute(const StepArgs& sa, const Chain& ch, cudaStream_t st, bool forward) const {
  const StepItem* back = d_back + ch.back_first;
  const int nn = (int)ch.narrow_count, nw = (int)(ch.back_count - ch.narrow_count);
  cudaError_t e = cudaSuccess;
  if (nn)
    e = forward ? launch_forward(sa, back, nn, ch.narrow_nmax, 8, st) : launch_back(sa, back, nn, ch.narrow_nmax, 8, st);
  if (e == cudaSuccess && nw)
    e = forward ? launch_forward(sa, back + nn, nw, ch.nmax, 64, st) : launch_back(sa, back + nn, nw, ch.nmax, 64, st);
  return e;
}

int Plan::time_kernels(const Ptrs& p, cudaStream_t st, double* ms) const {
  for (int k = 0; k < kKinds; ++k) ms[k] = 0.0;
  cudaEvent_t e0, e1;
  NPPB_CUDA(cudaEventCreate(&e0), "event");
  NPPB_CUDA(cudaEventCreate(&e1), "event");
  cudaError_t err = cudaSuccess;
  auto timed = [&](int kind, auto&& launch) {
    if (err != cudaSuccess) return;
    err = cudaEventRecord(e0, st);
    if (err == cudaSuccess) err = launch();
    if (err == cudaSuccess) err = cudaEventRecord(e1, st);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float t = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
    ms[kind] += t;
  };
  for (int c = 0; c < (int)warp_classes.size(); ++c) timed(kKindWarp, [&] { return launch_warp(p, c, st); });
  const StepArgs sa = step_args(p);
  for (const Chain& ch : chains) {
    if (solve_only) {
      timed(kKindBack, [&] { return substitute(sa, ch, st, true); });
    } else {
      for (const Step& s : ch.steps) {
        for (const auto& pr : s.panels)
          timed(kKindPanel, [&] { return launch_panel(sa, d_step_list + pr.first, (int)pr.num, pr.mmax, s.k0, st); });
        timed(kKindUpdate, [&] { return launch_update(sa, d_items + s.item_first, (int)s.item_count, s.nmax, s.k0, st); });
      }
    }
    timed(kKindBack, [&] { return substitute(sa, ch, st, false); });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return cuda_status(err, "kernel timing");
  return NPPB_OK;
}

cudaError_t Plan::launch_steps(const Ptrs& p, cudaStream_t st) const {
  for (int c = 0; c < (int)chains.size(); ++c) {
    cudaError_t e = launch_chain(p, c, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int Plan::execute(const Ptrs& p, cudaStream_t st) {
  if (count == 0) return NPPB_OK;
  if (a_elems && !p.A && !p.LU) return arg_error("A is null");
  if ((flags & NPPB_WANT_SOLVE) && b_elems && (!p.B || !p.X)) return arg_error("solve needs B and X");
  if ((flags & NPPB_WANT_INV) && inv_elems && !p.Inv) return arg_error("inverse needs Inv");
  if ((flags & NPPB_WANT_DET) && !p.Det) return arg_error("det needs Det");
  if ((flags & NPPB_WANT_SLOGDET) && (!p.Sign || !p.Logabs)) return arg_error("slogdet needs Sign, Logabs");
  if ((lu_elems || !p.A) && !p.LU) return arg_error("plan workspace missing");
  if ((piv_elems || ext_factors) && !p.ipiv) return arg_error("plan pivot workspace missing");
  if (ext_factors && !p.LU) return arg_error("plan factor storage missing");
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != dev) return arg_error("plan used on a different device than it was created on");
  std::lock_guard<std::mutex> lk(mu);
  NPPB_CUDA(ensure_lookahead(), "look-ahead streams");
  const int nwarp = (int)warp_classes.size();
  const int branches = nwarp + (int)chains.size();
  // executions share the plan's workspace: each one starts after the previous
  if (!done) NPPB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming), "event");
  else NPPB_CUDA(cudaStreamWaitEvent(st, done, 0), "stream wait");
  if (!use_graph) {
    for (size_t c = 0; c < warp_classes.size(); ++c) NPPB_CUDA(launch_warp(p, (int)c, st), "warp class launch");
    NPPB_CUDA(launch_steps(p, st), "step launch");
    NPPB_CUDA(cudaEventRecord(done, st), "event record");
    return NPPB_OK;
  }
  if (!exec || std::memcmp(&p, &key, sizeof(Ptrs)) != 0) {
    if (!cap) {
      NPPB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream");
      NPPB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
      for (int i = 0; i < branches; ++i) {
        cudaStream_t s;
        cudaEvent_t e;
        NPPB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        NPPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        side.push_back(s);
        join.push_back(e);
      }
    }
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
    NPPB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaEventRecord(fork, cap);
    // the step chains are the long poles: start them first
    for (int b = 0; b < branches && err == cudaSuccess; ++b) {
      const int i = (b + nwarp) % branches;
      err = cudaStreamWaitEvent(side[i], fork, 0);
      if (err == cudaSuccess)
        err = (i < nwarp) ? launch_warp(p, i, side[i]) : launch_chain(p, i - nwarp, side[i]);
      if (err == cudaSuccess) err = cudaEventRecord(join[i], side[i]);
      if (err == cudaSuccess) err = cudaStreamWaitEvent(cap, join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(cap, &g);
    if (err == cudaSuccess) err = end;
    if (err != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return cuda_status(err, "graph capture");
    }
    graph = g;
    NPPB_CUDA(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    key = p;
  }
  NPPB_CUDA(cudaGraphLaunch(exec, st), "graph launch");
  NPPB_CUDA(cudaEventRecord(done, st), "event record");
  return NPPB_OK;
}

int Plan::num_kernel_groups() const { return (int)warp_classes.size() + (nstep_sys ? 1 : 0); }

int Plan::launches_per_execute() const {
  // mirrors launch_update (k_rows, plus k_update while rows remain below the
  // panel) and the windowed substitutions (a solve and, between windows, an
  // update launch per pass; k_permute first for getrs)
  auto windows = [](int nmax, int narrow, bool forward) {
    const int sb = narrow ? 128 : 256, passes = (nmax + sb - 1) / sb;
    return 2 * passes - 1 + (forward ? 1 : 0);
  };
  // wide strips: the chain's largest order bounds the passes
  int l = (int)warp_classes.size();
  for (const Chain& ch : chains) {
    const int nn = (int)ch.narrow_count, nw = (int)(ch.back_count - ch.narrow_count);
    for (int fwd = solve_only ? 1 : 0; fwd >= 0; --fwd) {
      if (nn) l += windows(ch.narrow_nmax, 1, fwd);
      if (nw) l += windows(ch.nmax, 0, fwd);
    }
    if (solve_only) continue;
    for (size_t k = 0; k < ch.steps.size(); ++k) {
      const Step& s = ch.steps[k];
      l += (int)s.panels.size() + 1 + (s.nmax - s.k0 - kStepNB > 0 ? 1 : 0);
      if (lookahead && k > 0 && k + 1 < ch.steps.size() && s.nfirst > 0) ++l;  // the look-ahead strip
    }
  }
  return l;
}

std::shared_ptr<Plan> uniform_plan(int64_t count, int32_t n, int32_t nrhs, int flags, bool solve_only,
                                   bool own_lu, int* rc) {
  using Key = std::tuple<int, int64_t, int32_t, int32_t, int, bool, bool>;
  static std::mutex mu;
  static std::list<std::pair<Key, std::shared_ptr<Plan>>> cache;
  int dev = -1;
  cudaGetDevice(&dev);
  const Key k{dev, count, n, nrhs, flags, solve_only, own_lu};
  {
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = cache.begin(); it != cache.end(); ++it) {
      if (it->first == k) {
        cache.splice(cache.begin(), cache, it);
        *rc = NPPB_OK;
        return cache.front().second;
      }
    }
  }
  std::vector<int32_t> nv(count, n), kv(count, nrhs);
  std::vector<int64_t> ao(count), bo(count), io(count);
  for (int64_t i = 0; i < count; ++i) {
    ao[i] = i * (int64_t)n * n;
    bo[i] = i * (int64_t)n * nrhs;
    io[i] = i * (int64_t)n * n;
  }
  auto p = std::make_shared<Plan>();
  p->use_graph = false;  // pointers change from call to call
  *rc = p->build(count, nv.data(), kv.data(), ao.data(), bo.data(), io.data(), flags, solve_only, own_lu);
  if (*rc != NPPB_OK) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  cache.emplace_front(k, p);
  if (cache.size() > 8) cache.pop_back();
  return p;
}

}  // namespace nppb

// ---------------------------------------------------------------------------
// C ABI
using nppb::Plan;

struct nppb_plan {
  std::unique_ptr<Plan> pp = std::make_unique<Plan>();
  // Host-buffer execution pipelined over chunks of systems: the copy of chunk
  // c+1 runs while chunk c computes (needs a packed layout: offsets ascending).
  struct Chunk {
    std::unique_ptr<Plan> plan;
    int64_t lo = 0, hi = 0;          // systems [lo, hi)
    int64_t a_lo = 0, a_hi = 0, b_lo = 0, b_hi = 0, i_lo = 0, i_hi = 0;
    cudaEvent_t in = nullptr, out = nullptr;
  };
  std::vector<int32_t> n, nrhs;
  std::vector<int64_t> a_off, b_off, inv_off;
  int flags = 0;
  bool packed = false;
  std::vector<Chunk> chunks;
  cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
  ~nppb_plan() {
    for (auto& c : chunks) {
      if (c.in) cudaEventDestroy(c.in);
      if (c.out) cudaEventDestroy(c.out);
    }
    for (cudaStream_t st : {s_in, s_comp, s_out})
      if (st) cudaStreamDestroy(st);
  }
};

namespace {

template <class F>
int guarded(F&& f) {
  try {
    nppb::clear_error();
    return f();
  } catch (const std::bad_alloc&) {
    nppb::set_error("host allocation failed");
    return NPPB_E_NOMEM;
  }
}

int ensure(void** p, size_t bytes) {
  if (*p || bytes == 0) return NPPB_OK;
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return nppb::cuda_status(e, "plan staging");
  return NPPB_OK;
}

Plan::Ptrs dev_ptrs(const Plan& pl, const double* dA, const double* dB, double* dX, double* dInv,
                    double* dDet, double* dSign, double* dLogabs, int32_t* dinfo) {
  Plan::Ptrs p{};
  p.A = dA;
  p.B = dB;
  p.X = dX;
  p.Inv = dInv;
  p.Det = dDet;
  p.Sign = dSign;
  p.Logabs = dLogabs;
  p.info = dinfo;
  p.LU = pl.d_lu;
  p.ipiv = pl.d_piv;
  return p;
}

}  // namespace

extern "C" {

int nppb_plan_create(nppb_plan** plan, int64_t count, const int32_t* n, const int32_t* nrhs,
                     const int64_t* a_off, const int64_t* b_off, const int64_t* inv_off, int flags) {
  return guarded([&]() -> int {
    if (!plan) {
      nppb::set_error("plan is null");
      return NPPB_E_ARG;
    }
    *plan = nullptr;
    auto* pl = new nppb_plan();
    if (const char* e = std::getenv("NPPB_CHAINS")) pl->pp->nchains = std::max(1, std::atoi(e));
    const int rc = pl->pp->build(count, n, nrhs, a_off, b_off, inv_off, flags & ~NPPB_WANT_LU, false, true);
    if (rc != NPPB_OK) {
      delete pl;
      return rc;
    }
    const bool solve = flags & NPPB_WANT_SOLVE, inv = flags & NPPB_WANT_INV;
    pl->flags = flags & ~NPPB_WANT_LU;
    pl->n.assign(n, n + count);
    pl->nrhs.assign(count, 0);
    pl->a_off.assign(a_off, a_off + count);
    pl->b_off.assign(count, 0);
    pl->inv_off.assign(count, -1);
    if (solve) {
      pl->nrhs.assign(nrhs, nrhs + count);
      pl->b_off.assign(b_off, b_off + count);
    }
    if (inv) pl->inv_off.assign(inv_off, inv_off + count);
    // packed: every system starts at or after the end of the previous one
    bool packed = true;
    int64_t ae = 0, be = 0, ie = 0;
    for (int64_t i = 0; i < count && packed; ++i) {
      const int64_t nn = (int64_t)n[i] * n[i];
      packed = pl->a_off[i] >= ae && pl->b_off[i] >= be;
      ae = pl->a_off[i] + nn;
      be = pl->b_off[i] + (int64_t)n[i] * pl->nrhs[i];
      if (pl->inv_off[i] >= 0) {
        packed = packed && pl->inv_off[i] >= ie;
        ie = pl->inv_off[i] + nn;
      }
    }
    pl->packed = packed;
    *plan = pl;
    return NPPB_OK;
  });
}

int nppb_plan_sizes(const nppb_plan* plan, int64_t* a_elems, int64_t* b_elems, int64_t* inv_elems) {
  if (!plan) {
    nppb::set_error("plan is null");
    return NPPB_E_ARG;
  }
  if (a_elems) *a_elems = plan->pp->a_elems;
  if (b_elems) *b_elems = plan->pp->b_elems;
  if (inv_elems) *inv_elems = plan->pp->inv_elems;
  return NPPB_OK;
}

int nppb_plan_execute(nppb_plan* plan, const double* dA, const double* dB, double* dX, double* dInv,
                      double* dDet, double* dSign, double* dLogabs, int32_t* dinfo, void* stream) {
  return guarded([&]() -> int {
    if (!plan) {
      nppb::set_error("plan is null");
      return NPPB_E_ARG;
    }
    if (plan->pp->a_elems && !dA) {
      nppb::set_error("A is null");
      return NPPB_E_ARG;
    }
    return plan->pp->execute(dev_ptrs(*plan->pp, dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo),
                           static_cast<cudaStream_t>(stream));
  });
}

namespace {

// Splits a packed plan into chunks of systems with their own sub-plans (built
// on first use).
int build_chunks(nppb_plan& P) {
  if (!P.chunks.empty()) return NPPB_OK;
  int K = 4;
  if (const char* e = std::getenv("NPPB_HOST_CHUNKS")) K = std::max(1, std::atoi(e));
  const int64_t count = P.pp->count;
  K = (int)std::min<int64_t>(K, std::max<int64_t>(1, count / 256));
  for (int c = 0; c < K; ++c) {
    nppb_plan::Chunk ch;
    ch.lo = count * c / K;
    ch.hi = count * (c + 1) / K;
    if (ch.hi <= ch.lo) continue;
    const int64_t m = ch.hi - ch.lo;
    ch.a_lo = P.a_off[ch.lo];
    ch.b_lo = P.b_off[ch.lo];
    ch.i_lo = -1;
    std::vector<int64_t> ao(m), bo(m), io(m);
    for (int64_t i = 0; i < m; ++i) {
      const int64_t s = ch.lo + i, nn = (int64_t)P.n[s] * P.n[s];
      ao[i] = P.a_off[s] - ch.a_lo;
      bo[i] = P.b_off[s] - ch.b_lo;
      ch.a_hi = P.a_off[s] + nn;
      ch.b_hi = std::max(ch.b_hi, P.b_off[s] + (int64_t)P.n[s] * P.nrhs[s]);
      if (P.inv_off[s] >= 0) {
        if (ch.i_lo < 0) ch.i_lo = P.inv_off[s];
        ch.i_hi = P.inv_off[s] + nn;
      }
    }
    if (ch.b_hi < ch.b_lo) ch.b_hi = ch.b_lo;
    if (ch.i_lo < 0) ch.i_lo = ch.i_hi = 0;
    for (int64_t i = 0; i < m; ++i) {
      const int64_t s = ch.lo + i;
      io[i] = P.inv_off[s] >= 0 ? P.inv_off[s] - ch.i_lo : -1;
    }
    ch.plan = std::make_unique<Plan>();
    const int rc = ch.plan->build(m, P.n.data() + ch.lo, P.nrhs.data() + ch.lo, ao.data(), bo.data(),
                                  io.data(), P.flags, false, true);
    if (rc != NPPB_OK) {
      P.chunks.clear();
      return rc;
    }
    NPPB_CUDA(cudaEventCreateWithFlags(&ch.in, cudaEventDisableTiming), "event");
    NPPB_CUDA(cudaEventCreateWithFlags(&ch.out, cudaEventDisableTiming), "event");
    P.chunks.push_back(std::move(ch));
  }
  for (cudaStream_t* st : {&P.s_in, &P.s_comp, &P.s_out})
    NPPB_CUDA(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "stream");
  return NPPB_OK;
}

}  // namespace

namespace {

// ---- the autotuner's on-disk cache ----------------------------------------
// One line per tuned configuration: "<key>\t<chains>\t<ms>", chains negated
// when look-ahead is on; the last line for a key wins. The key names the
// device (name, compute capability, SM count), the plan flags and the batch's
// histogram over (order class, right-hand-side class), counts bucketed by
// powers of two, so that batches of the same make share an entry.
std::mutex g_tune_mu;

std::string tune_cache_path() {
  if (const char* p = std::getenv("NPPB_AUTOTUNE_CACHE")) return p;  // empty: no disk cache
  const char* xdg = std::getenv("XDG_CACHE_HOME");
  if (xdg && *xdg) return std::string(xdg) + "/numpp_b200/autotune.txt";
  const char* home = std::getenv("HOME");
  if (home && *home) return std::string(home) + "/.cache/numpp_b200/autotune.txt";
  return "";
}

bool make_parent_dirs(const std::string& path) {
  for (size_t i = 1; i < path.size(); ++i) {
    if (path[i] != '/') continue;
    const std::string d = path.substr(0, i);
    if (mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) return false;
  }
  return true;
}

int order_class(int n) {
  static const int kBounds[] = {8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096};
  for (int b : kBounds)
    if (n <= b) return b;
  return 1 << 30;
}
int rhs_class(int k) { return k <= 0 ? 0 : k == 1 ? 1 : k <= 8 ? 8 : k <= 32 ? 32 : k <= 64 ? 64 : 65; }

std::string device_signature() {
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    return "nodev";
  }
  std::ostringstream o;
  for (const char* c = prop.name; *c; ++c) o << (*c == ' ' || *c == '\t' ? '_' : *c);
  o << "/sm" << prop.major << prop.minor << "/x" << prop.multiProcessorCount;
  return o.str();
}

std::string tuning_key(int64_t count, const int32_t* n, const int32_t* nrhs, int flags) {
  std::map<std::pair<int, int>, int64_t> h;
  for (int64_t i = 0; i < count; ++i) ++h[{order_class(n[i]), rhs_class(nrhs ? nrhs[i] : 0)}];
  std::ostringstream o;
  o << device_signature() << "|f" << flags;
  for (const auto& [cls, c] : h) {
    int lg = 0;
    while ((int64_t{2} << lg) <= c) ++lg;
    o << "|n" << cls.first << "r" << cls.second << "c" << lg;
  }
  return o.str();
}

bool cache_get(const std::string& key, int* chains, float* ms) {
  const std::string path = tune_cache_path();
  if (path.empty()) return false;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::ifstream f(path);
  if (!f) return false;
  bool found = false;
  std::string line;
  while (std::getline(f, line)) {
    const size_t t1 = line.find('\t');
    if (t1 == std::string::npos || line.compare(0, t1, key) != 0 || t1 != key.size()) continue;
    int c = 0;
    float m = 0.f;
    if (std::sscanf(line.c_str() + t1 + 1, "%d\t%f", &c, &m) == 2 && c != 0) {
      *chains = c;
      *ms = m;
      found = true;
    }
  }
  return found;
}

bool cache_put(const std::string& key, int chains, float ms) {
  const std::string path = tune_cache_path();
  if (path.empty() || key.find_first_of("\t\n") != std::string::npos) return false;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (!make_parent_dirs(path)) return false;
  std::ofstream f(path, std::ios::app);
  if (!f) return false;
  f << key << '\t' << chains << '\t' << std::setprecision(9) << ms << '\n';
  return static_cast<bool>(f);
}

}  // namespace

int nppb_autotune_key(int64_t count, const int32_t* n, const int32_t* nrhs, int flags, char* buf, int64_t len) {
  return guarded([&]() -> int {
    if (count < 0 || (count && !n) || !buf || len <= 0) {
      nppb::set_error("autotune key: bad arguments");
      return NPPB_E_ARG;
    }
    const std::string k = tuning_key(count, n, nrhs, flags);
    if ((int64_t)k.size() >= len) {
      nppb::set_error("autotune key: buffer too small");
      return NPPB_E_RANGE;
    }
    std::memcpy(buf, k.c_str(), k.size() + 1);
    return NPPB_OK;
  });
}

int nppb_autotune_cache_get(const char* key, int32_t* chains, float* ms, int32_t* found) {
  return guarded([&]() -> int {
    if (!key || !chains || !ms || !found) {
      nppb::set_error("autotune cache: bad arguments");
      return NPPB_E_ARG;
    }
    int c = 0;
    float m = 0.f;
    *found = cache_get(key, &c, &m) ? 1 : 0;
    if (*found) {
      *chains = c;
      *ms = m;
    }
    return NPPB_OK;
  });
}

int nppb_autotune_cache_put(const char* key, int32_t chains, float ms) {
  return guarded([&]() -> int {
    if (!key || chains == 0) {
      nppb::set_error("autotune cache: bad arguments");
      return NPPB_E_ARG;
    }
    if (!cache_put(key, chains, ms)) {
      nppb::set_error("autotune cache: not written (no cache path, or the file cannot be written)");
      return NPPB_E_ARG;
    }
    return NPPB_OK;
  });
}

int nppb_plan_autotune(nppb_plan* plan, const double* dA, const double* dB, double* dX, double* dInv,
                       double* dDet, double* dSign, double* dLogabs, int32_t* dinfo, void* stream,
                       int32_t* chains_out, float* ms_out) {
  return guarded([&]() -> int {
    if (!plan) {
      nppb::set_error("plan is null");
      return NPPB_E_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
      return nppb::cuda_status(cudaGetLastError(), "event");
    struct Events {
      cudaEvent_t a, b;
      ~Events() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
      }
    } ev{e0, e1};
    // candidates are built fresh; the plan's own Plan stays in place until a
    // timed candidate replaces it
    const int64_t count = (int64_t)plan->n.size();
    const int64_t nstep = plan->pp->nstep_sys;
    std::unique_ptr<Plan> best;
    float best_ms = 0.f;
    int rc = NPPB_OK;
    const std::string key = tuning_key(count, plan->n.data(), plan->nrhs.data(), plan->flags);
    int cached_chains = 0;
    float cached_ms = 0.f;
    const char* refresh = std::getenv("NPPB_AUTOTUNE_REFRESH");
    const bool hit = !(refresh && *refresh && *refresh != '0') && cache_get(key, &cached_chains, &cached_ms);
    if (hit) {  // the cached configuration, built and run once (the outputs as documented), untimed
      auto cand = std::make_unique<Plan>();
      cand->nchains = cached_chains < 0 ? -cached_chains : cached_chains;
      cand->lookahead_mode = cached_chains < 0 ? 1 : 0;
      rc = cand->build(count, plan->n.data(), plan->nrhs.data(), plan->a_off.data(), plan->b_off.data(),
                       plan->inv_off.data(), plan->flags, false, true);
      if (rc == NPPB_OK) rc = cand->execute(dev_ptrs(*cand, dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo), st);
      if (rc == NPPB_OK) {
        cudaStreamSynchronize(st);
        plan->pp = std::move(cand);
        if (chains_out) *chains_out = plan->pp->nchains * (plan->pp->lookahead ? -1 : 1);
        if (ms_out) *ms_out = cached_ms;
        return NPPB_OK;
      }
      cudaStreamSynchronize(st);
      rc = NPPB_OK;  // tune afresh
    }
    static const int kChainCounts[5] = {1, 2, 3, 4, 6};
    for (int cfg = 0; cfg < 10; ++cfg) {
      const int c = kChainCounts[cfg / 2], la = cfg % 2;
      if (c > 1 && c > nstep) break;  // more chains than step-wise systems change nothing
      auto cand = std::make_unique<Plan>();
      cand->nchains = c;
      cand->lookahead_mode = la;
      rc = cand->build(count, plan->n.data(), plan->nrhs.data(), plan->a_off.data(), plan->b_off.data(),
                       plan->inv_off.data(), plan->flags, false, true);
      if (rc != NPPB_OK) break;
      const Plan::Ptrs p = dev_ptrs(*cand, dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo);
      rc = cand->execute(p, st);  // warm-up (and graph capture)
      if (rc == NPPB_OK && cudaEventRecord(e0, st) != cudaSuccess) rc = NPPB_E_CUDA;
      for (int r = 0; r < 2 && rc == NPPB_OK; ++r) rc = cand->execute(p, st);
      float ms = 0.f;
      if (rc == NPPB_OK) {
        cudaError_t x = cudaEventRecord(e1, st);
        if (x == cudaSuccess) x = cudaEventSynchronize(e1);
        if (x == cudaSuccess) x = cudaEventElapsedTime(&ms, e0, e1);
        if (x != cudaSuccess) rc = nppb::cuda_status(x, "autotune timing");
      }
      if (rc != NPPB_OK) break;
      ms /= 2.f;
      if (!best || ms < best_ms) {
        best_ms = ms;
        best = std::move(cand);
      }
    }
    // a failed candidate may still be in flight on `st`: drain before it is freed
    cudaStreamSynchronize(st);
    if (best) plan->pp = std::move(best);
    if (rc != NPPB_OK) return rc;
    if (chains_out) *chains_out = plan->pp->nchains * (plan->pp->lookahead ? -1 : 1);
    if (ms_out) *ms_out = best_ms;
    if (best_ms > 0.f) cache_put(key, plan->pp->nchains * (plan->pp->lookahead ? -1 : 1), best_ms);
    return NPPB_OK;
  });
}

int nppb_plan_execute_host(nppb_plan* plan, const double* A, const double* B, double* X, double* Inv,
                           double* Det, double* Sign, double* Logabs, int32_t* info) {
  return guarded([&]() -> int {
    if (!plan) {
      nppb::set_error("plan is null");
      return NPPB_E_ARG;
    }
    Plan& pl = *plan->pp;
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
    if (pl.a_elems && !A) {
      nppb::set_error("A is null");
      return NPPB_E_ARG;
    }
    if ((f & NPPB_WANT_SOLVE) && pl.b_elems && (!B || !X)) {
      nppb::set_error("solve needs B and X");
      return NPPB_E_ARG;
    }
    const bool pipelined = plan->packed && pl.count >= 512 && !std::getenv("NPPB_NO_HOST_PIPELINE");
    if (pipelined) {
      rc = build_chunks(*plan);
      if (rc != NPPB_OK) return rc;
    }
    if (pipelined && plan->chunks.size() > 1) {
      auto cp = [](void* dst, const void* src, size_t bytes, cudaMemcpyKind k, cudaStream_t st) {
        return (bytes && dst && src) ? cudaMemcpyAsync(dst, src, bytes, k, st) : cudaSuccess;
      };
      const size_t D = sizeof(double);
      for (auto& ch : plan->chunks) {
        NPPB_CUDA(cp(pl.hA + ch.a_lo, A + ch.a_lo, D * (ch.a_hi - ch.a_lo), cudaMemcpyHostToDevice, plan->s_in),
                  "host to device copy");
        if (f & NPPB_WANT_SOLVE)
          NPPB_CUDA(cp(pl.hB + ch.b_lo, B + ch.b_lo, D * (ch.b_hi - ch.b_lo), cudaMemcpyHostToDevice, plan->s_in),
                    "host to device copy");
        NPPB_CUDA(cudaEventRecord(ch.in, plan->s_in), "event record");
        NPPB_CUDA(cudaStreamWaitEvent(plan->s_comp, ch.in, 0), "stream wait");
        Plan::Ptrs p = dev_ptrs(*ch.plan, pl.hA + ch.a_lo, pl.hB ? pl.hB + ch.b_lo : nullptr,
                                pl.hX ? pl.hX + ch.b_lo : nullptr, pl.hInv ? pl.hInv + ch.i_lo : nullptr,
                                pl.hDet ? pl.hDet + ch.lo : nullptr, pl.hSign ? pl.hSign + ch.lo : nullptr,
                                pl.hLog ? pl.hLog + ch.lo : nullptr, pl.hInfo + ch.lo);
        rc = ch.plan->execute(p, plan->s_comp);
        if (rc != NPPB_OK) return rc;
        NPPB_CUDA(cudaEventRecord(ch.out, plan->s_comp), "event record");
        NPPB_CUDA(cudaStreamWaitEvent(plan->s_out, ch.out, 0), "stream wait");
        const size_t m = (size_t)(ch.hi - ch.lo);
        if (f & NPPB_WANT_SOLVE)
          NPPB_CUDA(cp(X + ch.b_lo, pl.hX + ch.b_lo, D * (ch.b_hi - ch.b_lo), cudaMemcpyDeviceToHost, plan->s_out),
                    "device to host copy");
        if (f & NPPB_WANT_INV)
          NPPB_CUDA(cp(Inv + ch.i_lo, pl.hInv + ch.i_lo, D * (ch.i_hi - ch.i_lo), cudaMemcpyDeviceToHost, plan->s_out),
                    "device to host copy");
        if (f & NPPB_WANT_DET)
          NPPB_CUDA(cp(Det + ch.lo, pl.hDet + ch.lo, D * m, cudaMemcpyDeviceToHost, plan->s_out), "device to host copy");
        if (f & NPPB_WANT_SLOGDET) {
          NPPB_CUDA(cp(Sign + ch.lo, pl.hSign + ch.lo, D * m, cudaMemcpyDeviceToHost, plan->s_out), "device to host copy");
          NPPB_CUDA(cp(Logabs + ch.lo, pl.hLog + ch.lo, D * m, cudaMemcpyDeviceToHost, plan->s_out), "device to host copy");
        }
        NPPB_CUDA(cp(info + ch.lo, pl.hInfo + ch.lo, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, plan->s_out),
                  "device to host copy");
      }
      NPPB_CUDA(cudaStreamSynchronize(plan->s_out), "stream synchronize");
      NPPB_CUDA(cudaStreamSynchronize(plan->s_comp), "stream synchronize");
      return NPPB_OK;
    }
    cudaStream_t st = nppb::thread_stream();
    auto h2d = [&](void* d, const void* h, size_t bytes) {
      return bytes ? cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    auto d2h = [&](void* h, const void* d, size_t bytes) {
      return (bytes && h) ? cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
    };
    NPPB_CUDA(h2d(pl.hA, A, sizeof(double) * pl.a_elems), "host to device copy");
    if (f & NPPB_WANT_SOLVE) NPPB_CUDA(h2d(pl.hB, B, sizeof(double) * pl.b_elems), "host to device copy");
    rc = pl.execute(dev_ptrs(pl, pl.hA, pl.hB, pl.hX, pl.hInv, pl.hDet, pl.hSign, pl.hLog, pl.hInfo), st);
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

int nppb_plan_destroy(nppb_plan* plan) {
  delete plan;
  return NPPB_OK;
}

int nppb_plan_num_classes(const nppb_plan* plan) { return plan ? plan->pp->num_kernel_groups() : 0; }

int nppb_plan_num_launches(const nppb_plan* plan) { return plan ? plan->pp->launches_per_execute() : 0; }

int nppb_plan_class_info(const nppb_plan* plan, int c, int* is_warp, int* bound, int64_t* systems,
                         double* flops, double* bytes) {
  if (!plan || c < 0 || c >= plan->pp->num_kernel_groups()) {
    nppb::set_error("bad plan or class index");
    return NPPB_E_ARG;
  }
  const Plan& pl = *plan->pp;
  if (c < (int)pl.warp_classes.size()) {
    const auto& w = pl.warp_classes[c];
    if (is_warp) *is_warp = 1;
    if (bound) *bound = w.bound;
    if (systems) *systems = w.num;
    if (flops) *flops = w.flops;
    if (bytes) *bytes = w.bytes;
  } else {
    if (is_warp) *is_warp = 0;
    if (bound) *bound = pl.step_nmax;
    if (systems) *systems = pl.nstep_sys;
    if (flops) *flops = pl.step_flops;
    if (bytes) *bytes = pl.step_bytes;
  }
  return NPPB_OK;
}

int nppb_plan_time_classes(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                           double* dInv, double* dDet, double* dSign, double* dLogabs, int32_t* dinfo,
                           void* stream, int reps, float* ms_out) {
  return guarded([&]() -> int {
    if (!plan || reps < 1 || !ms_out) {
      nppb::set_error("bad plan, reps or ms_out");
      return NPPB_E_ARG;
    }
    Plan& pl = *plan->pp;
    const Plan::Ptrs p = dev_ptrs(pl, dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    NPPB_CUDA(cudaEventCreate(&e0), "event");
    NPPB_CUDA(cudaEventCreate(&e1), "event");
    int rc = NPPB_OK;
    const int groups = pl.num_kernel_groups();
    for (int c = 0; c < groups && rc == NPPB_OK; ++c) {
      cudaError_t e = cudaEventRecord(e0, st);
      for (int r = 0; r < reps && e == cudaSuccess; ++r)
        e = (c < (int)pl.warp_classes.size()) ? pl.launch_warp(p, c, st) : pl.launch_steps(p, st);
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) rc = nppb::cuda_status(e, "class timing");
      ms_out[c] = ms / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
  });
}

int nppb_plan_time_kernels(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                           double* dInv, double* dDet, double* dSign, double* dLogabs, int32_t* dinfo,
                           void* stream, double* ms_out, double* flops_out) {
  return guarded([&]() -> int {
    if (!plan || !ms_out) {
      nppb::set_error("bad plan or ms_out");
      return NPPB_E_ARG;
    }
    Plan& pl = *plan->pp;
    if (flops_out)
      for (int k = 0; k < Plan::kKinds; ++k) flops_out[k] = pl.kind_flops[k];
    return pl.time_kernels(dev_ptrs(pl, dA, dB, dX, dInv, dDet, dSign, dLogabs, dinfo),
                           static_cast<cudaStream_t>(stream), ms_out);
  });
}

int nppb_solve_grouped(int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                       const int64_t* b_off, const int64_t* inv_off, int flags, const double* A,
                       const double* B, double* X, double* Inv, double* Det, double* Sign,
                       double* Logabs, int32_t* info) {
  nppb_plan* pl = nullptr;
  int rc = nppb_plan_create(&pl, count, n, nrhs, a_off, b_off, inv_off, flags);
  if (rc != NPPB_OK) return rc;
  pl->pp->use_graph = false;  // a one-shot call gains nothing from capture
  rc = nppb_plan_execute_host(pl, A, B, X, Inv, Det, Sign, Logabs, info);
  nppb_plan_destroy(pl);
  return rc;
}

}  // extern "C"
