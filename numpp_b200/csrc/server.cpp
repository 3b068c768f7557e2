// Serving loop: continuous batching of independent solve requests with
// resident factors. C++20.
//
// No counterpart in the reference, which solves one call at a time on the
// caller's thread (src/linalg/linalg.cpp:368-385). Clients submit requests
// from any thread; one worker thread per server drains the queue in batches:
//  * a batch closes when its oldest request has waited `window_us`, when it
//    holds `max_batch` requests, or when its inputs reach the byte cap;
//  * factor requests (a new A) run as one uneven plan (every order in one
//    launch sequence); their factors are written straight into the resident
//    factor arena, kept after the batch when the request asked for it;
//  * re-solve requests (new right-hand sides on a resident factor) run as one
//    solve-only plan after the factor plan, so a re-solve may follow its
//    factor request in the same batch;
//  * requests go to one of three lanes by order (<= 128, <= 512, larger),
//    each with its own queue, worker thread and stream, so small requests
//    never queue behind a large factorisation; a re-solve takes its
//    factor's lane, after the factor request;
//  * the factor arena is carved out of the memory budget at creation; when a
//    new factor does not fit, the least recently used resident factors that
//    this batch does not read are evicted, those no queued request reads
//    first (a later re-solve on an evicted factor completes with
//    NPPB_E_RANGE); a released factor is freed once no queued request reads
//    it.
// Inputs are read and outputs written with cudaMemcpyAsync straight from / to
// the client's buffers (pinned buffers take the fast DMA path); the client
// must keep them alive until its request completes. Latency = completion time
// minus submission time on the host's steady clock.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <exception>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/numpp_b200.h"
#include "plan.hpp"
#include "runtime.hpp"

namespace nppb {
namespace {

using Clock = std::chrono::steady_clock;

// First-fit allocator over [0, cap) elements; blocks rounded to 32 elements
// (256-byte aligned factors).
class RangeAlloc {
 public:
  void reset(int64_t cap) {
    free_.clear();
    if (cap > 0) free_[0] = cap;
    used_ = 0;
  }
  int64_t alloc(int64_t size) {
    size = round(size);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= size) {
        const int64_t off = it->first, rest = it->second - size;
        free_.erase(it);
        if (rest) free_[off + size] = rest;
        used_ += size;
        return off;
      }
    }
    return -1;
  }
  void release(int64_t off, int64_t size) {
    size = round(size);
    used_ -= size;
    auto it = free_.emplace(off, size).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t used() const { return used_; }

 private:
  static int64_t round(int64_t s) { return (s + 31) / 32 * 32; }
  std::map<int64_t, int64_t> free_;
  int64_t used_ = 0;
};

struct Req {
  int64_t id = 0;
  int32_t n = 0, nrhs = 0;
  const double* A = nullptr;
  const double* B = nullptr;
  double* X = nullptr;
  int64_t factor_in = -1;  // re-solve on this resident factor; -1: factor A
  bool keep = false;
  int64_t factor_out = -1;
  Clock::time_point t_submit, t_done;
  bool done = false;
  int status = NPPB_OK;
  int32_t info = 0;
  std::string error;
};

struct Factor {
  int32_t n = 0;
  int64_t lu_off = -1, piv_off = -1;
  bool ready = false;     // factored by a completed batch
  bool resident = false;  // holds arena slots
  bool released = false;  // the client let go of it
  int pins = 0;           // read or written by the batch in flight
  int refs = 0;           // queued re-solve requests that read it
  std::list<int64_t>::iterator lru;
};

// One batch on its lane's stream: copies in, the factor plan, the re-solve
// plan, copies out.
struct Sub {
  cudaStream_t st = nullptr;
  std::vector<Req*> F, R;
  std::vector<int64_t> f_lu, f_piv, r_lu, r_piv;
  std::vector<int32_t> finfo;
  std::vector<int64_t> transient_lu, transient_piv;  // factor slots freed after the batch
  std::vector<int32_t> transient_n;
  std::vector<int64_t> pinned;
  DevMem dA, dB, dX, dI;
  std::unique_ptr<Plan> pf, pr;
  int rc = NPPB_OK;
  bool ok = true;
  std::string err;
};

}  // namespace

class Server {
 public:
  ~Server() { shutdown(); }

  int init(int64_t budget, double window_us, int max_batch) {
    if (budget <= 0 || !(window_us >= 0.0) || max_batch <= 0) {
      set_error("budget, window and max_batch must be positive");
      return NPPB_E_ARG;
    }
    const Device* d = device();
    if (!d) return NPPB_E_NODEV;
    dev_ = d->id;
    window_ = std::chrono::microseconds((int64_t)window_us);
    max_batch_ = max_batch;
    // three quarters of the budget hold resident factors (LU: 15/16 of it,
    // pivots: 1/16); the rest bounds the inputs staged per batch
    const int64_t arena_bytes = budget / 4 * 3;
    lu_cap_ = std::max<int64_t>(arena_bytes / 16 * 15 / (int64_t)sizeof(double) / 32 * 32, 32);
    piv_cap_ = std::max<int64_t>(arena_bytes / 16 / (int64_t)sizeof(int32_t) / 32 * 32, 32 * 128);
    batch_bytes_ = std::max<int64_t>(budget - arena_bytes, 64 << 20);
    cudaError_t e = cudaSuccess;
    for (Lane& ln : lanes_)
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ln.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&lu_arena_, sizeof(double) * (size_t)lu_cap_);
    if (e == cudaSuccess) e = cudaMalloc(&piv_arena_, sizeof(int32_t) * (size_t)piv_cap_);
    if (e != cudaSuccess) return cuda_status(e, "server arena");
    lu_alloc_.reset(lu_cap_);
    piv_alloc_.reset(piv_cap_);
    for (int i = 0; i < kLanes; ++i) lanes_[i].worker = std::thread([this, i] { loop(i); });
    return NPPB_OK;
  }

  int submit(int32_t n, int32_t nrhs, const double* A, const double* B, double* X, int64_t factor_in, bool keep,
             int64_t* req_id, int64_t* factor_out) {
    if (n <= 0 || nrhs <= 0 || n > kStepMaxN || !B || !X || (!A && factor_in < 0)) {
      set_error("need 1 <= n <= " + std::to_string(kStepMaxN) + ", nrhs >= 1, B, X, and A or a resident factor");
      return NPPB_E_ARG;
    }
    if ((int64_t)n * n > lu_cap_) {
      set_error("matrix larger than the factor arena");
      return NPPB_E_RANGE;
    }
    auto r = std::make_unique<Req>();
    r->n = n;
    r->nrhs = nrhs;
    r->A = A;
    r->B = B;
    r->X = X;
    r->factor_in = A ? -1 : factor_in;
    r->keep = A && keep;
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) {
      set_error("server is shutting down");
      return NPPB_E_ARG;
    }
    if (r->factor_in >= 0) {
      auto it = factors_.find(r->factor_in);
      if (it == factors_.end() || it->second.released) {
        set_error("unknown or released factor");
        return NPPB_E_ARG;
      }
      if (it->second.n != n) {
        set_error("order differs from the factor's");
        return NPPB_E_ARG;
      }
      ++it->second.refs;
    }
    r->id = next_req_++;
    if (r->keep) {
      r->factor_out = next_factor_++;
      Factor f;
      f.n = n;
      factors_[r->factor_out] = f;
    }
    if (req_id) *req_id = r->id;
    if (factor_out) *factor_out = r->factor_out;
    r->t_submit = Clock::now();
    Lane& ln = lanes_[lane_of(n)];
    ln.queue.push_back(r.get());
    reqs_[r->id] = std::move(r);
    ln.cv.notify_one();
    return NPPB_OK;
  }

  int wait(int64_t id, double timeout_s, int32_t* info, double* latency_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) {
      set_error("unknown request (or already waited for)");
      return NPPB_E_ARG;
    }
    Req* r = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(std::max(timeout_s, 0.0)));
    if (!cv_done_.wait_until(lk, deadline, [&] { return r->done; })) {
      set_error("request not finished within the timeout");
      return NPPB_DECLINED;
    }
    if (info) *info = r->info;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    const int status = r->status;
    if (status != NPPB_OK) set_error(r->error);
    reqs_.erase(it);
    return status;
  }

  int release(int64_t fid) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = factors_.find(fid);
    if (it == factors_.end()) {
      set_error("unknown factor");
      return NPPB_E_ARG;
    }
    it->second.released = true;
    maybe_free(fid);
    return NPPB_OK;
  }

  void stats(int64_t* out) {
    std::lock_guard<std::mutex> lk(mu_);
    int64_t resident = 0;
    for (auto& kv : factors_) resident += kv.second.resident ? 1 : 0;
    out[0] = completed_;
    out[1] = batches_;
    out[2] = resident;
    out[3] = lu_alloc_.used() * (int64_t)sizeof(double);
    out[4] = evictions_;
    out[5] = 0;
    for (const Lane& ln : lanes_) out[5] += (int64_t)ln.queue.size();
  }

  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    for (Lane& ln : lanes_) ln.cv.notify_all();
    for (Lane& ln : lanes_)
      if (ln.worker.joinable()) ln.worker.join();
    if (dev_ >= 0) cudaSetDevice(dev_);
    for (Lane& ln : lanes_)
      if (ln.st) cudaStreamSynchronize(ln.st);
    if (lu_arena_) cudaFree(lu_arena_);
    if (piv_arena_) cudaFree(piv_arena_);
    for (Lane& ln : lanes_) {
      if (ln.st) cudaStreamDestroy(ln.st);
      ln.st = nullptr;
    }
    lu_arena_ = nullptr;
    piv_arena_ = nullptr;
  }

 private:
  // The helpers below run with mu_ held.
  void free_slots(Factor& f) {
    if (!f.resident) return;
    lu_alloc_.release(f.lu_off, (int64_t)f.n * f.n);
    piv_alloc_.release(f.piv_off, f.n);
    f.resident = false;
    f.ready = false;
    lru_.erase(f.lru);
  }
  void maybe_free(int64_t fid) {
    auto it = factors_.find(fid);
    if (it == factors_.end()) return;
    Factor& f = it->second;
    if (f.released && f.pins == 0 && f.refs == 0) {
      free_slots(f);
      factors_.erase(it);
    }
  }
  // Arena slots for an n x n factor, evicting unpinned completed factors
  // (least recently used first) while it does not fit.
  bool place(int32_t n, int64_t& lu_off, int64_t& piv_off) {
    for (;;) {
      lu_off = lu_alloc_.alloc((int64_t)n * n);
      piv_off = lu_off >= 0 ? piv_alloc_.alloc(n) : -1;
      if (lu_off >= 0 && piv_off >= 0) return true;
      if (lu_off >= 0) lu_alloc_.release(lu_off, (int64_t)n * n);
      int64_t victim = -1;
      for (int pass = 0; pass < 2 && victim < 0; ++pass) {
        for (auto it = lru_.rbegin(); it != lru_.rend(); ++it) {
          const Factor& f = factors_[*it];
          if (f.pins == 0 && f.ready && (pass == 1 || f.refs == 0)) {
            victim = *it;
            break;
          }
        }
      }
      if (victim < 0) return false;
      free_slots(factors_[victim]);
      ++evictions_;
    }
  }
  static void fail(Req* r, int status, const std::string& msg) {
    r->status = status;
    r->error = msg;
  }

  static int lane_of(int32_t n) { return n <= 128 ? 0 : n <= 512 ? 1 : 2; }

  void loop(int li) {
    cudaSetDevice(dev_);
    Lane& ln = lanes_[li];
    for (;;) {
      std::vector<Req*> batch;
      {
        std::unique_lock<std::mutex> lk(mu_);
        ln.cv.wait(lk, [&] { return stop_ || !ln.queue.empty(); });
        if (ln.queue.empty()) return;  // stopping, nothing left
        const auto deadline = ln.queue.front()->t_submit + window_;
        ln.cv.wait_until(lk, deadline, [&] { return stop_ || (int)ln.queue.size() >= max_batch_; });
        int64_t bytes = 0;
        while (!ln.queue.empty() && (int)batch.size() < max_batch_) {
          Req* r = ln.queue.front();
          const int64_t rb = 8 * ((r->A ? (int64_t)r->n * r->n : 0) + 2 * (int64_t)r->n * r->nrhs);
          if (!batch.empty() && bytes + rb > batch_bytes_) break;
          bytes += rb;
          batch.push_back(r);
          ln.queue.pop_front();
        }
      }
      try {
        run_batch(batch, ln.st);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu_);
        for (Req* r : batch) {
          if (!r->done) {
            fail(r, NPPB_E_NOMEM, std::string("batch failed on the host: ") + e.what());
            r->t_done = Clock::now();
            r->done = true;
          }
        }
        cv_done_.notify_all();
      }
    }
  }

  void run_batch(std::vector<Req*>& batch, cudaStream_t st) {
    Sub p;
    p.st = st;
    {
      std::lock_guard<std::mutex> lk(mu_);
      // factor requests first: a re-solve in the same batch may read them
      for (Req* r : batch) {
        if (r->factor_in >= 0) continue;
        int64_t lu, pv;
        if (!place(r->n, lu, pv)) {
          fail(r, NPPB_E_NOMEM, "factor arena full (every resident factor is in use)");
          if (r->keep) factors_.erase(r->factor_out);
          continue;
        }
        p.F.push_back(r);
        p.f_lu.push_back(lu);
        p.f_piv.push_back(pv);
        if (r->keep) {
          Factor& f = factors_[r->factor_out];
          f.lu_off = lu;
          f.piv_off = pv;
          f.resident = true;
          f.pins = 1;
          lru_.push_front(r->factor_out);
          f.lru = lru_.begin();
          p.pinned.push_back(r->factor_out);
        } else {
          p.transient_lu.push_back(lu);
          p.transient_piv.push_back(pv);
          p.transient_n.push_back(r->n);
        }
      }
      for (Req* r : batch) {
        if (r->factor_in < 0) continue;
        auto it = factors_.find(r->factor_in);
        if (it != factors_.end()) --it->second.refs;
        if (it == factors_.end() || !it->second.resident) {
          fail(r, NPPB_E_RANGE, "factor not resident (evicted, failed or released)");
          if (it != factors_.end()) maybe_free(r->factor_in);
          continue;
        }
        Factor& f = it->second;
        ++f.pins;
        p.pinned.push_back(r->factor_in);
        lru_.splice(lru_.begin(), lru_, f.lru);
        p.R.push_back(r);
        p.r_lu.push_back(f.lu_off);
        p.r_piv.push_back(f.piv_off);
      }
    }
    launch(p);
    if (!p.F.empty() || !p.R.empty()) {
      if (!check(p, cudaStreamSynchronize(p.st), "batch")) p.ok = false;
      if (p.rc == NPPB_OK && !p.ok) p.rc = NPPB_E_CUDA;
    }
    const auto t_done = Clock::now();
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t i = 0; i < p.F.size(); ++i) {
        Req* r = p.F[i];
        if (p.rc != NPPB_OK) fail(r, p.rc, p.err);
        r->info = p.rc == NPPB_OK ? p.finfo[i] : 0;
        if (r->keep) {
          Factor& f = factors_[r->factor_out];
          f.ready = p.rc == NPPB_OK && r->info == 0;
          if (!f.ready) f.released = true;  // a failed or singular factorisation is not kept
        }
      }
      for (Req* r : p.R)
        if (p.rc != NPPB_OK) fail(r, p.rc, p.err);
      for (size_t i = 0; i < p.transient_lu.size(); ++i) {
        lu_alloc_.release(p.transient_lu[i], (int64_t)p.transient_n[i] * p.transient_n[i]);
        piv_alloc_.release(p.transient_piv[i], p.transient_n[i]);
      }
      for (int64_t fid : p.pinned) {
        auto it = factors_.find(fid);
        if (it != factors_.end()) {
          --it->second.pins;
          maybe_free(fid);
        }
      }
      for (Req* r : batch) {
        r->t_done = t_done;
        r->done = true;
      }
      completed_ += (int64_t)batch.size();
      ++batches_;
    }
    cv_done_.notify_all();
  }

  static bool check(Sub& p, cudaError_t e, const char* what) {
    if (e != cudaSuccess && p.err.empty()) p.err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaSuccess;
  }

  // Enqueues one part on its stream; device memory is released
  // stream-ordered, so the part is complete once its stream has drained.
  void launch(Sub& p) {
    const size_t nf = p.F.size(), nr = p.R.size();
    if (!nf && !nr) return;
    // packed layout: A of the factor requests, then B / X of all requests
    std::vector<int32_t> fn(nf), fk(nf), rn(nr), rk(nr);
    std::vector<int64_t> fa(nf), fb(nf), rb(nr), fi(nf, -1), ri(nr, -1);
    int64_t a_elems = 0, b_elems = 0;
    for (size_t i = 0; i < nf; ++i) {
      fn[i] = p.F[i]->n;
      fk[i] = p.F[i]->nrhs;
      fa[i] = a_elems;
      a_elems += (int64_t)fn[i] * fn[i];
      fb[i] = b_elems;
      b_elems += (int64_t)fn[i] * fk[i];
    }
    const int64_t r_base = b_elems;
    for (size_t i = 0; i < nr; ++i) {
      rn[i] = p.R[i]->n;
      rk[i] = p.R[i]->nrhs;
      rb[i] = b_elems - r_base;
      b_elems += (int64_t)rn[i] * rk[i];
    }
    p.finfo.assign(nf, 0);
    cudaStream_t st = p.st;
    bool& ok = p.ok;
    if (a_elems) ok = ok && check(p, p.dA.alloc(sizeof(double) * a_elems, st), "batch A");
    ok = ok && check(p, p.dB.alloc(sizeof(double) * b_elems, st), "batch B");
    ok = ok && check(p, p.dX.alloc(sizeof(double) * b_elems, st), "batch X");
    if (nf) ok = ok && check(p, p.dI.alloc(sizeof(int32_t) * nf, st), "batch info");
    for (size_t i = 0; ok && i < nf; ++i) {
      ok = check(p, cudaMemcpyAsync(p.dA.as<double>() + fa[i], p.F[i]->A, sizeof(double) * fn[i] * fn[i],
                                    cudaMemcpyHostToDevice, st), "copy A") &&
           check(p, cudaMemcpyAsync(p.dB.as<double>() + fb[i], p.F[i]->B, sizeof(double) * fn[i] * fk[i],
                                    cudaMemcpyHostToDevice, st), "copy B");
    }
    for (size_t i = 0; ok && i < nr; ++i)
      ok = check(p, cudaMemcpyAsync(p.dB.as<double>() + r_base + rb[i], p.R[i]->B, sizeof(double) * rn[i] * rk[i],
                                    cudaMemcpyHostToDevice, st), "copy B");
    int& rc = p.rc;
    if (ok && nf) {
      p.pf = std::make_unique<Plan>();
      p.pf->use_graph = false;
      p.pf->alloc_stream = st;
      rc = p.pf->build((int64_t)nf, fn.data(), fk.data(), fa.data(), fb.data(), fi.data(),
                       NPPB_WANT_SOLVE | NPPB_WANT_LU, false, false, p.f_lu.data(), p.f_piv.data());
      if (rc == NPPB_OK) {
        Plan::Ptrs q{};
        q.A = p.dA.as<double>();
        q.B = p.dB.as<double>();
        q.X = p.dX.as<double>();
        q.info = p.dI.as<int32_t>();
        q.LU = lu_arena_;
        q.ipiv = piv_arena_;
        rc = p.pf->execute(q, st);
      }
    }
    if (ok && rc == NPPB_OK && nr) {
      p.pr = std::make_unique<Plan>();
      p.pr->use_graph = false;
      p.pr->alloc_stream = st;
      // a_off is not read in solve-only mode: the factor offsets stand in
      rc = p.pr->build((int64_t)nr, rn.data(), rk.data(), p.r_lu.data(), rb.data(), ri.data(), NPPB_WANT_SOLVE,
                       true, false, p.r_lu.data(), p.r_piv.data());
      if (rc == NPPB_OK) {
        Plan::Ptrs q{};
        q.B = p.dB.as<double>() + r_base;
        q.X = p.dX.as<double>() + r_base;
        q.LU = lu_arena_;
        q.ipiv = piv_arena_;
        rc = p.pr->execute(q, st);
      }
    }
    if (rc != NPPB_OK && p.err.empty()) p.err = last_error();
    for (size_t i = 0; ok && rc == NPPB_OK && i < nf; ++i)
      ok = check(p, cudaMemcpyAsync(p.F[i]->X, p.dX.as<double>() + fb[i], sizeof(double) * fn[i] * fk[i],
                                    cudaMemcpyDeviceToHost, st), "copy X");
    for (size_t i = 0; ok && rc == NPPB_OK && i < nr; ++i)
      ok = check(p, cudaMemcpyAsync(p.R[i]->X, p.dX.as<double>() + r_base + rb[i], sizeof(double) * rn[i] * rk[i],
                                    cudaMemcpyDeviceToHost, st), "copy X");
    if (ok && rc == NPPB_OK && nf)
      ok = check(p, cudaMemcpyAsync(p.finfo.data(), p.dI.as<int32_t>(), sizeof(int32_t) * nf,
                                    cudaMemcpyDeviceToHost, st), "copy info");
    p.pf.reset();
    p.pr.reset();
    p.dA.release();
    p.dB.release();
    p.dX.release();
    p.dI.release();
  }

  int dev_ = -1;
  static constexpr int kLanes = 3;
  struct Lane {
    std::deque<Req*> queue;
    std::condition_variable cv;
    std::thread worker;
    cudaStream_t st = nullptr;
  };
  Lane lanes_[kLanes];
  double* lu_arena_ = nullptr;
  int32_t* piv_arena_ = nullptr;
  int64_t lu_cap_ = 0, piv_cap_ = 0, batch_bytes_ = 0;
  std::chrono::microseconds window_{0};
  int max_batch_ = 1;

  std::mutex mu_;
  std::condition_variable cv_done_;
  std::unordered_map<int64_t, std::unique_ptr<Req>> reqs_;
  std::unordered_map<int64_t, Factor> factors_;
  std::list<int64_t> lru_;  // most recently used first
  RangeAlloc lu_alloc_, piv_alloc_;
  int64_t next_req_ = 0, next_factor_ = 0;
  int64_t completed_ = 0, batches_ = 0, evictions_ = 0;
  bool stop_ = false;
};

}  // namespace nppb

struct nppb_server {
  nppb::Server s;
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
  } catch (const std::system_error& e) {
    nppb::set_error(std::string("thread error: ") + e.what());
    return NPPB_E_ARG;
  }
}

int null_server() {
  nppb::set_error("srv is null");
  return NPPB_E_ARG;
}
}  // namespace

extern "C" {

int nppb_server_create(nppb_server** srv, int64_t budget_bytes, double window_us, int32_t max_batch) {
  return guarded([&]() -> int {
    if (!srv) return null_server();
    *srv = nullptr;
    auto s = std::make_unique<nppb_server>();
    const int rc = s->s.init(budget_bytes, window_us, max_batch);
    if (rc != NPPB_OK) return rc;
    *srv = s.release();
    return NPPB_OK;
  });
}

int nppb_server_submit(nppb_server* srv, int32_t n, int32_t nrhs, const double* A, const double* B, double* X,
                       int64_t factor_in, int32_t keep_factor, int64_t* request_id, int64_t* factor_out) {
  return guarded([&]() -> int {
    if (!srv) return null_server();
    return srv->s.submit(n, nrhs, A, B, X, factor_in, keep_factor != 0, request_id, factor_out);
  });
}

int nppb_server_wait(nppb_server* srv, int64_t request_id, double timeout_s, int32_t* info, double* latency_s) {
  return guarded([&]() -> int {
    if (!srv) return null_server();
    return srv->s.wait(request_id, timeout_s, info, latency_s);
  });
}

int nppb_server_release_factor(nppb_server* srv, int64_t factor_id) {
  return guarded([&]() -> int {
    if (!srv) return null_server();
    return srv->s.release(factor_id);
  });
}

int nppb_server_stats(nppb_server* srv, int64_t* out6) {
  return guarded([&]() -> int {
    if (!srv || !out6) return null_server();
    srv->s.stats(out6);
    return NPPB_OK;
  });
}

int nppb_server_destroy(nppb_server* srv) {
  return guarded([&]() -> int {
    delete srv;
    return NPPB_OK;
  });
}

}  // extern "C"
