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
//  * the factor arena is carved out of the memory budget at creation; when a
//    new factor does not fit, the least recently used resident factors that
//    this batch does not read are evicted (a later re-solve on an evicted
//    factor completes with NPPB_E_RANGE).
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
  std::list<int64_t>::iterator lru;
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
    cudaError_t e = cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&lu_arena_, sizeof(double) * (size_t)lu_cap_);
    if (e == cudaSuccess) e = cudaMalloc(&piv_arena_, sizeof(int32_t) * (size_t)piv_cap_);
    if (e != cudaSuccess) return cuda_status(e, "server arena");
    lu_alloc_.reset(lu_cap_);
    piv_alloc_.reset(piv_cap_);
    worker_ = std::thread([this] { loop(); });
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
    queue_.push_back(r.get());
    reqs_[r->id] = std::move(r);
    cv_work_.notify_one();
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
    out[5] = (int64_t)queue_.size();
  }

  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    if (worker_.joinable()) worker_.join();
    if (dev_ >= 0) cudaSetDevice(dev_);
    if (st_) cudaStreamSynchronize(st_);
    if (lu_arena_) cudaFree(lu_arena_);
    if (piv_arena_) cudaFree(piv_arena_);
    if (st_) cudaStreamDestroy(st_);
    lu_arena_ = nullptr;
    piv_arena_ = nullptr;
    st_ = nullptr;
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
    if (f.released && f.pins == 0) {
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
      for (auto it = lru_.rbegin(); it != lru_.rend(); ++it) {
        const Factor& f = factors_[*it];
        if (f.pins == 0 && f.ready) {
          victim = *it;
          break;
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

  void loop() {
    cudaSetDevice(dev_);
    for (;;) {
      std::vector<Req*> batch;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] { return stop_ || !queue_.empty(); });
        if (queue_.empty()) return;  // stopping, nothing left
        const auto deadline = queue_.front()->t_submit + window_;
        cv_work_.wait_until(lk, deadline, [&] { return stop_ || (int)queue_.size() >= max_batch_; });
        int64_t bytes = 0;
        while (!queue_.empty() && (int)batch.size() < max_batch_) {
          Req* r = queue_.front();
          const int64_t rb = 8 * ((r->A ? (int64_t)r->n * r->n : 0) + 2 * (int64_t)r->n * r->nrhs);
          if (!batch.empty() && bytes + rb > batch_bytes_) break;
          bytes += rb;
          batch.push_back(r);
          queue_.pop_front();
        }
      }
      try {
        run_batch(batch);
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

  void run_batch(std::vector<Req*>& batch) {
    std::vector<Req*> F, R;
    std::vector<int64_t> f_lu, f_piv, r_lu, r_piv;
    std::vector<int64_t> transient_lu, transient_piv;  // freed after the batch
    std::vector<int32_t> transient_n;
    std::vector<int64_t> pinned;
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
        F.push_back(r);
        f_lu.push_back(lu);
        f_piv.push_back(pv);
        if (r->keep) {
          Factor& f = factors_[r->factor_out];
          f.lu_off = lu;
          f.piv_off = pv;
          f.resident = true;
          f.pins = 1;
          lru_.push_front(r->factor_out);
          f.lru = lru_.begin();
          pinned.push_back(r->factor_out);
        } else {
          transient_lu.push_back(lu);
          transient_piv.push_back(pv);
          transient_n.push_back(r->n);
        }
      }
      for (Req* r : batch) {
        if (r->factor_in < 0) continue;
        auto it = factors_.find(r->factor_in);
        if (it == factors_.end() || !it->second.resident) {
          fail(r, NPPB_E_RANGE, "factor not resident (evicted, failed or released)");
          continue;
        }
        Factor& f = it->second;
        ++f.pins;
        pinned.push_back(r->factor_in);
        lru_.splice(lru_.begin(), lru_, f.lru);
        R.push_back(r);
        r_lu.push_back(f.lu_off);
        r_piv.push_back(f.piv_off);
      }
    }

    std::string err;
    int rc = NPPB_OK;
    std::vector<int32_t> finfo(F.size(), 0);
    if (!F.empty() || !R.empty()) rc = execute(F, R, f_lu, f_piv, r_lu, r_piv, finfo, err);

    const auto t_done = Clock::now();
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t i = 0; i < F.size(); ++i) {
        Req* r = F[i];
        if (rc != NPPB_OK) fail(r, rc, err);
        r->info = finfo[i];
        if (r->keep) {
          Factor& f = factors_[r->factor_out];
          f.ready = rc == NPPB_OK && finfo[i] == 0;
          if (!f.ready) f.released = true;  // a failed or singular factorisation is not kept
        }
      }
      for (Req* r : R)
        if (rc != NPPB_OK) fail(r, rc, err);
      for (size_t i = 0; i < transient_lu.size(); ++i) {
        lu_alloc_.release(transient_lu[i], (int64_t)transient_n[i] * transient_n[i]);
        piv_alloc_.release(transient_piv[i], transient_n[i]);
      }
      for (int64_t fid : pinned) {
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

  // One batch on the server stream: copies in, the factor plan, the re-solve
  // plan, copies out; returns after the stream has drained.
  int execute(const std::vector<Req*>& F, const std::vector<Req*>& R, const std::vector<int64_t>& f_lu,
              const std::vector<int64_t>& f_piv, const std::vector<int64_t>& r_lu, const std::vector<int64_t>& r_piv,
              std::vector<int32_t>& finfo, std::string& err) {
    // packed layout: A of the factor requests, then B / X of all requests
    const size_t nf = F.size(), nr = R.size();
    std::vector<int32_t> fn(nf), fk(nf), rn(nr), rk(nr);
    std::vector<int64_t> fa(nf), fb(nf), rb(nr), fi(nf, -1), ri(nr, -1);
    int64_t a_elems = 0, b_elems = 0;
    for (size_t i = 0; i < nf; ++i) {
      fn[i] = F[i]->n;
      fk[i] = F[i]->nrhs;
      fa[i] = a_elems;
      a_elems += (int64_t)fn[i] * fn[i];
      fb[i] = b_elems;
      b_elems += (int64_t)fn[i] * fk[i];
    }
    const int64_t r_base = b_elems;
    for (size_t i = 0; i < nr; ++i) {
      rn[i] = R[i]->n;
      rk[i] = R[i]->nrhs;
      rb[i] = b_elems - r_base;
      b_elems += (int64_t)rn[i] * rk[i];
    }
    DevMem dA, dB, dX, dI;
    auto cuda = [&](cudaError_t e, const char* what) {
      if (e != cudaSuccess && err.empty()) err = std::string(what) + ": " + cudaGetErrorString(e);
      return e == cudaSuccess;
    };
    bool ok = true;
    if (a_elems) ok = ok && cuda(dA.alloc(sizeof(double) * a_elems, st_), "batch A");
    ok = ok && cuda(dB.alloc(sizeof(double) * b_elems, st_), "batch B");
    ok = ok && cuda(dX.alloc(sizeof(double) * b_elems, st_), "batch X");
    if (nf) ok = ok && cuda(dI.alloc(sizeof(int32_t) * nf, st_), "batch info");
    for (size_t i = 0; ok && i < nf; ++i) {
      ok = cuda(cudaMemcpyAsync(dA.as<double>() + fa[i], F[i]->A, sizeof(double) * fn[i] * fn[i],
                                cudaMemcpyHostToDevice, st_), "copy A") &&
           cuda(cudaMemcpyAsync(dB.as<double>() + fb[i], F[i]->B, sizeof(double) * fn[i] * fk[i],
                                cudaMemcpyHostToDevice, st_), "copy B");
    }
    for (size_t i = 0; ok && i < nr; ++i)
      ok = cuda(cudaMemcpyAsync(dB.as<double>() + r_base + rb[i], R[i]->B, sizeof(double) * rn[i] * rk[i],
                                cudaMemcpyHostToDevice, st_), "copy B");
    int rc = NPPB_OK;
    std::unique_ptr<Plan> pf, pr;
    if (ok && nf) {
      pf = std::make_unique<Plan>();
      pf->use_graph = false;
      pf->alloc_stream = st_;
      rc = pf->build((int64_t)nf, fn.data(), fk.data(), fa.data(), fb.data(), fi.data(),
                     NPPB_WANT_SOLVE | NPPB_WANT_LU, false, false, f_lu.data(), f_piv.data());
      if (rc == NPPB_OK) {
        Plan::Ptrs p{};
        p.A = dA.as<double>();
        p.B = dB.as<double>();
        p.X = dX.as<double>();
        p.info = dI.as<int32_t>();
        p.LU = lu_arena_;
        p.ipiv = piv_arena_;
        rc = pf->execute(p, st_);
      }
    }
    if (ok && rc == NPPB_OK && nr) {
      pr = std::make_unique<Plan>();
      pr->use_graph = false;
      pr->alloc_stream = st_;
      // a_off is not read in solve-only mode: the factor offsets stand in
      rc = pr->build((int64_t)nr, rn.data(), rk.data(), r_lu.data(), rb.data(), ri.data(), NPPB_WANT_SOLVE, true,
                     false, r_lu.data(), r_piv.data());
      if (rc == NPPB_OK) {
        Plan::Ptrs p{};
        p.B = dB.as<double>() + r_base;
        p.X = dX.as<double>() + r_base;
        p.LU = lu_arena_;
        p.ipiv = piv_arena_;
        rc = pr->execute(p, st_);
      }
    }
    if (rc != NPPB_OK && err.empty()) err = last_error();
    for (size_t i = 0; ok && rc == NPPB_OK && i < nf; ++i)
      ok = cuda(cudaMemcpyAsync(F[i]->X, dX.as<double>() + fb[i], sizeof(double) * fn[i] * fk[i],
                                cudaMemcpyDeviceToHost, st_), "copy X");
    for (size_t i = 0; ok && rc == NPPB_OK && i < nr; ++i)
      ok = cuda(cudaMemcpyAsync(R[i]->X, dX.as<double>() + r_base + rb[i], sizeof(double) * rn[i] * rk[i],
                                cudaMemcpyDeviceToHost, st_), "copy X");
    if (ok && rc == NPPB_OK && nf)
      ok = cuda(cudaMemcpyAsync(finfo.data(), dI.as<int32_t>(), sizeof(int32_t) * nf, cudaMemcpyDeviceToHost, st_),
                "copy info");
    // plans and staging free their device memory stream-ordered; then wait for the batch
    pf.reset();
    pr.reset();
    dA.release();
    dB.release();
    dX.release();
    dI.release();
    ok = cuda(cudaStreamSynchronize(st_), "batch") && ok;
    if (rc != NPPB_OK) return rc;
    return ok ? NPPB_OK : NPPB_E_CUDA;
  }

  int dev_ = -1;
  cudaStream_t st_ = nullptr;
  double* lu_arena_ = nullptr;
  int32_t* piv_arena_ = nullptr;
  int64_t lu_cap_ = 0, piv_cap_ = 0, batch_bytes_ = 0;
  std::chrono::microseconds window_{0};
  int max_batch_ = 1;

  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Req*> queue_;
  std::unordered_map<int64_t, std::unique_ptr<Req>> reqs_;
  std::unordered_map<int64_t, Factor> factors_;
  std::list<int64_t> lru_;  // most recently used first
  RangeAlloc lu_alloc_, piv_alloc_;
  int64_t next_req_ = 0, next_factor_ = 0;
  int64_t completed_ = 0, batches_ = 0, evictions_ = 0;
  bool stop_ = false;
  std::thread worker_;
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
