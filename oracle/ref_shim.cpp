// REFERENCE SHIM — TEST INFRASTRUCTURE ONLY.
//
// extern "C" wrappers around the reference library's own public API
// (numpp::linalg::solve/inv/det/slogdet/cholesky/matrix_power/tensorsolve/tensorinv
// and numpp::matmul), compiled together
// with the reference's unmodified CPU sources into oracle/_ref/libnumpp_ref.so
// by oracle/Makefile. Tests use it to pin the C oracle and to make golden
// fixtures; bench.py's reference arm times it. The product never loads it.
//
// Error codes: 0 ok, 1 numpp::linalg_error, 2 any other numpp::error,
// 3 unexpected exception. The message is copied to err (if given).
#include <atomic>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "numpp/backend/backend.hpp"
#include "numpp/core/error.hpp"
#include "numpp/core/ndarray.hpp"
#include "numpp/linalg/linalg.hpp"
#include "numpp/random/random.hpp"

using numpp::DType;
using numpp::DTypeId;
using numpp::ndarray;
using numpp::Shape;

namespace {

ndarray make(int nd, const int64_t* shape, int dt, const void* data) {
  Shape s(shape, shape + nd);
  ndarray a(s, DType(static_cast<DTypeId>(dt)), numpp::Order::C);
  if (a.nbytes()) std::memcpy(a.bytes(), data, static_cast<size_t>(a.nbytes()));
  return a;
}

// Copies a result out in the dtype it came back with; reports that dtype and
// its element count so the caller can check the reference's dtype policy.
void put(const ndarray& r, void* out, int* out_dt, int64_t* out_size) {
  ndarray c = r.ascontiguousarray();
  if (c.nbytes() && out) std::memcpy(out, c.bytes(), static_cast<size_t>(c.nbytes()));
  if (out_dt) *out_dt = static_cast<int>(c.dtype().id());
  if (out_size) *out_size = c.size();
}

template <class F>
int guard(char* err, int errlen, F&& f) {
  auto msg = [&](const char* m) {
    if (err && errlen > 0) { std::strncpy(err, m, static_cast<size_t>(errlen - 1)); err[errlen - 1] = 0; }
  };
  try { f(); return 0; }
  catch (const numpp::linalg_error& e) { msg(e.what()); return 1; }
  catch (const numpp::error& e) { msg(e.what()); return 2; }
  catch (const std::exception& e) { msg(e.what()); return 3; }
}

}  // namespace

extern "C" {

int ref_solve(int nda, const int64_t* sa, int dta, const void* A, int ndb, const int64_t* sb,
              int dtb, const void* B, void* X, int* x_dt, int64_t* x_size, char* err, int errlen) {
  return guard(err, errlen, [&] {
    put(numpp::linalg::solve(make(nda, sa, dta, A), make(ndb, sb, dtb, B)), X, x_dt, x_size);
  });
}

int ref_inv(int nda, const int64_t* sa, int dta, const void* A, void* out, int* o_dt,
            int64_t* o_size, char* err, int errlen) {
  return guard(err, errlen, [&] { put(numpp::linalg::inv(make(nda, sa, dta, A)), out, o_dt, o_size); });
}

int ref_det(int nda, const int64_t* sa, int dta, const void* A, void* out, int* o_dt,
            int64_t* o_size, char* err, int errlen) {
  return guard(err, errlen, [&] { put(numpp::linalg::det(make(nda, sa, dta, A)), out, o_dt, o_size); });
}

int ref_slogdet(int nda, const int64_t* sa, int dta, const void* A, void* sign, void* logabs,
                int* o_dt, int64_t* o_size, char* err, int errlen) {
  return guard(err, errlen, [&] {
    numpp::linalg::SignLogDet r = numpp::linalg::slogdet(make(nda, sa, dta, A));
    put(r.sign, sign, o_dt, o_size);
    put(r.logabsdet, logabs, nullptr, nullptr);
  });
}

// lstsq (src/linalg/linalg.cpp:755-784): solution, residuals (size 0 or k),
// rank and singular values, each copied out with its element count.
int ref_lstsq(int nda, const int64_t* sa, const void* A, int ndb, const int64_t* sb, const void* B,
              double rcond, void* X, int64_t* x_size, void* R, int64_t* r_size, int64_t* rank, void* S,
              int64_t* s_size, char* err, int errlen) {
  return guard(err, errlen, [&] {
    numpp::linalg::LstsqResult r = numpp::linalg::lstsq(make(nda, sa, 11, A), make(ndb, sb, 11, B), rcond);
    put(r.solution, X, nullptr, x_size);
    put(r.residuals, R, nullptr, r_size);
    put(r.singular_values, S, nullptr, s_size);
    *rank = r.rank.astype(numpp::kInt64).item<int64_t>({});
  });
}

// cholesky (src/linalg/linalg.cpp:117-136; stacks batched.cpp:77).
int ref_cholesky(int nda, const int64_t* sa, int dta, const void* A, void* out, int* o_dt, int64_t* o_size,
                 char* err, int errlen) {
  return guard(err, errlen, [&] { put(numpp::linalg::cholesky(make(nda, sa, dta, A)), out, o_dt, o_size); });
}

// matrix_power (src/linalg/linalg.cpp:440-454; stacks batched.cpp:83-84).
int ref_matrix_power(int nda, const int64_t* sa, int dta, const void* A, int64_t p, void* out,
                     int* o_dt, int64_t* o_size, char* err, int errlen) {
  return guard(err, errlen, [&] {
    put(numpp::linalg::matrix_power(make(nda, sa, dta, A), p), out, o_dt, o_size);
  });
}

// tensorsolve / tensorinv (src/linalg/tensor_solve.cpp:10-49). naxes = 0: no axes.
int ref_tensorsolve(int nda, const int64_t* sa, int dta, const void* A, int ndb, const int64_t* sb,
                    int dtb, const void* B, int naxes, const int64_t* axes, void* X, int* x_dt,
                    int64_t* x_size, char* err, int errlen) {
  return guard(err, errlen, [&] {
    std::vector<int64_t> ax(axes, axes + naxes);
    put(numpp::linalg::tensorsolve(make(nda, sa, dta, A), make(ndb, sb, dtb, B), ax), X, x_dt, x_size);
  });
}

int ref_tensorinv(int nda, const int64_t* sa, int dta, const void* A, int64_t ind, void* out, int* o_dt,
                  int64_t* o_size, char* err, int errlen) {
  return guard(err, errlen, [&] { put(numpp::linalg::tensorinv(make(nda, sa, dta, A), ind), out, o_dt, o_size); });
}

int ref_matmul_cpu(int64_t m, int64_t n, int64_t k, int dt, const void* A, const void* B, void* C,
                   char* err, int errlen) {
  return guard(err, errlen, [&] {
    int64_t sa[2] = {m, k}, sb[2] = {k, n};
    put(numpp::matmul(make(2, sa, dt, A), make(2, sb, dt, B), numpp::Backend::Cpu), C, nullptr, nullptr);
  });
}

// Uneven batch through the reference's 2-D public calls, the way a caller of
// NumPP would loop over systems of different orders. System i: order n[i],
// nrhs[i] columns; A at a_off[i], B/X at b_off[i]; inverse into inv_off[i]
// when >= 0. sign/logabs may be null (no slogdet). The reference itself is
// single-threaded; `threads` > 1 fans disjoint systems out over std::threads,
// each running the unmodified single-matrix path. ok[i] = 1, or 0 on
// linalg_error for that system.
int ref_solve_grouped(int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                      const int64_t* b_off, const int64_t* inv_off, const double* A,
                      const double* B, double* X, double* sign, double* logabs, double* inv,
                      int32_t* ok, int threads) {
  std::atomic<int64_t> next{0};
  auto work = [&] {
    for (;;) {
      int64_t i = next.fetch_add(1);
      if (i >= count) break;
      int64_t sa[2] = {n[i], n[i]};
      int64_t sb[2] = {n[i], nrhs[i]};
      ok[i] = 1;
      try {
        ndarray a = make(2, sa, 11, A + a_off[i]);
        put(numpp::linalg::solve(a, make(2, sb, 11, B + b_off[i])), X + b_off[i], nullptr, nullptr);
        if (sign) {
          numpp::linalg::SignLogDet r = numpp::linalg::slogdet(a);
          put(r.sign, sign + i, nullptr, nullptr);
          put(r.logabsdet, logabs + i, nullptr, nullptr);
        }
        if (inv && inv_off[i] >= 0) put(numpp::linalg::inv(a), inv + inv_off[i], nullptr, nullptr);
      } catch (const numpp::linalg_error&) {
        ok[i] = 0;
      }
    }
  };
  if (threads <= 1) { work(); return 0; }
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  return 0;
}

// numpp::last_backend() (src/backend/backend.cpp:118-119), as its enum value
// (numpp::Backend: Auto 0, Cpu 1, Blas 2, Device 3, Metal 4, Vulkan 5, Cuda 6,
// OpenCL 7), and set_last_backend(Auto) to clear it between calls.
int ref_last_backend(void) { return static_cast<int>(numpp::last_backend()); }
void ref_clear_last_backend(void) { numpp::set_last_backend(numpp::Backend::Auto); }

// numpp::random::default_rng(seed): n1 standard normals, then n2 more from the
// same generator (the draw order of the uniform-batch workload: A, then b).
int ref_standard_normal2(uint64_t seed, int64_t n1, double* out1, int64_t n2, double* out2) {
  return guard(nullptr, 0, [&] {
    numpp::random::Generator g = numpp::random::default_rng(seed);
    put(g.standard_normal(Shape{n1}), out1, nullptr, nullptr);
    put(g.standard_normal(Shape{n2}), out2, nullptr, nullptr);
  });
}

// numpp::random::default_rng(seed).uniform(low, high, n).
int ref_uniform(uint64_t seed, double low, double high, int64_t n, double* out) {
  return guard(nullptr, 0, [&] {
    numpp::random::Generator g = numpp::random::default_rng(seed);
    put(g.uniform(low, high, Shape{n}), out, nullptr, nullptr);
  });
}

}  // extern "C"
