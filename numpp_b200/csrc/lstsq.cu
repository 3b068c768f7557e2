// Batched least squares and singular values through one-sided Jacobi. C++20.
//
// The reference solves lstsq through its economy SVD, a cyclic one-sided
// Jacobi on the tall orientation (A, or A^T when m < n), and returns the
// solution, the residuals (overdetermined and full rank only), the rank at
// tol = (rcond < 0 ? eps * max(m, n) : rcond) * s_max and the singular values
// (src/linalg/linalg.cpp:620-712, 755-784). Here one CTA runs the same
// cyclic sweeps for one problem of the batch with the tall matrix and V in
// shared memory (column-major, so a column is contiguous): per column pair,
// the two squared norms and the dot product are reduced over the CTA, the
// pair is rotated (after the sign flip that makes the dot product positive),
// up to 60 sweeps until the largest relative dot product is below 1e-15.
// Then the column norms (the singular values, sorted descending), the rank,
// x = V diag(1/s or 0) U^T b and the residuals. Sums run in a different order
// than the reference's (parallel partial sums, fused multiply-adds), so the
// results agree within rounding, not bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <new>

#include "../../include/numpp_b200.h"
#include "nppb_internal.hpp"
#include "runtime.hpp"

using namespace nppb;

namespace {

constexpr int LT = 256;               // threads per problem
constexpr int kLsqMaxN = 64;          // columns of the tall orientation
constexpr int kLsqMaxK = 64;          // right-hand sides
constexpr size_t kLsqMaxSmem = 220 * 1024;  // dynamic shared memory of one problem

#define NPPB_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)

size_t lsq_smem(int M, int N, int k) {
  return sizeof(double) * ((size_t)M * N + (size_t)N * N + (size_t)N * (k > 0 ? k : 1) + N + 3 * (LT / 32)) +
         sizeof(int) * (size_t)N;
}

// Sum of v over the CTA; every thread returns the same total (partials added
// in warp order by every thread).
__device__ __forceinline__ double cta_sum(double v, double* red, int slot) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[slot * (LT / 32) + warp] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < LT / 32; ++w) t += red[slot * (LT / 32) + w];
  return t;
}

// One problem per CTA. A (m x n), B (m x k) row-major in global memory; X
// (n x k), S (min(m, n)), rank, resid (k) and has_resid out. k = 0: singular
// values (and rank) only.
__global__ void __launch_bounds__(LT)
k_lstsq(int m, int n, int k, const double* __restrict__ A, const double* __restrict__ B, double rcond,
        double* __restrict__ X, double* __restrict__ S, int32_t* __restrict__ rank, double* __restrict__ resid,
        int32_t* __restrict__ has_resid) {
  extern __shared__ __align__(16) unsigned char lsq_raw[];
  const int wide = m < n, M = wide ? n : m, N = wide ? m : n, kk = N;
  double* W = reinterpret_cast<double*>(lsq_raw);  // column c at W + c * M
  double* V = W + (size_t)M * N;                     // column c at V + c * N
  double* T1 = V + (size_t)N * N;                    // N x k (row c at T1 + c * k)
  double* sig = T1 + (size_t)N * (k > 0 ? k : 1);
  double* red = sig + N;                             // 3 x warps
  int* ord = reinterpret_cast<int*>(red + 3 * (LT / 32));
  __shared__ double s_maxoff;
  __shared__ int s_rank;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t z = blockIdx.x;
  const double* Az = A + z * (int64_t)m * n;
  for (int idx = tid; idx < M * N; idx += LT) {
    const int c = idx / M, r = idx - c * M;  // W[c][r] = tall(r, c)
    W[idx] = wide ? Az[(int64_t)c * n + r] : Az[(int64_t)r * n + c];
  }
  for (int idx = tid; idx < N * N; idx += LT) V[idx] = (idx / N == idx % N) ? 1.0 : 0.0;
  __syncthreads();

  for (int sweep = 0; sweep < 60; ++sweep) {
    if (tid == 0) s_maxoff = 0.0;
    for (int i = 0; i < N; ++i) {
      for (int j = i + 1; j < N; ++j) {
        double* wi = W + (size_t)i * M;
        double* wj = W + (size_t)j * M;
        double aa = 0.0, bb = 0.0, cc = 0.0;
        for (int r = tid; r < M; r += LT) {
          const double xi = wi[r], xj = wj[r];
          aa = fma(xi, xi, aa);
          bb = fma(xj, xj, bb);
          cc = fma(xi, xj, cc);
        }
        aa = cta_sum(aa, red, 0);
        bb = cta_sum(bb, red, 1);
        cc = cta_sum(cc, red, 2);
        bool rot = aa != 0.0 && bb != 0.0;
        double w = 1.0, cs = 1.0, sn = 0.0;
        if (rot) {
          const double magc = fabs(cc), off = magc / sqrt(aa * bb);
          if (tid == 0 && off > s_maxoff) s_maxoff = off;
          rot = off >= 1e-300;
          if (rot) {
            w = cc / magc;
            const double zeta = (bb - aa) / (2.0 * magc);
            const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            cs = 1.0 / sqrt(1.0 + t * t);
            sn = cs * t;
          }
        }
        if (rot) {
          for (int r = tid; r < M; r += LT) {
            const double xi = wi[r], xj = wj[r] * w;
            wi[r] = cs * xi - sn * xj;
            wj[r] = sn * xi + cs * xj;
          }
          double* vi = V + (size_t)i * N;
          double* vj = V + (size_t)j * N;
          for (int r = tid; r < N; r += LT) {
            const double a = vi[r], b = vj[r] * w;
            vi[r] = cs * a - sn * b;
            vj[r] = sn * a + cs * b;
          }
        }
        __syncthreads();  // the pair's columns are final before any thread reads them again
      }
    }
    __syncthreads();
    if (s_maxoff < 1e-15) break;  // uniform: every thread read the same value after the barrier
    __syncthreads();              // nobody resets s_maxoff before every thread has read it
  }

  // singular values: the column norms; U's columns normalised in place
  for (int c = warp; c < N; c += LT / 32) {
    double s2 = 0.0;
    for (int r = lane; r < M; r += 32) s2 = fma(W[(size_t)c * M + r], W[(size_t)c * M + r], s2);
#pragma unroll
    for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    const double s = sqrt(s2);
    if (lane == 0) sig[c] = s;
    for (int r = lane; r < M; r += 32) W[(size_t)c * M + r] = s > 0.0 ? W[(size_t)c * M + r] / s : 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    for (int c = 0; c < N; ++c) ord[c] = c;
    for (int a = 1; a < N; ++a) {  // stable insertion sort, descending
      const int o = ord[a];
      int b = a - 1;
      while (b >= 0 && sig[ord[b]] < sig[o]) {
        ord[b + 1] = ord[b];
        --b;
      }
      ord[b + 1] = o;
    }
    const double smax = kk ? sig[ord[0]] : 0.0;
    const double tol = (rcond < 0 ? 2.220446049250313e-16 * (m > n ? m : n) : rcond) * smax;
    int rk = 0;
    for (int c = 0; c < kk; ++c) {
      S[z * kk + c] = sig[ord[c]];
      rk += sig[ord[c]] > tol;
    }
    rank[z] = rk;
    s_rank = rk;
    // sig becomes 1/s or 0 in sorted order
    double tmp[kLsqMaxN];
    for (int c = 0; c < kk; ++c) tmp[c] = sig[ord[c]] > tol ? 1.0 / sig[ord[c]] : 0.0;
    for (int c = 0; c < kk; ++c) sig[c] = tmp[c];
  }
  __syncthreads();
  if (k == 0) return;

  // T1 = diag(sinv) Um^T b (kk x k); Um = U (tall, M = m) or V (wide, m x m)
  const double* Bz = B + z * (int64_t)m * k;
  for (int q = warp; q < kk * k; q += LT / 32) {
    const int c = q / k, j = q - c * k;
    const double* uc = wide ? V + (size_t)ord[c] * N : W + (size_t)ord[c] * M;  // length m either way
    double t = 0.0;
    for (int p = lane; p < m; p += 32) t = fma(uc[p], Bz[(int64_t)p * k + j], t);
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) T1[(size_t)c * k + j] = sig[c] * t;
  }
  __syncthreads();
  // x = Vm T1 (n x k); Vm = V (tall, n x n) or U (wide, n x m)
  double* Xz = X + z * (int64_t)n * k;
  for (int q = tid; q < n * k; q += LT) {
    const int i = q / k, j = q - i * k;
    double t = 0.0;
    for (int c = 0; c < kk; ++c) {
      const double v = wide ? W[(size_t)ord[c] * M + i] : V[(size_t)ord[c] * N + i];
      t = fma(v, T1[(size_t)c * k + j], t);
    }
    Xz[(int64_t)i * k + j] = t;
  }
  const bool form = m > n && s_rank == n;
  if (tid == 0) has_resid[z] = form ? 1 : 0;
  if (!form) return;
  __syncthreads();  // x is in global memory for every thread
  // residuals: sum over rows of (b - A x)^2, per column
  for (int j = 0; j < k; ++j) {
    double acc = 0.0;
    for (int i = tid; i < m; i += LT) {
      double ax = 0.0;
      for (int p = 0; p < n; ++p) ax = fma(Az[(int64_t)i * n + p], Xz[(int64_t)p * k + j], ax);
      const double d = Bz[(int64_t)i * k + j] - ax;
      acc = fma(d, d, acc);
    }
    acc = cta_sum(acc, red, 0);
    if (tid == 0) resid[z * k + j] = acc;
    __syncthreads();  // red is reused by the next column
  }
}

int check(int64_t count, int32_t m, int32_t n, int32_t k) {
  if (count < 0 || m < 0 || n < 0 || k < 0) {
    set_error("negative count, shape or nrhs");
    return NPPB_E_ARG;
  }
  if (count > INT32_MAX) {
    set_error("batch count above 2^31-1");
    return NPPB_E_RANGE;
  }
  const int M = m > n ? m : n, N = m < n ? m : n;
  if (N > kLsqMaxN || k > kLsqMaxK || (int64_t)M * N > (int64_t)kLsqMaxSmem / 8 || lsq_smem(M, N, k) > kLsqMaxSmem) {
    set_error("least squares on the device: min(m, n) <= 64, nrhs <= 64 and the tall matrix, V and U^T b "
              "within 220 KiB of shared memory (about m * n + min(m, n)^2 <= 26000)");
    return NPPB_DECLINED;
  }
  return NPPB_OK;
}

int lstsq_device(int64_t count, int32_t m, int32_t n, int32_t k, const double* dA, const double* dB, double rcond,
                 double* dX, double* dS, int32_t* drank, double* dres, int32_t* dhas, cudaStream_t st) {
  const int M = m > n ? m : n, N = m < n ? m : n;
  const size_t smem = lsq_smem(M, N, k);
  NPPB_CUDA(cudaFuncSetAttribute(k_lstsq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attribute");
  k_lstsq<<<(unsigned)count, LT, smem, st>>>(m, n, k, dA, dB, rcond, dX, dS, drank, dres, dhas);
  NPPB_CUDA(cudaGetLastError(), "least squares");
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

}  // namespace

extern "C" {

int nppb_d_lstsq_batched(int64_t count, int32_t m, int32_t n, int32_t k, const double* dA, const double* dB,
                         double rcond, double* dX, double* dS, int32_t* drank, double* dres, int32_t* dhas,
                         void* stream) {
  return guarded([&]() -> int {
    const int rc = check(count, m, n, k);
    if (rc != NPPB_OK) return rc;
    if (!count || !m || !n) return NPPB_OK;
    if (!dA || !dS || !drank || (k && (!dB || !dX || !dres || !dhas))) {
      set_error("lstsq needs A, S, rank and, with right-hand sides, B, X, residuals and their flags");
      return NPPB_E_ARG;
    }
    if (!device()) return NPPB_E_NODEV;
    return lstsq_device(count, m, n, k, dA, dB, rcond, dX, dS, drank, dres, dhas, static_cast<cudaStream_t>(stream));
  });
}

int nppb_lstsq_batched(int64_t count, int32_t m, int32_t n, int32_t k, const double* A, const double* B,
                       double rcond, double* X, double* S, int32_t* rank, double* resid, int32_t* has_resid) {
  return guarded([&]() -> int {
    const int rc = check(count, m, n, k);
    if (rc != NPPB_OK) return rc;
    if (!count || !m || !n) return NPPB_OK;
    if (!A || !S || !rank || (k && (!B || !X || !resid || !has_resid))) {
      set_error("lstsq needs A, S, rank and, with right-hand sides, B, X, residuals and their flags");
      return NPPB_E_ARG;
    }
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t c = (size_t)count, kk = (size_t)(m < n ? m : n);
    DevMem dA, dB, dX, dS, dR, dres, dh;
    NPPB_CUDA(dA.alloc(sizeof(double) * c * m * n, st), "allocation");
    NPPB_CUDA(dS.alloc(sizeof(double) * c * kk, st), "allocation");
    NPPB_CUDA(dR.alloc(sizeof(int32_t) * c, st), "allocation");
    NPPB_CUDA(cudaMemcpyAsync(dA.as<double>(), A, sizeof(double) * c * m * n, cudaMemcpyHostToDevice, st), "copy");
    if (k) {
      NPPB_CUDA(dB.alloc(sizeof(double) * c * m * k, st), "allocation");
      NPPB_CUDA(dX.alloc(sizeof(double) * c * n * k, st), "allocation");
      NPPB_CUDA(dres.alloc(sizeof(double) * c * k, st), "allocation");
      NPPB_CUDA(dh.alloc(sizeof(int32_t) * c, st), "allocation");
      NPPB_CUDA(cudaMemcpyAsync(dB.as<double>(), B, sizeof(double) * c * m * k, cudaMemcpyHostToDevice, st), "copy");
    }
    const int r = lstsq_device(count, m, n, k, dA.as<double>(), k ? dB.as<double>() : nullptr, rcond,
                               k ? dX.as<double>() : nullptr, dS.as<double>(), dR.as<int32_t>(),
                               k ? dres.as<double>() : nullptr, k ? dh.as<int32_t>() : nullptr, st);
    if (r != NPPB_OK) return r;
    NPPB_CUDA(cudaMemcpyAsync(S, dS.as<double>(), sizeof(double) * c * kk, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaMemcpyAsync(rank, dR.as<int32_t>(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, st), "copy");
    if (k) {
      NPPB_CUDA(cudaMemcpyAsync(X, dX.as<double>(), sizeof(double) * c * n * k, cudaMemcpyDeviceToHost, st), "copy");
      NPPB_CUDA(cudaMemcpyAsync(resid, dres.as<double>(), sizeof(double) * c * k, cudaMemcpyDeviceToHost, st),
                "copy");
      NPPB_CUDA(cudaMemcpyAsync(has_resid, dh.as<int32_t>(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, st),
                "copy");
    }
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    NPPB_CUDA(cudaGetLastError(), "kernel");
    return NPPB_OK;
  });
}

}  // extern "C"
