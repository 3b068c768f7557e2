// Kernels of the mixed-precision solve (FP32 factors, FP64 refinement).
//
// No counterpart in the reference, which solves in double only
// (src/linalg/linalg.cpp:20-26,92-103). Per system of a uniform batch:
//  k_equil_rows / k_equil_apply
//                 power-of-two row and column scales r, c (exact in FP64) so
//                 that every row and column of diag(r) A diag(c) peaks in
//                 [1, 2); writes that matrix in FP32 and ||A||_inf
//  k_scale_rhs    r * B in FP32 (the first right-hand side), ||B||_max
//  k_apply        X = c * Y (first solution) or X += c * Y (correction), FP64
//  k_residual     R = B - A X in FP64 and r * R in FP32 for the next correction
//  k_refine_decide eta = max|R| / (||A||_inf max|X| + max|B|) (normwise
//                 backward error) and the convergence / stall decision
//                 (stalled: the contraction shown cannot reach tol in the
//                 corrections left)
//  k_ferr         forward error max|X - Xtrue| / max|Xtrue| when Xtrue is known
#include <cfloat>
#include <cmath>

#include "mixed.hpp"

namespace nppb {
namespace {

constexpr int MT = 256;

__device__ __forceinline__ double pow2_scale(double m) {
  // 2^-e with m * 2^-e in [1, 2); 1 for zero or non-finite rows
  if (!(m > 0.0) || !isfinite(m)) return 1.0;
  return ldexp(1.0, -ilogb(m));
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide max over MT threads (scratch: MT/32 doubles).
__device__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = lane < MT / 32 ? red[lane] : 0.0;
  return warp_max(r);
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* bits, double v) {
  // non-negative doubles (and NaN, which then wins) order like their bit patterns
  atomicMax(bits, (unsigned long long)__double_as_longlong(v));
}

// Row pass, one CTA per (system, kMixedRows rows): row scales, ||A||_inf, and
// the column maxima of diag(r) |A| over this CTA's rows.
__global__ void __launch_bounds__(MT)
k_equil_rows(const double* __restrict__ A, int n, int equil, double* __restrict__ rs,
             double* __restrict__ cmax, RefineState* __restrict__ st) {
  __shared__ double rsc[kMixedRows];
  __shared__ double red[MT / 32];
  const int s = blockIdx.x, r0 = blockIdx.y * kMixedRows;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rows = min(kMixedRows, n - r0);
  const double* a = A + (int64_t)s * n * n + (int64_t)r0 * n;
  double arow = 0.0;
  for (int i = warp; i < rows; i += MT / 32) {
    double m = 0.0, sum = 0.0;
#pragma unroll 8
    for (int j = lane; j < n; j += 32) {
      const double v = fabs(a[(int64_t)i * n + j]);
      m = fmax(m, v);
      sum += v;
    }
    m = warp_max(m);
    sum = warp_sum(sum);
    const double r = equil ? pow2_scale(m) : 1.0;
    if (lane == 0) {
      rsc[i] = r;
      rs[(int64_t)s * n + r0 + i] = r;
    }
    arow = fmax(arow, sum);
  }
  const double anorm = block_max(arow, red);  // includes the barrier publishing rsc
  if (tid == 0) atomic_max_nonneg(reinterpret_cast<unsigned long long*>(&st[s].anorm), anorm);
  if (!equil) return;
  for (int j = tid; j < n; j += MT) {
    double m = 0.0;
#pragma unroll 8
    for (int i = 0; i < rows; ++i) m = fmax(m, rsc[i] * fabs(a[(int64_t)i * n + j]));
    atomic_max_nonneg(reinterpret_cast<unsigned long long*>(&cmax[(int64_t)s * n + j]), m);
  }
}

// Column scales from the maxima, the scaled matrix in FP32, and the state of
// every system (by the CTA of its first rows).
__global__ void __launch_bounds__(MT)
k_equil_apply(const double* __restrict__ A, int n, int equil, const double* __restrict__ rs,
              const double* __restrict__ cmax, double* __restrict__ cs, float* __restrict__ A32,
              RefineState* __restrict__ st) {
  __shared__ double csc[kMixedMaxN];
  const int s = blockIdx.x, r0 = blockIdx.y * kMixedRows, tid = threadIdx.x;
  const int rows = min(kMixedRows, n - r0);
  for (int j = tid; j < n; j += MT) {
    const double c = equil ? pow2_scale(cmax[(int64_t)s * n + j]) : 1.0;
    csc[j] = c;
    if (blockIdx.y == 0) cs[(int64_t)s * n + j] = c;
  }
  __syncthreads();
  const double* a = A + (int64_t)s * n * n + (int64_t)r0 * n;
  float* a32 = A32 + (int64_t)s * n * n + (int64_t)r0 * n;
  for (int i = 0; i < rows; ++i) {
    const double r = rs[(int64_t)s * n + r0 + i];
    for (int j = tid; j < n; j += MT) a32[(int64_t)i * n + j] = (float)(r * a[(int64_t)i * n + j] * csc[j]);
  }
  if (blockIdx.y == 0 && tid == 0) {
    st[s].eta = INFINITY;
    st[s].prev = INFINITY;
    st[s].status = kRefineActive;
    st[s].iters = 0;
  }
}

__global__ void __launch_bounds__(MT)
k_scale_rhs(const double* __restrict__ B, int n, int nrhs, const double* __restrict__ rs,
            float* __restrict__ B32, RefineState* __restrict__ st) {
  __shared__ double red[MT / 32];
  const int s = blockIdx.x, tid = threadIdx.x;
  const int64_t nb = (int64_t)n * nrhs;
  const double* b = B ? B + (int64_t)s * nb : nullptr;  // null: R = -A X (the product alone)
  double m = 0.0;
  for (int64_t idx = tid; idx < nb; idx += MT) {
    const double v = b[idx];
    m = fmax(m, fabs(v));
    B32[(int64_t)s * nb + idx] = (float)(rs[(int64_t)s * n + idx / nrhs] * v);
  }
  m = block_max(m, red);
  if (tid == 0) st[s].bnorm = m;
}

__global__ void __launch_bounds__(MT)
k_apply(double* __restrict__ X, const float* __restrict__ Y, const double* __restrict__ cs, int n,
        int nrhs, const RefineState* __restrict__ st, int init) {
  const int s = blockIdx.x;
  if (!init && st[s].status != kRefineActive) return;
  const int64_t nb = (int64_t)n * nrhs;
  for (int64_t idx = threadIdx.x; idx < nb; idx += MT) {
    const double d = cs[(int64_t)s * n + idx / nrhs] * (double)Y[(int64_t)s * nb + idx];
    X[(int64_t)s * nb + idx] = init ? d : X[(int64_t)s * nb + idx] + d;
  }
}

// One CTA per (system, kMixedRows rows of A): R = B - A X for those rows,
// right-hand sides in chunks of RC (1, 2, 4 or 8: the smallest power of two
// covering nrhs, at most 8), X staged through shared memory in blocks of
// XS / RC rows; each warp keeps kMixedRows / 8 rows' sums in registers and
// reads its rows of A coalesced. max |R| (and, by the first CTA, max |X|) go
// to the system's running maxima; k_refine_decide turns them into eta. With
// rpos, row i of the scaled residual is stored at row rpos[i] (pivoted order).
constexpr int XS = 4096;                    // doubles of X staged per block
constexpr int RW = kMixedRows / (MT / 32);  // rows per warp

template <int RC>
__global__ void __launch_bounds__(MT)
k_residual(const double* __restrict__ A, const double* __restrict__ B, const double* __restrict__ X,
           int n, int nrhs, const double* __restrict__ rs, float* __restrict__ R32,
           const int32_t* __restrict__ rpos, double* __restrict__ R64, RefineState* __restrict__ st,
           int only_active, int stats) {
  constexpr int CB = XS / RC;
  __shared__ double xs[XS];
  __shared__ double red[MT / 32];
  __shared__ double ax_s[MT / 32][RW][RC];
  const int s = blockIdx.x, r0 = blockIdx.y * kMixedRows;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (only_active && st[s].status != kRefineActive) return;
  const int64_t nb = (int64_t)n * nrhs;
  const double* a = A + (int64_t)s * n * n;
  const double* b = B ? B + (int64_t)s * nb : nullptr;  // null: R = -A X (the product alone)
  const double* x = X + (int64_t)s * nb;
  const bool first = stats && blockIdx.y == 0;
  double rmax = 0.0, xmax = 0.0;
  for (int k0 = 0; k0 < nrhs; k0 += RC) {
    const int kc = min(RC, nrhs - k0);
    double acc[RW][RC];
#pragma unroll
    for (int q = 0; q < RW; ++q)
#pragma unroll
      for (int k = 0; k < RC; ++k) acc[q][k] = 0.0;
    for (int j0 = 0; j0 < n; j0 += CB) {
      const int jn = min(CB, n - j0);
      __syncthreads();
      for (int idx = tid; idx < jn * RC; idx += MT) {
        const int j = idx / RC, k = idx % RC;
        const double v = k < kc ? x[(int64_t)(j0 + j) * nrhs + k0 + k] : 0.0;
        xs[idx] = v;
        if (first) xmax = fmax(xmax, fabs(v));
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < RW; ++q) {
        const int i = r0 + warp * RW + q;
        if (i < n) {
          const double* ai = a + (int64_t)i * n + j0;
#pragma unroll 4
          for (int j = lane; j < jn; j += 32) {
            const double aij = ai[j];
#pragma unroll
            for (int k = 0; k < RC; ++k) acc[q][k] = fma(aij, xs[j * RC + k], acc[q][k]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < RW; ++q)
#pragma unroll
      for (int k = 0; k < RC; ++k) acc[q][k] = warp_sum(acc[q][k]);
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < RW; ++q)
#pragma unroll
        for (int k = 0; k < RC; ++k) ax_s[warp][q][k] = acc[q][k];
    }
    __syncwarp();
    if (lane < RW * RC) {
      const int q = lane / RC, k = lane % RC;
      const int i = r0 + warp * RW + q;
      if (i < n && k < kc) {
        const double r = (b ? b[(int64_t)i * nrhs + k0 + k] : 0.0) - ax_s[warp][q][k];
        rmax = fmax(rmax, fabs(r));
        if (R32) {
          const int p = rpos ? rpos[(int64_t)s * n + i] : i;
          R32[(int64_t)s * nb + (int64_t)p * nrhs + k0 + k] = (float)(rs[(int64_t)s * n + i] * r);
        }
        if (R64) R64[(int64_t)s * nb + (int64_t)i * nrhs + k0 + k] = rs[(int64_t)s * n + i] * r;
      }
    }
    __syncwarp();
  }
  if (!stats) return;
  rmax = block_max(rmax, red);
  if (tid == 0) atomic_max_nonneg(&st[s].rmax_bits, rmax);
  if (first) {
    xmax = block_max(xmax, red);
    if (tid == 0) atomic_max_nonneg(&st[s].xmax_bits, xmax);
  }
}

// eta = max|R| / (||A||_inf max|X| + max|B|) per system; with decide, the
// convergence / stall decision and the count of systems still refining.
// A system is stalled when eta stops decreasing (or is NaN), or when the
// contraction it has shown, rho = eta / previous eta, cannot bring eta down
// to tol within the corrections left (log(tol / eta) / log(rho) of them):
// slow but steady convergence continues, hopeless refinement stops at once.
// Clears the running maxima for the next residual pass.
__global__ void k_refine_decide(RefineState* __restrict__ st, int count, double tol, int iter, int max_iter,
                                int decide, int* __restrict__ active) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  RefineState& q = st[s];
  if (decide && q.status != kRefineActive) return;
  const double rmax = __longlong_as_double((long long)q.rmax_bits);
  const double xmax = __longlong_as_double((long long)q.xmax_bits);
  q.rmax_bits = 0;
  q.xmax_bits = 0;
  const double eta = rmax / (q.anorm * xmax + q.bnorm);
  q.eta = eta;
  if (!decide) return;
  q.iters = iter;
  bool stalled = false;
  if (!(eta <= tol) && iter > 0) {
    const double rho = eta / q.prev;
    stalled = !(rho < 1.0) || log(tol / eta) / log(rho) > (double)(max_iter - iter);
  }
  if (eta <= tol) {
    q.status = kRefineConverged;
  } else if (stalled || !(eta == eta)) {
    q.status = kRefineStalled;
  } else {
    atomicAdd(active, 1);
  }
  q.prev = eta;
}

__global__ void __launch_bounds__(MT)
k_ferr(const double* __restrict__ X, const double* __restrict__ Xt, int n, int nrhs, double* __restrict__ ferr) {
  __shared__ double red[MT / 32];
  const int s = blockIdx.x;
  const int64_t nb = (int64_t)n * nrhs;
  double d = 0.0, m = 0.0;
  for (int64_t idx = threadIdx.x; idx < nb; idx += MT) {
    const double t = Xt[(int64_t)s * nb + idx];
    d = fmax(d, fabs(X[(int64_t)s * nb + idx] - t));
    m = fmax(m, fabs(t));
  }
  d = block_max(d, red);
  m = block_max(m, red);
  if (threadIdx.x == 0) ferr[s] = m > 0.0 ? d / m : d;
}

// Position of every row in the pivoted order (the inverse of the row
// permutation a swap list applies), one CTA per system: the swaps are
// replayed serially from shared memory.
__global__ void __launch_bounds__(MT)
k_row_positions(const int32_t* __restrict__ ipiv, int n, int32_t* __restrict__ rpos) {
  extern __shared__ int prm[];  // perm, then the swap list
  int* piv = prm + n;
  const int s = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += MT) {
    prm[i] = i;
    piv[i] = ipiv[(int64_t)s * n + i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < n; ++k) {
      int p = piv[k];
      if (p < k || p >= n) p = k;
      const int t = prm[k]; prm[k] = prm[p]; prm[p] = t;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < n; q += MT) rpos[(int64_t)s * n + prm[q]] = q;
}

__global__ void k_mark_fp32_failures(const int32_t* __restrict__ info32, RefineState* __restrict__ st, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < count && info32[s]) st[s].status = kRefineStalled;
}

}  // namespace

cudaError_t mixed_equilibrate(const double* A, int count, int n, int equil, float* A32, double* rs, double* cs,
                              double* cmax, RefineState* st, cudaStream_t s) {
  const dim3 grid((unsigned)count, (unsigned)((n + kMixedRows - 1) / kMixedRows));
  k_equil_rows<<<grid, MT, 0, s>>>(A, n, equil, rs, cmax, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_equil_apply<<<grid, MT, 0, s>>>(A, n, equil, rs, cmax, cs, A32, st);
  return cudaGetLastError();
}
cudaError_t mixed_equil_scan(const double* A, int count, int n, int equil, double* rs, double* cmax,
                             RefineState* st, cudaStream_t s) {
  const dim3 grid((unsigned)count, (unsigned)((n + kMixedRows - 1) / kMixedRows));
  k_equil_rows<<<grid, MT, 0, s>>>(A, n, equil, rs, cmax, st);
  return cudaGetLastError();
}
cudaError_t mixed_scale_rhs(const double* B, int count, int n, int nrhs, const double* rs, float* B32,
                            RefineState* st, cudaStream_t s) {
  k_scale_rhs<<<count, MT, 0, s>>>(B, n, nrhs, rs, B32, st);
  return cudaGetLastError();
}
cudaError_t mixed_apply(double* X, const float* Y, const double* cs, int count, int n, int nrhs,
                        const RefineState* st, int init, cudaStream_t s) {
  k_apply<<<count, MT, 0, s>>>(X, Y, cs, n, nrhs, st, init);
  return cudaGetLastError();
}
namespace {
cudaError_t launch_residual(const double* A, const double* B, const double* X, int count, int n, int nrhs,
                            const double* rs, float* R32, const int32_t* rpos, double* R64, RefineState* st,
                            int only_active, int stats, cudaStream_t s) {
  const dim3 grid((unsigned)count, (unsigned)((n + kMixedRows - 1) / kMixedRows));
  if (nrhs == 1) k_residual<1><<<grid, MT, 0, s>>>(A, B, X, n, nrhs, rs, R32, rpos, R64, st, only_active, stats);
  else if (nrhs == 2) k_residual<2><<<grid, MT, 0, s>>>(A, B, X, n, nrhs, rs, R32, rpos, R64, st, only_active, stats);
  else if (nrhs <= 4) k_residual<4><<<grid, MT, 0, s>>>(A, B, X, n, nrhs, rs, R32, rpos, R64, st, only_active, stats);
  else k_residual<8><<<grid, MT, 0, s>>>(A, B, X, n, nrhs, rs, R32, rpos, R64, st, only_active, stats);
  return cudaGetLastError();
}
}  // namespace

cudaError_t mixed_residual(const double* A, const double* B, const double* X, int count, int n, int nrhs,
                           const double* rs, float* R32, const int32_t* rpos, RefineState* st, double tol,
                           int iter, int max_iter, int decide, int* active, cudaStream_t s, double* R64) {
  cudaError_t e = launch_residual(A, B, X, count, n, nrhs, rs, R32, rpos, R64, st, decide, 1, s);
  if (e != cudaSuccess) return e;
  k_refine_decide<<<(count + 255) / 256, 256, 0, s>>>(st, count, tol, iter, max_iter, decide, active);
  return cudaGetLastError();
}
cudaError_t mixed_matvec(const double* A, const double* X, int count, int n, int nrhs, const double* rs,
                         double* R64, RefineState* st, cudaStream_t s) {
  return launch_residual(A, nullptr, X, count, n, nrhs, rs, nullptr, nullptr, R64, st, 1, 0, s);
}
cudaError_t mixed_ferr(const double* X, const double* Xt, int count, int n, int nrhs, double* ferr,
                       cudaStream_t s) {
  k_ferr<<<count, MT, 0, s>>>(X, Xt, n, nrhs, ferr);
  return cudaGetLastError();
}
cudaError_t mixed_row_positions(const int32_t* ipiv, int count, int n, int32_t* rpos, cudaStream_t s) {
  k_row_positions<<<count, MT, 2 * sizeof(int) * (size_t)n, s>>>(ipiv, n, rpos);
  return cudaGetLastError();
}
cudaError_t mixed_mark_fp32_failures(const int32_t* info32, RefineState* st, int count, cudaStream_t s) {
  k_mark_fp32_failures<<<(count + 255) / 256, 256, 0, s>>>(info32, st, count);
  return cudaGetLastError();
}

}  // namespace nppb
