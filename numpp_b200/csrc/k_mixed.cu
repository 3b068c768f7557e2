// Kernels of the mixed-precision solve (FP32 factors, FP64 refinement).
//
// No counterpart in the reference, which solves in double only
// (src/linalg/linalg.cpp:20-26,92-103). Per system of a uniform batch:
//  k_equilibrate  power-of-two row and column scales r, c (exact in FP64) so
//                 that every row and column of diag(r) A diag(c) peaks in
//                 [1, 2); writes that matrix in FP32 and ||A||_inf
//  k_scale_rhs    r * B in FP32 (the first right-hand side), ||B||_max
//  k_apply        X = c * Y (first solution) or X += c * Y (correction), FP64
//  k_residual     R = B - A X in FP64, eta = max|R| / (||A||_inf max|X| + max|B|)
//                 (normwise backward error), r * R in FP32 for the next
//                 correction, and the convergence / stall decision
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

__global__ void __launch_bounds__(MT)
k_equilibrate(const double* __restrict__ A, int n, int equil, float* __restrict__ A32,
              double* __restrict__ rs, double* __restrict__ cs, RefineState* __restrict__ st) {
  __shared__ double rsc[kMixedMaxN];
  __shared__ double red[MT / 32];
  const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* a = A + (int64_t)s * n * n;
  double arow = 0.0;
  for (int i = warp; i < n; i += MT / 32) {
    double m = 0.0, sum = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double v = fabs(a[(int64_t)i * n + j]);
      m = fmax(m, v);
      sum += v;
    }
    m = warp_max(m);
    sum = warp_sum(sum);
    if (lane == 0) rsc[i] = equil ? pow2_scale(m) : 1.0;
    arow = fmax(arow, sum);
  }
  const double anorm = block_max(arow, red);  // includes the barrier publishing rsc
  for (int j = tid; j < n; j += MT) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, rsc[i] * fabs(a[(int64_t)i * n + j]));
    cs[(int64_t)s * n + j] = equil ? pow2_scale(m) : 1.0;
  }
  for (int i = tid; i < n; i += MT) rs[(int64_t)s * n + i] = rsc[i];
  __syncthreads();
  const double* c = cs + (int64_t)s * n;
  float* a32 = A32 + (int64_t)s * n * n;
  for (int64_t idx = tid; idx < (int64_t)n * n; idx += MT) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    a32[idx] = (float)(rsc[i] * a[idx] * c[j]);
  }
  if (tid == 0) {
    st[s].anorm = anorm;
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
  const double* b = B + (int64_t)s * nb;
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

// One CTA per system; right-hand sides in chunks of 8 held in shared memory,
// one warp per row of A (coalesced row reads, shuffle reductions).
constexpr int RC = 8;

__global__ void __launch_bounds__(MT)
k_residual(const double* __restrict__ A, const double* __restrict__ B, const double* __restrict__ X,
           int n, int nrhs, const double* __restrict__ rs, float* __restrict__ R32,
           RefineState* __restrict__ st, double tol, int iter, int decide, int* __restrict__ active) {
  __shared__ double xs[kMixedMaxN * RC];
  __shared__ double red[MT / 32];
  __shared__ double ax_s[MT / 32][RC];
  const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (decide && st[s].status != kRefineActive) return;
  const int64_t nb = (int64_t)n * nrhs;
  const double* a = A + (int64_t)s * n * n;
  const double* b = B + (int64_t)s * nb;
  const double* x = X + (int64_t)s * nb;
  double rmax = 0.0, xmax = 0.0;
  for (int k0 = 0; k0 < nrhs; k0 += RC) {
    const int kc = min(RC, nrhs - k0);
    __syncthreads();
    for (int idx = tid; idx < n * RC; idx += MT) {
      const int j = idx / RC, k = idx % RC;
      const double v = k < kc ? x[(int64_t)j * nrhs + k0 + k] : 0.0;
      xs[idx] = v;
      xmax = fmax(xmax, fabs(v));
    }
    __syncthreads();
    for (int i = warp; i < n; i += MT / 32) {
      double acc[RC];
#pragma unroll
      for (int k = 0; k < RC; ++k) acc[k] = 0.0;
      for (int j = lane; j < n; j += 32) {
        const double aij = a[(int64_t)i * n + j];
#pragma unroll
        for (int k = 0; k < RC; ++k) acc[k] = fma(aij, xs[j * RC + k], acc[k]);
      }
#pragma unroll
      for (int k = 0; k < RC; ++k) acc[k] = warp_sum(acc[k]);
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < RC; ++k) ax_s[warp][k] = acc[k];
      }
      __syncwarp();
      if (lane < kc) {
        const double ax = ax_s[warp][lane];
        const double r = b[(int64_t)i * nrhs + k0 + lane] - ax;
        rmax = fmax(rmax, fabs(r));
        if (R32) R32[(int64_t)s * nb + (int64_t)i * nrhs + k0 + lane] = (float)(rs[(int64_t)s * n + i] * r);
      }
      __syncwarp();
    }
  }
  rmax = block_max(rmax, red);
  xmax = block_max(xmax, red);
  if (tid == 0) {
    RefineState& q = st[s];
    const double eta = rmax / (q.anorm * xmax + q.bnorm);
    q.eta = eta;
    if (decide) {
      q.iters = iter;
      if (eta <= tol) {
        q.status = kRefineConverged;
      } else if (iter > 0 && !(eta <= 0.5 * q.prev)) {
        q.status = kRefineStalled;  // not halving any more (or NaN): refinement has stalled
      } else {
        atomicAdd(active, 1);
      }
      q.prev = eta;
    }
  }
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

__global__ void k_mark_fp32_failures(const int32_t* __restrict__ info32, RefineState* __restrict__ st, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < count && info32[s]) st[s].status = kRefineStalled;
}

}  // namespace

cudaError_t mixed_equilibrate(const double* A, int count, int n, int equil, float* A32, double* rs, double* cs,
                              RefineState* st, cudaStream_t s) {
  k_equilibrate<<<count, MT, 0, s>>>(A, n, equil, A32, rs, cs, st);
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
cudaError_t mixed_residual(const double* A, const double* B, const double* X, int count, int n, int nrhs,
                           const double* rs, float* R32, RefineState* st, double tol, int iter, int decide,
                           int* active, cudaStream_t s) {
  k_residual<<<count, MT, 0, s>>>(A, B, X, n, nrhs, rs, R32, st, tol, iter, decide, active);
  return cudaGetLastError();
}
cudaError_t mixed_ferr(const double* X, const double* Xt, int count, int n, int nrhs, double* ferr,
                       cudaStream_t s) {
  k_ferr<<<count, MT, 0, s>>>(X, Xt, n, nrhs, ferr);
  return cudaGetLastError();
}
cudaError_t mixed_mark_fp32_failures(const int32_t* info32, RefineState* st, int count, cudaStream_t s) {
  k_mark_fp32_failures<<<(count + 255) / 256, 256, 0, s>>>(info32, st, count);
  return cudaGetLastError();
}

}  // namespace nppb
