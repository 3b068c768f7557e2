// GMRES for the correction equation of the mixed solve: the Arnoldi step,
// the rotations and the final update, one CTA per instance (system,
// right-hand-side column). See gmres.hpp.
#include <cmath>

#include "gmres.hpp"

namespace nppb {
namespace {

constexpr int GT = 256;
constexpr int GW = GT / 32;

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum over GT threads (red: GW doubles); every thread gets the result.
__device__ double block_sum_d(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum_d(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = 0.0;
#pragma unroll
  for (int w = 0; w < GW; ++w) r += red[w];
  return r;
}

__device__ __forceinline__ bool refining(const RefineState* st, int s) { return st[s].status == kRefineActive; }

__global__ void __launch_bounds__(GT)
k_gm_start(const double* __restrict__ Z, double* __restrict__ V, GmState* __restrict__ gs,
           const RefineState* __restrict__ st, int n, int nrhs) {
  __shared__ double red[GW];
  const int inst = blockIdx.x, s = inst / nrhs, col = inst % nrhs, tid = threadIdx.x;
  GmState& g = gs[inst];
  if (!refining(st, s)) {
    if (tid == 0) {
      g.k = 0;
      g.done = 1;
    }
    return;
  }
  const int64_t base = (int64_t)s * n * nrhs + col;
  double m = 0.0;
  for (int i = tid; i < n; i += GT) m = fmax(m, fabs(Z[base + (int64_t)i * nrhs]));
  // max through the sum machinery: the largest magnitude first, for a scaled 2-norm
  {
    double v = m;
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    m = 0.0;
#pragma unroll
    for (int w = 0; w < GW; ++w) m = fmax(m, red[w]);
  }
  double ss = 0.0;
  if (m > 0.0 && isfinite(m))
    for (int i = tid; i < n; i += GT) {
      const double z = Z[base + (int64_t)i * nrhs] / m;
      ss = fma(z, z, ss);
    }
  const double beta = m > 0.0 && isfinite(m) ? m * sqrt(block_sum_d(ss, red)) : 0.0;
  const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
  for (int i = tid; i < n; i += GT) V[base + (int64_t)i * nrhs] = Z[base + (int64_t)i * nrhs] * inv;
  if (tid == 0) {
    g.beta = beta;
    g.g[0] = beta;
    for (int j = 1; j <= kGmM; ++j) g.g[j] = 0.0;
    g.k = 0;
    g.done = beta > 0.0 ? 0 : 1;
  }
}

// One Arnoldi step for instance (s, col): w = -W, orthogonalised against
// V_0..V_k twice (classical Gram-Schmidt: all k+1 dots from one sweep, then
// one update sweep), normalised into V_{k+1}; thread 0 rotates column k.
__global__ void __launch_bounds__(GT)
k_gm_arnoldi(const double* __restrict__ W, double* __restrict__ V, GmState* __restrict__ gs,
             const RefineState* __restrict__ st, int n, int nrhs, int k, double tau, int* __restrict__ active) {
  extern __shared__ double ws[];  // [n] the new vector
  __shared__ double red[GW][kGmM + 1];
  __shared__ double h[kGmM + 1], htot[kGmM + 1];
  __shared__ double nred[GW];
  const int inst = blockIdx.x, s = inst / nrhs, col = inst % nrhs, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  GmState& g = gs[inst];
  if (!refining(st, s) || g.done) return;
  const int64_t plane = (int64_t)gridDim.x / nrhs * n * nrhs;  // count * n * nrhs
  const int64_t base = (int64_t)s * n * nrhs + col;
  for (int i = tid; i < n; i += GT) ws[i] = -W[base + (int64_t)i * nrhs];
  if (tid <= k) htot[tid] = 0.0;
  __syncthreads();
  for (int pass = 0; pass < 2; ++pass) {
    for (int j = 0; j <= k; ++j) {
      const double* vj = V + j * plane + base;
      double p = 0.0;
      for (int i = tid; i < n; i += GT) p = fma(vj[(int64_t)i * nrhs], ws[i], p);
      p = warp_sum_d(p);
      if (lane == 0) red[warp][j] = p;
    }
    __syncthreads();
    if (tid <= k) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < GW; ++w) v += red[w][tid];
      h[tid] = v;
      htot[tid] += v;
    }
    __syncthreads();
    for (int i = tid; i < n; i += GT) {
      double x = ws[i];
      for (int j = 0; j <= k; ++j) x = fma(-h[j], V[j * plane + base + (int64_t)i * nrhs], x);
      ws[i] = x;
    }
    __syncthreads();
  }
  double ss = 0.0;
  for (int i = tid; i < n; i += GT) ss = fma(ws[i], ws[i], ss);
  const double hk1 = sqrt(block_sum_d(ss, nred));
  const double inv = hk1 > 0.0 ? 1.0 / hk1 : 0.0;
  double* vk1 = V + (k + 1) * plane + base;
  for (int i = tid; i < n; i += GT) vk1[(int64_t)i * nrhs] = ws[i] * inv;
  if (tid == 0) {
    double* Rk = g.R[k];
    for (int j = 0; j <= k; ++j) Rk[j] = htot[j];
    Rk[k + 1] = hk1;
    for (int j = 0; j < k; ++j) {  // the earlier rotations
      const double a = Rk[j], b = Rk[j + 1];
      Rk[j] = g.c[j] * a + g.sn[j] * b;
      Rk[j + 1] = -g.sn[j] * a + g.c[j] * b;
    }
    const double a = Rk[k], b = Rk[k + 1], r = hypot(a, b);
    bool fin = false;
    if (!(r > 0.0) || !isfinite(r)) {
      fin = true;  // singular least-squares column: keep the k steps before it
    } else {
      const double c = a / r, sn = b / r;
      g.c[k] = c;
      g.sn[k] = sn;
      Rk[k] = r;
      Rk[k + 1] = 0.0;
      g.g[k + 1] = -sn * g.g[k];
      g.g[k] = c * g.g[k];
      g.k = k + 1;
      fin = !(fabs(g.g[k + 1]) > tau * g.beta) || k + 1 == kGmM || !(hk1 > 0.0);
    }
    if (fin) g.done = 1;
    else atomicAdd(active, 1);
  }
}

__global__ void __launch_bounds__(GT)
k_gm_update(const double* __restrict__ V, double* __restrict__ X, const GmState* __restrict__ gs,
            const RefineState* __restrict__ st, int n, int nrhs) {
  __shared__ double y[kGmM];
  const int inst = blockIdx.x, s = inst / nrhs, col = inst % nrhs, tid = threadIdx.x;
  if (!refining(st, s)) return;
  const GmState& g = gs[inst];
  const int kk = g.k;
  if (kk == 0) return;
  if (tid == 0) {  // R y = g, upper triangular (column-major R[col][row])
    for (int i = kk - 1; i >= 0; --i) {
      double v = g.g[i];
      for (int j = i + 1; j < kk; ++j) v = fma(-g.R[j][i], y[j], v);
      y[i] = v / g.R[i][i];
    }
  }
  __syncthreads();
  const int64_t plane = (int64_t)gridDim.x / nrhs * n * nrhs;
  const int64_t base = (int64_t)s * n * nrhs + col;
  for (int i = tid; i < n; i += GT) {
    double d = 0.0;
    for (int j = 0; j < kk; ++j) d = fma(y[j], V[j * plane + base + (int64_t)i * nrhs], d);
    X[base + (int64_t)i * nrhs] += d;
  }
}

}  // namespace

cudaError_t gm_start(const double* Z, double* V, GmState* gs, const RefineState* st, int count, int n, int nrhs,
                     cudaStream_t s) {
  k_gm_start<<<(unsigned)(count * nrhs), GT, 0, s>>>(Z, V, gs, st, n, nrhs);
  return cudaGetLastError();
}

cudaError_t gm_arnoldi(const double* W, double* V, GmState* gs, const RefineState* st, int count, int n,
                       int nrhs, int k, double tau, int* active, cudaStream_t s) {
  // n <= 4096: the vector (32 KB) fits the default dynamic shared memory
  k_gm_arnoldi<<<(unsigned)(count * nrhs), GT, sizeof(double) * n, s>>>(W, V, gs, st, n, nrhs, k, tau, active);
  return cudaGetLastError();
}

cudaError_t gm_update(const double* V, double* X, const GmState* gs, const RefineState* st, int count, int n,
                      int nrhs, cudaStream_t s) {
  k_gm_update<<<(unsigned)(count * nrhs), GT, 0, s>>>(V, X, gs, st, n, nrhs);
  return cudaGetLastError();
}

}  // namespace nppb
