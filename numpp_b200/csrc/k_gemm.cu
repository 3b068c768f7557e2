// Row-major GEMM for the GpuVTable::gemm slot (include/numpp/backend/gpu_vtable.hpp
// in NumPP: C[m,n] = A[m,k] B[k,n], accumulated in k order per output element).
//
// FP64: 128x64 CTA tile, 8 warps of 32x32, DMMA m8n8k4; K is staged 8 deep in
// shared memory with a two-stage cp.async pipeline (global -> shared without a
// register round trip), so the next slab lands while the tensor pipe works on
// the current one.
// FP32: SIMT 64x64 tile, 4x4 outputs per thread (the float32 form of the slot).
#include <algorithm>

#include "dmma.cuh"
#include "nppb_internal.hpp"

namespace nppb {
namespace {

constexpr int BM = 128, BN = 64, BK = 8;
constexpr int NT = 256;
constexpr int AS = BK + 1;   // A slab row stride (doubles)
constexpr int BS = BN + 1;   // B slab row stride (doubles)

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int bytes = pred ? 8 : 0;  // 0 source bytes = zero fill
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// blockIdx.z walks a strided batch (sA, sB, sC elements apart; 0 for one GEMM)
__global__ void __launch_bounds__(NT)
k_gemm_f64(int64_t M, int64_t N, int64_t K, const double* __restrict__ A, int64_t lda,
           const double* __restrict__ B, int64_t ldb, double* __restrict__ C, int64_t ldc, int64_t sA,
           int64_t sB, int64_t sC, int64_t z0) {
  __shared__ double As[2][BM * AS];
  __shared__ double Bs[2][BK * BS];
  {
    const int64_t z = z0 + blockIdx.z;
    A += z * sA;
    B += z * sB;
    C += z * sC;
  }
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int64_t bm = (int64_t)blockIdx.y * BM, bn = (int64_t)blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // 4 x 2 warps

  auto load = [&](int stage, int64_t k0) {
    // A slab: BM x BK doubles
#pragma unroll
    for (int i = 0; i < (BM * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int r = idx / BK, c = idx % BK;
      const int64_t gr = bm + r, gc = k0 + c;
      const bool ok = gr < M && gc < K;
      cp_async8(&As[stage][r * AS + c], ok ? A + gr * lda + gc : A, ok);
    }
    // B slab: BK x BN doubles
#pragma unroll
    for (int i = 0; i < (BK * BN) / NT; ++i) {
      const int idx = tid + i * NT;
      const int r = idx / BN, c = idx % BN;
      const int64_t gr = k0 + r, gc = bn + c;
      const bool ok = gr < K && gc < N;
      cp_async8(&Bs[stage][r * BS + c], ok ? B + gr * ldb + gc : B, ok);
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;

  const int64_t nk = (K + BK - 1) / BK;
  if (nk > 0) load(0, 0);
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int st = kt & 1;
    if (kt + 1 < nk) {
      load(st ^ 1, (kt + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = As[st][(wm + mi * 8 + g) * AS + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[st][(kk + tq) * BS + wn + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], af[mi], bf[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int64_t row = bm + wm + mi * 8 + g;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t col = bn + wn + ni * 8 + 2 * tq + e;
        if (row < M && col < N) C[row * ldc + col] = acc[mi][ni][e];
      }
    }
  }
}

constexpr int FT = 64;
__global__ void __launch_bounds__(256)
k_gemm_f32(int64_t M, int64_t N, int64_t K, const float* __restrict__ A,
           const float* __restrict__ B, float* __restrict__ C) {
  __shared__ float As[16][FT + 1];
  __shared__ float Bs[16][FT + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t bm = (int64_t)blockIdx.y * FT, bn = (int64_t)blockIdx.x * FT;
  float acc[4][4] = {};
  for (int64_t k0 = 0; k0 < K; k0 += 16) {
    for (int i = threadIdx.x; i < FT * 16; i += 256) {
      const int r = i / 16, c = i % 16;
      const int64_t gr = bm + r, gc = k0 + c;
      As[c][r] = (gr < M && gc < K) ? A[gr * K + gc] : 0.f;
      const int rb = i / FT, cb = i % FT;
      const int64_t hr = k0 + rb, hc = bn + cb;
      Bs[rb][cb] = (hr < K && hc < N) ? B[hr * N + hc] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t r = bm + ty + 16 * i, c = bn + tx + 16 * j;
      if (r < M && c < N) C[r * N + c] = acc[i][j];
    }
}

}  // namespace

cudaError_t launch_gemm_f64(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda,
                            const double* B, int64_t ldb, double* C, int64_t ldc,
                            cudaStream_t st) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid((unsigned)((n + BN - 1) / BN), (unsigned)((m + BM - 1) / BM));
  k_gemm_f64<<<grid, NT, 0, st>>>(m, n, k, A, lda, B, ldb, C, ldc, 0, 0, 0, 0);
  return cudaGetLastError();
}

cudaError_t launch_gemm_f64_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* A,
                                    const double* B, double* C, cudaStream_t st) {
  if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
  const unsigned gx = (unsigned)((n + BN - 1) / BN), gy = (unsigned)((m + BM - 1) / BM);
  for (int64_t z0 = 0; z0 < batch; z0 += 65535) {
    const dim3 grid(gx, gy, (unsigned)std::min<int64_t>(65535, batch - z0));
    k_gemm_f64<<<grid, NT, 0, st>>>(m, n, k, A, k, B, n, C, n, m * k, k * n, m * n, z0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_gemm_f32(int64_t m, int64_t n, int64_t k, const float* A, const float* B,
                            float* C, cudaStream_t st) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid((unsigned)((n + FT - 1) / FT), (unsigned)((m + FT - 1) / FT));
  k_gemm_f32<<<grid, 256, 0, st>>>(m, n, k, A, B, C);
  return cudaGetLastError();
}

}  // namespace nppb
