// Batched LU with partial pivoting for 32 < n <= 512: one CTA (8 warps) per
// system, persistent over the systems of one size class.
//
// Blocked right-looking LU (panel width NB = 32) in the LU workspace in global
// memory (L2-resident while the CTA works on it):
//   1. the n-k0 x 32 panel is staged in shared memory and factored there with
//      the reference's pivot rule (first largest |a|, src/linalg/linalg.cpp:55-57);
//      two barriers per column: the rows a thread scans for the argmax are the
//      rows it updated in the previous column, so no barrier sits between them;
//   2. the panel's row exchanges are applied to the columns left and right of it;
//   3. U12 = L11^-1 A12 per 256-column strip (a thread per column, registers);
//   4. A22 -= L21 U12 on FP64 DMMA (mma.m8n8k4), 32x32 warp tiles whose
//      accumulators are loaded from and stored back to the workspace.
// det / slogdet come from the pivots kept in shared memory during step 1
// (product and log-sum in the reference's order i = 0..n-1, linalg.cpp:393-439).
// getrs (linalg.cpp:73-90) runs per 32-column chunk of the right-hand side in
// shared memory: gather through the row permutation, blocked forward
// substitution with unit L, blocked back substitution with U. The inverse is the
// same solve against I (linalg.cpp:105-115).
#include <cmath>

#include "dmma.cuh"
#include "nppb_internal.hpp"

namespace nppb {
namespace {

constexpr int NB = 32;         // panel width
constexpr int NT = 256;        // threads per CTA
constexpr int SW = 256;        // trailing strip width (one column per thread)
constexpr int PS = NB + 1;     // panel row stride (doubles)
constexpr int XS = 33;         // right-hand-side chunk row stride
constexpr int TS = 33;         // diagonal-block tile stride

struct Smem {
  double* P;      // (nmax + 32) x PS   panel, later the RHS chunk
  double* Us;     // NB x us            U12 strip, later the diagonal block / logs
  double* diag;   // nmax               pivots U[i,i]
  double* red_v;  // 8
  int* perm;      // nmax               original row at each position
  int* lpiv;      // NB                 panel-local pivot rows
  int* red_i;     // 8
  int* ctl;       // 4: [0] info, [1] swap count
  int us;         // U12 strip row stride: min(SW, nmax rounded to 32) + 1
};

__host__ __device__ inline int strip_stride(int nmax) {
  const int r = (nmax + 31) / 32 * 32;
  return (r < SW ? r : SW) + 1;
}

__host__ __device__ inline size_t smem_bytes(int nmax) {
  return sizeof(double) * ((size_t)(nmax + 32) * PS + (size_t)NB * strip_stride(nmax) + nmax + 8) +
         sizeof(int) * ((size_t)nmax + NB + 8 + 4);
}

__device__ inline Smem carve(double* base, int nmax) {
  Smem s;
  s.P = base;
  s.us = strip_stride(nmax);
  s.Us = s.P + (size_t)(nmax + 32) * PS;
  s.diag = s.Us + (size_t)NB * s.us;
  s.red_v = s.diag + nmax;
  s.perm = reinterpret_cast<int*>(s.red_v + 8);
  s.lpiv = s.perm + nmax;
  s.red_i = s.lpiv + NB;
  s.ctl = s.red_i + 8;
  return s;
}

// ---------------------------------------------------------------------------
// Factorisation. Returns info (0 or first zero-pivot position + 1).
__device__ int factor(const SysView& v, const Smem& s, bool keep_piv) {
  const int n = v.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* LU = v.LU;
  if (tid == 0) { s.ctl[0] = 0; s.ctl[1] = 0; }

  for (int k0 = 0; k0 < n; k0 += NB) {
    const int kb = min(NB, n - k0);
    const int m = n - k0;
    // -- 1. stage the panel
    for (int idx = tid; idx < m * NB; idx += NT) {
      const int r = idx >> 5, c = idx & 31;
      s.P[r * PS + c] = (c < kb) ? LU[(int64_t)(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    // -- factor it
    for (int j = 0; j < kb; ++j) {
      double best = -1.0;
      int bi = INT_MAX;
      for (int r = j + tid; r < m; r += NT) {
        const double x = fabs(s.P[r * PS + j]);
        if (x > best) { best = x; bi = r; }
      }
      warp_argmax(best, bi);
      if (lane == 0) { s.red_v[warp] = best; s.red_i[warp] = bi; }
      __syncthreads();
      if (warp == 0) {
        double b2 = lane < NT / 32 ? s.red_v[lane] : -1.0;
        int i2 = lane < NT / 32 ? s.red_i[lane] : INT_MAX;
        warp_argmax(b2, i2);
        if (b2 == 0.0) {
          if (lane == 0) s.ctl[0] = k0 + j + 1;
        } else {
          // row exchange inside the panel (all NB columns: L part included)
          if (i2 != j) {
            const double t = s.P[j * PS + lane];
            s.P[j * PS + lane] = s.P[i2 * PS + lane];
            s.P[i2 * PS + lane] = t;
          }
          __syncwarp();
          if (lane == 0) {
            s.lpiv[j] = i2;
            s.diag[k0 + j] = s.P[j * PS + j];
            if (keep_piv) v.ipiv[k0 + j] = k0 + i2;
            if (i2 != j) {
              s.ctl[1] += 1;
              const int t = s.perm[k0 + j];
              s.perm[k0 + j] = s.perm[k0 + i2];
              s.perm[k0 + i2] = t;
            }
          }
        }
      }
      __syncthreads();
      if (s.ctl[0]) return s.ctl[0];
      const double pv = s.P[j * PS + j];
      for (int r = j + 1 + tid; r < m; r += NT) {
        double* row = s.P + r * PS;
        const double f = row[j] / pv;
        row[j] = f;
        for (int c = j + 1; c < kb; ++c) row[c] = fma(-f, s.P[j * PS + c], row[c]);
      }
      // no barrier: the next argmax reads only rows this thread just updated
    }
    __syncthreads();
    // write the factored panel back
    for (int idx = tid; idx < m * NB; idx += NT) {
      const int r = idx >> 5, c = idx & 31;
      if (c < kb) LU[(int64_t)(k0 + r) * n + k0 + c] = s.P[r * PS + c];
    }
    // -- 2. apply the panel's exchanges to the other columns (column per thread)
    for (int c = tid; c < n; c += NT) {
      if (c >= k0 && c < k0 + kb) continue;
      for (int j = 0; j < kb; ++j) {
        const int p = s.lpiv[j];
        if (p != j) {
          double* a = LU + (int64_t)(k0 + j) * n + c;
          double* b = LU + (int64_t)(k0 + p) * n + c;
          const double t = *a; *a = *b; *b = t;
        }
      }
    }
    __syncthreads();
    if (k0 + kb >= n) break;
    // -- 3/4. trailing update in strips of SW columns (kb == NB here)
    const int mrows = m - NB;
    const int tm = (mrows + 31) >> 5;
    for (int cs = k0 + NB; cs < n; cs += SW) {
      const int sw = min(SW, n - cs);
      if (tid < sw) {
        const int c = cs + tid;
        double u[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) u[r] = LU[(int64_t)(k0 + r) * n + c];
#pragma unroll
        for (int r = 1; r < NB; ++r) {
#pragma unroll
          for (int q = 0; q < r; ++q) u[r] = fma(-s.P[r * PS + q], u[q], u[r]);
        }
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          LU[(int64_t)(k0 + r) * n + c] = u[r];
          s.Us[r * s.us + tid] = u[r];
        }
      }
      __syncthreads();
      const int tn = (sw + 31) >> 5;
      const int g = lane >> 2, tq = lane & 3;
      for (int t = warp; t < tm * tn; t += NT / 32) {
        const int r0 = (t / tn) * 32, c0 = (t % tn) * 32;
        double acc[4][4][2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          const int row = k0 + NB + r0 + mi * 8 + g;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = cs + c0 + ni * 8 + 2 * tq + e;
              acc[mi][ni][e] = (row < n && col < cs + sw) ? LU[(int64_t)row * n + col] : 0.0;
            }
          }
        }
#pragma unroll
        for (int kk = 0; kk < NB; kk += 4) {
          double af[4], bf[4];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) af[mi] = -s.P[(NB + r0 + mi * 8 + g) * PS + kk + tq];
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) bf[ni] = s.Us[(kk + tq) * s.us + c0 + ni * 8 + g];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], af[mi], bf[ni]);
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          const int row = k0 + NB + r0 + mi * 8 + g;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = cs + c0 + ni * 8 + 2 * tq + e;
              if (row < n && col < cs + sw) LU[(int64_t)row * n + col] = acc[mi][ni][e];
            }
          }
        }
      }
      __syncthreads();
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Triangular solves on a CW-column chunk Xs (n x XS) in shared memory.
template <int CW>
__device__ void trsv_chunk(const double* __restrict__ LU, int n, double* Xs, double* T, int cw) {
  const int tid = threadIdx.x;
  // forward: unit lower, top to bottom
  for (int kb0 = 0; kb0 < n; kb0 += 32) {
    const int kb1 = min(kb0 + 32, n), bw = kb1 - kb0;
    for (int idx = tid; idx < 32 * 32; idx += NT) {
      const int i = idx >> 5, q = idx & 31;
      T[i * TS + q] = (i < bw && q < bw) ? LU[(int64_t)(kb0 + i) * n + kb0 + q] : 0.0;
    }
    __syncthreads();
    if (tid < cw) {
      for (int i = 1; i < bw; ++i) {
        double x = Xs[(kb0 + i) * XS + tid];
        for (int q = 0; q < i; ++q) x = fma(-T[i * TS + q], Xs[(kb0 + q) * XS + tid], x);
        Xs[(kb0 + i) * XS + tid] = x;
      }
    }
    __syncthreads();
    for (int i = kb1 + tid; i < n; i += NT) {
      double acc[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) acc[c] = Xs[i * XS + c];
      const double* lrow = LU + (int64_t)i * n + kb0;
      for (int q = 0; q < bw; ++q) {
        const double l = lrow[q];
#pragma unroll
        for (int c = 0; c < CW; ++c) acc[c] = fma(-l, Xs[(kb0 + q) * XS + c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < CW; ++c) Xs[i * XS + c] = acc[c];
    }
    __syncthreads();
  }
  // back: upper, bottom to top
  for (int kb0 = ((n - 1) / 32) * 32; kb0 >= 0; kb0 -= 32) {
    const int kb1 = min(kb0 + 32, n), bw = kb1 - kb0;
    for (int idx = tid; idx < 32 * 32; idx += NT) {
      const int i = idx >> 5, q = idx & 31;
      T[i * TS + q] = (i < bw && q < bw) ? LU[(int64_t)(kb0 + i) * n + kb0 + q] : 0.0;
    }
    __syncthreads();
    if (tid < cw) {
      for (int i = bw - 1; i >= 0; --i) {
        double x = Xs[(kb0 + i) * XS + tid];
        for (int q = i + 1; q < bw; ++q) x = fma(-T[i * TS + q], Xs[(kb0 + q) * XS + tid], x);
        Xs[(kb0 + i) * XS + tid] = x / T[i * TS + i];
      }
    }
    __syncthreads();
    for (int i = tid; i < kb0; i += NT) {
      double acc[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) acc[c] = Xs[i * XS + c];
      const double* urow = LU + (int64_t)i * n + kb0;
      for (int q = 0; q < bw; ++q) {
        const double u = urow[q];
#pragma unroll
        for (int c = 0; c < CW; ++c) acc[c] = fma(-u, Xs[(kb0 + q) * XS + c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < CW; ++c) Xs[i * XS + c] = acc[c];
    }
    __syncthreads();
  }
}

// X[:, c0:c0+cw] for one right-hand-side chunk: gather, solve, scatter.
// src == nullptr means the identity (inverse).
__device__ void solve_chunk(const SysView& v, const Smem& s, const double* src, double* dst,
                            int ld, int c0, int cw) {
  const int n = v.n, tid = threadIdx.x;
  double* Xs = s.P;
  for (int idx = tid; idx < n * 32; idx += NT) {
    const int p = idx >> 5, c = idx & 31;
    double x = 0.0;
    if (c < cw) {
      const int r = s.perm[p];
      x = src ? src[(int64_t)r * ld + c0 + c] : (r == c0 + c ? 1.0 : 0.0);
    }
    Xs[p * XS + c] = x;
  }
  __syncthreads();
  if (cw == 1) trsv_chunk<1>(v.LU, n, Xs, s.Us, cw);
  else if (cw <= 8) trsv_chunk<8>(v.LU, n, Xs, s.Us, cw);
  else trsv_chunk<32>(v.LU, n, Xs, s.Us, cw);
  for (int idx = tid; idx < n * 32; idx += NT) {
    const int p = idx >> 5, c = idx & 31;
    if (c < cw) dst[(int64_t)p * ld + c0 + c] = Xs[p * XS + c];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(NT, 1)
k_lu_cta(Batch bt, const int32_t* __restrict__ order, int nsys, int nmax) {
  extern __shared__ __align__(16) double smem_raw[];
  const Smem s = carve(smem_raw, nmax);
  const int tid = threadIdx.x;
  const int flags = bt.flags;
  for (int w = blockIdx.x; w < nsys; w += gridDim.x) {
    const int sidx = order ? order[w] : w;
    const SysView v = sys_view(bt, sidx);
    const int n = v.n;
    int info = 0;
    if (flags & kSolveOnly) {
      if (tid == 0) {
        for (int i = 0; i < n; ++i) s.perm[i] = i;
        for (int k = 0; k < n; ++k) {
          int p = v.ipiv[k];
          if (p < k || p >= n) p = k;  // a swap list only names rows >= k; ignore anything else
          const int t = s.perm[k]; s.perm[k] = s.perm[p]; s.perm[p] = t;
        }
      }
      __syncthreads();
    } else {
      if (!(flags & kInPlace)) {
        const int64_t nn = (int64_t)n * n;
        for (int64_t i = tid; i < nn; i += NT) v.LU[i] = v.A[i];
      }
      for (int i = tid; i < n; i += NT) s.perm[i] = i;
      __syncthreads();
      info = factor(v, s, (flags & kWantLU) != 0);
      __syncthreads();
      if (flags & (kWantDet | kWantSlogdet)) {
        double* lg = s.Us;
        for (int i = tid; i < n; i += NT) lg[i] = log(fabs(s.diag[i]));
        __syncthreads();
        if (tid == 0) {
          double det = (s.ctl[1] & 1) ? -1.0 : 1.0, sgn = det, la = 0.0;
          if (!info) {
            for (int i = 0; i < n; ++i) {
              const double d = s.diag[i];
              det *= d;
              la += lg[i];
              sgn *= d / fabs(d);
            }
          }
          if (flags & kWantDet) bt.det[v.idx] = info ? 0.0 : det;
          if (flags & kWantSlogdet) {
            bt.sign[v.idx] = info ? 0.0 : sgn;
            bt.logabs[v.idx] = info ? -INFINITY : la;
          }
        }
      }
      if (tid == 0 && bt.info) bt.info[v.idx] = info;
      __syncthreads();
    }
    if (!info) {
      if ((flags & kWantSolve) && v.nrhs > 0) {
        const bool in_place = (flags & kSolveOnly) && v.B == v.X;
        for (int c0 = 0; c0 < v.nrhs; c0 += 32) {
          // in-place getrs: gather from X itself is safe only chunk-wise via smem
          solve_chunk(v, s, in_place ? v.X : v.B, v.X, v.nrhs, c0, min(32, v.nrhs - c0));
        }
      }
      if ((flags & kWantInv) && v.inv) {
        for (int c0 = 0; c0 < n; c0 += 32) solve_chunk(v, s, nullptr, v.inv, n, c0, min(32, n - c0));
      }
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t lu_cta_prepare() {
  return cudaFuncSetAttribute(k_lu_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_bytes(kCtaMaxN));
}

int lu_cta_blocks_per_sm(int nmax) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_cta, NT, smem_bytes(nmax)) !=
      cudaSuccess)
    return 1;
  return per_sm < 1 ? 1 : per_sm;
}

cudaError_t launch_lu_cta(const Batch& bt, const int32_t* order, int nsys, int nmax, int grid,
                          cudaStream_t st) {
  if (nsys <= 0) return cudaSuccess;
  if (nmax < 1 || nmax > kCtaMaxN || grid < 1) return cudaErrorInvalidValue;
  k_lu_cta<<<grid, NT, smem_bytes(nmax), st>>>(bt, order, nsys, nmax);
  return cudaGetLastError();
}

}  // namespace nppb
