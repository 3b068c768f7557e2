// Batched LU with partial pivoting for orders n <= 32: one warp per system.
//
// Lane r holds row r of A in registers for the whole factorisation. Rows never
// move: a row exchange only swaps the two lanes' `pos` labels (the row's
// position in the pivoted order), so a pivot step costs one warp argmax plus
// one shuffle per trailing column. The algorithm is the reference's unblocked
// right-looking elimination (src/linalg/linalg.cpp:48-71): at step k the pivot
// is the first position p >= k with the largest |a[p,k]| (ties go to the lower
// position, as the reference's strict '>' scan does), multipliers are
// a[i,k]/a[k,k] and the trailing update is a[i,j] -= f*a[k,j] (one FMA here).
//
// The same launch finishes the requested outputs from the registers:
//  * det  = permsign * prod U[i,i] in order i = 0..n-1   (linalg.cpp:393-407)
//  * slogdet sign / sum log|U[i,i]| in order               (linalg.cpp:408-439)
//  * X = A^-1 B: X[pos(r)] starts as B[r]; forward (unit L) and back (U)
//    substitution run across lanes, RC columns at a time  (linalg.cpp:73-90)
//  * inverse = the same solve against I                    (linalg.cpp:105-115)
//  * LU + ipiv (LAPACK-style swap list, 0-based) for getrf.
#include <cfloat>
#include <climits>
#include <cmath>

#include "nppb_internal.hpp"

namespace nppb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerCta = 4;

template <int NP, int RC>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
k_lu_warp(Batch bt, const int32_t* __restrict__ order, int nsys) {
  __shared__ int s_lane_of_pos[kWarpsPerCta][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int w = blockIdx.x * kWarpsPerCta + wib;
  if (w >= nsys) return;  // whole warp leaves together
  const int s = order ? order[w] : w;
  const SysView v = sys_view(bt, s);
  const int n = v.n;
  const int flags = bt.flags;
  const bool live = lane < n;

  double a[NP];
  if (flags & kSolveOnly) {
    // getrs from a stored factorisation: LU rows are already in pivoted order,
    // so lane r holds position r; the right-hand side is gathered through ipiv.
#pragma unroll 64
    for (int j = 0; j < NP; ++j) a[j] = (live && j < n) ? v.LU[(int64_t)lane * n + j] : 0.0;
  } else {
#pragma unroll 64
    for (int j = 0; j < NP; ++j) a[j] = (live && j < n) ? v.A[(int64_t)lane * n + j] : 0.0;
  }

  int pos = lane;
  int info = 0;
  int nswap = 0;
  double dg = 1.0;  // U[pos,pos]: set when this lane's row becomes the pivot row
  // Original row index held by each position, for getrs from stored factors.
  int orig = lane;

  if (!(flags & kSolveOnly)) {
#pragma unroll 64
    for (int k = 0; k < NP; ++k) {
      if (k >= n || info) continue;
      const bool nopiv = flags & kNoPivot;
      const bool cand = live && (nopiv ? pos == k : pos >= k);
      // without pivoting the diagonal is the only candidate; <= 0 counts as a zero pivot
      double best = cand ? (nopiv ? (a[k] > 0.0 ? a[k] : 0.0) : fabs(a[k])) : -1.0;
      int key = cand ? pos : INT_MAX;
#pragma unroll 64
      for (int off = 16; off; off >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, off);
        const int ok = __shfl_xor_sync(kFull, key, off);
        if (ob > best || (ob == best && ok < key)) { best = ob; key = ok; }
      }
      if (best == 0.0) { info = k + 1; continue; }  // exact zero pivot: singular
      const int pl = __ffs(__ballot_sync(kFull, live && pos == key)) - 1;
      const int kl = __ffs(__ballot_sync(kFull, live && pos == k)) - 1;
      if (key != k) {
        if (lane == pl) pos = k;
        else if (lane == kl) pos = key;
        ++nswap;
      }
      if ((flags & kWantLU) && lane == 0) v.ipiv[k] = key;
      const double pk = __shfl_sync(kFull, a[k], pl);
      if (lane == pl) dg = pk;
      const bool below = live && pos > k;
      double f = 0.0;
      if (below) { f = a[k] / pk; a[k] = f; }
#pragma unroll 64
      for (int j = k + 1; j < NP; ++j) {
        // columns j >= n are zero in every row, so the update leaves them zero
        const double pj = __shfl_sync(kFull, a[j], pl);
        if (below) a[j] = fma(-f, pj, a[j]);
      }
    }
  } else {
    // Replay the stored swap list to find which original row each position holds.
    // orig(lane) = perm[lane] where perm = swaps applied to the identity.
    if (lane == 0) {
      for (int i = 0; i < n; ++i) s_lane_of_pos[wib][i] = i;
      for (int k = 0; k < n; ++k) {
        int p = v.ipiv[k];
        if (p < k || p >= n) p = k;  // a swap list only names rows >= k; ignore anything else
        const int t = s_lane_of_pos[wib][k];
        s_lane_of_pos[wib][k] = s_lane_of_pos[wib][p];
        s_lane_of_pos[wib][p] = t;
      }
    }
    __syncwarp();
    orig = live ? s_lane_of_pos[wib][lane] : lane;
    __syncwarp();
  }

  if (live) s_lane_of_pos[wib][pos] = lane;
  __syncwarp();
  const int* lop = s_lane_of_pos[wib];

  if ((flags & kWantLU) && !(flags & kSolveOnly) && live) {
#pragma unroll 64
    for (int j = 0; j < NP; ++j)
      if (j < n) v.LU[(int64_t)pos * n + j] = a[j];
  }

  if ((flags & (kWantDet | kWantSlogdet)) && !(flags & kSolveOnly)) {
    const double lg = log(fabs(dg));
    double det = (nswap & 1) ? -1.0 : 1.0;
    double sgn = det;
    double logabs = 0.0;
    if (info == 0) {
      for (int i = 0; i < n; ++i) {
        const int l = lop[i];
        const double di = __shfl_sync(kFull, dg, l);
        const double li = __shfl_sync(kFull, lg, l);
        det *= di;
        logabs += li;
        sgn *= di / fabs(di);
      }
    }
    if (lane == 0) {
      if (flags & kWantDet) bt.det[v.idx] = info ? 0.0 : det;
      if (flags & kWantSlogdet) {
        bt.sign[v.idx] = info ? 0.0 : sgn;
        bt.logabs[v.idx] = info ? -INFINITY : logabs;
      }
    }
  }
  if (lane == 0 && bt.info && !(flags & kSolveOnly)) bt.info[v.idx] = info;
  if (info) return;

  // ---- substitution: X = U^-1 L^-1 P B, RC right-hand-side columns at a time ----
  for (int pass = 0; pass < 2; ++pass) {
    const bool is_inv = pass == 1;
    if (!is_inv && !(flags & kWantSolve)) continue;
    if (is_inv && (!(flags & kWantInv) || v.inv == nullptr)) continue;
    const int ncols = is_inv ? n : v.nrhs;
    for (int c0 = 0; c0 < ncols; c0 += RC) {
      double x[RC];
#pragma unroll 64
      for (int c = 0; c < RC; ++c) {
        const int col = c0 + c;
        double b = 0.0;
        if (live && col < ncols) {
          if (is_inv) b = (orig == col) ? 1.0 : 0.0;
          else b = v.B[(int64_t)orig * ncols + col];
        }
        x[c] = b;
      }
      __syncwarp();  // every lane has read its right-hand side before any lane writes X (getrs in place)
      // forward: unit lower, position order
#pragma unroll 64
      for (int k = 0; k < NP; ++k) {
        if (k >= n) continue;
        const int l = lop[k];
        const bool below = live && pos > k;
#pragma unroll 64
        for (int c = 0; c < RC; ++c) {
          const double xk = __shfl_sync(kFull, x[c], l);
          if (below) x[c] = fma(-a[k], xk, x[c]);
        }
      }
      // back: upper, divide by the diagonal when the row is final
#pragma unroll 64
      for (int k = NP - 1; k >= 0; --k) {
        if (k < n) {
          const int l = lop[k];
          if (lane == l) {
            const double rd = 1.0 / a[k];
#pragma unroll 64
            for (int c = 0; c < RC; ++c) x[c] *= rd;
          }
          const bool above = live && pos < k;
#pragma unroll 64
          for (int c = 0; c < RC; ++c) {
            const double xk = __shfl_sync(kFull, x[c], l);
            if (above) x[c] = fma(-a[k], xk, x[c]);
          }
        }
      }
      if (live) {
        double* out = is_inv ? v.inv : v.X;
#pragma unroll 64
        for (int c = 0; c < RC; ++c)
          if (c0 + c < ncols) out[(int64_t)pos * ncols + c0 + c] = x[c];
      }
    }
  }
}

template <int NP>
cudaError_t launch_np(const Batch& bt, const int32_t* order, int nsys, cudaStream_t st) {
  const int grid = (nsys + kWarpsPerCta - 1) / kWarpsPerCta;
  k_lu_warp<NP, 8><<<grid, kWarpsPerCta * 32, 0, st>>>(bt, order, nsys);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lu_warp(const Batch& bt, const int32_t* order, int nsys, int np,
                           cudaStream_t st) {
  if (nsys <= 0) return cudaSuccess;
  if (np <= 8) return launch_np<8>(bt, order, nsys, st);
  if (np <= 16) return launch_np<16>(bt, order, nsys, st);
  return launch_np<32>(bt, order, nsys, st);
}

}  // namespace nppb
