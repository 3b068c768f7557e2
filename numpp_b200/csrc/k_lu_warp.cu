// Batched LU with partial pivoting for orders n <= 32: one warp per system.
//
// Lane r owns row r of A, kept in shared memory (one 32 x 33 tile per warp,
// loaded coalesced) so that every loop is a rolled loop over a runtime index:
// fully unrolled code for 32 steps plus the substitutions was bound by
// instruction fetch. Rows never move: a row exchange only swaps the two lanes'
// `pos` labels (the row's position in the pivoted order). The algorithm is the
// reference's unblocked right-looking elimination (src/linalg/linalg.cpp:48-71):
// at step k the pivot is the first position p >= k with the largest |a[p,k]|
// (ties go to the lower position, as the reference's strict '>' scan does),
// found exactly by warp reductions on the bit patterns of |a| (non-negative
// doubles order like their patterns: high word, then low word, then the lowest
// position among the lanes holding both); multipliers are a[i,k]/a[k,k] and
// the trailing update is a[i,j] -= f*a[k,j] (one FMA here). NaN entries are
// never pivot candidates.
//
// The same launch finishes the requested outputs:
//  * det  = permsign * prod U[i,i] in order i = 0..n-1   (linalg.cpp:393-407)
//  * slogdet sign / sum log|U[i,i]| in order               (linalg.cpp:408-439)
//  * X = A^-1 B: X[pos(r)] starts as B[r]; forward (unit L) and back (U)
//    substitution run across lanes, up to RC columns at a time (linalg.cpp:73-90)
//  * inverse = the same solve against I                    (linalg.cpp:105-115)
//  * LU + ipiv (LAPACK-style swap list, 0-based) for getrf.
#include <cfloat>
#include <climits>
#include <cmath>

#include "nppb_internal.hpp"

namespace nppb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerCta = 2;  // small batches spread over more SMs
constexpr int kLd = 34;          // row stride of a warp's tile (doubles): columns 32, 33 are scratch

template <int NP, int RC>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
k_lu_warp(Batch bt, const int32_t* __restrict__ order, int nsys) {
  __shared__ int s_lane_of_pos[kWarpsPerCta][32];
  __shared__ __align__(16) double s_rows[kWarpsPerCta][32 * kLd];  // row r at r * kLd (16-byte aligned rows)
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int w = blockIdx.x * kWarpsPerCta + wib;
  if (w >= nsys) return;  // whole warp leaves together
  const int s = order ? order[w] : w;
  const SysView v = sys_view(bt, s);
  const int n = v.n;
  const int flags = bt.flags;
  const bool live = lane < n;
  double* R = s_rows[wib];
  double* row = R + lane * kLd;  // this lane's row

  {
    // coalesced: lane c reads column c of every row, all loads in flight before the stores
    const double* src = (flags & kSolveOnly) ? v.LU : v.A;
    double t[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) t[r] = (live && r < n) ? src[(int64_t)r * n + lane] : 0.0;
#pragma unroll
    for (int r = 0; r < 32; ++r)
      if (r < n) R[r * kLd + lane] = t[r];
  }
  __syncwarp();

  int pos = lane;
  int info = 0;
  int nswap = 0;
  double dg = 1.0;  // U[pos,pos]: set when this lane's row becomes the pivot row
  // Original row index held by each position, for getrs from stored factors.
  int orig = lane;

  if (!(flags & kSolveOnly)) {
    const bool nopiv = flags & kNoPivot;
#pragma unroll 1
    for (int k = 0; k < n; ++k) {
      const bool cand = live && (nopiv ? pos == k : pos >= k);
      const double akk = live ? row[k] : 0.0;
      // without pivoting the diagonal is the only candidate; <= 0 counts as a zero pivot
      const double mag = cand ? (nopiv ? (akk > 0.0 ? akk : 0.0) : fabs(akk)) : 0.0;
      const unsigned long long bits = (mag == mag) ? (unsigned long long)__double_as_longlong(mag) : 0ull;
      const uint32_t hi = (uint32_t)(bits >> 32), lo = (uint32_t)bits;
      const uint32_t mhi = __reduce_max_sync(kFull, hi);
      const uint32_t mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
      if ((mhi | mlo) == 0u) {  // no nonzero candidate: singular
        info = k + 1;
        break;
      }
      const bool top = cand && hi == mhi && lo == mlo;
      const int key = (int)__reduce_min_sync(kFull, top ? (uint32_t)pos : 0xffffffffu);
      const int pl = __ffs(__ballot_sync(kFull, live && pos == key)) - 1;
      const int kl = __ffs(__ballot_sync(kFull, live && pos == k)) - 1;
      if (key != k) {
        if (lane == pl) pos = k;
        else if (lane == kl) pos = key;
        ++nswap;
      }
      if ((flags & kWantLU) && lane == 0) v.ipiv[k] = key;
      const double* prow = R + pl * kLd;
      const double pk = prow[k];
      if (lane == pl) dg = pk;
      if (live && pos > k) {
        const double f = row[k] / pk;
        row[k] = f;
        // 16-byte pieces (rows start 16-byte aligned); the piece holding column k
        // keeps it, columns past n are padding
        double2* r2 = reinterpret_cast<double2*>(row);
        const double2* p2 = reinterpret_cast<const double2*>(prow);
#pragma unroll 4
        for (int q = (k + 1) >> 1; q < (n + 1) >> 1; ++q) {
          const double2 pv = p2[q];
          double2 rv = r2[q];
          if (2 * q > k) rv.x = fma(-f, pv.x, rv.x);
          rv.y = fma(-f, pv.y, rv.y);
          r2[q] = rv;
        }
      }
      __syncwarp();
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

  if ((flags & kWantLU) && !(flags & kSolveOnly)) {
    // row-major by position (the partial factors too when a pivot was zero), coalesced
#pragma unroll 4
    for (int p = 0; p < n; ++p)
      if (live) v.LU[(int64_t)p * n + lane] = R[lop[p] * kLd + lane];
  }

  if ((flags & (kWantDet | kWantSlogdet)) && !(flags & kSolveOnly)) {
    // the pivots and their logs by position (the tile's padding column), folded in
    // position order by lane 0: the reference's sequence of products and sums
    double* dgs = R + 32;  // column 32 of the tile: rows 0..n-1 hold the pivot of position r
    if (live) {
      dgs[pos * kLd] = dg;
      dgs[pos * kLd + 1] = log(fabs(dg));  // column 33
    }
    __syncwarp();
    double det = (nswap & 1) ? -1.0 : 1.0;
    double sgn = det;
    double logabs = 0.0;
    if (info == 0 && lane == 0) {
      for (int i = 0; i < n; ++i) {
        const double di = dgs[i * kLd], li = dgs[i * kLd + 1];
        det *= di;
        logabs += li;
        // d / |d| is exactly +-1 for finite nonzero d, NaN otherwise
        sgn = isfinite(di) ? (di < 0.0 ? -sgn : sgn) : NAN;
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

  // ---- substitution: X = U^-1 L^-1 P B, up to RC right-hand-side columns at a time ----
  const double rdg = live ? 1.0 / row[pos] : 0.0;  // this row's diagonal of U, inverted once
  for (int pass = 0; pass < 2; ++pass) {
    const bool is_inv = pass == 1;
    if (!is_inv && !(flags & kWantSolve)) continue;
    if (is_inv && (!(flags & kWantInv) || v.inv == nullptr)) continue;
    const int ncols = is_inv ? n : v.nrhs;
    for (int c0 = 0; c0 < ncols; c0 += RC) {
      const int nc = min(RC, ncols - c0);  // columns of this chunk (warp-uniform)
      double x[RC];
#pragma unroll
      for (int c = 0; c < RC; ++c) {
        const int col = c0 + c;
        double b = 0.0;
        if (live && c < nc) {
          if (is_inv) b = (orig == col) ? 1.0 : 0.0;
          else b = v.B[(int64_t)orig * ncols + col];
        }
        x[c] = b;
      }
      __syncwarp();  // every lane has read its right-hand side before any lane writes X (getrs in place)
      // forward: unit lower, position order
#pragma unroll 1
      for (int k = 0; k < n; ++k) {
        const int l = lop[k];
        const bool below = live && pos > k;
        const double lk = below ? row[k] : 0.0;
#pragma unroll
        for (int c = 0; c < RC; ++c) {
          if (c < nc) {
            const double xk = __shfl_sync(kFull, x[c], l);
            if (below) x[c] = fma(-lk, xk, x[c]);
          }
        }
      }
      // back: upper, multiply by the diagonal's reciprocal when the row is final
#pragma unroll 1
      for (int k = n - 1; k >= 0; --k) {
        const int l = lop[k];
        if (lane == l) {
#pragma unroll
          for (int c = 0; c < RC; ++c) x[c] *= rdg;
        }
        const bool above = live && pos < k;
        const double uk = above ? row[k] : 0.0;
#pragma unroll
        for (int c = 0; c < RC; ++c) {
          if (c < nc) {
            const double xk = __shfl_sync(kFull, x[c], l);
            if (above) x[c] = fma(-uk, xk, x[c]);
          }
        }
      }
      if (live) {
        double* out = is_inv ? v.inv : v.X;
#pragma unroll
        for (int c = 0; c < RC; ++c)
          if (c < nc) out[(int64_t)pos * ncols + c0 + c] = x[c];
      }
    }
  }
}

template <int NP>
cudaError_t launch_np(const Batch& bt, const int32_t* order, int nsys, cudaStream_t st) {
  const int grid = (nsys + kWarpsPerCta - 1) / kWarpsPerCta;
  // one right-hand-side column and no inverse (a uniform batch says so): the one-column substitution
  if (!bt.desc && bt.nrhs <= 1 && !(bt.flags & kWantInv))
    k_lu_warp<NP, 1><<<grid, kWarpsPerCta * 32, 0, st>>>(bt, order, nsys);
  else
    k_lu_warp<NP, 8><<<grid, kWarpsPerCta * 32, 0, st>>>(bt, order, nsys);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lu_warp(const Batch& bt, const int32_t* order, int nsys, int np,
                           cudaStream_t st) {
  if (nsys <= 0) return cudaSuccess;
  (void)np;  // one kernel for every order <= 32: its loops run over the order at run time
  return launch_np<32>(bt, order, nsys, st);
}

}  // namespace nppb
