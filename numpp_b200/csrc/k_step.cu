// Step-wise batched LU for orders n > 32 (any mix of orders in one batch).
//
// The reference factors one matrix at a time with an unblocked right-looking
// elimination (src/linalg/linalg.cpp:48-71) and then solves (:73-90). Here the
// same elimination is blocked by 32-column panels and run for every system of
// the batch at once, one step (panel) per pair of launches:
//
//  k_panel   one CTA (n - k0 <= 512) or one thread-block cluster of 2..8 CTAs
//            (up to 4096 rows) per active system: the (n-k0) x 32 panel lives in
//            registers (row r of the panel in thread r mod NT of CTA r / (NT*RPT)),
//            the pivot of each column is the first largest |a| in position order
//            (the reference's rule, linalg.cpp:55-57) found with one barrier per
//            column (plus one cluster barrier, the CTAs' candidates exchanged
//            through distributed shared memory); a row exchange only swaps the
//            two rows' position labels. It writes the panel at its pivoted
//            positions, the pivots, L11^-1 (for the update) and the row moves the
//            panel implies for every other column, and folds the pivots into
//            det / slogdet in the reference's order.
//  k_rows    one CTA per (system, 64-column strip) of the trailing matrix, of
//            the right-hand sides (augmented columns: forward substitution rides
//            along) and of the identity (inverse): apply the row moves and
//            write U12 = L11^-1 A12.
//  k_update  one CTA per (strip, 512 rows below the panel): A22 -= L21 U12.
//  k_back    one CTA per (system, 64-column strip) of X / inverse: blocked back
//            substitution with U (diagonal blocks by substitution) inside a
//            256-row window; k_back_update then applies the solved window to
//            every row above it, one CTA per (strip, 64-row tile). Windows run
//            from the bottom, one pass per window.
//  k_forward getrs from stored factors: k_permute gathers the rows through the
//            pivots, then windows from the top with the unit-lower L
//            (k_forward + k_forward_update).
//
// Every kernel is instantiated for FP64 factors (tile products on the FP64
// tensor pipe, mma.m8n8k4) and for FP32 factors (the mixed-precision path:
// tile products on FP32 FMA). Step 0 reads A / B / I directly and writes the
// workspace, so no copy pass is needed. Exact-zero pivots stop the system
// (info = k+1) and later launches skip it, as the reference stops
// (linalg.cpp:56).
#include <cooperative_groups.h>

#include <climits>
#include <cmath>
#include <type_traits>

#include <cuda_bf16.h>

#include "dmma.cuh"
#include "nppb_step.hpp"

namespace nppb {
namespace {

constexpr int NB = kStepNB;  // 32
constexpr int LS = NB + 1;   // 33: stride of 32-wide shared tiles
constexpr int WS = 64 + 1;   // 65: stride of 64-wide shared tiles
constexpr int UT = 128;      // threads of the strip kernels
constexpr int SB = 256;      // rows of one substitution window

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// System descriptor: from the list, or derived for a uniform batch.
template <class T>
__device__ __forceinline__ SysDesc step_desc(const StepArgsT<T>& sa, int s) {
  if (sa.desc) return sa.desc[s];
  SysDesc d;
  const int64_t n = sa.un, nn = n * n;
  d.n = sa.un;
  d.nrhs = sa.unrhs;
  d.idx = s;
  d.pad_ = s;
  d.a_off = s * nn;
  d.lu_off = s * nn;
  d.b_off = s * n * sa.unrhs;
  d.inv_off = sa.uinv ? s * nn : -1;
  d.piv_off = s * n;
  return d;
}

template <class T>
__device__ __forceinline__ StepItem uniform_item(const StepArgsT<T>& sa, int b, int k0, bool back) {
  const int n = sa.un;
  StepItem it;
  it.pad_ = 0;
  if (sa.utrail) {  // trailing pass of a two-level factorisation: matrix strips right of the block
    const int per = trailing_strips(n, sa.ubend);
    it.sys = b / per;
    it.kind = kSegMatrix;
    it.c0 = sa.ubend + 64 * (b % per);
    it.width = (int16_t)min(64, n - it.c0);
    return it;
  }
  const bool blk = sa.ubend > 0 && !back;
  const int mend = blk ? sa.ubend : n;  // matrix strips end here
  const int trail = mend - k0 - NB;
  const int nm = back ? 0 : (trail > 0 ? (trail + 63) / 64 : 0);
  const int nr = (sa.unrhs + 63) / 64;
  const int ni = sa.uinv ? (n + 63) / 64 : 0;
  const int lo = (blk && !sa.uleft) ? sa.ubbeg : 0;  // moves-only strips from here to the panel
  const int nl = (!back && (sa.uleft || blk) && k0 > lo) ? (k0 - lo + 63) / 64 : 0;
  const int per = nm + nr + ni + nl;
  it.sys = b / per;
  int r = b % per;
  if (r < nm) {
    it.kind = kSegMatrix;
    it.c0 = k0 + NB + 64 * r;
    it.width = (int16_t)min(64, mend - it.c0);
  } else if ((r -= nm) < nr) {
    it.kind = kSegRhs;
    it.c0 = 64 * r;
    it.width = (int16_t)min(64, sa.unrhs - it.c0);
  } else if ((r -= nr) < ni) {
    it.kind = kSegInv;
    it.c0 = 64 * r;
    it.width = (int16_t)min(64, n - it.c0);
  } else {
    r -= ni;
    it.kind = kSegLeft;
    it.c0 = lo + 64 * r;
    it.width = (int16_t)min(64, k0 - it.c0);
  }
  return it;
}

template <class T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };
template <class T>
__device__ __forceinline__ typename Pair<T>::type make_pair2(T x, T y) {
  typename Pair<T>::type p;
  p.x = x;
  p.y = y;
  return p;
}

// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool pred) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gmem), "n"(BYTES),
               "r"(pred ? BYTES : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Pivot candidate of one column among this warp's rows: the first largest
// |a| in position order over rows at or below position j (the reference's
// rule, linalg.cpp:55-57), reduced over the warp; without pivoting, the row at
// position j. The thread holding it also returns 1 / value in rp (the
// multiplier scale if it wins).
template <class T, int RPT>
__device__ __forceinline__ void column_candidate(const T (&v)[RPT], const int (&pos)[RPT], const bool (&valid)[RPT],
                                                 int j, T& best, int& key, T& rp, bool nopiv) {
  best = T(-1);
  key = INT_MAX;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (nopiv) {
      // no row exchanges (the LU behind cholesky): the diagonal is the only
      // candidate, and a value <= 0 counts as a zero pivot
      if (valid[q] && pos[q] == j) { best = v[q] > T(0) ? v[q] : T(0); key = j; }
    } else if (valid[q] && pos[q] >= j) {
      const T x = fabs(v[q]);
      if (x > best || (x == best && pos[q] < key)) { best = x; key = pos[q]; }
    }
  }
  warp_argmax_abs(best, key);
  rp = T(0);
#pragma unroll
  for (int q = 0; q < RPT; ++q)
    if (valid[q] && pos[q] == key) rp = T(1) / v[q];
}

// k_panel
// CS CTAs per system (a cluster when CS > 1); CTA `rank` holds panel rows
// [rank*NT*RPT, (rank+1)*NT*RPT). Rank 0 holds the top rows and does the
// per-panel bookkeeping (pivots, L11^-1, det, row moves of the top rows).
// The panel moves between global memory and registers through a shared
// staging tile (whole rows per warp: coalesced); the column loop is fully
// unrolled, so every register index and every column range is static.
template <class T, int NT, int RPT>
constexpr size_t panel_smem() {
  return sizeof(T) * (size_t)NT * RPT * (NB + 1) + sizeof(int) * (size_t)NT * RPT;
}

template <class T, int NT, int RPT, int CS>
__global__ void __launch_bounds__(NT, (RPT == 1 ? 65536 / (NT * 128) : 1))
k_panel(StepArgsT<T> sa, const int32_t* __restrict__ list, int k0) {
  using P2 = typename Pair<T>::type;
  constexpr int NW = NT / 32;
  constexpr int ROWS = NT * RPT;  // panel rows held by this CTA
  constexpr int PS = NB + 1;      // staging row stride: conflict-free row-per-thread access
  __shared__ __align__(16) T cand_row[2][NW][NB];
  __shared__ T cand_v[2][NW];
  __shared__ int cand_k[2][NW];
  __shared__ T cand_rp[2][NW];
  __shared__ __align__(16) T xc_row[2][CS][NB];  // each CTA's candidate, pushed by every CTA of the cluster
  __shared__ T xc_v[2][CS];
  __shared__ int xc_k[2][CS];
  __shared__ T xc_rp[2][CS];
  __shared__ T L11[NB][LS];
  __shared__ T Xinv[NB][LS];
  __shared__ T pvals[NB];
  __shared__ int s_ndisp;
  extern __shared__ __align__(16) unsigned char panel_dyn[];
  T* stage = reinterpret_cast<T*>(panel_dyn);                // ROWS x PS
  int* spos = reinterpret_cast<int*>(stage + (size_t)ROWS * PS);  // ROWS

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rank = CS > 1 ? (int)blockIdx.x % CS : 0;
  const int sysb = (int)blockIdx.x / CS;
  const SysDesc d = step_desc(sa, list ? list[sysb] : sysb);
  StepScratchT<T>* sc = sa.scratch + d.pad_;
  const int n = d.n, m = n - k0, kb = min(NB, m);
  if (k0 == 0) {
    if (tid == 0 && rank == 0) {
      sc->info = 0; sc->nswap = 0; sc->det = 1.0; sc->logabs = 0.0; sc->sign = 1.0;
    }
  } else if (sc->info) {
    return;  // the same for every CTA of the cluster
  }
  T* dst = sa.LU + d.lu_off;
  const T* src = (k0 == 0 && sa.A) ? sa.A + d.a_off : dst;
  if (rank == 0) {
    for (int idx = tid; idx < NB * NB; idx += NT) {
      const int i = idx / NB, c = idx % NB;
      L11[i][c] = (i == c) ? T(1) : T(0);
    }
  }

  // rows in: warp w copies rows w, w + NW, ... (lane = column; past kb and m zero)
  const int r0 = rank * ROWS;
#pragma unroll 4
  for (int rr = warp; rr < ROWS; rr += NW) {
    const int r = r0 + rr;
    const bool ok = r < m && lane < kb;
    cp_async<sizeof(T)>(&stage[rr * PS + lane], ok ? src + (int64_t)(k0 + r) * n + k0 + lane : src, ok);
  }
  cp_async_commit();
  if (tid == 0) s_ndisp = 0;
  cp_async_wait<0>();
  __syncthreads();
  T a[RPT][NB];
  int pos[RPT];
  bool valid[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = r0 + tid + q * NT;
    valid[q] = r < m;
    pos[q] = r;
#pragma unroll
    for (int c = 0; c < NB; ++c) a[q][c] = stage[(tid + q * NT) * PS + c];
  }

  // Column loop, software-pipelined: iteration j publishes the candidates of
  // column j (found at the end of iteration j-1), takes the winner after the
  // barrier, updates column j+1 first and searches it (the warp reductions and
  // the candidate owner's reciprocal overlap the rank-1 update of the columns
  // after it). The multiplier L (rows below the pivot) overwrites the column
  // entry it came from. Every element sees the same operations in the same
  // order as in a plain right-looking column loop.
  int info = 0;
  int nswap = 0;
  T nbest;
  int nkey;
  T nrp;  // 1 / (this thread's candidate value), valid in the owner of nkey
  {
    T v[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) v[q] = a[q][0];
    column_candidate<T, RPT>(v, pos, valid, 0, nbest, nkey, nrp, sa.unopiv != 0);
  }
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (j < kb && !info) {  // uniform across the CTA
      const int par = j & 1;
      if (lane == 0) { cand_v[par][warp] = nbest; cand_k[par][warp] = nkey; }
      // the candidate row from column j on (earlier columns are never read)
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        if (valid[q] && pos[q] == nkey) {
          P2* cr = reinterpret_cast<P2*>(cand_row[par][warp]);
#pragma unroll
          for (int c2 = j / 2; c2 < NB / 2; ++c2) cr[c2] = make_pair2<T>(a[q][2 * c2], a[q][2 * c2 + 1]);
          cand_rp[par][warp] = nrp;
        }
      }
      __syncthreads();
      T gb = T(-1);
      int gk = INT_MAX, gw = 0;
      if constexpr (NW > 4) {
        // lane w < NW holds warp w's candidate; the same rule by warp reductions
        const int ck = lane < NW ? cand_k[par][lane] : INT_MAX;
        gb = lane < NW ? cand_v[par][lane] : T(-1);
        gk = ck;
        warp_argmax_abs(gb, gk);
        gw = __ffs(__ballot_sync(0xffffffffu, lane < NW && ck == gk)) - 1;
        if (gw < 0) gw = 0;  // no candidate anywhere: gb is 0 and the column is singular
      } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          const T v = cand_v[par][w];
          const int k = cand_k[par][w];
          if (v > gb || (v == gb && k < gk)) { gb = v; gk = k; gw = w; }
        }
      }
      const T* prow = cand_row[par][gw];
      T rp = cand_rp[par][gw];
      if constexpr (CS > 1) {
        // every CTA pushes its candidate into slot `rank` of every CTA, then
        // one cluster barrier; the slots alternate with the column parity, so
        // a slot is rewritten only after every CTA has passed the next barrier
        cg::cluster_group cl = cg::this_cluster();
        if (warp == 0) {
          const T rv = lane >= (j & ~1) ? prow[lane] : T(0);
#pragma unroll 1
          for (int to = 0; to < CS; ++to) {
            cl.map_shared_rank(&xc_row[par][rank][0], to)[lane] = rv;
            if (lane == 0) {
              *cl.map_shared_rank(&xc_v[par][rank], to) = gb;
              *cl.map_shared_rank(&xc_k[par][rank], to) = gk;
              *cl.map_shared_rank(&xc_rp[par][rank], to) = rp;
            }
          }
        }
        cl.sync();
        gb = T(-1);
        gk = INT_MAX;
        int gr = 0;
#pragma unroll
        for (int r = 0; r < CS; ++r) {
          const T v = xc_v[par][r];
          const int k = xc_k[par][r];
          if (v > gb || (v == gb && k < gk)) { gb = v; gk = k; gr = r; }
        }
        prow = xc_row[par][gr];
        rp = xc_rp[par][gr];
      }
      if (gb == T(0)) {
        info = k0 + j + 1;
      } else {
        const P2* pr2 = reinterpret_cast<const P2*>(prow);
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          if (valid[q]) {
            if (pos[q] == j) pos[q] = gk;
            else if (pos[q] == gk) pos[q] = j;
          }
        }
        if (tid == 0 && rank == 0) {
          pvals[j] = prow[j];
          if (sa.ipiv) sa.ipiv[d.piv_off + k0 + j] = k0 + gk;
        }
        nswap += (gk != j);
        T f[RPT];
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          const bool below = valid[q] && pos[q] > j;
          f[q] = below ? a[q][j] * rp : T(0);
          if (below) a[q][j] = f[q];
        }
        if (j + 1 < NB) {
          // column j+1 first, then its candidates
          const T t = prow[j + 1];
          T v[RPT];
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            a[q][j + 1] = fma(-f[q], t, a[q][j + 1]);
            v[q] = a[q][j + 1];
          }
          if (j + 1 < kb) column_candidate<T, RPT>(v, pos, valid, j + 1, nbest, nkey, nrp, sa.unopiv != 0);
#pragma unroll
          for (int c2 = (j + 2) / 2; c2 < NB / 2; ++c2) {
            const P2 t2 = pr2[c2];
            const int c = 2 * c2;
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
              if (c > j + 1) a[q][c] = fma(-f[q], t2.x, a[q][c]);
              a[q][c + 1] = fma(-f[q], t2.y, a[q][c + 1]);
            }
          }
        }
      }
    }
  }

  if (info) {
    if (tid == 0 && rank == 0) {
      sc->info = info;
      if (sa.det) sa.det[d.idx] = 0.0;
      if (sa.sign) sa.sign[d.idx] = 0.0;
      if (sa.logabs) sa.logabs[d.idx] = -INFINITY;
      if (sa.info) sa.info[d.idx] = info;
    }
    return;
  }

  // panel back at the pivoted positions: each thread stages its rows with
  // their positions, then warps write whole rows; the strictly lower part of
  // L11 into rank 0's shared memory (identity-initialised before the loop)
  T(*L11r)[LS] = L11;
  if constexpr (CS > 1) L11r = reinterpret_cast<T(*)[LS]>(cg::this_cluster().map_shared_rank(&L11[0][0], 0));
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int sl = tid + q * NT;
    spos[sl] = valid[q] ? pos[q] : -1;
    if (valid[q]) {
#pragma unroll
      for (int c = 0; c < NB; ++c) stage[sl * PS + c] = a[q][c];
      if (pos[q] < kb) {
#pragma unroll
        for (int c = 0; c < NB; ++c)
          if (c < pos[q]) L11r[pos[q]][c] = a[q][c];
      }
      // row moves for the other columns (rows r < kb all live in rank 0)
      const int r = r0 + sl;
      if (pos[q] < kb) {
        sc->top_src[pos[q]] = r;
      } else if (r < kb) {
        const int k = atomicAdd(&s_ndisp, 1);
        sc->disp_dst[k] = pos[q];
        sc->disp_src[k] = r;
      }
    }
  }
  __syncthreads();
#pragma unroll 4
  for (int sl = warp; sl < ROWS; sl += NW) {
    const int p = spos[sl];
    if (p >= 0 && lane < kb) dst[(int64_t)(k0 + p) * n + k0 + lane] = stage[sl * PS + lane];
  }
  if constexpr (CS > 1) {
    cg::this_cluster().sync();  // no shared memory of another CTA is touched after this
    if (rank != 0) return;
  } else {
    __syncthreads();
  }
  if (tid == 0) sc->ndisp = s_ndisp;
  StepHistT<T>* hs = sa.hist ? sa.hist + d.pad_ : nullptr;
  if (hs && tid < NB) {
    // every CTA's writes of the row moves are visible after the barrier above
    hs->top_src[sa.hslot][tid] = sc->top_src[tid];
    hs->disp_dst[sa.hslot][tid] = sc->disp_dst[tid];
    hs->disp_src[sa.hslot][tid] = sc->disp_src[tid];
    if (tid == 0) hs->ndisp[sa.hslot] = s_ndisp;
  }

  // L11^-1 (unit lower, identity-padded past kb): lane c builds column c in
  // shared memory; four partial sums per entry shorten the dependent chain
  if (warp == 0) {
#pragma unroll 1
    for (int i = 0; i < NB; ++i) {
      T p0 = (i == lane) ? T(1) : T(0), p1 = T(0), p2 = T(0), p3 = T(0);
      int q = 0;
#pragma unroll 1
      for (; q + 3 < i; q += 4) {
        p0 = fma(-L11[i][q], Xinv[q][lane], p0);
        p1 = fma(-L11[i][q + 1], Xinv[q + 1][lane], p1);
        p2 = fma(-L11[i][q + 2], Xinv[q + 2][lane], p2);
        p3 = fma(-L11[i][q + 3], Xinv[q + 3][lane], p3);
      }
#pragma unroll 1
      for (; q < i; ++q) p0 = fma(-L11[i][q], Xinv[q][lane], p0);
      const T x = (p0 + p1) + (p2 + p3);
      Xinv[i][lane] = x;
      sc->linv[i * NB + lane] = x;
      if (hs) hs->linv[sa.hslot][i * NB + lane] = x;
    }
  }

  // det / slogdet: pivots folded in the reference's order (linalg.cpp:400-403, 425-431)
  if (warp == (NW > 1 ? 1 : 0)) {
    const double lg = lane < kb ? log(fabs((double)pvals[lane])) : 0.0;
    const int ns = nswap;  // every thread counted the same exchanges
    double det = sc->det, la = sc->logabs, sg = sc->sign;
    if (ns & 1) { det = -det; sg = -sg; }
    for (int j = 0; j < kb; ++j) {
      const double pj = pvals[j];
      const double lj = __shfl_sync(0xffffffffu, lg, j);
      det *= pj;
      la += lj;
      sg *= pj / fabs(pj);
    }
    if (lane == 0) {
      sc->det = det; sc->logabs = la; sc->sign = sg;
      sc->nswap += ns;
      if (k0 + kb >= n) {
        if (sa.det) sa.det[d.idx] = det;
        if (sa.sign) sa.sign[d.idx] = sg;
        if (sa.logabs) sa.logabs[d.idx] = la;
        if (sa.info) sa.info[d.idx] = 0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Shared helpers for the 64-column strip kernels.

template <class T>
struct Seg {
  T* dst;         // where the strip lives
  const T* src;   // where it is read from (== dst after step 0)
  int ld;
  bool ident;     // source is the identity (inverse at step 0)
};

template <class T>
__device__ inline Seg<T> segment(const StepArgsT<T>& sa, const SysDesc& d, int kind, int k0) {
  Seg<T> s;
  if (kind == kSegMatrix || kind == kSegLeft) {
    s.dst = sa.LU + d.lu_off;
    s.src = (k0 == 0 && sa.A) ? sa.A + d.a_off : s.dst;
    s.ld = d.n;
    s.ident = false;
  } else if (kind == kSegRhs) {
    s.dst = sa.X + d.b_off;
    s.src = (k0 == 0) ? sa.B + d.b_off : s.dst;
    s.ld = d.nrhs;
    s.ident = false;
  } else {
    s.dst = sa.inv + d.inv_off;
    s.src = s.dst;
    s.ld = d.n;
    s.ident = (k0 == 0);
  }
  return s;
}

template <class T>
__device__ __forceinline__ T seg_load(const Seg<T>& s, int row, int col) {
  return s.ident ? (row == col ? T(1) : T(0)) : s.src[(int64_t)row * s.ld + col];
}

// A 64 x 64 accumulator tile spread over the 128 threads of a strip kernel.
// each(f) visits (row, column, value&) of the thread's elements;
// sub_mma(As, Bs) does tile -= As(64 x 32, stride LS) * Bs(32 x 64, stride WS).
template <class T> struct Acc64;

template <> struct Acc64<double> {  // 2 x 2 warps of 32 x 32, DMMA fragments
  double v[4][4][2];
  template <class F>
  __device__ __forceinline__ void each(F&& f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) f(wm + mi * 8 + g, wn + ni * 8 + 2 * tq + e, v[mi][ni][e]);
  }
  // (row, even column, the two elements of that column pair)
  template <class F>
  __device__ __forceinline__ void pairs(F&& f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) f(wm + mi * 8 + g, wn + ni * 8 + 2 * tq, v[mi][ni][0], v[mi][ni][1]);
  }
  template <int AST = LS, int BST = WS>
  __device__ __forceinline__ void sub_mma(const double* As, const double* Bs) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = -As[(wm + mi * 8 + g) * AST + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[(kk + tq) * BST + wn + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(v[mi][ni], af[mi], bf[ni]);
    }
  }
};

template <> struct Acc64<float> {  // 4 x 8 elements per thread, FP32 FMA
  float v[4][8];
  template <class F>
  __device__ __forceinline__ void each(F&& f) {
    const int ty = threadIdx.x >> 3, tx = threadIdx.x & 7;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) f(ty * 4 + i, tx * 8 + j, v[i][j]);
  }
  template <class F>
  __device__ __forceinline__ void pairs(F&& f) {
    const int ty = threadIdx.x >> 3, tx = threadIdx.x & 7;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; j += 2) f(ty * 4 + i, tx * 8 + j, v[i][j], v[i][j + 1]);
  }
  template <int AST = LS, int BST = WS>
  __device__ __forceinline__ void sub_mma(const float* As, const float* Bs) {
    const int ty = threadIdx.x >> 3, tx = threadIdx.x & 7;
#pragma unroll 4
    for (int k = 0; k < NB; ++k) {
      float a[4], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[(ty * 4 + i) * AST + k];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[k * BST + tx * 8 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) v[i][j] = fmaf(-a[i], b[j], v[i][j]);
    }
  }
};

// The 32 x 64 tile of U12 = L11^-1 A12 (plain product, no negation).
template <class T> struct Acc32;

template <> struct Acc32<double> {  // warp w owns columns [16w, 16w+16)
  double v[4][2][2];
  template <class F>
  __device__ __forceinline__ void each(F&& f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) f(mi * 8 + g, warp * 16 + ni * 8 + 2 * tq + e, v[mi][ni][e]);
  }
  __device__ __forceinline__ void mma(const double* As, const double* Bs) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) v[mi][ni][0] = v[mi][ni][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = As[(mi * 8 + g) * LS + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) bf[ni] = Bs[(kk + tq) * WS + warp * 16 + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) dmma884(v[mi][ni], af[mi], bf[ni]);
    }
  }
};

template <> struct Acc32<float> {  // 4 x 4 elements per thread
  float v[4][4];
  template <class F>
  __device__ __forceinline__ void each(F&& f) {
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) f(ty * 4 + i, tx * 4 + j, v[i][j]);
  }
  __device__ __forceinline__ void mma(const float* As, const float* Bs) {
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) v[i][j] = 0.f;
#pragma unroll 4
    for (int k = 0; k < NB; ++k) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[(ty * 4 + i) * LS + k];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k * WS + tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) v[i][j] = fmaf(a[i], b[j], v[i][j]);
    }
  }
};

// FP32 factors with the trailing product on the tensor cores: operands
// rounded to TF32 (mma.m16n8k8) or BF16 (mma.m16n8k16), FP32 accumulation.
// Same 64 x 64 tile and 2 x 2 warp split as Acc64; a warp holds 2 x 4
// m16n8 accumulators.
// kUpd3xTf32: each FP32 operand split as x = hi + lo with hi = tf32(x) and
// lo = tf32(x - hi), the product taken as hi*hi + hi*lo + lo*hi (three
// tensor-core products, the lo*lo term dropped): close to FP32 accuracy at
// tensor-core speed (the error-compensated TF32 scheme of Ootomo and Yokota,
// 2022, and of CUTLASS's 3xTF32 kernels).
// kUpdTcTf32 / kUpdTc3xTf32: the same TF32 / 3xTF32 products on the
// tcgen05 tensor cores with TMEM accumulators (k_update_tc).
enum : int { kUpdFp32 = 0, kUpdTf32 = 1, kUpdBf16 = 2, kUpd3xTf32 = 3, kUpdTcTf32 = 4, kUpdTc3xTf32 = 5 };

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

template <int MODE>
struct AccTC {
  float v[2][4][4];
  template <class F>
  __device__ __forceinline__ void pairs(F&& f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        f(wm + mi * 16 + g, wn + ni * 8 + 2 * tq, v[mi][ni][0], v[mi][ni][1]);
        f(wm + mi * 16 + g + 8, wn + ni * 8 + 2 * tq, v[mi][ni][2], v[mi][ni][3]);
      }
  }
  __device__ __forceinline__ void mma_tf32(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
  }
  template <int AST, int BST>
  __device__ __forceinline__ void sub_mma(const float* As, const float* Bs) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    if constexpr (MODE == kUpd3xTf32) {
#pragma unroll
      for (int kk = 0; kk < NB; kk += 8) {
        uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          const float* r0 = As + (wm + mi * 16 + g) * AST + kk + tq;
          const float* r1 = r0 + 8 * AST;
          const float x[4] = {-r0[0], -r1[0], -r0[4], -r1[4]};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            ah[mi][e] = to_tf32(x[e]);
            al[mi][e] = to_tf32(x[e] - __uint_as_float(ah[mi][e]));
          }
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const float* c = Bs + (kk + tq) * BST + wn + ni * 8 + g;
          const float y[2] = {c[0], c[4 * BST]};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            bh[ni][e] = to_tf32(y[e]);
            bl[ni][e] = to_tf32(y[e] - __uint_as_float(bh[ni][e]));
          }
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            mma_tf32(v[mi][ni], al[mi], bh[ni]);  // small terms first
            mma_tf32(v[mi][ni], ah[mi], bl[ni]);
            mma_tf32(v[mi][ni], ah[mi], bh[ni]);
          }
      }
    } else
    if constexpr (MODE == kUpdTf32) {
#pragma unroll
      for (int kk = 0; kk < NB; kk += 8) {
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          const float* r0 = As + (wm + mi * 16 + g) * AST + kk + tq;
          const float* r1 = r0 + 8 * AST;
          a[mi][0] = to_tf32(-r0[0]);
          a[mi][1] = to_tf32(-r1[0]);
          a[mi][2] = to_tf32(-r0[4]);
          a[mi][3] = to_tf32(-r1[4]);
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const float* c = Bs + (kk + tq) * BST + wn + ni * 8 + g;
          b[ni][0] = to_tf32(c[0]);
          b[ni][1] = to_tf32(c[4 * BST]);
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
            asm volatile(
                "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(v[mi][ni][0]), "+f"(v[mi][ni][1]), "+f"(v[mi][ni][2]), "+f"(v[mi][ni][3])
                : "r"(a[mi][0]), "r"(a[mi][1]), "r"(a[mi][2]), "r"(a[mi][3]), "r"(b[ni][0]), "r"(b[ni][1]));
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < NB; kk += 16) {
        uint32_t a[2][4], b[4][2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          const float* r0 = As + (wm + mi * 16 + g) * AST + kk + 2 * tq;
          const float* r1 = r0 + 8 * AST;
          const float2 x0 = *reinterpret_cast<const float2*>(r0);
          const float2 x1 = *reinterpret_cast<const float2*>(r1);
          const float2 x2 = *reinterpret_cast<const float2*>(r0 + 8);
          const float2 x3 = *reinterpret_cast<const float2*>(r1 + 8);
          a[mi][0] = pack_bf16(-x0.x, -x0.y);
          a[mi][1] = pack_bf16(-x1.x, -x1.y);
          a[mi][2] = pack_bf16(-x2.x, -x2.y);
          a[mi][3] = pack_bf16(-x3.x, -x3.y);
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const float* c = Bs + (kk + 2 * tq) * BST + wn + ni * 8 + g;
          b[ni][0] = pack_bf16(c[0], c[BST]);
          b[ni][1] = pack_bf16(c[8 * BST], c[9 * BST]);
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni)
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(v[mi][ni][0]), "+f"(v[mi][ni][1]), "+f"(v[mi][ni][2]), "+f"(v[mi][ni][3])
                : "r"(a[mi][0]), "r"(a[mi][1]), "r"(a[mi][2]), "r"(a[mi][3]), "r"(b[ni][0]), "r"(b[ni][1]));
      }
    }
  }
};

template <class T, int MODE> struct AccSel { using type = Acc64<T>; };
template <> struct AccSel<float, kUpdTf32> { using type = AccTC<kUpdTf32>; };
template <> struct AccSel<float, kUpdBf16> { using type = AccTC<kUpdBf16>; };
template <> struct AccSel<float, kUpd3xTf32> { using type = AccTC<kUpd3xTf32>; };

// C[rows r0.., 64 cols] -= As * Bs for rows [r0, rend), columns < w, one tile.
template <class T, class Load, class Store>
__device__ __forceinline__ void tile_update(const T* As, const T* Bs, int r0, int rend, int w, Load cload,
                                            Store cstore) {
  Acc64<T> acc;
  acc.each([&](int r, int cc, T& x) { x = (r0 + r < rend && cc < w) ? cload(r0 + r, cc) : T(0); });
  acc.sub_mma(As, Bs);
  acc.each([&](int r, int cc, T& x) {
    if (r0 + r < rend && cc < w) cstore(r0 + r, cc, x);
  });
}

// The work item of an update CTA. Uniform batches can split one step's update
// for look-ahead: part 1 = only the first matrix strip of every system (it
// holds the next panel's columns; grid.x = systems), part 2 = every other
// strip, part 0 = all. Returns false for a CTA with nothing to do.
template <class T>
__device__ __forceinline__ bool update_item(const StepArgsT<T>& sa, const StepItem* items, int k0, int part,
                                            StepItem& it) {
  if (items) {
    it = items[blockIdx.x];
    return true;
  }
  if (part == 0) {
    it = uniform_item(sa, blockIdx.x, k0, false);
    return true;
  }
  const int per = sa.ubend > 0 ? blocked_update_strips(sa.un, sa.unrhs, sa.uinv, k0, sa.uleft, sa.ubbeg, sa.ubend)
                               : uniform_update_strips(sa.un, sa.unrhs, sa.uinv, k0, sa.uleft);
  if (part == 1) {
    it = uniform_item(sa, (int)blockIdx.x * per, k0, false);
    return it.kind == kSegMatrix;
  }
  it = uniform_item(sa, blockIdx.x, k0, false);
  return !((int)blockIdx.x % per == 0 && it.kind == kSegMatrix);
}

// ---------------------------------------------------------------------------
// k_rows: one CTA per strip item of step k0. Applies the panel's row moves to
// the strip (top rows from their sources, displaced old top rows to their new
// positions) and, except for strips left of the panel, writes
// U12 = L11^-1 A12 over the top rows. After it, k_update reads every row of the
// strip in its final place, except at step 0 out of place, where only the
// displaced rows have been written to the destination yet.
template <class T>
__global__ void __launch_bounds__(UT)
k_rows(StepArgsT<T> sa, const StepItem* __restrict__ items, int k0) {
  __shared__ T Tm[NB * WS];
  __shared__ T D[NB * WS];
  __shared__ T Li[NB * LS];
  __shared__ int tsrc[NB], ddst[NB], dsrc[NB];
  const int tid = threadIdx.x;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, k0, false);
  const SysDesc d = step_desc(sa, it.sys);
  const StepScratchT<T>* sc = sa.scratch + d.pad_;
  if (sc->info) return;
  const int n = d.n, m = n - k0, kb = min(NB, m), w = it.width, c0 = it.c0;
  const Seg<T> s = segment(sa, d, it.kind, k0);
  // the trailing pass of a two-level factorisation replays a recorded panel
  const StepHistT<T>* hs = sa.utrail ? sa.hist + d.pad_ : nullptr;
  const int hsl = sa.hslot;
  const int mv = hs ? sa.umoves : 0;  // 1: row moves only, 2: U12 of rows already in place
  const int nd = mv == 2 ? 0 : hs ? hs->ndisp[hsl] : sc->ndisp;
  if (tid < NB) {
    tsrc[tid] = tid < kb ? (mv == 2 ? tid : hs ? hs->top_src[hsl][tid] : sc->top_src[tid]) : 0;
    ddst[tid] = tid < nd ? (hs ? hs->disp_dst[hsl][tid] : sc->disp_dst[tid]) : 0;
    dsrc[tid] = tid < nd ? (hs ? hs->disp_src[hsl][tid] : sc->disp_src[tid]) : 0;
  }
  const bool u12 = !(it.kind == kSegLeft || mv == 1);  // else row moves only
  if (u12) {  // L11^-1 comes in together with the move lists (one round trip fewer)
    const T* linv = hs ? hs->linv[hsl] : sc->linv;
#pragma unroll
    for (int it_ = 0; it_ < NB * NB / UT; ++it_) {
      const int idx = tid + it_ * UT;
      Li[(idx >> 5) * LS + (idx & 31)] = linv[idx];
    }
  }
  __syncthreads();
  // fixed trip counts, fully unrolled: every load of the gather is in flight at once
#pragma unroll
  for (int it = 0; it < NB * 64 / UT; ++it) {
    const int idx = tid + it * UT, i = idx >> 6, c = idx & 63;
    const bool in = c < w;
    Tm[i * WS + c] = (in && i < kb) ? seg_load(s, k0 + tsrc[i], c0 + c) : T(0);
    D[i * WS + c] = (in && i < nd) ? seg_load(s, k0 + dsrc[i], c0 + c) : T(0);
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < NB * 64 / UT; ++it) {
    const int idx = tid + it * UT, i = idx >> 6, c = idx & 63;
    if (c < w && i < nd) s.dst[(int64_t)(k0 + ddst[i]) * s.ld + c0 + c] = D[i * WS + c];
  }
  if (!u12) {
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      if (c < w && i < kb) s.dst[(int64_t)(k0 + i) * s.ld + c0 + c] = Tm[i * WS + c];
    }
    return;
  }
  Acc32<T> u;  // Tm and Li are complete since the barrier after the gather
  u.mma(Li, Tm);
  u.each([&](int i, int c, T& x) {
    if (i < kb && c < w) s.dst[(int64_t)(k0 + i) * s.ld + c0 + c] = x;
  });
}

// ---------------------------------------------------------------------------
// k_update: A22 -= L21 U12 on one strip, rows [k0+32 + RG*blockIdx.y, +RG), in
// 64-row tiles: while tile t is multiplied, tile t+1's L21 rows stream into
// shared memory (cp.async, 16-byte pieces when aligned); each tile's
// accumulator inputs are read when the tile starts (paired loads when
// aligned). At 128 registers four CTAs fit on an SM and hide those reads from
// one another (measured faster than prefetching them into a second register
// tile at three CTAs per SM).
constexpr int RG = 512;
constexpr int RG1 = 128;  // rows per CTA of the look-ahead strip (part 1): short critical path

// Shared row strides (elements) for bank-conflict-free fragment reads; every
// row starts on a 16-byte boundary.
template <class T, int MODE> struct TileCfg;
template <> struct TileCfg<double, kUpdFp32> {
  static constexpr int AS = 36;  // L21 tile: banks 8g + 2tq (8-byte reads)
  static constexpr int US = 68;  // U12: banks 8tq + 2g
};
template <> struct TileCfg<float, kUpdFp32> {
  static constexpr int AS = 34;  // SIMT reads: banks 8 * (row group)
  static constexpr int US = 68;
};
template <> struct TileCfg<float, kUpdTf32> {
  static constexpr int AS = 36;  // banks 4g + tq
  static constexpr int US = 72;  // banks 8tq + g
};
template <> struct TileCfg<float, kUpd3xTf32> {
  static constexpr int AS = 36;
  static constexpr int US = 72;
};
template <> struct TileCfg<float, kUpdBf16> {
  static constexpr int AS = 40;  // 8-byte reads: banks 8g + 2tq
  static constexpr int US = 68;  // banks 8tq + g
};

template <class T, int MODE>
size_t update_smem() {
  return sizeof(T) * (NB * TileCfg<T, MODE>::US + 2 * 64 * TileCfg<T, MODE>::AS) + RG;
}

__device__ __forceinline__ void cp_async_pair(void* smem, const void* gmem, int bytes, int valid) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid));
}

// sm[r][c] <- g[r*gld + c] for r < rows, c < cols of a nr x nc tile (zero
// elsewhere); vec: element pairs (rows and base aligned to two elements).
template <class T>
__device__ __forceinline__ void async_tile(T* sm, int sld, const T* g, int64_t gld, int rows, int cols, int nr,
                                           int nc, bool vec) {
  if (vec) {
    const int cpr = nc / 2;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < nr * cpr; idx += UT) {
      const int r = idx / cpr, c = (idx % cpr) * 2;
      const int ok = r < rows ? max(0, min(2, cols - c)) : 0;
      cp_async_pair(sm + r * sld + c, ok ? g + (int64_t)r * gld + c : g, 2 * (int)sizeof(T), ok * (int)sizeof(T));
    }
  } else {
#pragma unroll 4
    for (int idx = threadIdx.x; idx < nr * nc; idx += UT) {
      const int r = idx / nc, c = idx % nc;
      const bool ok = r < rows && c < cols;
      cp_async<sizeof(T)>(sm + r * sld + c, ok ? g + (int64_t)r * gld + c : g, ok);
    }
  }
  cp_async_commit();
}

template <class T>
__device__ __forceinline__ bool pair_aligned(const T* p, int64_t ld) {
  return ((reinterpret_cast<uintptr_t>(p) % (2 * sizeof(T))) == 0) && (ld % 2 == 0);
}

template <class T, int MODE>
__global__ void __launch_bounds__(UT, 4)
k_update(StepArgsT<T> sa, const StepItem* __restrict__ items, int k0, int part) {
  using P2 = typename Pair<T>::type;
  using Acc = typename AccSel<T, MODE>::type;
  constexpr int AS = TileCfg<T, MODE>::AS, US = TileCfg<T, MODE>::US;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Us = reinterpret_cast<T*>(smem_raw);  // U12, 32 x 64
  T* As0 = Us + NB * US;                   // L21 tiles, 64 x 32, two buffers
  T* As1 = As0 + 64 * AS;
  unsigned char* moved = reinterpret_cast<unsigned char*>(As1 + 64 * AS);  // RG flags

  const int tid = threadIdx.x;
  StepItem it;
  if (!update_item(sa, items, k0, part, it)) return;
  if (it.kind == kSegLeft) return;
  const SysDesc d = step_desc(sa, it.sys);
  const StepScratchT<T>* sc = sa.scratch + d.pad_;
  if (sc->info) return;
  const int n = d.n;
  const int rg = part == 1 ? RG1 : RG;  // rows per CTA
  const int rb = k0 + NB + (int)blockIdx.y * rg;
  const int rlim = sa.urow_end > 0 ? min(n, sa.urow_end) : n;
  if (rb >= rlim) return;  // includes the last panel (nothing below it)
  const int re = min(rlim, rb + rg), w = it.width, c0 = it.c0;
  const Seg<T> s = segment(sa, d, it.kind, k0);
  const int64_t ld = s.ld;
  // step 0 out of place: rows holding a displaced row are already in dst
  const bool first = s.ident || s.src != s.dst;
  if (first) {
    for (int i = tid; i < re - rb; i += UT) moved[i] = 0;
    __syncthreads();
    if (tid < sc->ndisp) {
      const int r = k0 + sc->disp_dst[tid];
      if (r >= rb && r < re) moved[r - rb] = 1;
    }
    __syncthreads();
  }
  const T* L = sa.LU + d.lu_off;
  T* const dst = s.dst + c0;
  const T* const src = s.src + c0;
  const bool dvec = pair_aligned(dst, ld), svec = !s.ident && pair_aligned(src, ld);

  async_tile<T>(Us, US, dst + (int64_t)k0 * ld, ld, NB, w, NB, 64, dvec);
  auto prefetch_a = [&](T* buf, int r0) {
    async_tile<T>(buf, AS, L + (int64_t)r0 * d.n + k0, d.n, re - r0, NB, 64, NB, pair_aligned(L + k0, d.n));
  };
  auto load_c = [&](Acc& c, int r0) {
    c.pairs([&](int rr, int cc, T& v0, T& v1) {
      const int r = r0 + rr;
      v0 = v1 = T(0);
      if (r < re && cc < w) {
        const bool two = cc + 1 < w;
        const bool fromdst = !first || moved[r - rb];
        if (!fromdst && s.ident) {
          v0 = (r == c0 + cc) ? T(1) : T(0);
          v1 = (two && r == c0 + cc + 1) ? T(1) : T(0);
        } else {
          const T* p = (fromdst ? dst : src) + (int64_t)r * ld + cc;
          if (two && (fromdst ? dvec : svec)) {
            const P2 t = *reinterpret_cast<const P2*>(p);
            v0 = t.x;
            v1 = t.y;
          } else {
            v0 = p[0];
            if (two) v1 = p[1];
          }
        }
      }
    });
  };
  Acc cur;
  prefetch_a(As0, rb);
  bool b1 = false;
  for (int r0 = rb; r0 < re; r0 += 64) {
    const bool more = r0 + 64 < re;
    load_c(cur, r0);
    if (more) {
      prefetch_a(b1 ? As0 : As1, r0 + 64);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    cur.template sub_mma<AS, US>(b1 ? As1 : As0, Us);
    cur.pairs([&](int rr, int cc, T& v0, T& v1) {
      const int r = r0 + rr;
      if (r < re && cc < w) {
        T* p = dst + (int64_t)r * ld + cc;
        if (cc + 1 < w && dvec) {
          *reinterpret_cast<P2*>(p) = make_pair2<T>(v0, v1);
        } else {
          p[0] = v0;
          if (cc + 1 < w) p[1] = v1;
        }
      }
    });
    b1 = !b1;
    __syncthreads();  // the buffer just read is refilled by the next iteration's prefetch
  }
}

// ---------------------------------------------------------------------------
// k_update_tc: the FP32 factors' trailing update on the 5th-generation tensor
// cores. One CTA per (strip, 512 rows below the panel), 128-row tiles:
//  * U12^T (64 x 32) and each L21 tile (128 x 32) are staged in shared memory
//    in the canonical K-major layout without swizzle: 8-row x 16-byte core
//    matrices, K-adjacent cores 128 bytes apart (leading byte offset), 8-row
//    groups 1024 bytes apart (stride byte offset);
//  * one thread issues tcgen05.mma.kind::tf32 (M = 128, N = 64, K = 8, four
//    per tile; three per K slice for 3xTF32: lo*hi + hi*lo + hi*hi on split
//    copies) into a 64-column TMEM accumulator and commits to an mbarrier;
//  * while the tensor core runs, the C tile (128 x 64) streams into shared
//    memory in 16-byte pieces, piece c of row r stored at piece c ^ (r & 15)
//    (conflict-free both for the coalesced copies and for one thread reading
//    a whole row), and the next L21 tile behind it; then tcgen05.ld brings P
//    back (thread = row), each thread subtracts its row in shared memory, and
//    the tile is stored coalesced.
// The mbarrier wait is bounded: past the limit the kernel records a timeout
// in g_tc_timeouts, skips its stores, frees its TMEM and returns.
constexpr int TC_M = 128;
constexpr int TC_LBO = 128;   // bytes between K-adjacent core matrices
constexpr int TC_SBO = 1024;  // bytes between 8-row groups (8 K-cores of 128 bytes)
constexpr int TC_TILE_A = TC_M * NB * 4;  // 16 KB: one 128 x 32 FP32 operand
constexpr int TC_TILE_B = 64 * NB * 4;    //  8 KB: U12^T
constexpr uint32_t TC_COLS = 64;          // TMEM columns (FP32 accumulator, N = 64)
__device__ __forceinline__ int tc_csw(int row, int piece) {  // float offset of a staged C piece
  return row * 64 + ((piece ^ (row & 15)) << 2);
}

__device__ int g_tc_timeouts = 0;

// byte offset of element (row, k) in a core-matrix K-major operand
__device__ __forceinline__ int tc_off(int row, int k) {
  return (row >> 3) * TC_SBO + (k >> 2) * TC_LBO + (row & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((TC_LBO >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((TC_SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);  // descriptor version 1, no swizzle
}

// kind::tf32 instruction descriptor: FP32 accumulator, TF32 A and B, both
// K-major, N = 64, M = 128
constexpr uint32_t TC_IDESC =
    (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(TC_IDESC), "r"(acc));
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int MODE>
size_t update_tc_smem() {
  // alignment slack, A raw x2 (prefetch), [A lo], B hi, [B lo], mbarrier +
  // TMEM slot + abort flag, row flags
  const int splits = MODE == kUpd3xTf32 ? 1 : 0;
  return 1024 + (size_t)(2 + splits) * TC_TILE_A + (size_t)(1 + splits) * TC_TILE_B + 64 + RG +
         sizeof(float) * TC_M * 64;
}

template <int MODE>
__global__ void __launch_bounds__(UT)
k_update_tc(StepArgsT<float> sa, const StepItem* __restrict__ items, int k0, int part) {
  constexpr bool SPLIT = MODE == kUpd3xTf32;
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char* Araw[2] = {base, base + TC_TILE_A};
  unsigned char* Alo = base + 2 * TC_TILE_A;
  unsigned char* Bhi = Alo + (SPLIT ? TC_TILE_A : 0);
  unsigned char* Blo = Bhi + TC_TILE_B;
  unsigned char* tail = Blo + (SPLIT ? TC_TILE_B : 0);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tail);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tail + 8);
  int* abort_flag = reinterpret_cast<int*>(tail + 16);
  unsigned char* moved = tail + 64;
  float* Cs = reinterpret_cast<float*>(moved + RG);  // staged C tile, TC_M x 64, swizzled pieces

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  StepItem it;
  if (!update_item(sa, items, k0, part, it)) return;
  if (it.kind == kSegLeft) return;
  const SysDesc d = step_desc(sa, it.sys);
  const StepScratchT<float>* sc = sa.scratch + d.pad_;
  if (sc->info) return;
  const int n = d.n;
  const int rg = part == 1 ? RG1 : RG;  // rows per CTA
  const int rb = k0 + NB + (int)blockIdx.y * rg;
  const int rlim = sa.urow_end > 0 ? min(n, sa.urow_end) : n;
  if (rb >= rlim) return;  // includes the last panel (nothing below it)
  const int re = min(rlim, rb + rg), w = it.width, c0 = it.c0;
  const Seg<float> s = segment(sa, d, it.kind, k0);
  const int64_t ld = s.ld;
  // step 0 out of place: rows holding a displaced row are already in dst
  const bool first = s.ident || s.src != s.dst;
  if (tid == 0) *abort_flag = 0;
  if (first) {
    for (int i = tid; i < re - rb; i += UT) moved[i] = 0;
    __syncthreads();
    if (tid < sc->ndisp) {
      const int r = k0 + sc->disp_dst[tid];
      if (r >= rb && r < re) moved[r - rb] = 1;
    }
  }
  float* const dst = s.dst + c0;
  const float* const src = s.src + c0;
  const float* L = sa.LU + d.lu_off;
  const bool lvec = ((reinterpret_cast<uintptr_t>(L + k0) & 15) == 0) && (n % 4 == 0);
  // C rows in 16-byte pieces (both the source and the destination of every row)
  const bool cvec = ld % 4 == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0 &&
                    (s.ident || (reinterpret_cast<uintptr_t>(src) & 15) == 0);

  // TMEM accumulator (one warp allocates) and the completion barrier
  if (warp == 0) {
    const uint32_t slot = static_cast<uint32_t>(__cvta_generic_to_shared(tslot));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  const uint32_t mbar_addr = static_cast<uint32_t>(__cvta_generic_to_shared(mbar));
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_addr));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }

  // A tile: rows r0 .. r0+127 of L21 (zero past re) into the core layout
  auto stage_a = [&](unsigned char* buf, int r0) {
    if (lvec) {
      for (int idx = tid; idx < TC_M * (NB / 4); idx += UT) {
        const int r = idx >> 3, q = (idx & 7) * 4;
        const bool ok = r0 + r < re;
        cp_async_pair(buf + tc_off(r, q), ok ? L + (int64_t)(r0 + r) * n + k0 + q : L + k0, 16, ok ? 16 : 0);
      }
    } else {
      for (int idx = tid; idx < TC_M * NB; idx += UT) {
        const int r = idx >> 5, q = idx & 31;
        const bool ok = r0 + r < re;
        cp_async<4>(buf + tc_off(r, q), ok ? L + (int64_t)(r0 + r) * n + k0 + q : L, ok);
      }
    }
    cp_async_commit();
  };
  // U12^T (64 x 32, K-major) from the strip's top rows, split for 3xTF32
#pragma unroll
  for (int it_ = 0; it_ < 64 * NB / UT; ++it_) {
    const int idx = tid + it_ * UT;
    const int c = idx >> 5, q = idx & 31;  // column of the strip, row of U12
    const float u = c < w ? dst[(int64_t)(k0 + q) * ld + c] : 0.f;
    if constexpr (SPLIT) {
      const float hi = __uint_as_float(to_tf32(u));
      *reinterpret_cast<float*>(Bhi + tc_off(c, q)) = hi;
      *reinterpret_cast<float*>(Blo + tc_off(c, q)) = __uint_as_float(to_tf32(u - hi));
    } else {
      *reinterpret_cast<float*>(Bhi + tc_off(c, q)) = u;
    }
  }
  stage_a(Araw[0], rb);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tslot;
  const uint32_t a_s[2] = {static_cast<uint32_t>(__cvta_generic_to_shared(Araw[0])),
                           static_cast<uint32_t>(__cvta_generic_to_shared(Araw[1]))};
  const uint32_t alo_s = static_cast<uint32_t>(__cvta_generic_to_shared(Alo));
  const uint32_t bhi_s = static_cast<uint32_t>(__cvta_generic_to_shared(Bhi));
  const uint32_t blo_s = static_cast<uint32_t>(__cvta_generic_to_shared(Blo));

  int t = 0;
  for (int r0 = rb; r0 < re; r0 += TC_M, ++t) {
    const int cur = t & 1;
    cp_async_wait<0>();
    __syncthreads();
    if constexpr (SPLIT) {
      for (int idx = tid; idx < TC_M * NB; idx += UT) {
        const int off = tc_off(idx >> 5, idx & 31);
        float* x = reinterpret_cast<float*>(Araw[cur] + off);
        const float v = *x;
        const float hi = __uint_as_float(to_tf32(v));
        *x = hi;
        *reinterpret_cast<float*>(Alo + off) = __uint_as_float(to_tf32(v - hi));
      }
    }
    // shared-memory writes of the generic proxy become visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll
      for (int kk = 0; kk < NB; kk += 8) {
        const uint32_t koff = (uint32_t)(kk / 4) * TC_LBO;
        if constexpr (SPLIT) {
          tc_mma(tmem, tc_desc(alo_s + koff), tc_desc(bhi_s + koff), kk > 0);  // small terms first
          tc_mma(tmem, tc_desc(a_s[cur] + koff), tc_desc(blo_s + koff), 1);
          tc_mma(tmem, tc_desc(a_s[cur] + koff), tc_desc(bhi_s + koff), 1);
        } else {
          tc_mma(tmem, tc_desc(a_s[cur] + koff), tc_desc(bhi_s + koff), kk > 0);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_addr));
    }
    // C tile into shared memory (one commit group), then the next A tile
    // behind it (its buffer was read by the previous tile's products)
    for (int idx = tid; idx < TC_M * 16; idx += UT) {
      const int rr = idx >> 4, pc = idx & 15, j = pc * 4, r = r0 + rr;
      float* cs = Cs + tc_csw(rr, pc);
      const int valid = (r < re) ? max(0, min(4, w - j)) : 0;
      const bool fromdst = valid && (!first || moved[r - rb]);
      if (valid && !fromdst && s.ident) {
#pragma unroll
        for (int e = 0; e < 4; ++e) cs[e] = (e < valid && r == c0 + j + e) ? 1.f : 0.f;
      } else if (cvec) {
        const float* g = valid ? (fromdst ? dst : src) + (int64_t)r * ld + j : dst;
        cp_async_pair(cs, g, 16, valid * 4);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (e < valid) cp_async<4>(cs + e, (fromdst ? dst : src) + (int64_t)r * ld + j + e, true);
          else cs[e] = 0.f;
        }
      }
    }
    cp_async_commit();
    if (r0 + TC_M < re) stage_a(Araw[cur ^ 1], r0 + TC_M);
    else cp_async_commit();  // keep one group behind the C tile either way
    const int row = warp * 32 + lane;  // TMEM lane = tile row
    const int r = r0 + row;
    const bool live = r < re;

    // wait for the products, bounded
    uint32_t done = 0;
    for (int spin = 0; spin < (1 << 22) && !done; ++spin) {
      asm volatile(
          "{\n\t.reg .pred q;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, q;\n\t}\n"
          : "=r"(done)
          : "r"(mbar_addr), "r"((uint32_t)(t & 1))
          : "memory");
    }
    if (!done) {
      *abort_flag = 1;
      atomicAdd(&g_tc_timeouts, 1);
    }
    cp_async_wait<1>();  // the C tile has landed (the next A tile may still be in flight)
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    __syncthreads();
    if (*abort_flag) break;
    {
      float pv[64];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
      for (int j = 0; j < 64; j += 16) tc_ld16(taddr + (uint32_t)j, pv + j);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
      if (live) {
#pragma unroll
        for (int pc = 0; pc < 16; ++pc) {
          float4* q = reinterpret_cast<float4*>(Cs + tc_csw(row, pc));
          float4 v = *q;
          v.x -= pv[4 * pc];
          v.y -= pv[4 * pc + 1];
          v.z -= pv[4 * pc + 2];
          v.w -= pv[4 * pc + 3];
          *q = v;
        }
      }
    }
    __syncthreads();
    for (int idx = tid; idx < TC_M * 16; idx += UT) {
      const int rr = idx >> 4, pc = idx & 15, j = pc * 4, rg = r0 + rr;
      if (rg >= re || j >= w) continue;
      const float4 v = *reinterpret_cast<const float4*>(Cs + tc_csw(rr, pc));
      float* o = dst + (int64_t)rg * ld + j;
      if (cvec && j + 4 <= w) {
        *reinterpret_cast<float4*>(o) = v;
      } else {
        const float e4[4] = {v.x, v.y, v.z, v.w};
        for (int e = 0; e < 4 && j + e < w; ++e) o[e] = e4[e];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();  // TMEM read and A lo consumed before the next tile's products
  }
  cp_async_wait<0>();
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_COLS));
  }
}

// ---------------------------------------------------------------------------
// Substitution windows: rows [jw*SB, min(n, (jw+1)*SB)) of a system. Back
// substitution takes window jw = (n-1)/SB - pass (from the bottom), forward
// substitution window jw = pass (from the top); a system without that window
// skips the pass.
__device__ __forceinline__ bool back_window(int n, int pass, int& lo, int& hi, int sb = SB) {
  const int jw = (n - 1) / sb - pass;
  lo = jw * sb;
  hi = min(n, lo + sb);
  return jw >= 0;
}
__device__ __forceinline__ bool forward_window(int n, int pass, int& lo, int& hi, int sb = SB) {
  lo = pass * sb;
  hi = min(n, lo + sb);
  return lo < n;
}

template <class T>
__device__ __forceinline__ T* strip_base(const StepArgsT<T>& sa, const StepItem& it, const SysDesc& d, int& ld) {
  ld = (it.kind == kSegRhs) ? d.nrhs : d.n;
  return (it.kind == kSegRhs) ? sa.X + d.b_off : sa.inv + d.inv_off;
}

// Solve rows [lo, hi) of one strip in place: back substitution with U (UPPER,
// 32-row blocks from the bottom) or forward substitution with the unit-lower
// L (blocks from the top). After each diagonal block, the rest of the window
// is updated with the block just solved. Strips of up to 8 columns solve a
// diagonal block with one warp per column (lane i holds row i, the solved
// value is broadcast by shuffle) and update row by row from shared memory;
// wider strips use one thread per column and DMMA tiles.
template <class T, bool UPPER>
__device__ __forceinline__ void window_solve(const T* __restrict__ M, int n, T* X, int ld, int c0, int w, int lo,
                                             int hi) {
  __shared__ T Db[NB * LS];
  __shared__ T Xb[NB * WS];
  __shared__ T As[64 * LS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool narrow = w <= 8;
  const int nblk = (hi - lo + NB - 1) / NB;
  for (int bi = 0; bi < nblk; ++bi) {
    const int kb0 = UPPER ? lo + (nblk - 1 - bi) * NB : lo + bi * NB;
    const int bw = min(NB, hi - kb0);
#pragma unroll
    for (int it_ = 0; it_ < NB * NB / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 5, q = idx & 31;
      Db[i * LS + q] = (i < bw && q < bw) ? M[(int64_t)(kb0 + i) * n + kb0 + q] : (i == q ? T(1) : T(0));
    }
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      Xb[i * WS + c] = (i < bw && c < w) ? X[(int64_t)(kb0 + i) * ld + c0 + c] : T(0);
    }
    __syncthreads();
    if (narrow) {
      if (warp < min(w, 4)) {
        T u[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) u[j] = Db[lane * LS + j];
        const bool two = warp + 4 < w;
        T x0 = Xb[lane * WS + warp], x1 = two ? Xb[lane * WS + warp + 4] : T(0);
        if constexpr (UPPER) {
#pragma unroll
          for (int j = NB - 1; j >= 0; --j) {
            if (lane == j) {
              x0 = x0 / u[j];
              x1 = x1 / u[j];
            }
            const T y0 = __shfl_sync(0xffffffffu, x0, j), y1 = __shfl_sync(0xffffffffu, x1, j);
            if (lane < j) {
              x0 = fma(-u[j], y0, x0);
              x1 = fma(-u[j], y1, x1);
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < NB; ++j) {
            const T y0 = __shfl_sync(0xffffffffu, x0, j), y1 = __shfl_sync(0xffffffffu, x1, j);
            if (lane > j) {
              x0 = fma(-u[j], y0, x0);
              x1 = fma(-u[j], y1, x1);
            }
          }
        }
        Xb[lane * WS + warp] = x0;
        if (two) Xb[lane * WS + warp + 4] = x1;
      }
    } else if (tid < w) {
      if constexpr (UPPER) {
        for (int i = bw - 1; i >= 0; --i) {
          T x = Xb[i * WS + tid];
          for (int q = i + 1; q < bw; ++q) x = fma(-Db[i * LS + q], Xb[q * WS + tid], x);
          Xb[i * WS + tid] = x / Db[i * LS + i];
        }
      } else {
        for (int i = 1; i < bw; ++i) {
          T x = Xb[i * WS + tid];
          for (int q = 0; q < i; ++q) x = fma(-Db[i * LS + q], Xb[q * WS + tid], x);
          Xb[i * WS + tid] = x;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      if (i < bw && c < w) X[(int64_t)(kb0 + i) * ld + c0 + c] = Xb[i * WS + c];
    }
    // the rest of the window: above the block (UPPER) or below it
    const int r_lo = UPPER ? lo : kb0 + bw, r_hi = UPPER ? kb0 : hi;
    for (int r0 = r_lo; r0 < r_hi; r0 += 64) {
#pragma unroll
      for (int it_ = 0; it_ < 64 * NB / UT; ++it_) {
        const int idx = tid + it_ * UT;
        const int i = idx >> 5, q = idx & 31;
        As[i * LS + q] = (r0 + i < r_hi && q < bw) ? M[(int64_t)(r0 + i) * n + kb0 + q] : T(0);
      }
      __syncthreads();
      if (narrow) {
        for (int p = tid; p < 64 * w; p += UT) {
          const int r = p / w, c = p - r * w;
          if (r0 + r < r_hi) {
            T acc = T(0);
#pragma unroll 8
            for (int j = 0; j < NB; ++j) acc = fma(As[r * LS + j], Xb[j * WS + c], acc);
            X[(int64_t)(r0 + r) * ld + c0 + c] -= acc;
          }
        }
      } else {
        tile_update<T>(
            As, Xb, r0, r_hi, w, [&](int r, int cc) { return X[(int64_t)r * ld + c0 + cc]; },
            [&](int r, int cc, T v) { X[(int64_t)r * ld + c0 + cc] = v; });
      }
      __syncthreads();
    }
  }
}

// k_back: X = U^-1 Y on a strip, the window of this pass.
// four CTAs per SM: the substitution is a latency chain per strip, and the
// uneven batches launch thousands of strips
template <class T>
__global__ void __launch_bounds__(UT, 4)
k_back(StepArgsT<T> sa, const StepItem* __restrict__ items, int pass) {
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  if (!sa.solve_only && sa.scratch[d.pad_].info) return;
  int lo, hi, ld;
  if (!back_window(d.n, pass, lo, hi)) return;
  T* X = strip_base(sa, it, d, ld);
  window_solve<T, true>(sa.LU + d.lu_off, d.n, X, ld, it.c0, it.width, lo, hi);
}

// X[r0 .. r0+63] -= M[r0 .. r0+63, lo:hi] X[lo:hi] on one strip (rows < rend):
// the solved window applied to a 64-row tile outside it.
template <class T>
__device__ __forceinline__ void window_apply(const T* __restrict__ M, int n, T* X, int ld, int c0, int w, int r0,
                                             int rend, int lo, int hi) {
  __shared__ T As[64 * LS];
  __shared__ T Bs[NB * WS];
  const int tid = threadIdx.x;
  if (w <= 8) {
    // few columns: a warp takes 4 rows at a time, each row of M read
    // coalesced through the read-only path (all 4 rows' loads in flight
    // together), the window's solved values from shared memory
    constexpr int RPW = 4, JT = SB / 32;
    const int lane = tid & 31, warp = tid >> 5, kw = hi - lo;
    T* xs = As;  // SB x w, zero past kw  (256 x 8 <= 64 x LS elements)
    for (int idx = tid; idx < SB * w; idx += UT) {
      const int j = idx / w, c = idx - j * w;
      xs[idx] = j < kw ? X[(int64_t)(lo + j) * ld + c0 + c] : T(0);
    }
    __syncthreads();
    for (int g0 = warp * RPW; g0 < 64; g0 += (UT / 32) * RPW) {
      if (r0 + g0 >= rend) break;
      T m[RPW][JT];
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        const int r = r0 + g0 + q;
        const T* mr = M + (int64_t)min(r, rend - 1) * n + lo;
#pragma unroll
        for (int t = 0; t < JT; ++t) {
          const int j = t * 32 + lane;
          m[q][t] = (r < rend && j < kw) ? __ldg(mr + j) : T(0);
        }
      }
#pragma unroll
      for (int q = 0; q < RPW; ++q) {
        T mine = T(0);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (c < w) {
            T v = T(0);
#pragma unroll
            for (int t = 0; t < JT; ++t) v = fma(m[q][t], xs[(t * 32 + lane) * w + c], v);
#pragma unroll
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == c) mine = v;
          }
        }
        const int r = r0 + g0 + q;
        if (r < rend && lane < w) X[(int64_t)r * ld + c0 + lane] -= mine;
      }
    }
    return;
  }
  Acc64<T> acc;
  acc.each([&](int r, int cc, T& x) { x = (r0 + r < rend && cc < w) ? X[(int64_t)(r0 + r) * ld + c0 + cc] : T(0); });
  for (int kc = lo; kc < hi; kc += NB) {
    const int kw = min(NB, hi - kc);
#pragma unroll
    for (int it_ = 0; it_ < 64 * NB / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 5, q = idx & 31;
      As[i * LS + q] = (r0 + i < rend && q < kw) ? M[(int64_t)(r0 + i) * n + kc + q] : T(0);
    }
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      Bs[i * WS + c] = (i < kw && c < w) ? X[(int64_t)(kc + i) * ld + c0 + c] : T(0);
    }
    __syncthreads();
    acc.sub_mma(As, Bs);
    __syncthreads();
  }
  acc.each([&](int r, int cc, T& x) {
    if (r0 + r < rend && cc < w) X[(int64_t)(r0 + r) * ld + c0 + cc] = x;
  });
}

// Rows above the window of this pass: one CTA per (strip, 64-row tile = blockIdx.y).
template <class T>
__global__ void __launch_bounds__(UT)
k_back_update(StepArgsT<T> sa, const StepItem* __restrict__ items, int pass, int sb) {
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  if (!sa.solve_only && sa.scratch[d.pad_].info) return;
  int lo, hi, ld;
  if (!back_window(d.n, pass, lo, hi, sb)) return;
  const int r0 = (int)blockIdx.y * 64;
  if (r0 >= lo) return;
  T* X = strip_base(sa, it, d, ld);
  window_apply<T>(sa.LU + d.lu_off, d.n, X, ld, it.c0, it.width, r0, lo, lo, hi);
}

// ---------------------------------------------------------------------------
// getrs from stored factors. k_permute: X[p] = B[perm[p]], perm from the swap
// list; then forward windows with the unit-lower L. X must not alias B.
template <class T>
__global__ void __launch_bounds__(UT)
k_permute(StepArgsT<T> sa, const StepItem* __restrict__ items) {
  extern __shared__ int perm[];
  const int tid = threadIdx.x;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  const int n = d.n, w = it.width, c0 = it.c0, ld = d.nrhs;
  const int32_t* ipiv = sa.ipiv + d.piv_off;
  const T* B = sa.B + d.b_off;
  T* X = sa.X + d.b_off;
  int* piv = perm + n;
  for (int i = tid; i < n; i += UT) {
    perm[i] = i;
    piv[i] = ipiv[i];
  }
  __syncthreads();
  if (tid == 0) {
    for (int k = 0; k < n; ++k) {
      int p = piv[k];
      if (p < k || p >= n) p = k;  // a swap list only names rows >= k
      const int t = perm[k]; perm[k] = perm[p]; perm[p] = t;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < n * 64; idx += UT) {
    const int p = idx >> 6, c = idx & 63;
    if (c < w) X[(int64_t)p * ld + c0 + c] = B[(int64_t)perm[p] * ld + c0 + c];
  }
}

template <class T>
__global__ void __launch_bounds__(UT)
k_forward(StepArgsT<T> sa, const StepItem* __restrict__ items, int pass) {
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  int lo, hi;
  if (!forward_window(d.n, pass, lo, hi)) return;
  window_solve<T, false>(sa.LU + d.lu_off, d.n, sa.X + d.b_off, d.nrhs, it.c0, it.width, lo, hi);
}

// Strips of at most 8 columns (few right-hand sides): the whole window of M
// (SBN x SBN) is staged into shared memory once, then the window is solved
// from shared memory: each 32-row diagonal block by one warp per column
// (lane i holds row i; the solved value is broadcast by shuffle), the rest of
// the window by one warp per row. UPPER: back substitution with U from the
// bottom; else forward substitution with the unit-lower L from the top.
constexpr int SBN = 128;
constexpr int MSN = SBN + 2;  // row stride of the staged window (16-byte rows)

template <class T>
size_t narrow_smem() {
  return sizeof(T) * ((size_t)SBN * MSN + 8 * SBN);
}

template <class T, bool UPPER>
__global__ void __launch_bounds__(UT)
k_tri_narrow(StepArgsT<T> sa, const StepItem* __restrict__ items, int pass) {
  extern __shared__ __align__(16) unsigned char tri_raw[];
  T* Ms = reinterpret_cast<T*>(tri_raw);  // window of M, stride MSN
  T* xt = Ms + SBN * MSN;                 // window of X, column-major: xt[c * SBN + row]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  if (UPPER && !sa.solve_only && sa.scratch[d.pad_].info) return;
  const int n = d.n;
  int lo, hi;
  if (!(UPPER ? back_window(n, pass, lo, hi, SBN) : forward_window(n, pass, lo, hi, SBN))) return;
  int ld;
  T* X;
  if constexpr (UPPER) {
    X = strip_base(sa, it, d, ld);
  } else {
    X = sa.X + d.b_off;
    ld = d.nrhs;
  }
  const int kw = hi - lo, w = it.width, c0 = it.c0;
  const T* M = sa.LU + d.lu_off + (int64_t)lo * n + lo;
  async_tile<T>(Ms, MSN, M, n, kw, kw, kw, (kw + 1) & ~1, pair_aligned(M, n));  // only the live window
  for (int idx = tid; idx < 8 * SBN; idx += UT) {
    const int c = idx / SBN, j = idx - c * SBN;
    xt[idx] = (c < w && j < kw) ? X[(int64_t)(lo + j) * ld + c0 + c] : T(0);
  }
  cp_async_wait<0>();
  __syncthreads();
  const int nblk = (kw + NB - 1) / NB;
  for (int bi = 0; bi < nblk; ++bi) {
    const int b0 = UPPER ? (nblk - 1 - bi) * NB : bi * NB;  // window-relative
    const int bw = min(NB, kw - b0);
    if (warp < min(w, 4)) {
      const bool two = warp + 4 < w, in = lane < bw;
      T u[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) u[j] = (in && j < bw) ? Ms[(b0 + lane) * MSN + b0 + j] : (lane == j ? T(1) : T(0));
      T* x0p = xt + warp * SBN + b0;
      T* x1p = xt + (warp + 4) * SBN + b0;
      T x0 = in ? x0p[lane] : T(0), x1 = (in && two) ? x1p[lane] : T(0);
      if constexpr (UPPER) {
        // every lane takes the reciprocal of its own diagonal entry up front
        const T rd = T(1) / (in ? Ms[(b0 + lane) * MSN + b0 + lane] : T(1));
#pragma unroll
        for (int j = NB - 1; j >= 0; --j) {
          if (lane == j) {
            x0 *= rd;
            x1 *= rd;
          }
          const T y0 = __shfl_sync(0xffffffffu, x0, j), y1 = __shfl_sync(0xffffffffu, x1, j);
          if (lane < j) {
            x0 = fma(-u[j], y0, x0);
            x1 = fma(-u[j], y1, x1);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          const T y0 = __shfl_sync(0xffffffffu, x0, j), y1 = __shfl_sync(0xffffffffu, x1, j);
          if (lane > j) {
            x0 = fma(-u[j], y0, x0);
            x1 = fma(-u[j], y1, x1);
          }
        }
      }
      if (in) {
        x0p[lane] = x0;
        if (two) x1p[lane] = x1;
      }
    }
    __syncthreads();
    const int r_lo = UPPER ? 0 : b0 + bw, r_hi = UPPER ? b0 : kw;
    for (int r = r_lo + warp; r < r_hi; r += UT / 32) {
      const T m = lane < bw ? Ms[r * MSN + b0 + lane] : T(0);
      for (int c = 0; c < w; ++c) {
        T v = m * xt[c * SBN + b0 + lane];
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) xt[c * SBN + r] -= v;
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < w * SBN; idx += UT) {
    const int c = idx / SBN, j = idx - c * SBN;
    if (j < kw) X[(int64_t)(lo + j) * ld + c0 + c] = xt[idx];
  }
}

// Rows below the window of this pass: one CTA per (strip, 64-row tile = blockIdx.y).
template <class T>
__global__ void __launch_bounds__(UT)
k_forward_update(StepArgsT<T> sa, const StepItem* __restrict__ items, int pass, int sb) {
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  int lo, hi;
  if (!forward_window(d.n, pass, lo, hi, sb)) return;
  const int r0 = hi + (int)blockIdx.y * 64;
  if (r0 >= d.n) return;
  window_apply<T>(sa.LU + d.lu_off, d.n, sa.X + d.b_off, d.nrhs, it.c0, it.width, r0, d.n, lo, hi);
}

template <class T, int MODE>
cudaError_t prepare_update() {
  return cudaFuncSetAttribute(k_update<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)update_smem<T, MODE>());
}

// Passes over windows (SB rows, or SBN for strips of at most 8 columns of
// systems above 2 * SB);
// between two windows, the solved one is applied to the rows on the far side
// (tiles of 64 rows: blockIdx.y).
template <class T>
cudaError_t windowed(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int wmax, bool forward,
                     cudaStream_t st) {
  // the narrow kernels pay off once a system needs more than two wide windows
  const bool narrow = wmax <= 8 && nmax > 2 * SB;
  const int sb = narrow ? SBN : SB;
  const int passes = (nmax + sb - 1) / sb;
  for (int p = 0; p < passes; ++p) {
    if (narrow) {
      if (forward) k_tri_narrow<T, false><<<nitems, UT, narrow_smem<T>(), st>>>(sa, items, p);
      else k_tri_narrow<T, true><<<nitems, UT, narrow_smem<T>(), st>>>(sa, items, p);
    } else {
      if (forward) k_forward<T><<<nitems, UT, 0, st>>>(sa, items, p);
      else k_back<T><<<nitems, UT, 0, st>>>(sa, items, p);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // rows left on the far side of this pass's window, largest system first
    const int far = forward ? nmax - (p + 1) * sb : ((nmax - 1) / sb - p) * sb;
    if (p + 1 < passes && far > 0) {
      const dim3 grid((unsigned)nitems, (unsigned)((far + 63) / 64));
      if (forward) k_forward_update<T><<<grid, UT, 0, st>>>(sa, items, p, sb);
      else k_back_update<T><<<grid, UT, 0, st>>>(sa, items, p, sb);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// k_block_rows: the trailing pass after an outer block of the two-level
// factorisation, one CTA per (system, 64-column strip right of the block).
// First the block's recorded row moves, panel by panel, on the strip in
// global memory (rows no update has touched yet, as LAPACK's laswp); then the
// block's rows of the strip in shared memory: per panel, U12 = L11^-1 A12
// (DMMA) and the update of the block rows below that panel; then the rows go
// back. What is left below the block is one GEMM (k_block_gemm).
template <class T>
constexpr size_t block_rows_smem() {
  return sizeof(T) * ((size_t)kStepNBO * WS + 64 * LS + NB * LS);
}

template <class T>
__global__ void __launch_bounds__(UT)
k_block_rows(StepArgsT<T> sa, int bbeg, int bend) {
  extern __shared__ __align__(16) unsigned char br_raw[];
  T* X = reinterpret_cast<T*>(br_raw);  // the block's rows of the strip, kStepNBO x WS
  T* Lt = X + kStepNBO * WS;            // L rows below a panel inside the block, 64 x LS
  T* Li = Lt + 64 * LS;                 // L11^-1 of a panel, NB x LS
  __shared__ int tsrc[NB], ddst[NB], dsrc[NB];
  const int tid = threadIdx.x;
  const StepItem it = uniform_item(sa, blockIdx.x, bbeg, false);
  const SysDesc d = step_desc(sa, it.sys);
  if (sa.scratch[d.pad_].info) return;
  const StepHistT<T>* hs = sa.hist + d.pad_;
  const int n = d.n, w = it.width, c0 = it.c0, bw = bend - bbeg;
  const int64_t ld = n;
  T* const F = sa.LU + d.lu_off + c0;  // column c0 of row 0
  // 1. row moves, in panel order (all reads of a panel before its writes)
  for (int s = 0; s * NB < bw; ++s) {
    const int k0 = bbeg + s * NB, kb = min(NB, n - k0), nd = hs->ndisp[s];
    if (tid < NB) {
      tsrc[tid] = tid < kb ? hs->top_src[s][tid] : 0;
      ddst[tid] = tid < nd ? hs->disp_dst[s][tid] : 0;
      dsrc[tid] = tid < nd ? hs->disp_src[s][tid] : 0;
    }
    __syncthreads();
    T* Tm = X;
    T* D = X + NB * WS;
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      const bool in = c < w;
      Tm[i * WS + c] = (in && i < kb) ? F[(int64_t)(k0 + tsrc[i]) * ld + c] : T(0);
      D[i * WS + c] = (in && i < nd) ? F[(int64_t)(k0 + dsrc[i]) * ld + c] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int it_ = 0; it_ < NB * 64 / UT; ++it_) {
      const int idx = tid + it_ * UT;
      const int i = idx >> 6, c = idx & 63;
      if (c < w && i < nd) F[(int64_t)(k0 + ddst[i]) * ld + c] = D[i * WS + c];
      if (c < w && i < kb) F[(int64_t)(k0 + i) * ld + c] = Tm[i * WS + c];
    }
    __syncthreads();
  }
  // 2. the block's rows into shared memory
  for (int idx = tid; idx < kStepNBO * 64; idx += UT) {
    const int i = idx >> 6, c = idx & 63;
    X[i * WS + c] = (i < bw && c < w) ? F[(int64_t)(bbeg + i) * ld + c] : T(0);
  }
  // 3. per panel: U12, then the block rows below it
  for (int s = 0; s * NB < bw; ++s) {
    const int k0 = bbeg + s * NB;
    const T* linv = hs->linv[s];
#pragma unroll
    for (int it_ = 0; it_ < NB * NB / UT; ++it_) {
      const int idx = tid + it_ * UT;
      Li[(idx >> 5) * LS + (idx & 31)] = linv[idx];
    }
    __syncthreads();
    T* Xs = X + s * NB * WS;
    {
      Acc32<T> u;
      u.mma(Li, Xs);
      __syncthreads();
      u.each([&](int i, int c, T& x) { Xs[i * WS + c] = x; });
    }
    for (int r0 = (s + 1) * NB; r0 < bw; r0 += 64) {
      const int rows = min(64, bw - r0);
      __syncthreads();
#pragma unroll
      for (int it_ = 0; it_ < 64 * NB / UT; ++it_) {
        const int idx = tid + it_ * UT;
        const int i = idx >> 5, c = idx & 31;
        Lt[i * LS + c] = i < rows ? sa.LU[d.lu_off + (int64_t)(bbeg + r0 + i) * ld + k0 + c] : T(0);
      }
      __syncthreads();
      Acc64<T> acc;
      acc.each([&](int r, int c, T& v) { v = r < rows ? X[(r0 + r) * WS + c] : T(0); });
      acc.sub_mma(Lt, Xs);
      acc.each([&](int r, int c, T& v) {
        if (r < rows) X[(r0 + r) * WS + c] = v;
      });
    }
    __syncthreads();
  }
  // 4. back
  for (int idx = tid; idx < kStepNBO * 64; idx += UT) {
    const int i = idx >> 6, c = idx & 63;
    if (i < bw && c < w) F[(int64_t)(bbeg + i) * ld + c] = X[i * WS + c];
  }
}

// ---------------------------------------------------------------------------
// k_block_gemm: the trailing update after an outer block of the two-level
// factorisation, C -= L U with C = rows [bend, n) x columns [cbeg, cend), L =
// rows [bend, n) x columns [bbeg, bend), U = rows [bbeg, bend) x [cbeg, cend),
// all in place in the system's factor matrix (row-major, leading dimension n).
// One CTA per 128 x 64 tile of C (grid.z = system); K = bend - bbeg <= 128 in
// 8-deep slabs double-buffered through shared memory (cp.async), C read once
// into the DMMA accumulators and written once.
constexpr int GBM = 128, GBN = 64, GBK = 8, GNT = 256;
constexpr int GAS = GBK + 1, GBS = GBN + 1;

__global__ void __launch_bounds__(GNT, 2)
k_block_gemm(StepArgsT<double> sa, int bbeg, int bend, int cbeg, int cend) {
  __shared__ double As[2][GBM * GAS];
  __shared__ double Bs[2][GBK * GBS];
  const SysDesc d = step_desc(sa, (int)blockIdx.z);
  if (sa.scratch[d.pad_].info) return;
  const int n = d.n;
  const int M = n - bend, N = cend - cbeg, K = bend - bbeg;
  double* const F = sa.LU + d.lu_off;
  const double* const Lp = F + (int64_t)bend * n + bbeg;  // M x K
  const double* const Up = F + (int64_t)bbeg * n + cbeg;  // K x N
  double* const Cp = F + (int64_t)bend * n + cbeg;        // M x N
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int bm = (int)blockIdx.y * GBM, bn = (int)blockIdx.x * GBN;
  if (bm >= M || bn >= N) return;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

  auto load = [&](int stage, int k0) {
#pragma unroll
    for (int i = 0; i < (GBM * GBK) / GNT; ++i) {
      const int idx = tid + i * GNT;
      const int r = idx / GBK, c = idx % GBK;
      const bool ok = bm + r < M && k0 + c < K;
      cp_async<8>(&As[stage][r * GAS + c], ok ? Lp + (int64_t)(bm + r) * n + k0 + c : Lp, ok);
    }
#pragma unroll
    for (int i = 0; i < (GBK * GBN) / GNT; ++i) {
      const int idx = tid + i * GNT;
      const int r = idx / GBN, c = idx % GBN;
      const bool ok = k0 + r < K && bn + c < N;
      cp_async<8>(&Bs[stage][r * GBS + c], ok ? Up + (int64_t)(k0 + r) * n + bn + c : Up, ok);
    }
    cp_async_commit();
  };

  const int nk = (K + GBK - 1) / GBK;
  load(0, 0);
  double acc[4][4][2];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int row = bm + wm + mi * 8 + g;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = bn + wn + ni * 8 + 2 * tq + e;
        acc[mi][ni][e] = (row < M && col < N) ? Cp[(int64_t)row * n + col] : 0.0;
      }
    }
  }
  for (int kt = 0; kt < nk; ++kt) {
    const int st = kt & 1;
    if (kt + 1 < nk) {
      load(st ^ 1, (kt + 1) * GBK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = -As[st][(wm + mi * 8 + g) * GAS + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[st][(kk + tq) * GBS + wn + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], af[mi], bf[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int row = bm + wm + mi * 8 + g;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = bn + wn + ni * 8 + 2 * tq + e;
        if (row < M && col < N) Cp[(int64_t)row * n + col] = acc[mi][ni][e];
      }
    }
  }
}

}  // namespace

int tc_timeouts_take() {
  int h = 0;
  if (cudaMemcpyFromSymbol(&h, g_tc_timeouts, sizeof(int)) != cudaSuccess) return -1;
  if (h) {
    const int z = 0;
    cudaMemcpyToSymbol(g_tc_timeouts, &z, sizeof(int));
  }
  return h;
}

template <class T>
cudaError_t prepare_narrow() {
  cudaError_t e = cudaFuncSetAttribute(k_tri_narrow<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)narrow_smem<T>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tri_narrow<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)narrow_smem<T>());
}

template <class T, int NT, int RPT, int CS>
cudaError_t prepare_panel1() {
  return cudaFuncSetAttribute(k_panel<T, NT, RPT, CS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)panel_smem<T, NT, RPT>());
}

template <class T>
cudaError_t prepare_panel() {
  cudaError_t e = prepare_panel1<T, 64, 1, 1>();
  if (e == cudaSuccess) e = prepare_panel1<T, 128, 1, 1>();
  if (e == cudaSuccess) e = prepare_panel1<T, 256, 1, 1>();
  if (e == cudaSuccess) e = prepare_panel1<T, 512, 1, 1>();
  if (e == cudaSuccess) e = prepare_panel1<T, 512, 1, 2>();
  if (e == cudaSuccess) e = prepare_panel1<T, 512, 1, 4>();
  if (e == cudaSuccess) e = prepare_panel1<T, 512, 1, 8>();
  return e;
}

cudaError_t step_prepare() {
  cudaError_t e = prepare_narrow<double>();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_block_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_rows_smem<double>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_block_rows<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)block_rows_smem<float>());
  if (e == cudaSuccess) e = prepare_panel<double>();
  if (e == cudaSuccess) e = prepare_panel<float>();
  if (e == cudaSuccess) e = prepare_narrow<float>();
  if (e == cudaSuccess) e = prepare_update<double, kUpdFp32>();
  if (e == cudaSuccess) e = prepare_update<float, kUpdFp32>();
  if (e == cudaSuccess) e = prepare_update<float, kUpdTf32>();
  if (e == cudaSuccess) e = prepare_update<float, kUpdBf16>();
  if (e == cudaSuccess) e = prepare_update<float, kUpd3xTf32>();
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tc<kUpdTf32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)update_tc_smem<kUpdTf32>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tc<kUpd3xTf32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)update_tc_smem<kUpd3xTf32>());
  return e;
}

template <class T, int CS>
cudaError_t launch_cluster_panel(const StepArgsT<T>& sa, const int32_t* list, int nsys, int k0, cudaStream_t st) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)nsys * CS);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = panel_smem<T, 512, 1>();
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_panel<T, 512, 1, CS>, sa, list, k0);
}

template <class T>
cudaError_t launch_panel(const StepArgsT<T>& sa, const int32_t* list, int nsys, int mmax, int k0,
                         cudaStream_t st) {
  if (nsys <= 0) return cudaSuccess;
  if (mmax <= 64) k_panel<T, 64, 1, 1><<<nsys, 64, panel_smem<T, 64, 1>(), st>>>(sa, list, k0);
  else if (mmax <= 128) k_panel<T, 128, 1, 1><<<nsys, 128, panel_smem<T, 128, 1>(), st>>>(sa, list, k0);
  else if (mmax <= 256) k_panel<T, 256, 1, 1><<<nsys, 256, panel_smem<T, 256, 1>(), st>>>(sa, list, k0);
  else if (mmax <= 512) k_panel<T, 512, 1, 1><<<nsys, 512, panel_smem<T, 512, 1>(), st>>>(sa, list, k0);
  else if (mmax <= 1024) return launch_cluster_panel<T, 2>(sa, list, nsys, k0, st);
  else if (mmax <= 2048) return launch_cluster_panel<T, 4>(sa, list, nsys, k0, st);
  else if (mmax <= 4096) return launch_cluster_panel<T, 8>(sa, list, nsys, k0, st);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_rows(const StepArgsT<T>& sa, const StepItem* items, int nitems, int k0, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  k_rows<T><<<nitems, UT, 0, st>>>(sa, items, k0);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_trailing(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int k0, int part,
                            cudaStream_t st) {
  const int below = nmax - k0 - NB;
  if (nitems <= 0 || below <= 0) return cudaSuccess;
  const int rg = part == 1 ? RG1 : RG;
  const dim3 grid((unsigned)nitems, (unsigned)((below + rg - 1) / rg));
  if constexpr (std::is_same_v<T, float>) {
    switch (sa.umode) {
      case kUpdTf32:
        k_update<T, kUpdTf32><<<grid, UT, update_smem<T, kUpdTf32>(), st>>>(sa, items, k0, part);
        return cudaGetLastError();
      case kUpdBf16:
        k_update<T, kUpdBf16><<<grid, UT, update_smem<T, kUpdBf16>(), st>>>(sa, items, k0, part);
        return cudaGetLastError();
      case kUpd3xTf32:
        k_update<T, kUpd3xTf32><<<grid, UT, update_smem<T, kUpd3xTf32>(), st>>>(sa, items, k0, part);
        return cudaGetLastError();
      case kUpdTcTf32:
        k_update_tc<kUpdTf32><<<grid, UT, update_tc_smem<kUpdTf32>(), st>>>(sa, items, k0, part);
        return cudaGetLastError();
      case kUpdTc3xTf32:
        k_update_tc<kUpd3xTf32><<<grid, UT, update_tc_smem<kUpd3xTf32>(), st>>>(sa, items, k0, part);
        return cudaGetLastError();
      default:
        break;
    }
  }
  k_update<T, kUpdFp32><<<grid, UT, update_smem<T, kUpdFp32>(), st>>>(sa, items, k0, part);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_update(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int k0,
                          cudaStream_t st) {
  cudaError_t e = launch_rows(sa, items, nitems, k0, st);
  if (e != cudaSuccess) return e;
  return launch_trailing(sa, items, nitems, nmax, k0, 0, st);
}

template <class T>
cudaError_t launch_block_gemm(const StepArgsT<T>& sa, int count, int bbeg, int bend, int cbeg, int cend,
                              cudaStream_t st) {
  const int M = sa.un - bend, N = cend - cbeg;
  if (M <= 0 || N <= 0 || count <= 0) return cudaSuccess;
  if constexpr (!std::is_same_v<T, double>) {
    return cudaErrorInvalidValue;  // FP32 factors keep the one-level schedule
  } else {
    const dim3 grid((unsigned)((N + GBN - 1) / GBN), (unsigned)((M + GBM - 1) / GBM), (unsigned)count);
    k_block_gemm<<<grid, GNT, 0, st>>>(sa, bbeg, bend, cbeg, cend);
    return cudaGetLastError();
  }
}

template <class T>
cudaError_t launch_block_rows(const StepArgsT<T>& sa, int count, int bbeg, int bend, cudaStream_t st) {
  const int64_t items = (int64_t)count * trailing_strips(sa.un, bend);
  if (items <= 0) return cudaSuccess;
  if (items > INT32_MAX) return cudaErrorInvalidValue;
  StepArgsT<T> tr = sa;
  tr.utrail = 1;
  tr.ubend = bend;
  k_block_rows<T><<<(unsigned)items, UT, block_rows_smem<T>(), st>>>(tr, bbeg, bend);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_back(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int wmax,
                        cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  return windowed<T>(sa, items, nitems, nmax, wmax, false, st);
}

template <class T>
cudaError_t launch_forward(const StepArgsT<T>& sa, const StepItem* items, int nitems, int nmax, int wmax,
                           cudaStream_t st, bool permute) {
  if (nitems <= 0) return cudaSuccess;
  if (permute) {
    k_permute<T><<<nitems, UT, 2 * sizeof(int) * (size_t)nmax, st>>>(sa, items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return windowed<T>(sa, items, nitems, nmax, wmax, true, st);
}

#define NPPB_STEP_INSTANTIATE(T)                                                                          \
  template cudaError_t launch_panel<T>(const StepArgsT<T>&, const int32_t*, int, int, int, cudaStream_t);     \
  template cudaError_t launch_update<T>(const StepArgsT<T>&, const StepItem*, int, int, int, cudaStream_t);   \
  template cudaError_t launch_block_gemm<T>(const StepArgsT<T>&, int, int, int, int, int, cudaStream_t);    \
  template cudaError_t launch_block_rows<T>(const StepArgsT<T>&, int, int, int, cudaStream_t);              \
  template cudaError_t launch_rows<T>(const StepArgsT<T>&, const StepItem*, int, int, cudaStream_t);          \
  template cudaError_t launch_trailing<T>(const StepArgsT<T>&, const StepItem*, int, int, int, int,          \
                                          cudaStream_t);                                                     \
  template cudaError_t launch_back<T>(const StepArgsT<T>&, const StepItem*, int, int, int, cudaStream_t);          \
  template cudaError_t launch_forward<T>(const StepArgsT<T>&, const StepItem*, int, int, int, cudaStream_t, bool);
NPPB_STEP_INSTANTIATE(double)
NPPB_STEP_INSTANTIATE(float)
#undef NPPB_STEP_INSTANTIATE

}  // namespace nppb
