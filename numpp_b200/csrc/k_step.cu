// Step-wise batched LU for orders n > 32 (any mix of orders in one batch).
//
// The reference factors one matrix at a time with an unblocked right-looking
// elimination (src/linalg/linalg.cpp:48-71) and then solves (:73-90). Here the
// same elimination is blocked by 32-column panels and run for every system of
// the batch at once, one step (panel) per pair of launches:
//
//  k_panel   one CTA per active system: the (n-k0) x 32 panel lives in
//            registers (row r of the panel in thread r mod NT), the pivot of each
//            column is the first largest |a| in position order (the reference's
//            rule, linalg.cpp:55-57) found with one barrier per column; a row
//            exchange only swaps the two rows' position labels. It writes the
//            panel at its pivoted positions, the pivots, L11^-1 (for the update)
//            and the row moves the panel implies for every other column, and
//            folds the pivots into det / slogdet in the reference's order.
//  k_update  one CTA per (system, 64-column strip) of the trailing matrix, of
//            the right-hand sides (augmented columns: forward substitution rides
//            along) and of the identity (inverse): apply the row moves,
//            U12 = L11^-1 A12 and A22 -= L21 U12 on FP64 DMMA (mma.m8n8k4).
//  k_back    one CTA per (system, 64-column strip) of X / inverse: blocked back
//            substitution with U (diagonal blocks by substitution, the rest DMMA).
//  k_forward getrs from stored factors: row gather through the pivots and
//            blocked forward substitution with the unit-lower L.
//
// Step 0 reads A / B / I directly and writes the workspace, so no copy pass is
// needed. Exact-zero pivots stop the system (info = k+1) and later launches
// skip it, as the reference stops (linalg.cpp:56).
#include <climits>
#include <cmath>

#include "dmma.cuh"
#include "nppb_step.hpp"

namespace nppb {
namespace {

constexpr int NB = kStepNB;  // 32
constexpr int LS = NB + 1;   // 33: stride of 32-wide shared tiles
constexpr int WS = 64 + 1;   // 65: stride of 64-wide shared tiles

// ---------------------------------------------------------------------------
// System descriptor: from the list, or derived for a uniform batch.
__device__ __forceinline__ SysDesc step_desc(const StepArgs& sa, int s) {
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

__device__ __forceinline__ StepItem uniform_item(const StepArgs& sa, int b, int k0, bool back) {
  const int n = sa.un;
  const int trail = n - k0 - NB;
  const int nm = back ? 0 : (trail > 0 ? (trail + 63) / 64 : 0);
  const int nr = (sa.unrhs + 63) / 64;
  const int ni = sa.uinv ? (n + 63) / 64 : 0;
  const int per = nm + nr + ni;
  StepItem it;
  it.sys = b / per;
  int r = b % per;
  it.pad_ = 0;
  if (r < nm) {
    it.kind = kSegMatrix;
    it.c0 = k0 + NB + 64 * r;
    it.width = (int16_t)min(64, n - it.c0);
  } else if ((r -= nm) < nr) {
    it.kind = kSegRhs;
    it.c0 = 64 * r;
    it.width = (int16_t)min(64, sa.unrhs - it.c0);
  } else {
    r -= nr;
    it.kind = kSegInv;
    it.c0 = 64 * r;
    it.width = (int16_t)min(64, n - it.c0);
  }
  return it;
}

// ---------------------------------------------------------------------------
// k_panel
template <int NT, int RPT>
__global__ void __launch_bounds__(NT, (RPT == 1 ? 65536 / (NT * 128) : 1))
k_panel(StepArgs sa, const int32_t* __restrict__ list, int k0) {
  constexpr int NW = NT / 32;
  __shared__ __align__(16) double cand_row[2][NW][NB];
  __shared__ double cand_v[2][NW];
  __shared__ int cand_k[2][NW];
  __shared__ double L11[NB][LS];
  __shared__ double Xinv[NB][LS];
  __shared__ double pvals[NB];
  __shared__ int s_ndisp;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const SysDesc d = step_desc(sa, list ? list[blockIdx.x] : (int)blockIdx.x);
  StepScratch* sc = sa.scratch + d.pad_;
  const int n = d.n, m = n - k0, kb = min(NB, m);
  if (k0 == 0) {
    if (tid == 0) {
      sc->info = 0; sc->nswap = 0; sc->det = 1.0; sc->logabs = 0.0; sc->sign = 1.0;
    }
    __syncthreads();
  } else if (sc->info) {
    return;
  }
  double* dst = sa.LU + d.lu_off;
  const double* src = (k0 == 0 && sa.A) ? sa.A + d.a_off : dst;

  double a[RPT][NB];
  int pos[RPT];
  bool valid[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = tid + q * NT;
    valid[q] = r < m;
    pos[q] = r;
    const double* row = src + (int64_t)(k0 + r) * n + k0;
#pragma unroll
    for (int c = 0; c < NB; ++c) a[q][c] = (valid[q] && c < kb) ? row[c] : 0.0;
  }
  if (tid == 0) s_ndisp = 0;

  // Column loop. Each row is kept rotated so that the current block of 8
  // columns always sits in a[q][0..7]: the body below is written once for 8
  // columns (compile-time register indices) and run 4 times, with an 8-place
  // circular rotation in between; after the 4th rotation the row is back in
  // column order. The multiplier L (rows below the pivot) overwrites the
  // column entry it came from. Small code, few moves per column.
  int info = 0;
  int nswap = 0;
#pragma unroll 1
  for (int jb = 0; jb < NB; jb += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int j = jb + u;
      if (j < kb && !info) {  // uniform across the CTA
        double best = -1.0;
        int key = INT_MAX;
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          if (valid[q] && pos[q] >= j) {
            const double v = fabs(a[q][u]);
            if (v > best || (v == best && pos[q] < key)) { best = v; key = pos[q]; }
          }
        }
        warp_argmax_abs(best, key);
        const int par = j & 1;
        if (lane == 0) { cand_v[par][warp] = best; cand_k[par][warp] = key; }
        // the candidate row is published with its finished columns (rotated
        // slots past lim) zeroed, so the update below needs no predicates
        const int lim = NB - 1 - jb;
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          if (valid[q] && pos[q] == key) {
            double2* cr = reinterpret_cast<double2*>(cand_row[par][warp]);
#pragma unroll
            for (int c = 0; c < NB / 2; ++c)
              cr[c] = make_double2(2 * c <= lim ? a[q][2 * c] : 0.0, 2 * c + 1 <= lim ? a[q][2 * c + 1] : 0.0);
          }
        }
        __syncthreads();
        double gb = -1.0;
        int gk = INT_MAX, gw = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          const double v = cand_v[par][w];
          const int k = cand_k[par][w];
          if (v > gb || (v == gb && k < gk)) { gb = v; gk = k; gw = w; }
        }
        if (gb == 0.0) {
          info = k0 + j + 1;
        } else {
          const double2* pr2 = reinterpret_cast<const double2*>(cand_row[par][gw]);
          const double pj = cand_row[par][gw][u];
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            if (valid[q]) {
              if (pos[q] == j) pos[q] = gk;
              else if (pos[q] == gk) pos[q] = j;
            }
          }
          if (tid == 0) {
            pvals[j] = pj;
            if (sa.ipiv) sa.ipiv[d.piv_off + k0 + j] = k0 + gk;
          }
          nswap += (gk != j);
          // rotated columns u+1 .. lim hold the trailing columns j+1 .. 31; the
          // published pivot row is zero beyond lim, so those slots stay as they are
          const double rp = 1.0 / pj;
          double f[RPT];
#pragma unroll
          for (int q = 0; q < RPT; ++q) {
            const bool below = valid[q] && pos[q] > j;
            f[q] = below ? a[q][u] * rp : 0.0;
            if (below) a[q][u] = f[q];
          }
#pragma unroll
          for (int c2 = (u + 1) / 2; c2 < NB / 2; ++c2) {
            const double2 t = pr2[c2];
            const int c = 2 * c2;
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
              if (c > u) a[q][c] = fma(-f[q], t.x, a[q][c]);
              a[q][c + 1] = fma(-f[q], t.y, a[q][c + 1]);
            }
          }
        }
      }
    }
    // circular rotation by 8
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      double t[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) t[c] = a[q][c];
#pragma unroll
      for (int c = 0; c < NB - 8; ++c) a[q][c] = a[q][c + 8];
#pragma unroll
      for (int c = 0; c < 8; ++c) a[q][NB - 8 + c] = t[c];
    }
  }

  if (info) {
    if (tid == 0) {
      sc->info = info;
      if (sa.det) sa.det[d.idx] = 0.0;
      if (sa.sign) sa.sign[d.idx] = 0.0;
      if (sa.logabs) sa.logabs[d.idx] = -INFINITY;
      if (sa.info) sa.info[d.idx] = info;
    }
    return;
  }

  // panel back at the pivoted positions; L11 into shared memory
  for (int idx = tid; idx < NB * NB; idx += NT) {
    const int i = idx / NB, c = idx % NB;
    L11[i][c] = (i == c) ? 1.0 : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (valid[q]) {
      double* row = dst + (int64_t)(k0 + pos[q]) * n + k0;
#pragma unroll 32
      for (int c = 0; c < NB; ++c)
        if (c < kb) row[c] = a[q][c];
      if (pos[q] < kb) {
#pragma unroll 32
        for (int c = 0; c < NB; ++c)
          if (c < pos[q]) L11[pos[q]][c] = a[q][c];
      }
      // row moves for the other columns
      const int r = tid + q * NT;
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
  if (tid == 0) sc->ndisp = s_ndisp;

  // L11^-1 (unit lower, identity-padded past kb): lane c builds column c in
  // shared memory; four partial sums per entry shorten the dependent chain
  if (warp == 0) {
#pragma unroll 1
    for (int i = 0; i < NB; ++i) {
      double p0 = (i == lane) ? 1.0 : 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
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
      const double x = (p0 + p1) + (p2 + p3);
      Xinv[i][lane] = x;
      sc->linv[i * NB + lane] = x;
    }
  }

  // det / slogdet: pivots folded in the reference's order (linalg.cpp:400-403, 425-431)
  if (warp == (NW > 1 ? 1 : 0)) {
    const double lg = lane < kb ? log(fabs(pvals[lane])) : 0.0;
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
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(pred ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

struct Seg {
  double* dst;         // where the strip lives
  const double* src;   // where it is read from (== dst after step 0)
  int ld;
  bool ident;          // source is the identity (inverse at step 0)
};

__device__ inline Seg segment(const StepArgs& sa, const SysDesc& d, int kind, int k0) {
  Seg s;
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

__device__ __forceinline__ double seg_load(const Seg& s, int row, int col) {
  return s.ident ? (row == col ? 1.0 : 0.0) : s.src[(int64_t)row * s.ld + col];
}

// C[rows r0.., 64 cols] -= A[rows r0.., 32] * Bs[32][64] for rows [r0, rend), one
// 64x64 tile per call, 4 warps in 2x2. As holds the A rows (64 x LS), Bs the
// 32 x 64 right operand (WS stride). `crow(r, cc)` reads the input value of row
// r, column cc; `cstore(r, cc, v)` writes it.
template <class Load, class Store>
__device__ __forceinline__ void tile_update(const double* As, const double* Bs, int r0, int rend,
                                            int w, Load cload, Store cstore) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  double acc[4][4][2];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int r = r0 + wm + mi * 8 + g;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cc = wn + ni * 8 + 2 * tq + e;
        acc[mi][ni][e] = (r < rend && cc < w) ? cload(r, cc) : 0.0;
      }
    }
  }
#pragma unroll
  for (int kk = 0; kk < NB; kk += 4) {
    double af[4], bf[4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) af[mi] = -As[(wm + mi * 8 + g) * LS + kk + tq];
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[(kk + tq) * WS + wn + ni * 8 + g];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], af[mi], bf[ni]);
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi) {
    const int r = r0 + wm + mi * 8 + g;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cc = wn + ni * 8 + 2 * tq + e;
        if (r < rend && cc < w) cstore(r, cc, acc[mi][ni][e]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_update
constexpr int UT = 128;

__global__ void __launch_bounds__(UT)
k_update(StepArgs sa, const StepItem* __restrict__ items, int k0) {
  extern __shared__ __align__(16) double smem[];
  double* Us = smem;                 // 32 x WS   U12 strip
  double* D = Us + NB * WS;          // 32 x WS   displaced rows
  double* T = D + NB * WS;           // 64 x LS   A12 (permuted, 32 x WS), then L21 buffer 1
  double* As = T + 64 * LS;          // 64 x LS   L11^-1, then L21 buffer 0
  int* tsrc = reinterpret_cast<int*>(As + 64 * LS);
  int* ddst = tsrc + NB;
  int* dsrc = ddst + NB;
  int* dmap = dsrc + NB;             // m entries: displaced index of each row, or -1

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, k0, false);
  const SysDesc d = step_desc(sa, it.sys);
  const StepScratch* sc = sa.scratch + d.pad_;
  if (sc->info) return;
  const int n = d.n, m = n - k0, kb = min(NB, m), w = it.width, c0 = it.c0;
  const Seg s = segment(sa, d, it.kind, k0);
  const int nd = sc->ndisp;

  if (tid < NB) {
    tsrc[tid] = tid < kb ? sc->top_src[tid] : 0;
    ddst[tid] = tid < nd ? sc->disp_dst[tid] : 0;
    dsrc[tid] = tid < nd ? sc->disp_src[tid] : 0;
  }
  __syncthreads();
  // rows moved by this step's pivots: top rows from their sources, displaced rows
  for (int idx = tid; idx < NB * 64; idx += UT) {
    const int i = idx >> 6, c = idx & 63;
    const bool in = c < w;
    T[i * WS + c] = (in && i < kb) ? seg_load(s, k0 + tsrc[i], c0 + c) : 0.0;
    D[i * WS + c] = (in && i < nd) ? seg_load(s, k0 + dsrc[i], c0 + c) : 0.0;
  }
  if (it.kind == kSegLeft) {
    __syncthreads();
    for (int idx = tid; idx < NB * 64; idx += UT) {
      const int i = idx >> 6, c = idx & 63;
      if (c < w && i < kb) s.dst[(int64_t)(k0 + i) * s.ld + c0 + c] = T[i * WS + c];
      if (c < w && i < nd) s.dst[(int64_t)(k0 + ddst[i]) * s.ld + c0 + c] = D[i * WS + c];
    }
    return;
  }
  for (int r = tid; r < m - kb; r += UT) dmap[r] = -1;
  for (int idx = tid; idx < NB * NB; idx += UT) As[(idx >> 5) * LS + (idx & 31)] = sc->linv[idx];
  __syncthreads();
  if (tid < nd) dmap[ddst[tid] - kb] = tid;

  // U12 = L11^-1 T (32 x 64): warp w owns columns [16w, 16w+16)
  {
    const int g = lane >> 2, tq = lane & 3;
    double acc[4][2][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = As[(mi * 8 + g) * LS + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) bf[ni] = T[(kk + tq) * WS + warp * 16 + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) dmma884(acc[mi][ni], af[mi], bf[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int i = mi * 8 + g;
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = warp * 16 + ni * 8 + 2 * tq + e;
          const double v = (i < kb) ? acc[mi][ni][e] : 0.0;
          Us[i * WS + c] = v;
          if (i < kb && c < w) s.dst[(int64_t)(k0 + i) * s.ld + c0 + c] = v;
        }
      }
    }
  }
  __syncthreads();
  if (kb < NB) return;  // last panel: nothing below it
  // A22 strip -= L21 U12 in 64-row tiles, software-pipelined: while the tensor
  // pipe works on tile t, tile t+1's L21 rows stream into shared memory
  // (cp.async) and its accumulator inputs into registers.
  const double* L = sa.LU + d.lu_off;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  // L21 buffers: As (L11^-1 is consumed) and T (A12 is consumed once U12 is in Us)
  auto prefetch_a = [&](int buf, int r0) {
    double* dstb = buf ? T : As;
#pragma unroll 4
    for (int idx = tid; idx < 64 * NB; idx += UT) {
      const int i = idx >> 5, q = idx & 31;
      const bool ok = r0 + i < n;
      cp_async8(dstb + i * LS + q, ok ? L + (int64_t)(r0 + i) * n + k0 + q : L, ok);
    }
    cp_async_commit();
  };
  auto load_c = [&](double (&c)[4][4][2], int r0) {
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int r = r0 + wm + mi * 8 + g;
      const int dm = r < n ? dmap[r - k0 - kb] : -1;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int cc = wn + ni * 8 + 2 * tq + e;
          double v = 0.0;
          if (r < n && cc < w) v = dm >= 0 ? D[dm * WS + cc] : seg_load(s, r, c0 + cc);
          c[mi][ni][e] = v;
        }
      }
    }
  };
  const int r_first = k0 + NB;
  double cur[4][4][2], nxt[4][4][2];
  prefetch_a(0, r_first);
  load_c(cur, r_first);
  int buf = 0;
  for (int r0 = r_first; r0 < n; r0 += 64) {
    const bool more = r0 + 64 < n;
    if (more) {
      prefetch_a(buf ^ 1, r0 + 64);
      load_c(nxt, r0 + 64);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* Ab = buf ? T : As;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = -Ab[(wm + mi * 8 + g) * LS + kk + tq];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = Us[(kk + tq) * WS + wn + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma884(cur[mi][ni], af[mi], bf[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int r = r0 + wm + mi * 8 + g;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int cc = wn + ni * 8 + 2 * tq + e;
          if (r < n && cc < w) s.dst[(int64_t)r * s.ld + c0 + cc] = cur[mi][ni][e];
        }
      }
    }
    if (more) {
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          cur[mi][ni][0] = nxt[mi][ni][0];
          cur[mi][ni][1] = nxt[mi][ni][1];
        }
    }
    buf ^= 1;
    __syncthreads();  // buffer `buf` is refilled by the next iteration's prefetch
  }
}

// ---------------------------------------------------------------------------
// k_back: X = U^-1 Y on a 64-column strip, blocks from the bottom.
__global__ void __launch_bounds__(UT)
k_back(StepArgs sa, const StepItem* __restrict__ items) {
  __shared__ double Ub[NB * LS];
  __shared__ double Xb[NB * WS];
  __shared__ double As[64 * LS];
  const int tid = threadIdx.x;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  if (!sa.solve_only && sa.scratch[d.pad_].info) return;
  const int n = d.n, w = it.width, c0 = it.c0;
  const double* U = sa.LU + d.lu_off;
  double* X = (it.kind == kSegRhs) ? sa.X + d.b_off : sa.inv + d.inv_off;
  const int ld = (it.kind == kSegRhs) ? d.nrhs : n;
  for (int kb0 = ((n - 1) / NB) * NB; kb0 >= 0; kb0 -= NB) {
    const int bw = min(NB, n - kb0);
    for (int idx = tid; idx < NB * NB; idx += UT) {
      const int i = idx >> 5, q = idx & 31;
      Ub[i * LS + q] = (i < bw && q < bw) ? U[(int64_t)(kb0 + i) * n + kb0 + q] : 0.0;
    }
    for (int idx = tid; idx < NB * 64; idx += UT) {
      const int i = idx >> 6, c = idx & 63;
      Xb[i * WS + c] = (i < bw && c < w) ? X[(int64_t)(kb0 + i) * ld + c0 + c] : 0.0;
    }
    __syncthreads();
    if (tid < w) {
      for (int i = bw - 1; i >= 0; --i) {
        double x = Xb[i * WS + tid];
        for (int q = i + 1; q < bw; ++q) x = fma(-Ub[i * LS + q], Xb[q * WS + tid], x);
        Xb[i * WS + tid] = x / Ub[i * LS + i];
      }
    }
    __syncthreads();
    for (int idx = tid; idx < NB * 64; idx += UT) {
      const int i = idx >> 6, c = idx & 63;
      if (i < bw && c < w) X[(int64_t)(kb0 + i) * ld + c0 + c] = Xb[i * WS + c];
    }
    for (int r0 = 0; r0 < kb0; r0 += 64) {
      for (int idx = tid; idx < 64 * NB; idx += UT) {
        const int i = idx >> 5, q = idx & 31;
        As[i * LS + q] = (r0 + i < kb0 && q < bw) ? U[(int64_t)(r0 + i) * n + kb0 + q] : 0.0;
      }
      __syncthreads();
      tile_update(
          As, Xb, r0, kb0, w, [&](int r, int cc) { return X[(int64_t)r * ld + c0 + cc]; },
          [&](int r, int cc, double v) { X[(int64_t)r * ld + c0 + cc] = v; });
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// k_forward: getrs from stored factors, X[p] = B[perm[p]] then unit-lower
// substitution, blocks from the top. X must not alias B.
__global__ void __launch_bounds__(UT)
k_forward(StepArgs sa, const StepItem* __restrict__ items) {
  extern __shared__ __align__(16) double fsm[];
  double* Lb = fsm;              // 32 x LS
  double* Xb = Lb + NB * LS;     // 32 x WS
  double* As = Xb + NB * WS;     // 64 x LS
  int* perm = reinterpret_cast<int*>(As + 64 * LS);
  const int tid = threadIdx.x;
  const StepItem it = items ? items[blockIdx.x] : uniform_item(sa, blockIdx.x, 0, true);
  const SysDesc d = step_desc(sa, it.sys);
  const int n = d.n, w = it.width, c0 = it.c0, ld = d.nrhs;
  const double* L = sa.LU + d.lu_off;
  const int32_t* ipiv = sa.ipiv + d.piv_off;
  const double* B = sa.B + d.b_off;
  double* X = sa.X + d.b_off;
  if (tid == 0) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) {
      int p = ipiv[k];
      if (p < k || p >= n) p = k;  // a swap list only names rows >= k
      const int t = perm[k]; perm[k] = perm[p]; perm[p] = t;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < n * 64; idx += UT) {
    const int p = idx >> 6, c = idx & 63;
    if (c < w) X[(int64_t)p * ld + c0 + c] = B[(int64_t)perm[p] * ld + c0 + c];
  }
  __syncthreads();
  for (int kb0 = 0; kb0 < n; kb0 += NB) {
    const int bw = min(NB, n - kb0), kb1 = kb0 + bw;
    for (int idx = tid; idx < NB * NB; idx += UT) {
      const int i = idx >> 5, q = idx & 31;
      Lb[i * LS + q] = (i < bw && q < bw) ? L[(int64_t)(kb0 + i) * n + kb0 + q] : 0.0;
    }
    for (int idx = tid; idx < NB * 64; idx += UT) {
      const int i = idx >> 6, c = idx & 63;
      Xb[i * WS + c] = (i < bw && c < w) ? X[(int64_t)(kb0 + i) * ld + c0 + c] : 0.0;
    }
    __syncthreads();
    if (tid < w) {
      for (int i = 1; i < bw; ++i) {
        double x = Xb[i * WS + tid];
        for (int q = 0; q < i; ++q) x = fma(-Lb[i * LS + q], Xb[q * WS + tid], x);
        Xb[i * WS + tid] = x;
      }
    }
    __syncthreads();
    for (int idx = tid; idx < NB * 64; idx += UT) {
      const int i = idx >> 6, c = idx & 63;
      if (i < bw && c < w) X[(int64_t)(kb0 + i) * ld + c0 + c] = Xb[i * WS + c];
    }
    for (int r0 = kb1; r0 < n; r0 += 64) {
      for (int idx = tid; idx < 64 * NB; idx += UT) {
        const int i = idx >> 5, q = idx & 31;
        As[i * LS + q] = (r0 + i < n && q < bw) ? L[(int64_t)(r0 + i) * n + kb0 + q] : 0.0;
      }
      __syncthreads();
      tile_update(
          As, Xb, r0, n, w, [&](int r, int cc) { return X[(int64_t)r * ld + c0 + cc]; },
          [&](int r, int cc, double v) { X[(int64_t)r * ld + c0 + cc] = v; });
      __syncthreads();
    }
  }
}

size_t update_smem(int nmax) {
  return sizeof(double) * (2 * NB * WS + 2 * 64 * LS) + sizeof(int) * (3 * NB + (size_t)nmax);
}
size_t forward_smem(int nmax) {
  return sizeof(double) * (NB * LS + NB * WS + 64 * LS) + sizeof(int) * (size_t)nmax;
}

}  // namespace

cudaError_t step_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)update_smem(kStepMaxN));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)forward_smem(kStepMaxN));
}

cudaError_t launch_panel(const StepArgs& sa, const int32_t* list, int nsys, int mmax, int k0,
                         cudaStream_t st) {
  if (nsys <= 0) return cudaSuccess;
  if (mmax <= 64) k_panel<64, 1><<<nsys, 64, 0, st>>>(sa, list, k0);
  else if (mmax <= 128) k_panel<128, 1><<<nsys, 128, 0, st>>>(sa, list, k0);
  else if (mmax <= 256) k_panel<256, 1><<<nsys, 256, 0, st>>>(sa, list, k0);
  else if (mmax <= 512) k_panel<256, 2><<<nsys, 256, 0, st>>>(sa, list, k0);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_update(const StepArgs& sa, const StepItem* items, int nitems, int nmax, int k0,
                          cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  k_update<<<nitems, UT, update_smem(nmax), st>>>(sa, items, k0);
  return cudaGetLastError();
}

cudaError_t launch_back(const StepArgs& sa, const StepItem* items, int nitems, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  k_back<<<nitems, UT, 0, st>>>(sa, items);
  return cudaGetLastError();
}

cudaError_t launch_forward(const StepArgs& sa, const StepItem* items, int nitems, int nmax,
                           cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  k_forward<<<nitems, UT, forward_smem(nmax), st>>>(sa, items);
  return cudaGetLastError();
}

}  // namespace nppb
