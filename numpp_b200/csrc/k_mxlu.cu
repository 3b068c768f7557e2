// Randomised blocked LU in FP32 on tcgen05 (the mixed solve's factorisation)
// and its triangular solves. See mxlu.hpp for the algorithm.
//
// Kernels, per system of a uniform batch padded to order N (multiple of 128):
//  k_mx_build      M = U^T (Dr A Dc) V in FP64, rounded once to FP32. A depth-2
//                  butterfly restricted to the rows {r, r+N/4, r+N/2, r+3N/4}
//                  is a 4x4 matrix, so each thread maps one 4x4 quad of A to
//                  one quad of M.
//  k_mx_diag       LU of the 256 x 128 window panel (the diagonal block's
//                  rows and the next block's) with partial pivoting (one CTA,
//                  the window in shared memory, 32-column panels with the
//                  rows in registers, two per thread), then L^-1, U^-1 and U^-T of the block by
//                  blocked inversion in shared memory, and the window's order.
//  k_mx_permute    that order applied to the rest of the window's rows; the
//                  new panel row transposed (A12^T).
//  k_mx_rowpos     the windows' orders composed: the final position of each row.
//  k_mx_gemm       C (=|-=) A B^T for 128 x 128 tiles with K = 128: operands
//                  by TMA in 128-byte-swizzled boxes (two stages of 32-column
//                  chunks), split into TF32 hi / lo in shared memory, one
//                  thread issues tcgen05.mma.kind::tf32 (M = N = 128) into a
//                  TMEM accumulator, tcgen05.ld epilogue against the C tile
//                  (loaded by TMA behind the products), TMA store.
//  k_mx_trsv_c     forward and back substitution by 128-row blocks with the
//                  stored diagonal-block inverses: a cluster of 1..8 CTAs per
//                  system and right-hand-side chunk, each holding its blocks'
//                  right-hand sides in shared memory, block solutions passed
//                  through distributed shared memory.
//  k_mx_rhs_in / k_mx_apply   U^T applied to a right-hand side, V and the
//                  column scales applied to a solution (FP64 accumulation).
// Every wait on an mbarrier is bounded (about a second of SM clock): past it the
// CTA counts a timeout, skips its stores, releases its TMEM and returns.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <vector>

#include "mxlu.hpp"

namespace nppb {
namespace {

// ---------------------------------------------------------------------------
// Random butterflies.

__device__ __forceinline__ uint32_t mx_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}

// Diagonal entry i of butterfly factor `stage`: exp(u / 10), u uniform in
// [-1/2, 1/2) (the distribution of the RBT papers), from a counter hash so that
// every kernel reproduces the same transform.
__device__ __forceinline__ double rbt_d(uint32_t stage, uint32_t i) {
  const uint32_t h = mx_hash(mx_hash(i * 2u + 1u) ^ (0x9e3779b9u * (stage + 1u)));
  const double u = (double)(h >> 8) * (1.0 / 16777216.0) - 0.5;
  return exp(0.1 * u);
}

// The butterflies' diagonals, computed once per call: tab[stage][i] =
// rbt_d(stage, i) for the 12 stages and i < N / 2.
__global__ void k_mx_rbt_table(double* __restrict__ tab, int half) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < 12 * half) tab[idx] = rbt_d((uint32_t)(idx / half), (uint32_t)(idx % half));
}

// The depth-2 butterfly W = D2 B_N (B_N = 2^-1/2 [R S; R -S], D2 = two such
// blocks of order N/2) restricted to the quad {r, r+q, r+2q, r+3q}, q = N/4.
// side 0: the left transform U, side 1: the right transform V; diagonals
// from the table (rows of length 2q).
__device__ __forceinline__ void rbt_quad(const double* __restrict__ tab, int side, int r, int q, double Q[4][4]) {
  const double* t = tab + (size_t)(6 * side) * (2 * q);
  const int h = 2 * q;
  const double R0 = t[r], S0 = t[h + r], R1 = t[r + q], S1 = t[h + r + q];
  const double Ra = t[2 * h + r], Sa = t[3 * h + r], Rb = t[4 * h + r], Sb = t[5 * h + r];
  Q[0][0] = 0.5 * Ra * R0;  Q[0][1] = 0.5 * Sa * R1;  Q[0][2] = 0.5 * Ra * S0;  Q[0][3] = 0.5 * Sa * S1;
  Q[1][0] = 0.5 * Ra * R0;  Q[1][1] = -0.5 * Sa * R1; Q[1][2] = 0.5 * Ra * S0;  Q[1][3] = -0.5 * Sa * S1;
  Q[2][0] = 0.5 * Rb * R0;  Q[2][1] = 0.5 * Sb * R1;  Q[2][2] = -0.5 * Rb * S0; Q[2][3] = -0.5 * Sb * S1;
  Q[3][0] = 0.5 * Rb * R0;  Q[3][1] = -0.5 * Sb * R1; Q[3][2] = -0.5 * Rb * S0; Q[3][3] = 0.5 * Sb * S1;
}

__device__ __forceinline__ double pow2_scale(double m) {
  if (!(m > 0.0) || !isfinite(m)) return 1.0;
  return ldexp(1.0, -ilogb(m));
}

constexpr int BQX = 128, BQY = 2;  // a block reads 1 KB runs of each of its rows; quads in registers

__global__ void __launch_bounds__(BQX * BQY, 3)
k_mx_build(const double* __restrict__ A, const double* __restrict__ rs, const double* __restrict__ cmax, int equil,
           double* __restrict__ cs, RefineState* __restrict__ st, float* __restrict__ M, int n, int N,
           const double* __restrict__ tab) {
  const int s = blockIdx.z, q = N / 4;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    st[s].eta = INFINITY;
    st[s].prev = INFINITY;
    st[s].status = kRefineActive;
    st[s].iters = 0;
  }
  const int cq = blockIdx.x * BQX + threadIdx.x, rq = blockIdx.y * BQY + threadIdx.y;
  if (cq >= q || rq >= q) return;
  double csb[4], rsa[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int j = cq + b * q;
    csb[b] = (j < n && equil) ? pow2_scale(cmax[(int64_t)s * n + j]) : 1.0;
    if (j < n && blockIdx.y == 0 && threadIdx.y == 0) cs[(int64_t)s * n + j] = csb[b];
    const int i = rq + b * q;
    rsa[b] = i < n ? rs[(int64_t)s * n + i] : 1.0;
  }
  const double* As = A + (int64_t)s * n * n;
  double a[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int i = rq + x * q;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int j = cq + y * q;
      a[x][y] = (i < n && j < n) ? rsa[x] * As[(int64_t)i * n + j] * csb[y] : (i == j ? 1.0 : 0.0);
    }
  }
  double t[4][4];  // A V
  {
    double Vq[4][4];  // this thread's column quad (consecutive threads: consecutive table entries)
    rbt_quad(tab, 1, cq, q, Vq);
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        double v = 0.0;
#pragma unroll
        for (int z = 0; z < 4; ++z) v = fma(a[x][z], Vq[z][y], v);
        t[x][y] = v;
      }
  }
  double Uq[4][4];  // the row quad (one per warp: broadcast loads)
  rbt_quad(tab, 0, rq, q, Uq);
  float* Ms = M + (int64_t)s * N * N;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      double v = 0.0;  // (U^T A V)[x][y]
#pragma unroll
      for (int z = 0; z < 4; ++z) v = fma(Uq[z][x], t[z][y], v);
      Ms[(int64_t)(rq + x * q) * N + cq + y * q] = (float)v;
    }
}

// ---------------------------------------------------------------------------
// Diagonal block: LU of the 256-row window panel with partial pivoting over
// the window, then L^-1, U^-1 and U^-T of the 128 rows chosen.
//
// LU, in shared memory, blocked by 32-column panels. Rows never move: each
// physical row of the block gets its position when it is chosen as a pivot
// (pos_of / phys_of), so the multipliers left of a panel stay with their row
// as in LAPACK's getrf. Panel p (columns 32p .. 32p+31) is factored by one
// warp with the panel in registers (diag_panel: no block-wide barrier inside
// a panel). After the panel: U12 = L11^-1 A12 over the panel's pivot rows
// (thread = column), and A22 -= L21 U12 over the rows not yet chosen (4 x 4
// register tiles).
// The packed factors are then gathered into position order.
// Inverses, from the packed factors: the eight 32 x 32 diagonal blocks of L
// and U inverted by one warp each (lane = column, substitution down / up the
// block), then two levels of block products, [L00 0; L10 L11]^-1 =
// [L00^-1 0; -L11^-1 L10 L00^-1 L11^-1] and [U00 U01; 0 U11]^-1 =
// [U00^-1 -U00^-1 U01 U11^-1; 0 U11^-1], as 32^3 and 64^3 shared-memory GEMMs
// (temporaries in the quadrants the results leave zero, and at the last level
// in the factors' diagonal quadrants).
// Out: in M's window rows (position order), the packed LU of the 128 rows
// chosen and the other rows' multipliers; L^-1, U^-1 and U^-T; the window
// order (the physical window row of each position). The window rows outside
// the panel columns are reordered by k_mx_permute.
constexpr int DT = 256;
constexpr int DLD = 132;  // leading dimension of the shared 128 x 128 arrays (16-byte rows, 4-bank row offset)
// shared state of the LU besides the window (256 x DLD) and U^-1 (128 x DLD)
constexpr int kMxWin = 2 * kMxNB;  // pivot window: the block's rows and the next block's
struct DiagAux {
  int pos_of[kMxWin];    // position of each physical row, -1 until chosen as a pivot
  int phys_of[kMxWin];   // physical row of each position
  int act[kMxWin];       // rows not yet chosen, after a panel
  uint32_t keys[2][8];   // per warp: the key of its winner; two buffers (alternating steps)
  float crow[2][8][32];  // per warp: its winner's panel values
  float lcol[32][32];    // the panel's L11 columns below the diagonal (shifted to index 0)
  int fail;  // 1 + first position whose pivot failed, INT_MAX if none
};
constexpr size_t kDiagSmem = sizeof(float) * (kMxWin * DLD) + sizeof(DiagAux);

// Inverse of one 32 x 32 diagonal block of the packed factors at (o, o), one
// warp, lane = column: unit lower (L) by substitution down, upper (U) up.
__device__ __forceinline__ void inv_lower32(const float* LU, float* Li, int o, int lane) {
  float x[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    float s = r == lane ? 1.f : 0.f;
#pragma unroll
    for (int m = 0; m < r; ++m) s = fmaf(-LU[(o + r) * DLD + o + m], x[m], s);
    x[r] = s;
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) Li[(o + r) * DLD + o + lane] = x[r];
}
__device__ __forceinline__ void inv_upper32(const float* LU, float* Ui, int o, int lane) {
  float x[32];
#pragma unroll
  for (int r = 31; r >= 0; --r) {
    float s = r == lane ? 1.f : 0.f;
#pragma unroll
    for (int m = r + 1; m < 32; ++m) s = fmaf(-LU[(o + r) * DLD + o + m], x[m], s);
    x[r] = s / LU[(o + r) * DLD + o + r];
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) Ui[(o + r) * DLD + o + lane] = x[r];
}

// C = alpha A B for S x S blocks of the shared arrays (leading dimension DLD),
// thread t of a group of (S/TM) * (S/4) threads computing the 4 columns c0 ..
// c0+3 of the TM rows g, g + S/TM, ... (adjacent threads: adjacent rows, so the
// 16-byte loads of A along k and of B along c hit distinct banks).
template <int S, int TM>
__device__ __forceinline__ void sgemm(const float* A, const float* B, float* C, float alpha, int t) {
  constexpr int CG = S / 4, RG = S / TM;
  const int g = t / CG, c0 = (t % CG) * 4;
  float acc[TM][4];
#pragma unroll
  for (int r = 0; r < TM; ++r)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[r][j] = 0.f;
#pragma unroll 2
  for (int k = 0; k < S; k += 4) {
    float4 bv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) bv[i] = *reinterpret_cast<const float4*>(B + (k + i) * DLD + c0);
#pragma unroll
    for (int r = 0; r < TM; ++r) {
      const float4 av = *reinterpret_cast<const float4*>(A + (g + RG * r) * DLD + k);
      const float a4[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        acc[r][0] = fmaf(a4[i], bv[i].x, acc[r][0]);
        acc[r][1] = fmaf(a4[i], bv[i].y, acc[r][1]);
        acc[r][2] = fmaf(a4[i], bv[i].z, acc[r][2]);
        acc[r][3] = fmaf(a4[i], bv[i].w, acc[r][3]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < TM; ++r)
    *reinterpret_cast<float4*>(C + (g + RG * r) * DLD + c0) =
        make_float4(alpha * acc[r][0], alpha * acc[r][1], alpha * acc[r][2], alpha * acc[r][3]);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void st_shared_u32_if(bool c, uint32_t addr, uint32_t x) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.u32 p, %0, 0;\n @p st.shared.u32 [%1], %2;\n}\n" ::"r"((uint32_t)c),
      "r"(addr), "r"(x)
      : "memory");
}
// the 32 values v[0..31] to 128 bytes of shared memory at addr (16-byte aligned), if c
__device__ __forceinline__ void st_shared_row_if(bool c, uint32_t addr, const float (&v)[32]) {
#pragma unroll
  for (int q = 0; q < 8; ++q)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.u32 p, %0, 0;\n @p st.shared.v4.f32 [%1], {%2, %3, %4, %5};\n}\n" ::"r"(
            (uint32_t)c),
        "r"(addr + 16u * q), "f"(v[4 * q]), "f"(v[4 * q + 1]), "f"(v[4 * q + 2]), "f"(v[4 * q + 3])
        : "memory");
}
// 1 / x to about an ulp (the hardware approximation; subnormal x flushes to zero)
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Panel of the LU (columns c0 .. c0+31) on warps 0-3: thread t owns the
// physical rows t and t + 128 of the window (R rows), in a rolled loop over
// the steps (the code stays small). At step j a row's 32 registers hold its
// values in columns c0 + j .. c0 + j + 31 (shifted left by one every step
// while the row is not chosen, so register indices are static). Step j: each
// warp's largest key (magnitude with its 8 low mantissa bits dropped, plus
// one) << 8 | (255 - row) over its rows not yet chosen by one warp reduction;
// lane 0 publishes it and the owner of the warp's winner that row's values
// (predicated stores); one barrier over the four warps; the overall winner
// (the largest |a[j]| up to a relative 2^-15, the lowest row among those)
// takes position c0 + j, and every row not yet chosen stores l = a[j] / pivot
// and updates its values right of j. Keys and rows sit in two alternating
// buffers, so one barrier per step suffices.
__device__ __forceinline__ void diag_panel(float* LU, DiagAux& ax, int c0, int t, int R) {
  constexpr unsigned FULL = 0xffffffffu;
  const int w = t >> 5, lane = t & 31;
  bool was[2], done[2];
  int jd[2] = {0, 0};  // step at which each row was chosen
  int bad = INT_MAX;   // 1 + position of a row of this thread whose pivot failed
  float v[2][32];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = t + 128 * h;
    was[h] = r >= R || ax.pos_of[r] >= 0;  // rows past the window never compete
    done[h] = was[h];
    const float4* src = reinterpret_cast<const float4*>(LU + r * DLD + c0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 x = src[q];
      v[h][4 * q] = x.x;
      v[h][4 * q + 1] = x.y;
      v[h][4 * q + 2] = x.z;
      v[h][4 * q + 3] = x.w;
    }
  }
#pragma unroll 1
  for (int j = 0; j < 32; ++j) {
    const int b = j & 1;
    uint32_t key = 0u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t kh =
          done[h] ? 0u : ((((__float_as_uint(fabsf(v[h][0])) >> 8) + 1u) << 8) | (uint32_t)(255 - (t + 128 * h)));
      key = max(key, kh);
    }
    const uint32_t wkey = __reduce_max_sync(FULL, key);
    const int wrow = 255 - (int)(wkey & 255u);
    // predicated stores, not a divergent branch (a one-lane branch around
    // these stores costs several times their latency)
    st_shared_u32_if(lane == 0, smem_addr(&ax.keys[b][w]), wkey);
    st_shared_row_if(wkey != 0u && wrow == t, smem_addr(ax.crow[b][w]), v[0]);
    st_shared_row_if(wkey != 0u && wrow == t + 128, smem_addr(ax.crow[b][w]), v[1]);
    asm volatile("bar.sync 1, 128;\n" ::: "memory");
    const uint4 kk = *reinterpret_cast<const uint4*>(ax.keys[b]);
    const uint32_t best = max(max(kk.x, kk.y), max(kk.z, kk.w));
    const int prow = 255 - (int)(best & 255u);
    const float* pr = ax.crow[b][(prow & 127) >> 5];
    // the winner's bookkeeping without a branch
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const bool win = t + 128 * h == prow;
      st_shared_u32_if(win, smem_addr(&ax.pos_of[t + 128 * h]), (uint32_t)(c0 + j));
      st_shared_u32_if(win, smem_addr(&ax.phys_of[c0 + j]), (uint32_t)(t + 128 * h));
      // the approximate reciprocal below flushes subnormals: such a pivot fails too
      if (win && !(fabsf(v[h][0]) >= FLT_MIN && isfinite(v[h][0]))) bad = min(bad, c0 + j + 1);
      jd[h] = win ? j : jd[h];
      done[h] = done[h] || win;
    }
    if (!(done[0] && done[1])) {
      const float rp = rcp_approx(pr[0]);
      float u[32];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 x = reinterpret_cast<const float4*>(pr)[q];
        u[4 * q] = x.x;
        u[4 * q + 1] = x.y;
        u[4 * q + 2] = x.z;
        u[4 * q + 3] = x.w;
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!done[h]) {
          const float l = v[h][0] * rp;
          LU[(t + 128 * h) * DLD + c0 + j] = l;
#pragma unroll
          for (int c = 0; c < 31; ++c) v[h][c] = fmaf(-l, u[c + 1], v[h][c + 1]);
          v[h][31] = 0.f;
        }
      }
    }
  }
  if (bad != INT_MAX) atomicMin(&ax.fail, bad);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (done[h] && !was[h]) {  // the row's U values, columns c0 + jd .. c0 + 31
#pragma unroll
      for (int c = 0; c < 32; ++c)
        if (c < 32 - jd[h]) LU[(t + 128 * h) * DLD + c0 + jd[h] + c] = v[h][c];
    }
  }
}

__global__ void __launch_bounds__(DT, 1)
k_mx_diag(float* __restrict__ M, int32_t* __restrict__ perm, int32_t* __restrict__ info, int N, int k) {
  extern __shared__ __align__(16) float dsm[];
  float* W0 = dsm;                    // [256][DLD] the window by physical row
  DiagAux& ax = *reinterpret_cast<DiagAux*>(W0 + kMxWin * DLD);
  const int s = blockIdx.x, K = k * kMxNB, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int R = min(kMxWin, N - K);  // window rows: this block's and the next block's
  constexpr unsigned FULL = 0xffffffffu;
  float* Mb = M + (int64_t)s * N * N + (int64_t)K * N + K;
#pragma unroll 8  // several rows' loads in flight
  for (int idx = tid; idx < R * 32; idx += DT) {
    const int r = idx >> 5, c = (idx & 31) * 4;
    *reinterpret_cast<float4*>(W0 + r * DLD + c) = *reinterpret_cast<const float4*>(Mb + (int64_t)r * N + c);
  }
  ax.pos_of[tid] = -1;  // DT == kMxWin: one entry per thread
  if (tid == 0) ax.fail = INT_MAX;
  __syncthreads();
#pragma unroll 1
  for (int p = 0; p < 4; ++p) {
    const int c0 = 32 * p;
    if (warp < 4) diag_panel(W0, ax, c0, tid, R);
    __syncthreads();
    const int W = kMxNB - c0 - 32;  // trailing columns of the block
    const int Rn = R - c0 - 32;     // rows not yet chosen
    if (tid < W) {
      // U12 = L11^-1 A12 on the panel's pivot rows, thread = column, in a
      // rolled loop: v[i] holds position c0 + j + i at step j (shifted like
      // the panel); the columns of L11 below the diagonal are staged first,
      // shifted: lcol[j][i] = L(c0 + j + 1 + i, c0 + j)
      for (int idx = tid; idx < 32 * 32; idx += W) {
        const int j = idx >> 5, i = idx & 31;
        ax.lcol[j][i] = i < 31 - j ? W0[ax.phys_of[c0 + j + 1 + i] * DLD + c0 + j] : 0.f;
      }
      asm volatile("bar.sync 2, %0;\n" ::"r"(W) : "memory");
      const int c = c0 + 32 + tid;
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = W0[ax.phys_of[c0 + j] * DLD + c];
#pragma unroll 1
      for (int j = 0; j < 31; ++j) {
        const float x = v[0];
        W0[ax.phys_of[c0 + j] * DLD + c] = x;
        float lc[32];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 y = reinterpret_cast<const float4*>(ax.lcol[j])[q];
          lc[4 * q] = y.x;
          lc[4 * q + 1] = y.y;
          lc[4 * q + 2] = y.z;
          lc[4 * q + 3] = y.w;
        }
#pragma unroll
        for (int i = 0; i < 31; ++i) v[i] = fmaf(-lc[i], x, v[i + 1]);
      }
      W0[ax.phys_of[c0 + 31] * DLD + c] = v[0];
    } else if (warp == 4) {
      // the rows not yet chosen, in physical order (also after the last panel:
      // the window's rows that stay below the block)
      int base = 0;
#pragma unroll
      for (int q = 0; q < kMxWin / 32; ++q) {
        const int r = 32 * q + lane;
        const bool nd = r < R && ax.pos_of[r] < 0;
        const unsigned m = __ballot_sync(FULL, nd);
        if (nd) ax.act[base + __popc(m & ((1u << lane) - 1u))] = r;
        base += __popc(m);
      }
    }
    __syncthreads();
    if (p == 3) break;
    // A22 -= L21 U12: 4 rows (of act) x 4 columns per task
    {
      const int ngc = W >> 2, ntask = (Rn >> 2) * ngc;
      for (int task = tid; task < ntask; task += DT) {
        const int rg = task / ngc, cc = c0 + 32 + 4 * (task - rg * ngc);
        float* rp[4];
        float4 acc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          rp[i] = W0 + ax.act[4 * rg + i] * DLD;
          acc[i] = *reinterpret_cast<const float4*>(rp[i] + cc);
        }
#pragma unroll 8
        for (int m = 0; m < 32; ++m) {
          const float4 u = *reinterpret_cast<const float4*>(W0 + ax.phys_of[c0 + m] * DLD + cc);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float l = rp[i][c0 + m];
            acc[i].x = fmaf(-l, u.x, acc[i].x);
            acc[i].y = fmaf(-l, u.y, acc[i].y);
            acc[i].z = fmaf(-l, u.z, acc[i].z);
            acc[i].w = fmaf(-l, u.w, acc[i].w);
          }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) *reinterpret_cast<float4*>(rp[i] + cc) = acc[i];
      }
    }
    __syncthreads();
  }
  // the window's order: positions 0..127 the pivots, 128..R-1 the other rows
  // (their panel values are now their multipliers, L21 = A21 U11^-1)
  int32_t* pw = perm + ((int64_t)s * (N / kMxNB) + k) * kMxWin;
  if (tid < R) pw[tid] = tid < kMxNB ? ax.phys_of[tid] : ax.act[tid - kMxNB];
#pragma unroll 4
  for (int idx = tid; idx < R * 32; idx += DT) {
    const int r = idx >> 5, c = (idx & 31) * 4;
    const int ph = r < kMxNB ? ax.phys_of[r] : ax.act[r - kMxNB];
    *reinterpret_cast<float4*>(Mb + (int64_t)r * N + c) = *reinterpret_cast<const float4*>(W0 + ph * DLD + c);
  }
  if (tid == 0 && ax.fail != INT_MAX && info[s] == 0) info[s] = K + ax.fail;
}

// The diagonal block's inverses from its packed factors (written by k_mx_diag
// into M, position order): L^-1, U^-1 and U^-T. A kernel of its own so that it
// runs beside the window permute (which does not need them). The eight 32 x 32
// diagonal blocks of L and U inverted by one warp each (lane = column,
// substitution down / up the block), then two levels of block products,
// [L00 0; L10 L11]^-1 = [L00^-1 0; -L11^-1 L10 L00^-1 L11^-1] and
// [U00 U01; 0 U11]^-1 = [U00^-1 -U00^-1 U01 U11^-1; 0 U11^-1], as 32^3 and
// 64^3 shared-memory GEMMs (temporaries in the quadrants the results leave
// zero, and at the last level in the factors' diagonal quadrants).
constexpr size_t kInvSmem = sizeof(float) * 3 * kMxNB * DLD;
__global__ void __launch_bounds__(DT, 1)
k_mx_diag_inv(const float* __restrict__ M, float* __restrict__ Linv, float* __restrict__ Uinv,
              float* __restrict__ UinvT, int N, int k) {
  extern __shared__ __align__(16) float ism[];
  float* LU = ism;                  // [128][DLD] the packed factors (position order)
  float* Li = LU + kMxNB * DLD;     // [128][DLD] L^-1
  float* Ui = Li + kMxNB * DLD;     // [128][DLD] U^-1
  const int s = blockIdx.x, K = k * kMxNB, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float* Mb = M + (int64_t)s * N * N + (int64_t)K * N + K;
#pragma unroll 4
  for (int idx = tid; idx < kMxNB * 32; idx += DT) {
    const int r = idx >> 5, c = (idx & 31) * 4;
    *reinterpret_cast<float4*>(LU + r * DLD + c) = *reinterpret_cast<const float4*>(Mb + (int64_t)r * N + c);
  }
  for (int idx = tid; idx < kMxNB * DLD; idx += DT) {
    Li[idx] = 0.f;
    Ui[idx] = 0.f;
  }
  __syncthreads();
  // level 1: the eight 32 x 32 diagonal blocks
  if (warp < 4) inv_lower32(LU, Li, 32 * warp, lane);
  else inv_upper32(LU, Ui, 32 * (warp - 4), lane);
  __syncthreads();
  // level 2: 64 x 64 diagonal quadrants; four chains of 64 threads (one call
  // site per level in a rolled loop over the two products: compact code)
  {
    const int ch = tid >> 6, t = tid & 63, p = ch & 1, o = 64 * p;
    const bool isL = ch < 2;
    float* tmp = isL ? Li + (32 * p) * DLD + 64   // temporaries in Li's upper-right quadrant
                     : Ui + (64 + 32 * p) * DLD;  //   ... and Ui's lower-left quadrant
#pragma unroll 1
    for (int ph = 0; ph < 2; ++ph) {
      const float* A = ph == 0 ? (isL ? LU + (o + 32) * DLD + o : LU + o * DLD + o + 32)
                               : (isL ? Li + (o + 32) * DLD + o + 32 : Ui + o * DLD + o);
      const float* B = ph == 0 ? (isL ? Li + o * DLD + o : Ui + (o + 32) * DLD + o + 32) : tmp;
      float* C = ph == 0 ? tmp : (isL ? Li + (o + 32) * DLD + o : Ui + o * DLD + o + 32);
      sgemm<32, 4>(A, B, C, ph == 0 ? 1.f : -1.f, t);
      __syncthreads();
    }
  }
  // level 3: the off-diagonal quadrants; two chains of 128 threads, temporaries in LU's diagonal quadrants
  {
    const int ch = tid >> 7, t = tid & 127;
    const bool isL = ch == 0;
    float* tmp = isL ? LU : LU + 64 * DLD + 64;
#pragma unroll 1
    for (int ph = 0; ph < 2; ++ph) {
      const float* A = ph == 0 ? (isL ? LU + 64 * DLD : LU + 64) : (isL ? Li + 64 * DLD + 64 : Ui);
      const float* B = ph == 0 ? (isL ? Li : Ui + 64 * DLD + 64) : tmp;
      float* C = ph == 0 ? tmp : (isL ? Li + 64 * DLD : Ui + 64);
      sgemm<64, 8>(A, B, C, ph == 0 ? 1.f : -1.f, t);
      __syncthreads();
    }
  }
  float* Lb = Linv + (int64_t)s * N * kMxNB + (int64_t)K * kMxNB;
  float* Ub = Uinv + (int64_t)s * N * kMxNB + (int64_t)K * kMxNB;
  float* UTb = UinvT + (int64_t)s * N * kMxNB + (int64_t)K * kMxNB;
  for (int idx = tid; idx < kMxNB * kMxNB; idx += DT) {
    const int r = idx >> 7, c = idx & 127;
    Lb[idx] = c <= r ? Li[r * DLD + c] : 0.f;        // L^-1[r][c]
    Ub[idx] = c >= r ? Ui[r * DLD + c] : 0.f;        // U^-1[r][c]
    UTb[idx] = r >= c ? Ui[c * DLD + r] : 0.f;       // U^-T[r][c]
  }
}

// ---------------------------------------------------------------------------
// tcgen05 GEMM: one 128 x 128 tile of C, K = 128, per CTA.

constexpr int GT = 256;
constexpr int BOX = 128 * 128;  // bytes of one 128-row x 32-float swizzled box
constexpr size_t kGemmSmem = 1024 + 12 * (size_t)BOX + 128;

struct MxGemmArgs {
  int ax, ay, az;  // A box origin of tile (mt = 0, chunk 0): x = K column, y = row, z = plane offset
  int bx, by, bz;  // B (stored as B^T: row = output column) of tile (nt = 0)
  int cx, cy, cz;  // C tile (0, 0)
  int split3;
  // tile (mt, nt) of this CTA: cross = 1: the first two tile rows and the
  // first tile column (x < tiles: (0, x); x < 2 tiles: (1, x - tiles); else
  // (x - 2 tiles + 2, 0)); cross = 0: (blockIdx.y + moff, blockIdx.x + noff)
  int cross, tiles, moff, noff;
  // optional transposed copy of each result element (r, c) of tile (mt, nt):
  // tr + s * tr_sys + (tr_r0 + 128 mt + r) * tr_row + (tr_c0 + 128 nt + c) * tr_col
  float* tr;
  int64_t tr_sys, tr_col, tr_row;
  int tr_c0, tr_r0, tr_mt0_only;
};

__device__ int g_mx_timeouts = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait for phase `parity` of an mbarrier: about a second of the SM's
// own cycle counter (cheap to read, unlike the global timer).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  const long long t0 = clock64();
  while (true) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > (2ll << 30)) return false;
  }
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tma_store(const CUtensorMap* map, uint32_t src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(src), "r"(x), "r"(y), "r"(z)
               : "memory");
}

// K-major operand, 128-byte swizzle: 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// kind::tf32, FP32 accumulator, A and B K-major, N = 128, M = 128
constexpr uint32_t MX_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mx_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(MX_IDESC), "r"(acc));
}

__device__ __forceinline__ void mx_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void mx_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(r[e]);
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// In place x -> tf32(x) and lo = x - tf32(x) for one 16 KB box.
__device__ __forceinline__ void split_box(float* raw, float* lo, int tid) {
  float4* r4 = reinterpret_cast<float4*>(raw);
  float4* l4 = reinterpret_cast<float4*>(lo);
#pragma unroll 4
  for (int e = tid; e < BOX / 16; e += GT) {
    const float4 x = r4[e];
    float4 h;
    h.x = tf32_hi(x.x);
    h.y = tf32_hi(x.y);
    h.z = tf32_hi(x.z);
    h.w = tf32_hi(x.w);
    r4[e] = h;
    l4[e] = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
  }
}

template <int SUB>
__global__ void __launch_bounds__(GT, 1)
k_mx_gemm(const __grid_constant__ CUtensorMap mA1, const __grid_constant__ CUtensorMap mB1,
          const __grid_constant__ CUtensorMap mC1, const MxGemmArgs g1,
          const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB2,
          const __grid_constant__ CUtensorMap mC2, const MxGemmArgs g2, int rows1) {
  // two independent products in one launch: grid rows y < rows1 run the first
  // (maps 1, args 1), the others the second (tile row y - rows1)
  const bool second = (int)blockIdx.y >= rows1;
  const CUtensorMap& mA = second ? mA2 : mA1;
  const CUtensorMap& mB = second ? mB2 : mB1;
  const CUtensorMap& mC = second ? mC2 : mC1;
  const MxGemmArgs& g = second ? g2 : g1;
  const int by_ = (int)blockIdx.y - (second ? rows1 : 0);
  extern __shared__ __align__(1024) unsigned char gsm_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  // stage st (0, 1): A hi at base + st*4*BOX, B hi + BOX, A lo + 2 BOX, B lo + 3 BOX; C tile: 4 boxes
  unsigned char* Cs = base + 8 * BOX;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + 12 * BOX);  // full[2], freed[2], cfull, done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 6);
  int* abort_flag = reinterpret_cast<int*>(bars + 7);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = blockIdx.z;
  const int bx = (int)blockIdx.x;
  const int mt = !g.cross ? by_ + g.moff : bx < g.tiles ? 0 : bx < 2 * g.tiles ? 1 : bx - 2 * g.tiles + 2;
  const int nt = !g.cross ? bx + g.noff : bx < g.tiles ? bx : bx < 2 * g.tiles ? bx - g.tiles : 0;
  const uint32_t bar0 = smem_u32(bars);
  auto full = [&](int st) { return bar0 + 8u * st; };
  auto freed = [&](int st) { return bar0 + 16u + 8u * st; };
  const uint32_t cfull = bar0 + 32u, done = bar0 + 40u;

  if (warp == 0) {  // the whole warp, converged: TMEM for the 128 x 128 FP32 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;\n" ::"r"(smem_u32(tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int b = 0; b < 6; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0 + 8u * b));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    *abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tslot;

  const int ay = g.ay + 128 * mt, az = g.az + s;
  const int by = g.by + 128 * nt, bz = g.bz + s;
  const int cx = g.cx + 128 * nt, cy = g.cy + 128 * mt, cz = g.cz + s;
  auto stage = [&](int st) { return base + (size_t)st * 4 * BOX; };
  if (tid == 0) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      mbar_expect_tx(full(c), 2 * BOX);
      tma_load(smem_u32(stage(c)), &mA, full(c), g.ax + 32 * c, ay, az);
      tma_load(smem_u32(stage(c) + BOX), &mB, full(c), g.bx + 32 * c, by, bz);
    }
    if (SUB) {
      mbar_expect_tx(cfull, 4 * BOX);
#pragma unroll
      for (int b = 0; b < 4; ++b) tma_load(smem_u32(Cs + b * BOX), &mC, cfull, cx + 32 * b, cy, cz);
    }
  }
  bool ok = true;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    const int st = c & 1;
    const uint32_t par = (uint32_t)(c >> 1) & 1u;
    unsigned char* sb = stage(st);
    if (!mbar_wait(full(st), par)) ok = false;
    if (g.split3) {
      split_box(reinterpret_cast<float*>(sb), reinterpret_cast<float*>(sb + 2 * BOX), tid);
      split_box(reinterpret_cast<float*>(sb + BOX), reinterpret_cast<float*>(sb + 3 * BOX), tid);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint64_t dA = sw128_desc(smem_u32(sb)), dB = sw128_desc(smem_u32(sb + BOX));
      const uint64_t dAl = sw128_desc(smem_u32(sb + 2 * BOX)), dBl = sw128_desc(smem_u32(sb + 3 * BOX));
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const uint64_t o = (uint64_t)(2 * ks);  // 32 bytes along K, in 16-byte units
        const uint32_t acc0 = (c | ks) != 0;
        if (g.split3) {
          mx_mma(tmem, dAl + o, dB + o, acc0);  // small terms first
          mx_mma(tmem, dA + o, dBl + o, 1u);
          mx_mma(tmem, dA + o, dB + o, 1u);
        } else {
          mx_mma(tmem, dA + o, dB + o, acc0);
        }
      }
      mx_commit(freed(st));
      if (c + 2 < 4) {
        // the stage is reloaded once the products reading it are done
        if (!mbar_wait(freed(st), par)) {
          ok = false;
        } else {
          mbar_expect_tx(full(st), 2 * BOX);
          tma_load(smem_u32(sb), &mA, full(st), g.ax + 32 * (c + 2), ay, az);
          tma_load(smem_u32(sb + BOX), &mB, full(st), g.bx + 32 * (c + 2), by, bz);
        }
      }
    }
  }
  if (tid == 0) mx_commit(done);
  if (!mbar_wait(done, 0)) ok = false;
  if (SUB && !mbar_wait(cfull, 0)) ok = false;
  if (!ok) {
    *abort_flag = 1;
    atomicAdd(&g_mx_timeouts, 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  __syncthreads();
  const bool live = *abort_flag == 0;
  {
    const int qw = warp & 3, hf = warp >> 2, r = 32 * qw + lane;
    float acc[64];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 4; ++i) mx_ld16(tmem + ((uint32_t)(32 * qw) << 16) + (uint32_t)(64 * hf + 16 * i), acc + 16 * i);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
    const bool tr = live && g.tr != nullptr && (!g.tr_mt0_only || mt == 0);
    float* trp = tr ? g.tr + (int64_t)s * g.tr_sys + (int64_t)(g.tr_r0 + 128 * mt + r) * g.tr_row +
                          (int64_t)(g.tr_c0 + 128 * nt) * g.tr_col
                    : nullptr;
#pragma unroll
    for (int cc = 0; cc < 16; ++cc) {
      const int c = 64 * hf + 4 * cc, b = c >> 5, ch = ((c & 31) >> 2) ^ (r & 7);
      float4* p = reinterpret_cast<float4*>(Cs + b * BOX + r * 128 + ch * 16);
      float4 v;
      if (SUB) {
        v = *p;
        v.x -= acc[4 * cc];
        v.y -= acc[4 * cc + 1];
        v.z -= acc[4 * cc + 2];
        v.w -= acc[4 * cc + 3];
      } else {
        v = make_float4(acc[4 * cc], acc[4 * cc + 1], acc[4 * cc + 2], acc[4 * cc + 3]);
      }
      *p = v;
      if (tr) {
        float* t = trp + (int64_t)c * g.tr_col;
        t[0] = v.x;
        t[g.tr_col] = v.y;
        t[2 * g.tr_col] = v.z;
        t[3 * g.tr_col] = v.w;
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (tid == 0 && live) {
#pragma unroll
    for (int b = 0; b < 4; ++b) tma_store(&mC, smem_u32(Cs + b * BOX), cx + 32 * b, cy, cz);
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
  }
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;\n" ::"r"(tmem));
  }
}

// ---------------------------------------------------------------------------
// Triangular solves with the block factors.

// Cluster form of the triangular solves: C CTAs per (system, chunk of W
// right-hand sides), C = 1, 2, 4 or 8. CTA r owns the 128-row blocks b with
// b % C == r and keeps their right-hand sides in its shared memory. Block
// step k: the owner computes y_k = D_k c_k (D_k the stored inverse of the
// diagonal block), writes y_k into every CTA's shared memory (distributed
// shared memory), and one cluster barrier publishes it; each CTA then
// updates its own blocks, c_j -= M[block j][block k] y_k. y is
// double-buffered: a CTA reaches step k's barrier only after finishing step
// k-1's updates, so step k+1's owner may overwrite step k-1's buffer after it.
constexpr int TS = 512;  // threads per CTA: 16 warps
constexpr size_t kTrsv64Smem = 160 * 1024;  // shared-memory cap of the FP64-vector substitution

// tmp[i][w] = sum_m D[i][m] y[m][w] for the block's 128 rows, 16 warps
template <int W, class VT>
__device__ __forceinline__ void block_apply16(const float* __restrict__ D, const VT* y, VT* tmp, int warp,
                                              int lane) {
  VT yv[4][W];
#pragma unroll
  for (int e = 0; e < 4; ++e)
#pragma unroll
    for (int w = 0; w < W; ++w) yv[e][w] = y[(4 * lane + e) * W + w];
#pragma unroll
  for (int rr = 0; rr < 8; ++rr) {
    const int i = warp + 16 * rr;
    const float4 d = *reinterpret_cast<const float4*>(D + i * kMxNB + 4 * lane);
    VT sum[W];
#pragma unroll
    for (int w = 0; w < W; ++w) sum[w] = d.x * yv[0][w] + d.y * yv[1][w] + d.z * yv[2][w] + d.w * yv[3][w];
#pragma unroll
    for (int o = 16; o; o >>= 1)
#pragma unroll
      for (int w = 0; w < W; ++w) sum[w] += __shfl_xor_sync(0xffffffffu, sum[w], o);
    if (lane == 0)
#pragma unroll
      for (int w = 0; w < W; ++w) tmp[i * W + w] = sum[w];
  }
}

// c[i] -= M[J + i][K:K+128] . y for the 128 rows of block J (local copy c), 16 warps
template <int W, class VT>
__device__ __forceinline__ void block_update16(const float* __restrict__ Ms, int N, int J, int K, const VT* y,
                                               VT* c, int warp, int lane) {
  VT yv[4][W];
#pragma unroll
  for (int e = 0; e < 4; ++e)
#pragma unroll
    for (int w = 0; w < W; ++w) yv[e][w] = y[(4 * lane + e) * W + w];
  float4 m[8];  // rows warp + 16 u: all eight loads in flight before the sums
#pragma unroll
  for (int u = 0; u < 8; ++u)
    m[u] = __ldcs(reinterpret_cast<const float4*>(Ms + (int64_t)(J + warp + 16 * u) * N + K + 4 * lane));
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int i = warp + 16 * u;
    VT sum[W];
#pragma unroll
    for (int w = 0; w < W; ++w)
      sum[w] = m[u].x * yv[0][w] + m[u].y * yv[1][w] + m[u].z * yv[2][w] + m[u].w * yv[3][w];
#pragma unroll
    for (int o = 16; o; o >>= 1)
#pragma unroll
      for (int w = 0; w < W; ++w) sum[w] += __shfl_xor_sync(0xffffffffu, sum[w], o);
    if (lane == 0)
#pragma unroll
      for (int w = 0; w < W; ++w) c[i * W + w] -= sum[w];
  }
}

template <int W, class VT>
__global__ void __launch_bounds__(TS, 1)
k_mx_trsv_c(const float* __restrict__ M, const float* __restrict__ Linv, const float* __restrict__ Uinv,
            VT* __restrict__ Y, int N, int nrhs, int C, const RefineState* __restrict__ st, int only_active) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  VT* tsm = reinterpret_cast<VT*>(tsm_raw);
  const int rank = (int)cluster.block_rank();
  const int s = blockIdx.x / C, c0 = blockIdx.y * W;
  if (only_active && st[s].status != kRefineActive) return;  // every CTA of the cluster: same system, same answer
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nb = N / kMxNB, nbl = (nb - rank + C - 1) / C;  // blocks this CTA owns
  VT* cl = tsm;                                  // [nbl][128][W] owned right-hand sides
  VT* yb = cl + (size_t)((nb + C - 1) / C) * kMxNB * W;  // [2][128][W] broadcast block solutions
  VT* tmp = yb + 2 * kMxNB * W;                  // [128][W]
  const float* Ms = M + (int64_t)s * N * N;
  VT* Ys = Y + (int64_t)s * N * nrhs;
  for (int idx = tid; idx < nbl * kMxNB * W; idx += TS) {
    const int lb = idx / (kMxNB * W), rem = idx % (kMxNB * W), i = (lb * C + rank) * kMxNB + rem / W, w = rem % W;
    cl[idx] = c0 + w < nrhs ? Ys[(int64_t)i * nrhs + c0 + w] : VT(0);
  }
  const float* Ls = Linv + (int64_t)s * N * kMxNB;
  const float* Us = Uinv + (int64_t)s * N * kMxNB;
  for (int pass = 0; pass < 2; ++pass) {  // L y = P c, then U x = y
    for (int t = 0; t < nb; ++t) {
      const int k = pass == 0 ? t : nb - 1 - t, K = k * kMxNB, buf = (pass * nb + t) & 1;
      VT* yk = yb + buf * kMxNB * W;
      __syncthreads();  // this CTA's updates of the previous step are in
      if (k % C == rank) {
        VT* ck = cl + (k / C) * kMxNB * W;
        block_apply16<W, VT>((pass == 0 ? Ls : Us) + (int64_t)K * kMxNB, ck, tmp, warp, lane);
        __syncthreads();
        for (int q = 0; q < C; ++q) {
          VT* dst = cluster.map_shared_rank(yk, q);
          for (int idx = tid; idx < kMxNB * W; idx += TS) dst[idx] = tmp[idx];
        }
        for (int idx = tid; idx < kMxNB * W; idx += TS) ck[idx] = tmp[idx];
      }
      cluster.sync();  // y_k in every CTA
      if (t + 1 < nb) {  // the next step's panel rows of this CTA's blocks into L2, behind this step's loads
        const int kn = pass == 0 ? k + 1 : k - 1;
        for (int idx = tid; idx < nbl * kMxNB * 4; idx += TS) {
          const int lb = idx / (kMxNB * 4), j = lb * C + rank;
          if (pass == 0 ? j > kn : j < kn) {
            const int row = j * kMxNB + (idx / 4) % kMxNB;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(Ms + (int64_t)row * N + kn * kMxNB + 32 * (idx & 3)));
          }
        }
      }
      for (int lb = 0; lb < nbl; ++lb) {
        const int j = lb * C + rank;
        if (pass == 0 ? j > k : j < k)
          block_update16<W, VT>(Ms, N, j * kMxNB, K, yk, cl + lb * kMxNB * W, warp, lane);
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nbl * kMxNB * W; idx += TS) {
    const int lb = idx / (kMxNB * W), rem = idx % (kMxNB * W), i = (lb * C + rank) * kMxNB + rem / W, w = rem % W;
    if (c0 + w < nrhs) Ys[(int64_t)i * nrhs + c0 + w] = cl[idx];
  }
  cluster.sync();  // no CTA leaves while a peer may still write into its shared memory
}

// Window k's row order applied to the rest of its rows (the row interchanges
// of LAPACK's getrf, left of the block as well as right of it, so that the
// factors end in one global row order), and the block's new panel row,
// transposed, into T[buf]: CTA per (64-column chunk, system), the chunk's
// window rows staged in shared memory; the panel columns themselves were
// written in order by the diagonal kernel.
constexpr int PC = 64, PLD = PC + 4;  // columns per CTA; row stride of 16-byte pieces, padded by one piece
constexpr size_t kPermSmem = sizeof(float) * kMxWin * PLD;
__global__ void __launch_bounds__(256)
k_mx_permute(float* __restrict__ M, float* __restrict__ T, const int32_t* __restrict__ perm, int N, int k,
             int count, int buf) {
  __shared__ int pw[kMxWin];
  extern __shared__ __align__(16) float psm[];  // [R][PLD]
  const int s = blockIdx.y, c0 = blockIdx.x * PC, K = k * kMxNB, R = min(kMxWin, N - K);
  if (c0 >= K && c0 < K + kMxNB) return;
  const int32_t* pp = perm + ((int64_t)s * (N / kMxNB) + k) * kMxWin;
  for (int i = threadIdx.x; i < R; i += 256) pw[i] = pp[i];
  float* Ms = M + (int64_t)s * N * N + (int64_t)K * N + c0;
#pragma unroll 8  // several rows' loads in flight
  for (int idx = threadIdx.x; idx < R * (PC / 4); idx += 256) {
    const int r = idx / (PC / 4), c = (idx % (PC / 4)) * 4;
    *reinterpret_cast<float4*>(psm + r * PLD + c) = *reinterpret_cast<const float4*>(Ms + (int64_t)r * N + c);
  }
  __syncthreads();
#pragma unroll 8
  for (int idx = threadIdx.x; idx < R * (PC / 4); idx += 256) {
    const int r = idx / (PC / 4), c = (idx % (PC / 4)) * 4;
    *reinterpret_cast<float4*>(Ms + (int64_t)r * N + c) = *reinterpret_cast<const float4*>(psm + pw[r] * PLD + c);
  }
  if (c0 >= K + kMxNB) {  // T[col][row] for the block's 128 rows: thread = (row, 4 columns), rows fastest
    float* Tz = T + ((int64_t)buf * count + s) * N * kMxNB + (int64_t)c0 * kMxNB;
    for (int idx = threadIdx.x; idx < kMxNB * (PC / 4); idx += 256) {
      const int r = idx % kMxNB, c = (idx / kMxNB) * 4;
      const float4 v = *reinterpret_cast<const float4*>(psm + pw[r] * PLD + c);
      Tz[(int64_t)c * kMxNB + r] = v.x;
      Tz[(int64_t)(c + 1) * kMxNB + r] = v.y;
      Tz[(int64_t)(c + 2) * kMxNB + r] = v.z;
      Tz[(int64_t)(c + 3) * kMxNB + r] = v.w;
    }
  }
}

// Position of every row of M in the final order: the windows' orders
// composed in sequence (one CTA per system).
__global__ void __launch_bounds__(256)
k_mx_rowpos(const int32_t* __restrict__ perm, int32_t* __restrict__ rowpos, int N) {
  extern __shared__ int at[];  // [N] the original row now at each position, then [kMxWin] scratch
  int* tmp = at + N;
  const int s = blockIdx.x, nb = N / kMxNB;
  for (int i = threadIdx.x; i < N; i += 256) at[i] = i;
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const int K = k * kMxNB, R = min(kMxWin, N - K);
    const int32_t* pw = perm + ((int64_t)s * nb + k) * kMxWin;
    for (int j = threadIdx.x; j < R; j += 256) tmp[j] = at[K + pw[j]];
    __syncthreads();
    for (int j = threadIdx.x; j < R; j += 256) at[K + j] = tmp[j];
    __syncthreads();
  }
  for (int i = threadIdx.x; i < N; i += 256) rowpos[(int64_t)s * N + at[i]] = i;
}

// Y = P U^T pad(R) (P: the factorisation's row order): thread per (row quad, right-hand side).
template <class TR, class TY>
__global__ void __launch_bounds__(256)
k_mx_rhs_in(const TR* __restrict__ R, TY* __restrict__ Y, int n, int N, int nrhs,
            const RefineState* __restrict__ st, int only_active, const double* __restrict__ tab,
            const int32_t* __restrict__ rowpos) {
  const int s = blockIdx.y;
  if (only_active && st[s].status != kRefineActive) return;
  const int q = N / 4;
  const int idx = blockIdx.x * 256 + threadIdx.x;
  if (idx >= q * nrhs) return;
  const int r = idx / nrhs, col = idx % nrhs;
  double U[4][4];
  rbt_quad(tab, 0, r, q, U);
  double x[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = r + a * q;
    x[a] = i < n ? (double)R[((int64_t)s * n + i) * nrhs + col] : 0.0;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) v = fma(U[b][a], x[b], v);
    Y[((int64_t)s * N + rowpos[(int64_t)s * N + r + a * q]) * nrhs + col] = (TY)v;
  }
}

// X (=|+=) cs * (V Y)[0:n] in FP64: thread per (column quad, right-hand side).
template <class TY>
__global__ void __launch_bounds__(256)
k_mx_apply(const TY* __restrict__ Y, double* __restrict__ X, const double* __restrict__ cs, int n, int N,
           int nrhs, const RefineState* __restrict__ st, int init, const double* __restrict__ tab) {
  const int s = blockIdx.y;
  if (!init && st[s].status != kRefineActive) return;
  const int q = N / 4;
  const int idx = blockIdx.x * 256 + threadIdx.x;
  if (idx >= q * nrhs) return;
  const int c = idx / nrhs, col = idx % nrhs;
  double V[4][4];
  rbt_quad(tab, 1, c, q, V);
  double y[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) y[b] = (double)Y[((int64_t)s * N + c + b * q) * nrhs + col];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = c + a * q;
    if (i >= n) continue;
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) v = fma(V[a][b], y[b], v);
    double* x = X + ((int64_t)s * n + i) * nrhs + col;
    const double d = cs[(int64_t)s * n + i] * v;
    *x = init ? d : *x + d;
  }
}

// ---------------------------------------------------------------------------
// Host side: tensor maps and launches.

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// 3-D FP32 map {inner, rows, planes} (row-major planes), 32 x 128 boxes, 128-byte swizzle.
bool make_map(CUtensorMap* m, const float* base, uint64_t inner, uint64_t rows, uint64_t planes) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {inner, rows, planes};
  const cuuint64_t strides[2] = {inner * sizeof(float), inner * rows * sizeof(float)};
  const cuuint32_t box[3] = {32, 128, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

size_t mx_workspace_bytes(int count, int n) {
  const size_t N = (size_t)mx_padded(n), c = (size_t)count;
  return align256(4 * c * N * N) + align256(4 * 2 * c * N * kMxNB) + 3 * align256(4 * c * N * kMxNB) +
         align256(4 * c) + align256(sizeof(double) * 12 * (N / 2)) + align256(4 * c * (N / kMxNB) * kMxWin) +
         align256(4 * c * N);
}

void mx_carve(MxBufs& b, void* base, int count, int n) {
  const size_t N = (size_t)mx_padded(n), c = (size_t)count;
  unsigned char* p = static_cast<unsigned char*>(base);
  b.count = count;
  b.n = n;
  b.N = (int)N;
  b.M = reinterpret_cast<float*>(p);
  p += align256(4 * c * N * N);
  b.T = reinterpret_cast<float*>(p);
  p += align256(4 * 2 * c * N * kMxNB);
  b.Linv = reinterpret_cast<float*>(p);
  p += align256(4 * c * N * kMxNB);
  b.Uinv = reinterpret_cast<float*>(p);
  p += align256(4 * c * N * kMxNB);
  b.UinvT = reinterpret_cast<float*>(p);
  p += align256(4 * c * N * kMxNB);
  b.info = reinterpret_cast<int32_t*>(p);
  p += align256(4 * c);
  b.rbt = reinterpret_cast<double*>(p);
  p += align256(sizeof(double) * 12 * (N / 2));
  b.perm = reinterpret_cast<int32_t*>(p);
  p += align256(4 * c * (N / kMxNB) * kMxWin);
  b.rowpos = reinterpret_cast<int32_t*>(p);
}

cudaError_t mx_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_mx_gemm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_gemm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_permute, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPermSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_diag_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem);
  const int csm = (int)(sizeof(float) * ((size_t)4096 * 8 + 3 * kMxNB * 8));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mx_trsv_c<1, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mx_trsv_c<2, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mx_trsv_c<4, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mx_trsv_c<8, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, csm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_trsv_c<1, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsv64Smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_trsv_c<2, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsv64Smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mx_trsv_c<4, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsv64Smem);
  return e;
}

int mx_timeouts_take() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_mx_timeouts, sizeof(int)) != cudaSuccess) return -1;
  const int z = 0;
  if (cudaMemcpyToSymbol(g_mx_timeouts, &z, sizeof(int)) != cudaSuccess) return -1;
  return v;
}

cudaError_t mx_build(const double* A, const double* rs, const double* cmax, int equil, double* cs, RefineState* st,
                     const MxBufs& b, cudaStream_t s) {
  const int q = b.N / 4, half = b.N / 2;
  k_mx_rbt_table<<<(12 * half + 255) / 256, 256, 0, s>>>(b.rbt, half);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((q + BQX - 1) / BQX), (unsigned)((q + BQY - 1) / BQY), (unsigned)b.count);
  k_mx_build<<<grid, dim3(BQX, BQY), 0, s>>>(A, rs, cmax, equil, cs, st, b.M, b.n, b.N, b.rbt);
  return cudaGetLastError();
}

namespace {

// Streams and events of the look-ahead (per thread and device, made on first use).
struct MxStreams {
  cudaStream_t panel = nullptr;  // the next block's diagonal factor and triangular solves, highest priority
  cudaStream_t side = nullptr;   // the bulk of the trailing update
  cudaStream_t inv = nullptr;    // the diagonal block's inverses, beside the window permute
  cudaEvent_t ev[6] = {};
};

MxStreams* mx_streams() {
  struct Holder {
    std::vector<MxStreams> per_dev;
    ~Holder() {
      for (auto& m : per_dev) {
        for (cudaStream_t t : {m.panel, m.side, m.inv})
          if (t) cudaStreamDestroy(t);
        for (cudaEvent_t e : m.ev)
          if (e) cudaEventDestroy(e);
      }
    }
  };
  thread_local Holder h;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  if ((int)h.per_dev.size() <= dev) h.per_dev.resize(dev + 1);
  MxStreams& m = h.per_dev[dev];
  if (!m.side) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    bool ok = cudaStreamCreateWithPriority(&m.panel, cudaStreamNonBlocking, greatest) == cudaSuccess &&
              cudaStreamCreateWithPriority(&m.inv, cudaStreamNonBlocking, greatest) == cudaSuccess &&
              cudaStreamCreateWithFlags(&m.side, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t& e : m.ev) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      return nullptr;
    }
  }
  return &m;
}

}  // namespace

// Blocked factorisation with look-ahead. Per block k, on the panel stream:
// the diagonal kernel (pivots from the 256-row window), the window's row
// order applied to the rest of its rows (and the new panel row transposed),
// L21 for the rows below the window, U12, and the part of the trailing update
// the next window needs (its two 128-row tile rows and the next panel column);
// on the side stream, once U12 is in, the rest of the trailing update. Block
// k+1's diagonal factor, row order and solves therefore run beside the bulk of
// block k's update; block k+1's trailing update waits for it. Every element
// sees the same operations in the same order either way.
cudaError_t mx_factor(const MxBufs& b, cudaStream_t s) {
  const int N = b.N, count = b.count, nb = N / kMxNB;
  CUtensorMap mM, mT, mL, mUT;
  if (!make_map(&mM, b.M, N, N, count) || !make_map(&mT, b.T, kMxNB, N, 2 * (uint64_t)count) ||
      !make_map(&mL, b.Linv, kMxNB, N, count) || !make_map(&mUT, b.UinvT, kMxNB, N, count))
    return cudaErrorInvalidValue;
  MxStreams* ms = mx_streams();
  cudaStream_t ps = ms ? ms->panel : s, ss = ms ? ms->side : s;
  cudaError_t e = cudaMemsetAsync(b.info, 0, sizeof(int32_t) * count, s);
  if (e != cudaSuccess) return e;
  if (ms) {  // the panel stream starts behind everything queued on s
    if ((e = cudaEventRecord(ms->ev[0], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ps, ms->ev[0], 0)) != cudaSuccess) return e;
  }
  bool rest_pending = false;
  int buf = 0;
  for (int k = 0; k < nb; ++k) {
    const int K = k * kMxNB, tiles = nb - k - 1;
    // block k's window was last written by block k-1's cross update, earlier on ps
    k_mx_diag<<<count, DT, kDiagSmem, ps>>>(b.M, b.perm, b.info, N, k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the inverses beside the permute (they read the diagonal tile, which the permute leaves alone)
    cudaStream_t is = ms ? ms->inv : ps;
    if (ms) {
      if ((e = cudaEventRecord(ms->ev[4], ps)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(is, ms->ev[4], 0)) != cudaSuccess) return e;
    }
    k_mx_diag_inv<<<count, DT, kInvSmem, is>>>(b.M, b.Linv, b.Uinv, b.UinvT, N, k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_mx_permute<<<dim3((unsigned)(N / PC), (unsigned)count), 256, kPermSmem, ps>>>(b.M, b.T, b.perm, N, k, count,
                                                                                   buf);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ms) {
      if ((e = cudaEventRecord(ms->ev[5], is)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(ps, ms->ev[5], 0)) != cudaSuccess) return e;
    }
    if (tiles == 0) break;
    // one launch for the two triangular solves (independent of each other):
    // L21 = A21 U11^-1 below the window (the window's rows got theirs from the
    // diagonal kernel): B^T = U11^-T (block k of UinvT); and
    // U12^T = A12^T L11^-T: B^T = L11^-1 (block k of Linv), U12 also written back into M's panel row
    MxGemmArgs gl{}, gu{};
    gl.split3 = gu.split3 = b.split3;
    gl.ax = K; gl.ay = K + 2 * kMxNB; gl.az = 0;
    gl.bx = 0; gl.by = K; gl.bz = 0;
    gl.cx = K; gl.cy = K + 2 * kMxNB; gl.cz = 0;
    gu.ax = 0; gu.ay = K + kMxNB; gu.az = buf * count;
    gu.bx = 0; gu.by = K; gu.bz = 0;
    gu.cx = 0; gu.cy = K + kMxNB; gu.cz = buf * count;
    gu.tr = b.M; gu.tr_sys = (int64_t)N * N; gu.tr_col = N; gu.tr_row = 1; gu.tr_c0 = K; gu.tr_r0 = K + kMxNB;
    const int lrows = tiles - 1;
    k_mx_gemm<0><<<dim3(1, (unsigned)(lrows + tiles), (unsigned)count), GT, kGemmSmem, ps>>>(mM, mUT, mM, gl, mT, mL,
                                                                                           mT, gu, lrows);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // A22 -= L21 U12 over the trailing tiles
    MxGemmArgs g{};
    g.split3 = b.split3;
    g.ax = K; g.ay = K + kMxNB; g.az = 0;
    g.bx = 0; g.by = K + kMxNB; g.bz = buf * count;
    g.cx = K + kMxNB; g.cy = K + kMxNB; g.cz = 0;
    g.tr = nullptr;
    g.tiles = tiles;
    if (ms && tiles > 2) {
      // the bulk (tile rows >= 2, tile columns >= 1) on the side stream once
      // the solves are in; the previous bulk is ahead of it on the same stream
      if ((e = cudaEventRecord(ms->ev[1], ps)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(ss, ms->ev[1], 0)) != cudaSuccess) return e;
      MxGemmArgs gr = g;
      gr.cross = 0;
      gr.moff = 2;
      gr.noff = 1;
      k_mx_gemm<1><<<dim3((unsigned)(tiles - 1), (unsigned)(tiles - 2), (unsigned)count), GT, kGemmSmem, ss>>>(
          mM, mT, mM, gr, mM, mT, mM, gr, 1 << 30);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      // the cross on the panel stream; it touches tiles the previous bulk updated
      if (rest_pending && (e = cudaStreamWaitEvent(ps, ms->ev[2], 0)) != cudaSuccess) return e;
      g.cross = 1;
      k_mx_gemm<1><<<dim3((unsigned)(3 * tiles - 2), 1, (unsigned)count), GT, kGemmSmem, ps>>>(mM, mT, mM, g, mM, mT,
                                                                                              mM, g, 1 << 30);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = cudaEventRecord(ms->ev[2], ss)) != cudaSuccess) return e;
      rest_pending = true;
    } else {
      if (rest_pending && (e = cudaStreamWaitEvent(ps, ms->ev[2], 0)) != cudaSuccess) return e;
      rest_pending = false;
      g.cross = 0;
      g.moff = g.noff = 0;
      k_mx_gemm<1><<<dim3((unsigned)tiles, (unsigned)tiles, (unsigned)count), GT, kGemmSmem, ps>>>(mM, mT, mM, g, mM,
                                                                                               mT, mM, g, 1 << 30);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    buf ^= 1;
  }
  // the global row order of the factors, for the substitutions' right-hand sides
  k_mx_rowpos<<<count, 256, sizeof(int) * (N + kMxWin), ps>>>(b.perm, b.rowpos, N);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (ms) {  // s resumes behind both streams
    if (rest_pending && (e = cudaStreamWaitEvent(ps, ms->ev[2], 0)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ms->ev[3], ps)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, ms->ev[3], 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t mx_rhs_in(const float* R, float* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b,
                      cudaStream_t s) {
  const int work = b.N / 4 * nrhs;
  k_mx_rhs_in<float, float><<<dim3((unsigned)((work + 255) / 256), (unsigned)b.count), 256, 0, s>>>(
      R, Y, b.n, b.N, nrhs, st, only_active, b.rbt, b.rowpos);
  return cudaGetLastError();
}

// Cluster size of the triangular solves: enough CTAs per system to cover the
// GPU's SMs when the batch is small, at most 8 (the portable cluster size) and
// no more than the blocks.
int trsv_cluster(int count, int chunks, int nb) {
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  int c = 1;
  while (c < 8 && 2 * c <= nb && (int64_t)count * chunks * 2 * c <= sms) c *= 2;
  return c;
}

template <int W, class VT>
cudaError_t launch_trsv_c(VT* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b, int C,
                          cudaStream_t s) {
  const int nb = b.N / kMxNB;
  const size_t sm = sizeof(VT) * ((size_t)((nb + C - 1) / C) * kMxNB * W + 3 * kMxNB * W);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(b.count * C), (unsigned)((nrhs + W - 1) / W));
  cfg.blockDim = dim3(TS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_mx_trsv_c<W, VT>, (const float*)b.M, (const float*)b.Linv,
                            (const float*)b.Uinv, Y, b.N, nrhs, C, st, only_active);
}

cudaError_t mx_solve(float* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b, cudaStream_t s) {
  const int W = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : 8;
  const int C = trsv_cluster(b.count, (nrhs + W - 1) / W, b.N / kMxNB);
  switch (W) {
    case 1: return launch_trsv_c<1, float>(Y, nrhs, st, only_active, b, C, s);
    case 2: return launch_trsv_c<2, float>(Y, nrhs, st, only_active, b, C, s);
    case 4: return launch_trsv_c<4, float>(Y, nrhs, st, only_active, b, C, s);
    default: return launch_trsv_c<8, float>(Y, nrhs, st, only_active, b, C, s);
  }
}

// FP64 vectors: chunks of at most 4 right-hand sides (2 at order 4096 with a
// one-CTA cluster), so that a CTA's share of the vectors fits shared memory.
cudaError_t mx_solve64(double* Y, int nrhs, const RefineState* st, int only_active, const MxBufs& b,
                       cudaStream_t s) {
  const int nb = b.N / kMxNB;
  int W = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : 4;
  int C = trsv_cluster(b.count, (nrhs + W - 1) / W, nb);
  while (W > 1 && sizeof(double) * ((size_t)((nb + C - 1) / C) * kMxNB * W + 3 * kMxNB * W) > kTrsv64Smem) {
    W >>= 1;
    C = trsv_cluster(b.count, (nrhs + W - 1) / W, nb);
  }
  switch (W) {
    case 1: return launch_trsv_c<1, double>(Y, nrhs, st, only_active, b, C, s);
    case 2: return launch_trsv_c<2, double>(Y, nrhs, st, only_active, b, C, s);
    default: return launch_trsv_c<4, double>(Y, nrhs, st, only_active, b, C, s);
  }
}

cudaError_t mx_rhs_in64(const double* R, double* Y, int nrhs, const RefineState* st, int only_active,
                        const MxBufs& b, cudaStream_t s) {
  const int work = b.N / 4 * nrhs;
  k_mx_rhs_in<double, double><<<dim3((unsigned)((work + 255) / 256), (unsigned)b.count), 256, 0, s>>>(
      R, Y, b.n, b.N, nrhs, st, only_active, b.rbt, b.rowpos);
  return cudaGetLastError();
}

cudaError_t mx_apply64(const double* Y, double* X, const double* cs, int nrhs, const RefineState* st, int init,
                       const MxBufs& b, cudaStream_t s) {
  const int work = b.N / 4 * nrhs;
  k_mx_apply<double><<<dim3((unsigned)((work + 255) / 256), (unsigned)b.count), 256, 0, s>>>(
      Y, X, cs, b.n, b.N, nrhs, st, init, b.rbt);
  return cudaGetLastError();
}

cudaError_t mx_apply(const float* Y, double* X, const double* cs, int nrhs, const RefineState* st, int init,
                     const MxBufs& b, cudaStream_t s) {
  const int work = b.N / 4 * nrhs;
  k_mx_apply<float><<<dim3((unsigned)((work + 255) / 256), (unsigned)b.count), 256, 0, s>>>(
      Y, X, cs, b.n, b.N, nrhs, st, init, b.rbt);
  return cudaGetLastError();
}

}  // namespace nppb
