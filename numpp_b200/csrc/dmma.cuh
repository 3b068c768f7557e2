// FP64 tensor-core (DMMA) and warp helpers for sm_100a.
#pragma once

#include <climits>

namespace nppb {

// D(8x8) += A(8x4) * B(4x8), FP64, one warp. Lane l = 4*g + t holds
// A[g][t], B[t][g] and D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Warp-wide argmax of (v, i): the largest v wins, ties go to the smaller i.
// Every lane ends with the same pair.
__device__ __forceinline__ void warp_argmax(double& v, int& i) {
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
  }
}

// Warp-wide argmax for magnitudes (v >= 0; v < 0 marks "no candidate"): the
// largest v wins, ties go to the smaller key. IEEE bit patterns of non-negative
// doubles order like the values, so three redux instructions replace the
// shuffle butterfly. Every lane ends with the same pair.
__device__ __forceinline__ void warp_argmax_abs(double& v, int& key) {
  const unsigned long long bits = v > 0.0 ? (unsigned long long)__double_as_longlong(v) : 0ull;
  const unsigned hi = (unsigned)(bits >> 32), lo = (unsigned)bits;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool top = hi == mhi && lo == mlo;
  const int k = __reduce_min_sync(0xffffffffu, top ? key : INT_MAX);
  v = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
  key = k;
}

// The same for FP32 magnitudes: one 32-bit key.
__device__ __forceinline__ void warp_argmax_abs(float& v, int& key) {
  const unsigned bits = v > 0.f ? __float_as_uint(v) : 0u;
  const unsigned m = __reduce_max_sync(0xffffffffu, bits);
  const int k = __reduce_min_sync(0xffffffffu, bits == m ? key : INT_MAX);
  v = __uint_as_float(m);
  key = k;
}

}  // namespace nppb
