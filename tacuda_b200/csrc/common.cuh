// Shared device primitives of the batched indicator engine (sm_100a).
//
// Layout conventions used by every kernel in this library:
//  * Input/output planes are series-major: bar t of series s lives at
//    plane[row_base(s) + t], row_base = s*T (uniform) or offsets[s] (ragged).
//  * A warp processes one series at a time in "rounds" of TILE = 32*K bars.
//    Lane l owns bars [t0 + l*K, t0 + l*K + K) of the round (blocked layout),
//    which keeps per-lane recurrences sequential and lets a warp-level affine
//    scan stitch lanes together.
//  * Rounds are staged in shared memory with a HALO of earlier bars so window
//    families never leave the warp. Staged arrays are padded by one word every
//    32 (pad(i) = i + i/32) which makes both the blocked per-lane reads (stride
//    K) and the coalesced copy loops bank-conflict free.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tb {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fffffff); }
__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7fffffffffffffffll); }

__host__ __device__ __forceinline__ int pad(int i) { return i + (i >> 5); }
__host__ __device__ __forceinline__ int padded_len(int n) { return n + (n >> 5) + 1; }

// Warp-level inclusive scan of 1-D affine maps y -> A*y + B in FP64, lanes in
// bar order. After the call (A, B) of lane l is the composition of lanes
// 0..l; exclusive() shifts it by one lane with the identity at lane 0.
struct Affine1 {
  double A, B;
};

__device__ __forceinline__ void warp_scan_affine(double& A, double& B, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double pA = __shfl_up_sync(kFull, A, d);
    const double pB = __shfl_up_sync(kFull, B, d);
    if (lane >= d) {
      B = fma(A, pB, B);
      A = A * pA;
    }
  }
}

// Same scan for NC channels that share the multiplier A.
template <int NC>
__device__ __forceinline__ void warp_scan_affine_shared(double& A, double (&B)[NC], int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double pA = __shfl_up_sync(kFull, A, d);
    double pB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) pB[c] = __shfl_up_sync(kFull, B[c], d);
    if (lane >= d) {
#pragma unroll
      for (int c = 0; c < NC; ++c) B[c] = fma(A, pB[c], B[c]);
      A = A * pA;
    }
  }
}

__device__ __forceinline__ double shfl_excl(double v, double ident, int lane) {
  const double u = __shfl_up_sync(kFull, v, 1);
  return lane == 0 ? ident : u;
}

__device__ __forceinline__ int warp_min_int(int v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_xor_sync(kFull, v, d));
  return v;
}

__device__ __forceinline__ int warp_max_int(int v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(kFull, v, d));
  return v;
}

// TA-Lib TRUE_RANGE in FP64: the greatest of H-L, |prevC-H|, |prevC-L| chosen
// with strict comparisons in that order.
__device__ __forceinline__ double true_range(double hi, double lo, double yc) {
  double g = hi - lo;
  const double a = fabs(yc - hi);
  if (a > g) g = a;
  const double b = fabs(yc - lo);
  if (b > g) g = b;
  return g;
}

// TA-Lib's EMA coefficients (talib08:5546-5627 TA_EMA): beta = (p-1)/(p+1),
// k = 1 - beta, and beta = 1 - k when beta < 0.5.
__host__ __device__ inline void talib_ema_coeffs(int p, double& beta, double& k) {
  double b = (double)(p - 1) / (double)(p + 1);
  double kk = 1.0 - b;
  if (b < 0.5) b = 1.0 - kk;
  beta = b;
  k = kk;
}

// One AROON line as the reference's kernels round it (src/indicators/Aroon.cu:
// 37, 49): 100.0f times the bars left in the window, divided by the period.
__device__ __forceinline__ float aroon_line(int p, int since) { return 100.0f * (float)(p - since) / (float)p; }

}  // namespace tb
