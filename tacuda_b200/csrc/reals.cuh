// Arithmetic types of the precision variants (job precision field):
//   double - FP64 (the default, reference-parity path),
//   float  - plain FP32,
//   F2     - compensated FP32: an unevaluated float pair hi + lo kept with
//            error-free transformations (Knuth two-sum, FMA two-product),
//            about 44 significant bits from FP32 operations only.
// Code templated on the type uses the overloads below; the library is
// compiled without FMA contraction, so a + b and a * b are single roundings
// as the transformations require.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace tb {

struct F2 {
  float hi, lo;
};

__device__ __forceinline__ F2 two_sum(float a, float b) {
  const float s = a + b;
  const float bb = s - a;
  const float e = (a - (s - bb)) + (b - bb);
  return F2{s, e};
}

__device__ __forceinline__ F2 fast_two_sum(float a, float b) {  // |a| >= |b|
  const float s = a + b;
  return F2{s, b - (s - a)};
}

__device__ __forceinline__ F2 operator+(F2 x, F2 y) {
  F2 s = two_sum(x.hi, y.hi);
  const F2 t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ F2 operator-(F2 x) { return F2{-x.hi, -x.lo}; }
__device__ __forceinline__ F2 operator-(F2 x, F2 y) { return x + (-y); }
__device__ __forceinline__ F2 operator*(F2 x, F2 y) {
  const float p = x.hi * y.hi;
  float e = fmaf(x.hi, y.hi, -p);
  e += x.hi * y.lo + x.lo * y.hi;
  return fast_two_sum(p, e);
}
__device__ __forceinline__ F2 operator/(F2 x, F2 y) {
  const float q1 = x.hi / y.hi;
  const F2 r = x - y * F2{q1, 0.0f};
  const float q2 = r.hi / y.hi;
  return fast_two_sum(q1, q2);
}
__device__ __forceinline__ F2& operator+=(F2& x, F2 y) { return x = x + y; }
__device__ __forceinline__ F2& operator-=(F2& x, F2 y) { return x = x - y; }
__device__ __forceinline__ bool operator>(F2 x, F2 y) { return x.hi > y.hi || (x.hi == y.hi && x.lo > y.lo); }
__device__ __forceinline__ bool operator!=(F2 x, F2 y) { return x.hi != y.hi || x.lo != y.lo; }

// Uniform helpers over double / float / F2.
template <class R>
struct Real;

template <>
struct Real<double> {
  __device__ static __forceinline__ double of(double v) { return v; }
  __device__ static __forceinline__ double to_d(double v) { return v; }
  __device__ static __forceinline__ double sqrt_r(double v) { return sqrt(v); }
  __device__ static __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }
  __device__ static __forceinline__ bool is_nan(double v) { return isnan(v); }
};

template <>
struct Real<float> {
  __device__ static __forceinline__ float of(double v) { return (float)v; }
  __device__ static __forceinline__ double to_d(float v) { return (double)v; }
  __device__ static __forceinline__ float sqrt_r(float v) { return sqrtf(v); }
  __device__ static __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }
  __device__ static __forceinline__ bool is_nan(float v) { return isnan(v); }
};

template <>
struct Real<F2> {
  // exact split of a double with at most 48 significant bits (float inputs,
  // their differences and products); other doubles round to about 2^-48
  __device__ static __forceinline__ F2 of(double v) {
    const float hi = (float)v;
    return F2{hi, (float)(v - (double)hi)};
  }
  __device__ static __forceinline__ double to_d(F2 v) { return (double)v.hi + (double)v.lo; }
  __device__ static __forceinline__ F2 sqrt_r(F2 v) {
    if (!(v.hi > 0.0f)) return F2{0.0f, 0.0f};
    const float s = sqrtf(v.hi);
    const F2 r = v - F2{s, 0.0f} * F2{s, 0.0f};
    return fast_two_sum(s, r.hi / (2.0f * s));
  }
  __device__ static __forceinline__ F2 fma_r(F2 a, F2 b, F2 c) { return a * b + c; }
  __device__ static __forceinline__ bool is_nan(F2 v) { return isnan(v.hi); }
};

// Warp shuffles of the three types.
__device__ __forceinline__ double shfl_up_r(double v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ float shfl_up_r(float v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ F2 shfl_up_r(F2 v, int d) {
  return F2{__shfl_up_sync(kFull, v.hi, d), __shfl_up_sync(kFull, v.lo, d)};
}
__device__ __forceinline__ double shfl_r(double v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ float shfl_r(float v, int src) { return __shfl_sync(kFull, v, src); }
__device__ __forceinline__ F2 shfl_r(F2 v, int src) {
  return F2{__shfl_sync(kFull, v.hi, src), __shfl_sync(kFull, v.lo, src)};
}

}  // namespace tb
