// real.cuh -- arithmetic types for the narrowphase templates.
//
// xf64 is an FP64 value whose + - * / and sqrt each round once (IEEE round-to-nearest)
// and are never contracted into an FMA, whatever -fmad says.  Code written over xf64
// therefore performs exactly the rounded operations a C++ compiler emits for the same
// expression without contraction, which is how the reference is compiled for the
// oracle.  float is used as is (FMA contraction allowed).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace delta {

struct xf64 {
  double v;
  xf64() = default;
  __host__ __device__ __forceinline__ constexpr xf64(double x) : v(x) {}
};

__device__ __forceinline__ xf64 operator+(xf64 a, xf64 b) { return xf64(__dadd_rn(a.v, b.v)); }
__device__ __forceinline__ xf64 operator-(xf64 a, xf64 b) { return xf64(__dsub_rn(a.v, b.v)); }
__device__ __forceinline__ xf64 operator*(xf64 a, xf64 b) { return xf64(__dmul_rn(a.v, b.v)); }
__device__ __forceinline__ xf64 operator/(xf64 a, xf64 b) { return xf64(__ddiv_rn(a.v, b.v)); }
__device__ __forceinline__ xf64 operator-(xf64 a) { return xf64(-a.v); }
__device__ __forceinline__ xf64 &operator+=(xf64 &a, xf64 b) { a = a + b; return a; }
__device__ __forceinline__ xf64 &operator-=(xf64 &a, xf64 b) { a = a - b; return a; }
__device__ __forceinline__ xf64 &operator*=(xf64 &a, xf64 b) { a = a * b; return a; }
__device__ __forceinline__ xf64 &operator/=(xf64 &a, xf64 b) { a = a / b; return a; }
__device__ __forceinline__ bool operator<(xf64 a, xf64 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(xf64 a, xf64 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(xf64 a, xf64 b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(xf64 a, xf64 b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(xf64 a, xf64 b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(xf64 a, xf64 b) { return a.v != b.v; }

__device__ __forceinline__ xf64 sqrt_(xf64 a) { return xf64(__dsqrt_rn(a.v)); }
__device__ __forceinline__ xf64 fabs_(xf64 a) { return xf64(fabs(a.v)); }
__device__ __forceinline__ float sqrt_(float a) { return sqrtf(a); }
__device__ __forceinline__ float fabs_(float a) { return fabsf(a); }

template <class R> __device__ __forceinline__ double to_f64(R x);
template <> __device__ __forceinline__ double to_f64<xf64>(xf64 x) { return x.v; }
template <> __device__ __forceinline__ double to_f64<float>(float x) { return (double)x; }
template <class R> __device__ __forceinline__ R from_f64(double x);
template <> __device__ __forceinline__ xf64 from_f64<xf64>(double x) { return xf64(x); }
template <> __device__ __forceinline__ float from_f64<float>(double x) { return (float)x; }

template <class R> __device__ __forceinline__ R dot3(const R *a, const R *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

}  // namespace delta
