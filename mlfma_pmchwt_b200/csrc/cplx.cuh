// complex128 helpers on double2 (x = real, y = imaginary), and the complex64
// subset the mixed-precision operator uses on float2.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace mlfma {

__host__ __device__ __forceinline__ double2 c2(double re, double im) { return make_double2(re, im); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a * b + c
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// s * a + c (s real)
__host__ __device__ __forceinline__ double2 cfmas(double s, double2 a, double2 c) {
  return make_double2(fma(s, a.x, c.x), fma(s, a.y, c.y));
}
__host__ __device__ __forceinline__ double2 cmulj(double2 a) { return make_double2(-a.y, a.x); }  // j * a
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__host__ __device__ __forceinline__ double2 cexp(double2 z) {
  double s, c;
#ifdef __CUDA_ARCH__
  sincos(z.y, &s, &c);
#else
  s = ::sin(z.y);
  c = ::cos(z.y);
#endif
  const double e = exp(z.x);
  return make_double2(e * c, e * s);
}
// exp(-j * k * t) for complex k and real t
__host__ __device__ __forceinline__ double2 cexp_mjkt(double2 k, double t) {
  return cexp(make_double2(k.y * t, -k.x * t));
}

// complex64 counterparts on float2, for the mixed-precision operator
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__host__ __device__ __forceinline__ float2 cfmas(float s, float2 a, float2 c) {
  return make_float2(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y));
}

__host__ __device__ __forceinline__ float2 cdiv(float2 a, float2 b) {
  if (fabsf(b.x) >= fabsf(b.y)) {
    const float r = b.y / b.x, d = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const float r = b.x / b.y, d = b.x * r + b.y;
  return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

// Storage-type traits of the apply kernels: the complex type C (double2 or
// float2), its real type, zero and conversions from / to complex128.
template <class C>
struct Cx;
template <>
struct Cx<double2> {
  using real = double;
  __host__ __device__ static __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
  __host__ __device__ static __forceinline__ double2 from(double2 v) { return v; }
  __host__ __device__ static __forceinline__ double2 to64(double2 v) { return v; }
};
template <>
struct Cx<float2> {
  using real = float;
  __host__ __device__ static __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  __host__ __device__ static __forceinline__ float2 from(double2 v) {
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
  }
  __host__ __device__ static __forceinline__ double2 to64(float2 v) { return make_double2(v.x, v.y); }
};

}  // namespace mlfma
