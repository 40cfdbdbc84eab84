// Forward-mode dual numbers for tangent (Jacobian-vector) products of
// scalar device code: Dual<N> carries a float value and N directional
// derivatives.  Code written against the small set of functions below
// (arithmetic, vsqrt, vexp, vlog, vpow with a constant exponent, vmin, vmax,
// vabs, sel, val) runs both on float (the plain value) and on Dual<N> (the
// value and N tangents at once).  Comparisons take the value, so branches and
// selections follow the value path exactly: the derivative is that of the
// branch taken.
#pragma once
#include "wrf_common.cuh"

namespace wrf {

template <int N>
struct Dual {
  float v;
  float d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(float x) {
  Dual<N> r;
  r.v = x;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = 0.f;
  return r;
}

// the value of a float or a dual
__device__ __forceinline__ float val(float x) { return x; }
template <int N>
__device__ __forceinline__ float val(const Dual<N>& x) { return x.v; }

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a.d[n] + b.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a.d[n] - b.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = -a.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a.d[n] * b.v + a.v * b.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const float ib = 1.0f / b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = (a.d[n] - r.v * b.d[n]) * ib;
  return r;
}
// mixed with a constant
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, float b) {
  Dual<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(float a, const Dual<N>& b) {
  return b + a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, float b) {
  Dual<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(float a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = -b.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, float b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a.d[n] * b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(float a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a * b.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, float b) {
  Dual<N> r;
  r.v = a.v / b;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = a.d[n] / b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(float a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a / b.v;
  const float s = -r.v / b.v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = s * b.d[n];
  return r;
}

// elementary functions: the value by the library's float function, the
// derivative from its closed form
__device__ __forceinline__ float vsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float vexp(float x) { return wexp(x); }
__device__ __forceinline__ float vlog(float x) { return wlog(x); }
__device__ __forceinline__ float vpow(float x, float e) { return wpow(x, e); }
__device__ __forceinline__ float vabs(float x) { return fabsf(x); }
__device__ __forceinline__ float vmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float vmax(float a, float b) { return b > a ? b : a; }

template <int N>
__device__ __forceinline__ Dual<N> scale_d(float v, const Dual<N>& x, float dv) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int n = 0; n < N; ++n) r.d[n] = dv * x.d[n];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> vsqrt(const Dual<N>& x) {
  const float v = sqrtf(x.v);
  return scale_d(v, x, v > 0.f ? 0.5f / v : 0.f);
}
template <int N>
__device__ __forceinline__ Dual<N> vexp(const Dual<N>& x) {
  const float v = wexp(x.v);
  return scale_d(v, x, v);
}
template <int N>
__device__ __forceinline__ Dual<N> vlog(const Dual<N>& x) {
  return scale_d(wlog(x.v), x, 1.0f / x.v);
}
// x^e for a constant e: d = e x^(e-1), formed as e x^e / x (0 at x = 0
// for e > 1)
template <int N>
__device__ __forceinline__ Dual<N> vpow(const Dual<N>& x, float e) {
  const float v = wpow(x.v, e);
  return scale_d(v, x, x.v != 0.f ? e * v / x.v : 0.f);
}
template <int N>
__device__ __forceinline__ Dual<N> vabs(const Dual<N>& x) {
  return x.v < 0.f ? -x : x;
}
template <int N>
__device__ __forceinline__ Dual<N> vmin(const Dual<N>& a, const Dual<N>& b) {
  return b.v < a.v ? b : a;
}
template <int N>
__device__ __forceinline__ Dual<N> vmax(const Dual<N>& a, const Dual<N>& b) {
  return b.v > a.v ? b : a;
}
template <int N>
__device__ __forceinline__ Dual<N> vmin(const Dual<N>& a, float b) {
  return b < a.v ? dconst<N>(b) : a;
}
template <int N>
__device__ __forceinline__ Dual<N> vmax(const Dual<N>& a, float b) {
  return b > a.v ? dconst<N>(b) : a;
}
template <int N>
__device__ __forceinline__ Dual<N> vmin(float a, const Dual<N>& b) {
  return b.v < a ? b : dconst<N>(a);
}
template <int N>
__device__ __forceinline__ Dual<N> vmax(float a, const Dual<N>& b) {
  return b.v > a ? b : dconst<N>(a);
}

// a constant of the scalar type
template <class T>
struct Lift;
template <>
struct Lift<float> {
  __device__ static float c(float x) { return x; }
};
template <int N>
struct Lift<Dual<N>> {
  __device__ static Dual<N> c(float x) { return dconst<N>(x); }
};

// cond ? a : b on either type (a constant operand lifted)
template <class T>
__device__ __forceinline__ T sel(bool c, const T& a, const T& b) {
  return c ? a : b;
}

}  // namespace wrf
