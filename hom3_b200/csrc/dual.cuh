// dual.cuh -- forward-mode dual numbers with K derivative directions for
// device code: a value and K partial derivatives, propagated by the chain rule
// through the library's templated flux functions (make_prim, ausm, viscous),
// so an adjoint can take exact local derivatives of the GPU's own arithmetic.
// Comparisons look at values only: branches are those of the double path.
#pragma once
#include <cuda_runtime.h>

namespace h3c {

// keep the double overloads visible beside the dual ones below
using ::fabs;
using ::sqrt;

template <int K> struct DN {
  double v;
  double d[K];
  __device__ __forceinline__ DN() : v(0.0) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }
  __device__ __forceinline__ DN(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }
};

template <int K> __device__ __forceinline__ DN<K> operator+(const DN<K>& a, const DN<K>& b) {
  DN<K> r(a.v + b.v);
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator-(const DN<K>& a, const DN<K>& b) {
  DN<K> r(a.v - b.v);
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator-(const DN<K>& a) {
  DN<K> r(-a.v);
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator*(const DN<K>& a, const DN<K>& b) {
  DN<K> r(a.v * b.v);
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator/(const DN<K>& a, const DN<K>& b) {
  DN<K> r(a.v / b.v);
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator+(const DN<K>& a, double b) { return a + DN<K>(b); }
template <int K> __device__ __forceinline__ DN<K> operator+(double a, const DN<K>& b) { return DN<K>(a) + b; }
template <int K> __device__ __forceinline__ DN<K> operator-(const DN<K>& a, double b) { return a - DN<K>(b); }
template <int K> __device__ __forceinline__ DN<K> operator-(double a, const DN<K>& b) { return DN<K>(a) - b; }
template <int K> __device__ __forceinline__ DN<K> operator*(const DN<K>& a, double b) {
  DN<K> r(a.v * b);
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <int K> __device__ __forceinline__ DN<K> operator*(double a, const DN<K>& b) { return b * a; }
template <int K> __device__ __forceinline__ DN<K> operator/(const DN<K>& a, double b) { return a / DN<K>(b); }
template <int K> __device__ __forceinline__ DN<K> operator/(double a, const DN<K>& b) { return DN<K>(a) / b; }
#define H3C_DN_CMP(op)                                                                                      \
  template <int K> __device__ __forceinline__ bool operator op(const DN<K>& a, const DN<K>& b) {         \
    return a.v op b.v;                                                                                     \
  }                                                                                                        \
  template <int K> __device__ __forceinline__ bool operator op(const DN<K>& a, double b) { return a.v op b; } \
  template <int K> __device__ __forceinline__ bool operator op(double a, const DN<K>& b) { return a op b.v; }
H3C_DN_CMP(<)
H3C_DN_CMP(>)
H3C_DN_CMP(<=)
H3C_DN_CMP(>=)
#undef H3C_DN_CMP

template <int K> __device__ __forceinline__ DN<K> fabs(const DN<K>& a) { return a.v < 0.0 ? -a : a; }
template <int K> __device__ __forceinline__ DN<K> sqrt(const DN<K>& a) {
  DN<K> r(::sqrt(a.v));
  const double s = 0.5 / r.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
  return r;
}

}  // namespace h3c
