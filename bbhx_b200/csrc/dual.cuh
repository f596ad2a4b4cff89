// Forward-mode dual numbers for the gradient kernels.
//
// Dual<N> carries a value and N tangents (directional derivatives with respect to N seeded
// inputs).  The model code in phenomhm_model.cuh / response_model.cuh is templated on its
// scalar type; instantiated with Dual<N> it propagates d(output)/d(theta) for all N source
// parameters in one pass.  Arithmetic follows the chain rule exactly (no finite
// differences): for f(x) the value is f(v) and each tangent is f'(v) * dx.
//
// The overloads live in namespace bbhx::ad and are found by argument-dependent lookup, so
// unqualified calls such as sqrt(x) keep resolving to CUDA's double functions for double
// arguments.  Comparisons compare values (branches of the piecewise model follow the
// value, as in the FP64 code).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace bbhx {
namespace ad {

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ __forceinline__ Dual() {}
  __host__ __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
};

// a * x + b * y helpers keep the tangent loops in one place
template <int N>
__device__ __forceinline__ Dual<N> lin1(double fv, double dfdx, const Dual<N>& x) {
  Dual<N> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = dfdx * x.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> lin2(double fv, double a, const Dual<N>& x, double b,
                                        const Dual<N>& y) {
  Dual<N> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a * x.d[i] + b * y.d[i];
  return r;
}

// ---------------------------------------------------------------- arithmetic
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  return lin2(a.v + b.v, 1.0, a, 1.0, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  return lin2(a.v - b.v, 1.0, a, -1.0, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  return lin2(a.v * b.v, b.v, a, a.v, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  const double ib = 1.0 / b.v;
  const double q = a.v * ib;
  return lin2(q, ib, a, -q * ib, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  return lin1(-a.v, -1.0, a);
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v += b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
  return b + a;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v -= b;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
  return lin1(a - b.v, -1.0, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
  return lin1(a.v * b, b, a);
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
  return lin1(a * b.v, a, b);
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
  const double ib = 1.0 / b;
  return lin1(a.v * ib, ib, a);
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
  const double q = a / b.v;
  return lin1(q, -q / b.v, b);
}
template <int N, typename S>
__device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const S& b) {
  a = a + b;
  return a;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const S& b) {
  a = a - b;
  return a;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N>& operator*=(Dual<N>& a, const S& b) {
  a = a * b;
  return a;
}
template <int N, typename S>
__device__ __forceinline__ Dual<N>& operator/=(Dual<N>& a, const S& b) {
  a = a / b;
  return a;
}

// ---------------------------------------------------------------- comparisons (by value)
#define BBHX_DUAL_CMP(op)                                                                    \
  template <int N>                                                                           \
  __device__ __forceinline__ bool operator op(const Dual<N>& a, const Dual<N>& b) {          \
    return a.v op b.v;                                                                       \
  }                                                                                          \
  template <int N>                                                                           \
  __device__ __forceinline__ bool operator op(const Dual<N>& a, double b) {                  \
    return a.v op b;                                                                         \
  }                                                                                          \
  template <int N>                                                                           \
  __device__ __forceinline__ bool operator op(double a, const Dual<N>& b) {                  \
    return a op b.v;                                                                         \
  }
BBHX_DUAL_CMP(<)
BBHX_DUAL_CMP(>)
BBHX_DUAL_CMP(<=)
BBHX_DUAL_CMP(>=)
BBHX_DUAL_CMP(==)
BBHX_DUAL_CMP(!=)
#undef BBHX_DUAL_CMP

// ---------------------------------------------------------------- elementary functions
template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& x) {
  const double s = ::sqrt(x.v);
  return lin1(s, 0.5 / s, x);
}
template <int N>
__device__ __forceinline__ Dual<N> cbrt(const Dual<N>& x) {
  const double c = ::cbrt(x.v);
  return lin1(c, 1.0 / (3.0 * c * c), x);
}
template <int N>
__device__ __forceinline__ Dual<N> log(const Dual<N>& x) {
  return lin1(::log(x.v), 1.0 / x.v, x);
}
template <int N>
__device__ __forceinline__ Dual<N> exp(const Dual<N>& x) {
  const double e = ::exp(x.v);
  return lin1(e, e, x);
}
template <int N>
__device__ __forceinline__ Dual<N> pow(const Dual<N>& x, double p) {
  const double r = ::pow(x.v, p);
  return lin1(r, p * ::pow(x.v, p - 1.0), x);
}
template <int N>
__device__ __forceinline__ Dual<N> atan(const Dual<N>& x) {
  return lin1(::atan(x.v), 1.0 / (1.0 + x.v * x.v), x);
}
template <int N>
__device__ __forceinline__ Dual<N> sin(const Dual<N>& x) {
  double s, c;
  ::sincos(x.v, &s, &c);
  return lin1(s, c, x);
}
template <int N>
__device__ __forceinline__ Dual<N> cos(const Dual<N>& x) {
  double s, c;
  ::sincos(x.v, &s, &c);
  return lin1(c, -s, x);
}
template <int N>
__device__ __forceinline__ void sincos(const Dual<N>& x, Dual<N>* s, Dual<N>* c) {
  double sv, cv;
  ::sincos(x.v, &sv, &cv);
  *s = lin1(sv, cv, x);
  *c = lin1(cv, -sv, x);
}
template <int N>
__device__ __forceinline__ Dual<N> fabs(const Dual<N>& x) {
  return x.v < 0.0 ? -x : x;
}
template <int N>
__device__ __forceinline__ Dual<N> hypot(const Dual<N>& a, const Dual<N>& b) {
  const double h = ::hypot(a.v, b.v);
  if (h == 0.0) return Dual<N>(0.0);
  return lin2(h, a.v / h, a, b.v / h, b);
}
// piecewise-constant functions: value only, zero tangents
template <int N>
__device__ __forceinline__ double floor(const Dual<N>& x) {
  return ::floor(x.v);
}

}  // namespace ad

// value part of a scalar (identity for plain floating types)
__device__ __forceinline__ double value_of(double x) { return x; }
__device__ __forceinline__ float value_of(float x) { return x; }
template <int N>
__device__ __forceinline__ double value_of(const ad::Dual<N>& x) {
  return x.v;
}

}  // namespace bbhx
