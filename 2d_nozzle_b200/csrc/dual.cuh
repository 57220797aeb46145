// dual.cuh -- forward-mode dual numbers for exact flux Jacobians.
//
// A Dual<N> carries a value and N partial derivatives.  The pointwise physics
// (physics.cuh) is written once over a scalar type; instantiated with double it
// is the forward flux, with Dual<N> seeded on N inputs it also yields those N
// columns of the flux Jacobian, exactly (no finite differences).  Branches
// compare values, as the reference's own branches do, so a derivative is the
// derivative of the branch the value takes.
#pragma once
#include <cmath>

namespace nzb {

// The Dual overloads below would hide the global math functions for plain
// doubles inside this namespace; bring those back in.
using ::fabs;
using ::fmax;
using ::fmin;
using ::pow;
using ::sqrt;

template <int N>
struct Dual {
  double v;
  double d[N];
  __device__ __forceinline__ Dual() {}
  __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = 0.0;
  }
  static __device__ __forceinline__ Dual seed(double x, int k) {
    Dual r(x);
    r.d[k] = 1.0;
    return r;
  }
};

#define NZB_DUAL_BINOP(OP, VAL, DER)                                                   \
  template <int N>                                                                     \
  __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) { \
    Dual<N> r;                                                                         \
    r.v = VAL;                                                                         \
    _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DER;                        \
    return r;                                                                          \
  }
NZB_DUAL_BINOP(+, a.v + b.v, a.d[k] + b.d[k])
NZB_DUAL_BINOP(-, a.v - b.v, a.d[k] - b.d[k])
NZB_DUAL_BINOP(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef NZB_DUAL_BINOP

template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double inv = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
// Mixed with plain numbers.  A plain operand has no derivative, and these
// overloads skip the products with its zero derivative part outright: IEEE
// arithmetic does not let the compiler drop x * 0.0 or x + 0.0 by itself.  The
// values are the same as with a Dual of zero derivative.
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v + b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v - b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a * b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v / b;
  const double inv = 1.0 / b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * inv;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a / b.v;
  const double inv = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -(r.v * b.d[k]) * inv;
  return r;
}

// The type of an expression mixing A and B: Dual<N> when either is one.
template <class A, class B>
using Mix = decltype(*(A*)nullptr + *(B*)nullptr);
template <class A, class B, class C>
using Mix3 = Mix<Mix<A, B>, C>;

// x's type holding the plain number v (a constant branch of a selection).
template <class X>
__device__ __forceinline__ X like(const X&, double v) {
  return X(v);
}

#define NZB_DUAL_CMP(OP)                                                                                      \
  template <int N> __device__ __forceinline__ bool operator OP(const Dual<N>& a, const Dual<N>& b) {          \
    return a.v OP b.v;                                                                                        \
  }                                                                                                           \
  template <int N> __device__ __forceinline__ bool operator OP(const Dual<N>& a, double b) { return a.v OP b; } \
  template <int N> __device__ __forceinline__ bool operator OP(double a, const Dual<N>& b) { return a OP b.v; }
NZB_DUAL_CMP(<)
NZB_DUAL_CMP(>)
NZB_DUAL_CMP(<=)
NZB_DUAL_CMP(>=)
#undef NZB_DUAL_CMP

template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double h = 0.5 / r.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * h;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, const Dual<N>& b) {
  return b.v < a.v ? b : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, const Dual<N>& b) {
  return b.v > a.v ? b : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, double b) {
  return b < a.v ? Dual<N>(b) : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmin(double a, const Dual<N>& b) {
  return b.v < a ? b : Dual<N>(a);
}
template <int N>
__device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, double b) {
  return b > a.v ? Dual<N>(b) : a;
}
template <int N>
__device__ __forceinline__ Dual<N> fmax(double a, const Dual<N>& b) {
  return b.v > a ? b : Dual<N>(a);
}
template <int N>
__device__ __forceinline__ Dual<N> pow(const Dual<N>& a, double c) {
  Dual<N> r;
  r.v = ::pow(a.v, c);
  const double dv = c * ::pow(a.v, c - 1.0);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * dv;
  return r;
}

}  // namespace nzb
