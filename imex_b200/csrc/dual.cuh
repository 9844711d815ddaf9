// Forward-mode dual numbers with L derivative lanes.  The per-cell physics of the
// stage is written once as templates on its scalar type: double for the forward
// kernels, Dual<L> for the adjoint, which evaluates a cell function with L of its
// inputs seeded and so reads L columns of the cell's local Jacobian per pass.
// Non-smooth points (|x| at 0, min/max ties, sqrt at 0) take the one-sided
// derivative of the branch the double evaluation takes.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace imex {

// the double overloads stay visible beside the Dual ones declared below
using ::fabs;
using ::fmax;
using ::fmin;
using ::log;
using ::sqrt;

template <int L>
struct Dual {
  double v;
  double d[L];
  __device__ __forceinline__ Dual() : v(0.0) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = 0.0;
  }
  __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int l = 0; l < L; ++l) d[l] = 0.0;
  }
  __device__ __forceinline__ Dual& operator+=(const Dual& b) { return *this = *this + b; }
  __device__ __forceinline__ Dual& operator-=(const Dual& b) { return *this = *this - b; }
  __device__ __forceinline__ Dual& operator*=(const Dual& b) { return *this = *this * b; }
  __device__ __forceinline__ Dual& operator/=(const Dual& b) { return *this = *this / b; }
  friend __device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
    Dual r(a.v + b.v);
#pragma unroll
    for (int l = 0; l < L; ++l) r.d[l] = a.d[l] + b.d[l];
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
    Dual r(a.v - b.v);
#pragma unroll
    for (int l = 0; l < L; ++l) r.d[l] = a.d[l] - b.d[l];
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual& a) {
    Dual r(-a.v);
#pragma unroll
    for (int l = 0; l < L; ++l) r.d[l] = -a.d[l];
    return r;
  }
  friend __device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
    Dual r(a.v * b.v);
#pragma unroll
    for (int l = 0; l < L; ++l) r.d[l] = a.d[l] * b.v + a.v * b.d[l];
    return r;
  }
  friend __device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
    const double q = a.v / b.v;
    Dual r(q);
#pragma unroll
    for (int l = 0; l < L; ++l) r.d[l] = (a.d[l] - q * b.d[l]) / b.v;
    return r;
  }
  friend __device__ __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
  friend __device__ __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
  friend __device__ __forceinline__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
  friend __device__ __forceinline__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
};

template <int L>
__device__ __forceinline__ Dual<L> sqrt(const Dual<L>& a) {
  const double s = ::sqrt(a.v);
  Dual<L> r(s);
  const double g = s > 0.0 ? 0.5 / s : 0.0;
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = g * a.d[l];
  return r;
}
template <int L>
__device__ __forceinline__ Dual<L> fabs(const Dual<L>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int L>
__device__ __forceinline__ Dual<L> fmax(const Dual<L>& a, const Dual<L>& b) {
  return (b.v > a.v) ? b : a;
}
template <int L>
__device__ __forceinline__ Dual<L> fmin(const Dual<L>& a, const Dual<L>& b) {
  return (b.v < a.v) ? b : a;
}
template <int L>
__device__ __forceinline__ Dual<L> log(const Dual<L>& a) {
  Dual<L> r(::log(a.v));
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] / a.v;
  return r;
}
template <int L>
__device__ __forceinline__ double value_of(const Dual<L>& a) {
  return a.v;
}
__device__ __forceinline__ double value_of(double a) { return a; }

// a double operand on either side
template <int L>
__device__ __forceinline__ Dual<L> operator+(double a, const Dual<L>& b) { return Dual<L>(a) + b; }
template <int L>
__device__ __forceinline__ Dual<L> operator+(const Dual<L>& a, double b) { return a + Dual<L>(b); }
template <int L>
__device__ __forceinline__ Dual<L> operator-(double a, const Dual<L>& b) { return Dual<L>(a) - b; }
template <int L>
__device__ __forceinline__ Dual<L> operator-(const Dual<L>& a, double b) { return a - Dual<L>(b); }
template <int L>
__device__ __forceinline__ Dual<L> operator*(double a, const Dual<L>& b) {
  Dual<L> r(a * b.v);
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a * b.d[l];
  return r;
}
template <int L>
__device__ __forceinline__ Dual<L> operator*(const Dual<L>& a, double b) {
  Dual<L> r(a.v * b);
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] * b;
  return r;
}
template <int L>
__device__ __forceinline__ Dual<L> operator/(const Dual<L>& a, double b) {
  Dual<L> r(a.v / b);
#pragma unroll
  for (int l = 0; l < L; ++l) r.d[l] = a.d[l] / b;
  return r;
}
template <int L>
__device__ __forceinline__ Dual<L> operator/(double a, const Dual<L>& b) { return Dual<L>(a) / b; }
template <int L>
__device__ __forceinline__ bool operator<(const Dual<L>& a, double b) { return a.v < b; }
template <int L>
__device__ __forceinline__ bool operator>(const Dual<L>& a, double b) { return a.v > b; }
template <int L>
__device__ __forceinline__ bool operator<=(const Dual<L>& a, double b) { return a.v <= b; }
template <int L>
__device__ __forceinline__ bool operator>=(const Dual<L>& a, double b) { return a.v >= b; }
template <int L>
__device__ __forceinline__ bool operator<(double a, const Dual<L>& b) { return a < b.v; }
template <int L>
__device__ __forceinline__ bool operator>(double a, const Dual<L>& b) { return a > b.v; }
template <int L>
__device__ __forceinline__ bool operator<=(double a, const Dual<L>& b) { return a <= b.v; }
template <int L>
__device__ __forceinline__ bool operator>=(double a, const Dual<L>& b) { return a >= b.v; }

}  // namespace imex
