// Forward-mode dual numbers of the tangent-linear steps (nim_gpu_tangent_*).
//
// A DualD carries a value v and its derivative t along one seeded direction
// (of nu, alpha and the state fields).  Each operation computes v with the
// double operation itself, so a dual pass gives the FP64 pass's values bit
// for bit, and t by the chain rule, one rounded operation per term:
//   (a + b)' = a' + b'              (a b)' = a' b + a b'
//   (a / b)' = (a' - (a/b) b') / b  exp(a)' = exp(a) a'
//   |a|'     = sign(a) a'
// Comparisons look at the value only: the derivative is that of the branch
// the values take.
#pragma once

#include "nim_exp.cuh"

namespace nim {

struct DualD {
  double v, t;
  DualD() = default;
  __host__ __device__ constexpr DualD(double a) : v(a), t(0.0) {}  // constants, geometry: no derivative
  __host__ __device__ constexpr DualD(double a, double b) : v(a), t(b) {}
};

__host__ __device__ __forceinline__ DualD operator+(const DualD &a) { return a; }
__host__ __device__ __forceinline__ DualD operator-(const DualD &a) { return DualD(-a.v, -a.t); }
__host__ __device__ __forceinline__ DualD operator+(const DualD &a, const DualD &b) {
  return DualD(a.v + b.v, a.t + b.t);
}
__host__ __device__ __forceinline__ DualD operator-(const DualD &a, const DualD &b) {
  return DualD(a.v - b.v, a.t - b.t);
}
__host__ __device__ __forceinline__ DualD operator*(const DualD &a, const DualD &b) {
  return DualD(a.v * b.v, a.t * b.v + a.v * b.t);
}
__host__ __device__ __forceinline__ DualD operator/(const DualD &a, const DualD &b) {
  const double q = a.v / b.v;
  return DualD(q, (a.t - q * b.t) / b.v);
}
__host__ __device__ __forceinline__ bool operator<(const DualD &a, const DualD &b) { return a.v < b.v; }
__host__ __device__ __forceinline__ bool operator>(const DualD &a, const DualD &b) { return a.v > b.v; }
__host__ __device__ __forceinline__ bool operator<=(const DualD &a, const DualD &b) { return a.v <= b.v; }
__host__ __device__ __forceinline__ bool operator>=(const DualD &a, const DualD &b) { return a.v >= b.v; }

// (the global fabs overloads stay visible beside this one inside nim)
using ::fabs;
__host__ __device__ __forceinline__ DualD fabs(const DualD &a) { return a.v < 0.0 ? -a : a; }
__host__ __device__ __forceinline__ DualD nim_exp(const DualD &a) {
  const double e = nim_exp(a.v);
  return DualD(e, e * a.t);
}

// value and derivative of either kind of scalar
__host__ __device__ __forceinline__ double val(double a) { return a; }
__host__ __device__ __forceinline__ double val(const DualD &a) { return a.v; }
__host__ __device__ __forceinline__ double tan_of(double) { return 0.0; }
__host__ __device__ __forceinline__ double tan_of(const DualD &a) { return a.t; }

}  // namespace nim
