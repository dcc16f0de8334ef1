// Forward-mode dual numbers for the tangent-linear oracle -- TEST
// INFRASTRUCTURE ONLY.
//
// A Dual carries a value v and its derivative t along one direction of the
// inputs (the seeds).  Every operation computes v exactly as the double
// operation would (same operands, same order, one rounding), so a
// tangent-linear oracle run reproduces the FP64 oracle's values bit for bit
// and adds their directional derivatives:
//   (a + b)' = a' + b'          (a b)' = a' b + a b'
//   (a / b)' = (a' - (a/b) b') / b
//   exp(a)'  = exp(a) a'        sqrt(a)' = a' / (2 sqrt(a))
//   |a|'     = sign(a) a'
// Comparisons and branches look at the value only: the derivative is that
// of the branch the values take.
#ifndef NIM_DUAL_H
#define NIM_DUAL_H
#include <cmath>

namespace nimtl {

struct Dual {
  double v = 0.0, t = 0.0;
  Dual() = default;
  Dual(double a) : v(a), t(0.0) {}  // constants and FP64 inputs: zero derivative
  Dual(double a, double b) : v(a), t(b) {}
  Dual &operator+=(const Dual &b) { return *this = Dual(v + b.v, t + b.t); }
  Dual &operator-=(const Dual &b) { return *this = Dual(v - b.v, t - b.t); }
  Dual &operator*=(const Dual &b) { return *this = Dual(v * b.v, t * b.v + v * b.t); }
  Dual &operator/=(const Dual &b) {
    const double q = v / b.v;
    return *this = Dual(q, (t - q * b.t) / b.v);
  }
};

inline Dual operator+(const Dual &a) { return a; }
inline Dual operator-(const Dual &a) { return Dual(-a.v, -a.t); }
inline Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.t + b.t); }
inline Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.t - b.t); }
inline Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.t * b.v + a.v * b.t); }
inline Dual operator/(const Dual &a, const Dual &b) {
  const double q = a.v / b.v;
  return Dual(q, (a.t - q * b.t) / b.v);
}
inline bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
inline bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
inline bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
inline bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
inline bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
inline bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }

inline Dual exp(const Dual &a) {
  const double e = std::exp(a.v);
  return Dual(e, e * a.t);
}
// d sqrt at a zero value with a zero derivative stays zero (the geometry's
// square roots carry no derivative)
inline Dual sqrt(const Dual &a) {
  const double s = std::sqrt(a.v);
  return Dual(s, a.t == 0.0 ? 0.0 : a.t / (2.0 * s));
}
inline Dual fabs(const Dual &a) { return a.v < 0.0 ? -a : a; }
inline bool isfinite(const Dual &a) { return std::isfinite(a.v) && std::isfinite(a.t); }

inline double val(const Dual &a) { return a.v; }
inline double tan_of(const Dual &a) { return a.t; }

}  // namespace nimtl

#endif
