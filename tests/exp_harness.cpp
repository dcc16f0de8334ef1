// Test harness for nim_exp (nim-conv22-shared_b200/csrc/nim_exp.cuh): the
// host build of the same restatement the kernels use, and the host libm exp
// that the reference's gfortran build calls, side by side.  Built by the
// tests with g++ (no FMA contraction of the harness's own arithmetic).
#include <cmath>
#include <cstdint>

#include "nim_exp.cuh"

namespace {
uint64_t next(uint64_t &s) {
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return s;
}
}  // namespace

extern "C" {

void libm_exp_batch(const double *x, double *y, long n) {
  for (long i = 0; i < n; ++i) y[i] = std::exp(x[i]);
}

void nim_exp_batch(const double *x, double *y, long n) {
  for (long i = 0; i < n; ++i) y[i] = nim::nim_exp(x[i]);
}

// Arguments of kind 0: |x| log-uniform in [lo, hi], both signs; kind 1:
// uniformly random bit patterns (every double, NaN and inf included).
void make_args(double *x, long n, uint64_t seed, int kind, double lo, double hi) {
  uint64_t s = seed | 1;
  const double a = std::log(lo), b = std::log(hi);
  for (long i = 0; i < n; ++i) {
    const uint64_t r = next(s);
    if (kind == 1) {
      x[i] = nim::expd::from_bits(r);
    } else {
      const double u = (double)(r >> 11) * 0x1.0p-53;
      x[i] = ((r & 1) ? -1.0 : 1.0) * std::exp(a + u * (b - a));
    }
  }
}

// Number of arguments (generated as make_args) where nim_exp and libm's exp
// differ in any bit (two NaNs count as equal).
long count_mismatch(long n, uint64_t seed, int kind, double lo, double hi) {
  uint64_t s = seed | 1;
  const double a = std::log(lo), b = std::log(hi);
  long bad = 0;
  for (long i = 0; i < n; ++i) {
    const uint64_t r = next(s);
    double x;
    if (kind == 1) {
      x = nim::expd::from_bits(r);
    } else {
      const double u = (double)(r >> 11) * 0x1.0p-53;
      x = ((r & 1) ? -1.0 : 1.0) * std::exp(a + u * (b - a));
    }
    const double p = nim::nim_exp(x), q = std::exp(x);
    if (nim::expd::bits(p) != nim::expd::bits(q) && !(std::isnan(p) && std::isnan(q))) ++bad;
  }
  return bad;
}
}
