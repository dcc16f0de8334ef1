// exp(x) in FP64 with the same result, bit for bit, as the host's libm.
//
// Why: the NIM coefficients take exp of the cell Peclet number in their
// exponential form (nim.f90:190-194, 375-379), and just above the switch
// |Pe| = v_limit the differences there cancel so strongly that one ulp of
// exp becomes ~1e-7 relative in M_A(.,5).  The reference is gfortran on
// x86-64 glibc, whose exp is the table-driven algorithm of Arm's
// optimized-routines (Szabolcs Nagy, math/exp.c, MIT / Apache-2.0; in glibc
// since 2.28 as sysdeps/ieee754/dbl-64/e_exp.c).  On a CPU with FMA and AVX2
// glibc runs that C source compiled with FMA contraction (the x86-64
// multiarch __exp_fma), so this restatement takes every multiply-add the
// compiler fuses there as one fused operation and keeps the others apart.
// Device code calls CUDA's own __fma_rn for that; host code std::fma.
//
// The algorithm (published):
//   x = k ln2/N + r, N = 128, k integer, |r| <= ln2/(2N)
//   exp(x) = 2^(k/N) exp(r),  2^(k/N) = 2^floor(k/N) * H[k mod N] (1 + T[k mod N])
//   exp(r) - 1 ~ r + C2 r^2 + C3 r^3 + C4 r^4 + C5 r^5 (minimax on |r| <= ln2/256)
// The table holds, for j = 0..N-1, the bits of T[j] (the relative rounding
// error of H[j] = 2^(j/N) rounded to double) and the bits of H[j] with
// j << 45 subtracted, so that adding k << 45 to them puts the exponent of
// 2^floor(k/N) in place.  gen_exp_table.py recomputes it from 2^(j/128) in
// 80-digit decimal arithmetic.  The polynomial coefficients and the split of
// ln2/N into a 37-bit head and its tail are those of the published source.
// Results are bit-identical to glibc 2.39's exp on every double (tests cover
// 1e8 arguments in the NIM range, random bit patterns, the overflow and
// subnormal ranges).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define NIM_EXP_HD __host__ __device__ __forceinline__
#else
#define NIM_EXP_HD inline
#endif

namespace nim {

#define NIM_EXP_TABLE_INIT { \
    0x0000000000000000ULL, 0x3ff0000000000000ULL, 0x3c9b3b4f1a88bf6eULL, 0x3feff63da9fb3335ULL, \
    0xbc7160139cd8dc5dULL, 0x3fefec9a3e778061ULL, 0xbc905e7a108766d1ULL, 0x3fefe315e86e7f85ULL, \
    0x3c8cd2523567f613ULL, 0x3fefd9b0d3158574ULL, 0xbc8bce8023f98efaULL, 0x3fefd06b29ddf6deULL, \
    0x3c60f74e61e6c861ULL, 0x3fefc74518759bc8ULL, 0x3c90a3e45b33d399ULL, 0x3fefbe3ecac6f383ULL, \
    0x3c979aa65d837b6dULL, 0x3fefb5586cf9890fULL, 0x3c8eb51a92fdeffcULL, 0x3fefac922b7247f7ULL, \
    0x3c3ebe3d702f9cd1ULL, 0x3fefa3ec32d3d1a2ULL, 0xbc6a033489906e0bULL, 0x3fef9b66affed31bULL, \
    0xbc9556522a2fbd0eULL, 0x3fef9301d0125b51ULL, 0xbc5080ef8c4eea55ULL, 0x3fef8abdc06c31ccULL, \
    0xbc91c923b9d5f416ULL, 0x3fef829aaea92de0ULL, 0x3c80d3e3e95c55afULL, 0x3fef7a98c8a58e51ULL, \
    0xbc801b15eaa59348ULL, 0x3fef72b83c7d517bULL, 0xbc8f1ff055de323dULL, 0x3fef6af9388c8deaULL, \
    0x3c8b898c3f1353bfULL, 0x3fef635beb6fcb75ULL, 0xbc96d99c7611eb26ULL, 0x3fef5be084045cd4ULL, \
    0x3c9aecf73e3a2f60ULL, 0x3fef54873168b9aaULL, 0xbc8fe782cb86389dULL, 0x3fef4d5022fcd91dULL, \
    0x3c8a6f4144a6c38dULL, 0x3fef463b88628cd6ULL, 0x3c807a05b0e4047dULL, 0x3fef3f49917ddc96ULL, \
    0x3c968efde3a8a894ULL, 0x3fef387a6e756238ULL, 0x3c875e18f274487dULL, 0x3fef31ce4fb2a63fULL, \
    0x3c80472b981fe7f2ULL, 0x3fef2b4565e27cddULL, 0xbc96b87b3f71085eULL, 0x3fef24dfe1f56381ULL, \
    0x3c82f7e16d09ab31ULL, 0x3fef1e9df51fdee1ULL, 0xbc3d219b1a6fbffaULL, 0x3fef187fd0dad990ULL, \
    0x3c8b3782720c0ab4ULL, 0x3fef1285a6e4030bULL, 0x3c6e149289cecb8fULL, 0x3fef0cafa93e2f56ULL, \
    0x3c834d754db0abb6ULL, 0x3fef06fe0a31b715ULL, 0x3c864201e2ac744cULL, 0x3fef0170fc4cd831ULL, \
    0x3c8fdd395dd3f84aULL, 0x3feefc08b26416ffULL, 0xbc86a3803b8e5b04ULL, 0x3feef6c55f929ff1ULL, \
    0xbc924aedcc4b5068ULL, 0x3feef1a7373aa9cbULL, 0xbc9907f81b512d8eULL, 0x3feeecae6d05d866ULL, \
    0xbc71d1e83e9436d2ULL, 0x3feee7db34e59ff7ULL, 0xbc991919b3ce1b15ULL, 0x3feee32dc313a8e5ULL, \
    0x3c859f48a72a4c6dULL, 0x3feedea64c123422ULL, 0xbc9312607a28698aULL, 0x3feeda4504ac801cULL, \
    0xbc58a78f4817895bULL, 0x3feed60a21f72e2aULL, 0xbc7c2c9b67499a1bULL, 0x3feed1f5d950a897ULL, \
    0x3c4363ed60c2ac11ULL, 0x3feece086061892dULL, 0x3c9666093b0664efULL, 0x3feeca41ed1d0057ULL, \
    0x3c6ecce1daa10379ULL, 0x3feec6a2b5c13cd0ULL, 0x3c93ff8e3f0f1230ULL, 0x3feec32af0d7d3deULL, \
    0x3c7690cebb7aafb0ULL, 0x3feebfdad5362a27ULL, 0x3c931dbdeb54e077ULL, 0x3feebcb299fddd0dULL, \
    0xbc8f94340071a38eULL, 0x3feeb9b2769d2ca7ULL, 0xbc87deccdc93a349ULL, 0x3feeb6daa2cf6642ULL, \
    0xbc78dec6bd0f385fULL, 0x3feeb42b569d4f82ULL, 0xbc861246ec7b5cf6ULL, 0x3feeb1a4ca5d920fULL, \
    0x3c93350518fdd78eULL, 0x3feeaf4736b527daULL, 0x3c7b98b72f8a9b05ULL, 0x3feead12d497c7fdULL, \
    0x3c9063e1e21c5409ULL, 0x3feeab07dd485429ULL, 0x3c34c7855019c6eaULL, 0x3feea9268a5946b7ULL, \
    0x3c9432e62b64c035ULL, 0x3feea76f15ad2148ULL, 0xbc8ce44a6199769fULL, 0x3feea5e1b976dc09ULL, \
    0xbc8c33c53bef4da8ULL, 0x3feea47eb03a5585ULL, 0xbc845378892be9aeULL, 0x3feea34634ccc320ULL, \
    0xbc93cedd78565858ULL, 0x3feea23882552225ULL, 0x3c5710aa807e1964ULL, 0x3feea155d44ca973ULL, \
    0xbc93b3efbf5e2228ULL, 0x3feea09e667f3bcdULL, 0xbc6a12ad8734b982ULL, 0x3feea012750bdabfULL, \
    0xbc6367efb86da9eeULL, 0x3fee9fb23c651a2fULL, 0xbc80dc3d54e08851ULL, 0x3fee9f7df9519484ULL, \
    0xbc781f647e5a3ecfULL, 0x3fee9f75e8ec5f74ULL, 0xbc86ee4ac08b7db0ULL, 0x3fee9f9a48a58174ULL, \
    0xbc8619321e55e68aULL, 0x3fee9feb564267c9ULL, 0x3c909ccb5e09d4d3ULL, 0x3feea0694fde5d3fULL, \
    0xbc7b32dcb94da51dULL, 0x3feea11473eb0187ULL, 0x3c94ecfd5467c06bULL, 0x3feea1ed0130c132ULL, \
    0x3c65ebe1abd66c55ULL, 0x3feea2f336cf4e62ULL, 0xbc88a1c52fb3cf42ULL, 0x3feea427543e1a12ULL, \
    0xbc9369b6f13b3734ULL, 0x3feea589994cce13ULL, 0xbc805e843a19ff1eULL, 0x3feea71a4623c7adULL, \
    0xbc94d450d872576eULL, 0x3feea8d99b4492edULL, 0x3c90ad675b0e8a00ULL, 0x3feeaac7d98a6699ULL, \
    0x3c8db72fc1f0eab4ULL, 0x3feeace5422aa0dbULL, 0xbc65b6609cc5e7ffULL, 0x3feeaf3216b5448cULL, \
    0x3c7bf68359f35f44ULL, 0x3feeb1ae99157736ULL, 0xbc93091fa71e3d83ULL, 0x3feeb45b0b91ffc6ULL, \
    0xbc5da9b88b6c1e29ULL, 0x3feeb737b0cdc5e5ULL, 0xbc6c23f97c90b959ULL, 0x3feeba44cbc8520fULL, \
    0xbc92434322f4f9aaULL, 0x3feebd829fde4e50ULL, 0xbc85ca6cd7668e4bULL, 0x3feec0f170ca07baULL, \
    0x3c71affc2b91ce27ULL, 0x3feec49182a3f090ULL, 0x3c6dd235e10a73bbULL, 0x3feec86319e32323ULL, \
    0xbc87c50422622263ULL, 0x3feecc667b5de565ULL, 0x3c8b1c86e3e231d5ULL, 0x3feed09bec4a2d33ULL, \
    0xbc91bbd1d3bcbb15ULL, 0x3feed503b23e255dULL, 0x3c90cc319cee31d2ULL, 0x3feed99e1330b358ULL, \
    0x3c8469846e735ab3ULL, 0x3feede6b5579fdbfULL, 0xbc82dfcd978e9db4ULL, 0x3feee36bbfd3f37aULL, \
    0x3c8c1a7792cb3387ULL, 0x3feee89f995ad3adULL, 0xbc907b8f4ad1d9faULL, 0x3feeee07298db666ULL, \
    0xbc55c3d956dcaebaULL, 0x3feef3a2b84f15fbULL, 0xbc90a40e3da6f640ULL, 0x3feef9728de5593aULL, \
    0xbc68d6f438ad9334ULL, 0x3feeff76f2fb5e47ULL, 0xbc91eee26b588a35ULL, 0x3fef05b030a1064aULL, \
    0x3c74ffd70a5fddcdULL, 0x3fef0c1e904bc1d2ULL, 0xbc91bdfbfa9298acULL, 0x3fef12c25bd71e09ULL, \
    0x3c736eae30af0cb3ULL, 0x3fef199bdd85529cULL, 0x3c8ee3325c9ffd94ULL, 0x3fef20ab5fffd07aULL, \
    0x3c84e08fd10959acULL, 0x3fef27f12e57d14bULL, 0x3c63cdaf384e1a67ULL, 0x3fef2f6d9406e7b5ULL, \
    0x3c676b2c6c921968ULL, 0x3fef3720dcef9069ULL, 0xbc808a1883ccb5d2ULL, 0x3fef3f0b555dc3faULL, \
    0xbc8fad5d3ffffa6fULL, 0x3fef472d4a07897cULL, 0xbc900dae3875a949ULL, 0x3fef4f87080d89f2ULL, \
    0x3c74a385a63d07a7ULL, 0x3fef5818dcfba487ULL, 0xbc82919e2040220fULL, 0x3fef60e316c98398ULL, \
    0x3c8e5a50d5c192acULL, 0x3fef69e603db3285ULL, 0x3c843a59ac016b4bULL, 0x3fef7321f301b460ULL, \
    0xbc82d52107b43e1fULL, 0x3fef7c97337b9b5fULL, 0xbc892ab93b470dc9ULL, 0x3fef864614f5a129ULL, \
    0x3c74b604603a88d3ULL, 0x3fef902ee78b3ff6ULL, 0x3c83c5ec519d7271ULL, 0x3fef9a51fbc74c83ULL, \
    0xbc8ff7128fd391f0ULL, 0x3fefa4afa2a490daULL, 0xbc8dae98e223747dULL, 0x3fefaf482d8e67f1ULL, \
    0x3c8ec3bc41aa2008ULL, 0x3fefba1bee615a27ULL, 0x3c842b94c3a9eb32ULL, 0x3fefc52b376bba97ULL, \
    0x3c8a64a931d185eeULL, 0x3fefd0765b6e4540ULL, 0xbc8e37bae43be3edULL, 0x3fefdbfdad9cbe14ULL, \
    0x3c77893b4d91cd9dULL, 0x3fefe7c1819e90d8ULL, 0x3c5305c14160cc89ULL, 0x3feff3c22b8f71f1ULL \
}

#ifdef __CUDACC__
__device__ const uint64_t kExpTableDev[256] = NIM_EXP_TABLE_INIT;
#endif
static const uint64_t kExpTableHost[256] = NIM_EXP_TABLE_INIT;

namespace expd {
constexpr double kInvLn2N = 0x1.71547652b82fep0 * 128;  // N / ln2
constexpr double kNegLn2HiN = -0x1.62e42fefa0000p-8;    // -ln2/N, head (37 bits)
constexpr double kNegLn2LoN = -0x1.cf79abc9e3b3ap-47;   // -ln2/N, tail
constexpr double kShift = 0x1.8p52;                     // rounds k to an integer
constexpr double kC2 = 0x1.ffffffffffdbdp-2;
constexpr double kC3 = 0x1.555555555543cp-3;
constexpr double kC4 = 0x1.55555cf172b91p-5;
constexpr double kC5 = 0x1.1111167a4d017p-7;

NIM_EXP_HD double fma_(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
NIM_EXP_HD uint64_t bits(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
#endif
}
NIM_EXP_HD double from_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x;
  std::memcpy(&x, &u, 8);
  return x;
#endif
}
NIM_EXP_HD uint64_t table(unsigned i) {
#ifdef __CUDA_ARCH__
  return __ldg(reinterpret_cast<const unsigned long long *>(kExpTableDev) + i);
#else
  return kExpTableHost[i];
#endif
}
}  // namespace expd

// exp(x), bit-identical to glibc's (FMA build) for every double x.
NIM_EXP_HD double nim_exp(double x) {
  using namespace expd;
  // exponent field of |x|: 0x3c9 is 2^-54, 0x408 is 512, 0x409 is 1024
  const uint32_t ex = (uint32_t)(bits(x) >> 52) & 0x7ffu;
  bool wide = false;  // |x| in [512, 1024): the scale needs two factors
  if (ex - 0x3c9u >= 0x408u - 0x3c9u) {
    if (ex - 0x3c9u >= 0x80000000u) return 1.0 + x;  // |x| < 2^-54
    if (ex >= 0x409u) {                              // |x| >= 1024, inf, nan
      if (bits(x) == 0xfff0000000000000ull) return 0.0;
      if (ex >= 0x7ffu) return 1.0 + x;
      return (bits(x) >> 63) ? 0.0 : HUGE_VAL;
    }
    wide = true;
  }
  double kd = fma_(kInvLn2N, x, kShift);
  const uint64_t ki = bits(kd);
  kd -= kShift;
  const double r = fma_(kd, kNegLn2LoN, fma_(kd, kNegLn2HiN, x));
  const unsigned j = 2u * (unsigned)(ki % 128u);
  const double tail = from_bits(table(j));
  uint64_t sbits = table(j + 1) + (ki << 45);
  const double r2 = r * r;
  const double tmp = fma_(r2 * r2, fma_(r, kC5, kC4), fma_(r2, fma_(r, kC3, kC2), tail + r));
  if (wide) {
    if ((ki & 0x80000000u) == 0) {  // k > 0: scale by 2^1009 at the end
      sbits -= 1009ull << 52;
      const double s = from_bits(sbits);
      return 0x1p1009 * fma_(s, tmp, s);
    }
    // k < 0: the result may be subnormal; round once before scaling down
    sbits += 1022ull << 52;
    const double s = from_bits(sbits);
    const double st = s * tmp;  // used twice, so not fused
    double y = s + st;
    if (y < 1.0) {
      double lo = s - y + st;
      const double hi = 1.0 + y;
      lo = 1.0 - hi + y + lo;
      y = (hi + lo) - 1.0;
      if (y == 0.0) y = 0.0;
    }
    return 0x1p-1022 * y;
  }
  const double s = from_bits(sbits);
  return fma_(s, tmp, s);
}

}  // namespace nim
