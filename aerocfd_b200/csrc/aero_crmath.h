// Correctly rounded exp(x) and pow(x, y) for doubles, for host and device.
//
// The reference evaluates x**y and exp(x) with the platform libm (gfortran:
// glibc), whose results are not specified to the last bit; CUDA's pow and exp
// differ from glibc's in the last bit on a fraction of arguments, and in the
// iterated solver such one-ulp differences grow (the WENO weights amplify
// them).  The FP64 kernels and the CPU oracle therefore both call the
// functions of this header, which compute the result in double-double
// arithmetic (relative error below about 2^-94) and round it once, so they return
// the correctly rounded value (which glibc's pow and exp also return except on
// rare arguments within about 2^-14 ulp of a rounding boundary).  Every step
// is an IEEE-754 operation that rounds correctly (+, -, *, fma; the callers
// are built without contraction of separate multiplies and adds), so the host
// and the device give the same bits for the same arguments.
//
// Method (the textbook table-driven reductions, e.g. J.-M. Muller, Elementary
// Functions, 3rd ed., chapters 5-6; double-double arithmetic after
// T. J. Dekker, Numer. Math. 18 (1971) 224-242):
//  * ln x: x = 2^k m, m in [1, 2); i = the top 8 bits of m's fraction;
//    r = m c_i - 1 exactly (c_i ~ 1/m with 9 significant bits, one fma),
//    |r| < 2^-8; ln x = k ln 2 - ln c_i + ln(1 + r), the last by its Taylor
//    series to r^12 (terms from r^6 on in double, the rest in double-double);
//  * exp z (z double-double): n = nearest integer to 64 z / ln 2,
//    w = z - n ln(2)/64 (|w| < 2^-7), exp z = 2^(n div 64) 2^((n mod 64)/64)
//    exp w, exp w by its Taylor series to w^11 (terms from w^5 on in double);
//  * pow(x, y) = exp(y ln x) for finite x > 0 and finite y with
//    |y ln x| < 708.
// Tables (aero_crmath_tables.h, from gen_crmath_tables.py) hold c_i, -ln c_i,
// 2^(j/64) and the split constants.  Arguments outside the domains above
// (x <= 0, non-finite values, results near overflow or underflow) fall back to
// the platform's pow / exp; the solver's arguments never reach them.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define CRM_FN __host__ __device__ __forceinline__
#else
#define CRM_FN inline
#endif

namespace crm {

// The tables, once for host code and (in CUDA translation units) once in
// device global memory for device code (not constant memory: the threads of
// a warp index different entries, which constant memory would serialise);
// CRM_T(name) picks the copy of the side being compiled.
namespace host_tab {
#define CRM_TABLE static const
#define CRM_CONST static constexpr
#include "aero_crmath_tables.h"
#undef CRM_TABLE
#undef CRM_CONST
}  // namespace host_tab
#if defined(__CUDACC__)
namespace dev_tab {
#define CRM_TABLE static __device__ const
#define CRM_CONST static constexpr
#include "aero_crmath_tables.h"
#undef CRM_TABLE
#undef CRM_CONST
}  // namespace dev_tab
#endif
#if defined(__CUDA_ARCH__)
#define CRM_T(name) dev_tab::name
#else
#define CRM_T(name) host_tab::name
#endif

CRM_FN double crm_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return fma(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
CRM_FN uint64_t bits_of(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  std::memcpy(&u, &x, sizeof u);
  return u;
#endif
}
CRM_FN double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  std::memcpy(&x, &u, sizeof x);
  return x;
#endif
}
CRM_FN double nearest_int(double x) {
#if defined(__CUDA_ARCH__)
  return rint(x);
#else
  return std::nearbyint(x);
#endif
}
CRM_FN double libm_pow(double x, double y) {
#if defined(__CUDA_ARCH__)
  return pow(x, y);
#else
  return std::pow(x, y);
#endif
}
CRM_FN double libm_exp(double x) {
#if defined(__CUDA_ARCH__)
  return exp(x);
#else
  return std::exp(x);
#endif
}

// A double-double value hi + lo, |lo| <= ulp(hi) / 2.
struct dd {
  double hi, lo;
};
CRM_FN dd two_sum(double a, double b) {
  double s = a + b;
  double bp = s - a;
  double ap = s - bp;
  return {s, (a - ap) + (b - bp)};
}
// |a| >= |b| (or a = 0)
CRM_FN dd fast_two_sum(double a, double b) {
  double s = a + b;
  return {s, b - (s - a)};
}
CRM_FN dd two_prod(double a, double b) {
  double p = a * b;
  return {p, crm_fma(a, b, -p)};
}
CRM_FN dd add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  double lo = s.lo + t.hi;
  dd u = fast_two_sum(s.hi, lo);
  lo = t.lo + u.lo;
  return fast_two_sum(u.hi, lo);
}
CRM_FN dd add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  double lo = s.lo + a.lo;
  return fast_two_sum(s.hi, lo);
}
CRM_FN dd mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  double lo = p.lo + (a.hi * b.lo + a.lo * b.hi);
  return fast_two_sum(p.hi, lo);
}
CRM_FN dd mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  double lo = p.lo + a.lo * b;
  return fast_two_sum(p.hi, lo);
}
// a + b where |a.hi| >= |b.hi| (a Horner coefficient plus a much smaller
// product): one fast two-sum instead of two two-sums.
CRM_FN dd add_big(dd a, dd b) {
  dd s = fast_two_sum(a.hi, b.hi);
  double lo = s.lo + (a.lo + b.lo);
  return fast_two_sum(s.hi, lo);
}
CRM_FN dd add_big_d(double a, dd b) {
  dd s = fast_two_sum(a, b.hi);
  double lo = s.lo + b.lo;
  return fast_two_sum(s.hi, lo);
}

// ln x as a double-double, x finite and > 0.
CRM_FN dd log_dd(double x) {
  int k = 0;
  if (x < 0x1p-1022) {  // subnormal: scale into the normal range
    x *= 0x1p64;
    k = -64;
  }
  const uint64_t u = bits_of(x);
  k += (int)(u >> 52) - 1023;
  const int i = (int)((u >> 44) & 255);
  const double m = from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  const double r = crm_fma(m, CRM_T(kLogInv)[i], -1.0);  // exact
  // ln(1 + r) = sum_{n=1..12} (-1)^(n+1) r^n / n, Horner from n = 12: the
  // terms from r^6 on in double (their rounding is below 2^-103 of the
  // result), the rest in double-double; every coefficient outweighs the
  // product added to it (|r| < 2^-8), so each step is a fast two-sum
  double t = -1.0 / 12.0;
  t = t * r + 1.0 / 11.0;
  t = t * r - 1.0 / 10.0;
  t = t * r + 1.0 / 9.0;
  t = t * r - 1.0 / 8.0;
  t = t * r + 1.0 / 7.0;
  t = t * r - 1.0 / 6.0;
  dd a = add_big(dd{CRM_T(kInv5_hi), CRM_T(kInv5_lo)}, two_prod(t, r));
  a = add_big_d(-0.25, mul_d(a, r));
  a = add_big(dd{CRM_T(kInv3_hi), CRM_T(kInv3_lo)}, mul_d(a, r));
  a = add_big_d(-0.5, mul_d(a, r));
  a = add_big_d(1.0, mul_d(a, r));
  const dd lnr = mul_d(a, r);
  // k ln 2 (k * hi exact, k * mid exact as a pair)
  const double kd = (double)k;
  dd kl = two_prod(kd, CRM_T(kLn2_mid));
  kl = add_d(kl, kd * CRM_T(kLn2_lo));
  kl = add_d(kl, kd * CRM_T(kLn2_hi));
  const dd tab{CRM_T(kLogNegLnInv)[i][0], CRM_T(kLogNegLnInv)[i][1]};
  return add(add(kl, tab), lnr);
}

// exp z for a double-double z with |z.hi| < 708, rounded once to double.
CRM_FN double exp_dd_rounded(dd z) {
  const double fn = nearest_int(z.hi * CRM_T(k64OverLn2_hi));
  const int n = (int)fn;
  // w = z - n ln(2)/64: n * hi is exact and z.hi - n * hi is exact (the two
  // are within a factor of two of each other, or n = 0)
  dd w = two_sum(z.hi - fn * CRM_T(kLn2Over64_hi), z.lo);
  const dd nm = two_prod(fn, CRM_T(kLn2Over64_mid));
  w = add(w, dd{-nm.hi, -nm.lo});
  w = add_d(w, -(fn * CRM_T(kLn2Over64_lo)));
  // exp w = sum_{n=0..11} w^n / n!, Horner from n = 11: the terms from w^5 on
  // in double (their rounding is below 2^-97 of the result), the rest in
  // double-double; w's low part matters only in the linear term
  double t = 1.0 / 39916800.0;
  t = t * w.hi + 1.0 / 3628800.0;
  t = t * w.hi + 1.0 / 362880.0;
  t = t * w.hi + 1.0 / 40320.0;
  t = t * w.hi + 1.0 / 5040.0;
  t = t * w.hi + 1.0 / 720.0;
  t = t * w.hi + 1.0 / 120.0;
  dd a = add_big(dd{CRM_T(kInvFact4_hi), CRM_T(kInvFact4_lo)}, two_prod(t, w.hi));
  a = add_big(dd{CRM_T(kInvFact3_hi), CRM_T(kInvFact3_lo)}, mul_d(a, w.hi));
  a = add_big_d(0.5, mul_d(a, w.hi));
  a = add_big_d(1.0, mul_d(a, w.hi));
  a = add_big_d(1.0, mul(a, w));
  const int j = n & 63;
  const int e = (n - j) / 64;  // exact floor division
  const dd r = mul(a, dd{CRM_T(kExp2)[j][0], CRM_T(kExp2)[j][1]});
  // r.hi is r rounded to double; scaling by 2^e is exact in the normal range
  if (e > -1000 && e < 1000) return r.hi * from_bits((uint64_t)(e + 1023) << 52);
  return (r.hi * from_bits((uint64_t)(e / 2 + 1023) << 52)) * from_bits((uint64_t)(e - e / 2 + 1023) << 52);
}

// exp(x), correctly rounded for |x| < 708.
CRM_FN double exp(double x) {
  if (!(x > -708.0 && x < 708.0)) return libm_exp(x);
  if (x == 0.0) return 1.0;
  return exp_dd_rounded(dd{x, 0.0});
}

// x**y, correctly rounded for finite x > 0, finite y and |y ln x| < 708.
CRM_FN double pow(double x, double y) {
  if (!(x > 0.0 && x < INFINITY && y > -INFINITY && y < INFINITY)) return libm_pow(x, y);
  if (y == 0.0 || x == 1.0) return 1.0;
  const dd z = mul_d(log_dd(x), y);
  if (!(z.hi > -708.0 && z.hi < 708.0)) return libm_pow(x, y);
  return exp_dd_rounded(z);
}

}  // namespace crm
