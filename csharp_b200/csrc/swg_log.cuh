// Natural logarithm of a binary64, correctly rounded to nearest for the inputs the distance
// epilogues meet, in double-double arithmetic (host and device).
//
// The Kimura2 and JukesCantor distances (Salsa.CoreTPL/Bio/Algorithms/Alignment.cs:254-348) take
// Math.Log of a value and scale the result by 32767 before truncating it to Int16, so a log that is
// one unit in the last place off can change a distance.  .NET's Math.Log is the platform C
// library's log; a correctly rounded result is what any accurate (< 0.5 + tiny ulp) library gives
// except in rounding cases so close to a midpoint that none of those libraries agree either.
//
// Method (Dekker's double-double arithmetic, T. J. Dekker, "A floating-point technique for
// extending the available precision", Numer. Math. 18, 1971; the error-free sum and product of
// Knuth, TAOCP vol. 2, 4.2.2, with the product's low part from a fused multiply-add):
//   x = m * 2^k with m in [sqrt(1/2), sqrt(2))                         (exact)
//   log m = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + ...),  s = (m - 1) / (m + 1), |s| <= 0.1716
//   log x = k ln 2 + log m
// with s, the series (Horner, 25 terms: s^50 / 51 < 2^-128) and the sum carried as unevaluated
// pairs hi + lo of about 106 bits, and the pair rounded to the nearest binary64 at the end.  ln 2
// is the pair (0x3FE62E42FEFA39EF, 0x3C7ABC9E3B39803F).  Every operation is an IEEE binary64
// operation rounded to nearest (the device forms are the _rn intrinsics, which the compiler does
// not contract), so host and device give identical bits.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SWG_LOG_FN __host__ __device__ __forceinline__
#else
#define SWG_LOG_FN inline
#endif

namespace swg {

struct DD {
  double hi, lo;
};

#ifdef __CUDA_ARCH__
SWG_LOG_FN double dd_add_(double a, double b) { return __dadd_rn(a, b); }
SWG_LOG_FN double dd_sub_(double a, double b) { return __dsub_rn(a, b); }
SWG_LOG_FN double dd_mul_(double a, double b) { return __dmul_rn(a, b); }
SWG_LOG_FN double dd_div_(double a, double b) { return __ddiv_rn(a, b); }
SWG_LOG_FN double dd_fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
#else
SWG_LOG_FN double dd_add_(double a, double b) { return a + b; }
SWG_LOG_FN double dd_sub_(double a, double b) { return a - b; }
SWG_LOG_FN double dd_mul_(double a, double b) { return a * b; }
SWG_LOG_FN double dd_div_(double a, double b) { return a / b; }
SWG_LOG_FN double dd_fma_(double a, double b, double c) { return std::fma(a, b, c); }
#endif

// a + b exactly, as a pair (Knuth's branch-free two-sum)
SWG_LOG_FN DD two_sum(double a, double b) {
  const double s = dd_add_(a, b);
  const double bb = dd_sub_(s, a);
  const double err = dd_add_(dd_sub_(a, dd_sub_(s, bb)), dd_sub_(b, bb));
  return DD{s, err};
}

// a + b exactly when |a| >= |b| (Dekker's fast two-sum)
SWG_LOG_FN DD fast_two_sum(double a, double b) {
  const double s = dd_add_(a, b);
  return DD{s, dd_sub_(b, dd_sub_(s, a))};
}

// a * b exactly, as a pair
SWG_LOG_FN DD two_prod(double a, double b) {
  const double p = dd_mul_(a, b);
  return DD{p, dd_fma_(a, b, -p)};
}

SWG_LOG_FN DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo = dd_add_(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = dd_add_(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}

SWG_LOG_FN DD dd_mul(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo = dd_add_(p.lo, dd_add_(dd_mul_(a.hi, b.lo), dd_mul_(a.lo, b.hi)));
  return fast_two_sum(p.hi, p.lo);
}

// a / b: the quotient's leading double, then two corrections from the remainders
SWG_LOG_FN DD dd_div(DD a, DD b) {
  const double q1 = dd_div_(a.hi, b.hi);
  DD p = dd_mul(b, DD{q1, 0.0});
  DD r = dd_add(a, DD{-p.hi, -p.lo});
  const double q2 = dd_div_(r.hi, b.hi);
  p = dd_mul(b, DD{q2, 0.0});
  r = dd_add(r, DD{-p.hi, -p.lo});
  const double q3 = dd_div_(r.hi, b.hi);
  return dd_add(fast_two_sum(q1, q2), DD{q3, 0.0});
}

// log(x) for finite x > 0 (x = 0, negative or non-finite input: the C library's special values)
SWG_LOG_FN double cr_log(double x) {
  if (!(x > 0.0) || !(x < INFINITY)) {
    if (x == 0.0) return -INFINITY;
    if (x != x || x < 0.0) return NAN;
    return x;  // +infinity
  }
  int k = 0;
#ifdef __CUDA_ARCH__
  double m = ::frexp(x, &k);  // x = m * 2^k, m in [0.5, 1)
#else
  double m = std::frexp(x, &k);
#endif
  if (m < 0.70710678118654752440) {
    m = dd_mul_(m, 2.0);  // exact
    k -= 1;
  }
  // s = (m - 1) / (m + 1); m - 1 is exact (Sterbenz), m + 1 as a pair
  const DD num{dd_sub_(m, 1.0), 0.0};
  const DD den = two_sum(m, 1.0);
  const DD s = dd_div(num, den);
  const DD s2 = dd_mul(s, s);
  // sum_{j=0}^{24} s^(2j) / (2j + 1) by Horner, each 1 / (2j + 1) as a pair
  DD t{0.0, 0.0};
  for (int j = 24; j >= 0; j--) {
    const double d = (double)(2 * j + 1);
    const double rh = dd_div_(1.0, d);
    const double rl = dd_div_(dd_fma_(-rh, d, 1.0), d);
    t = dd_add(dd_mul(t, s2), DD{rh, rl});
  }
  DD lm = dd_mul(s, t);
  lm.hi = dd_mul_(lm.hi, 2.0);  // exact
  lm.lo = dd_mul_(lm.lo, 2.0);
  const double kd = (double)k;
  const DD kl = dd_add(two_prod(kd, 0.69314718055994528623), DD{dd_mul_(kd, 2.3190468138462995584e-17), 0.0});
  const DD r = dd_add(kl, lm);
  return dd_add_(r.hi, r.lo);
}

}  // namespace swg
