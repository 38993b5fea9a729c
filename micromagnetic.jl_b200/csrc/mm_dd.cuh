// mm_dd.cuh -- double-double arithmetic (about 106 significand bits) for the
// one-off Newell demag tensor assembly (internal).
//
// A value is the unevaluated sum hi + lo with |lo| <= ulp(hi)/2.  The
// error-free transformations are Knuth's two-sum and the FMA two-product;
// the sums, products and quotients follow the "accurate" double-double
// algorithms of Hida, Li and Bailey (QD library, 2001) and Shewchuk (1997).
// The transcendental functions are written here from the mathematics:
//   exp   argument reduction by ln 2 and 2^-10, Taylor series of expm1,
//         ten squarings in the expm1 form (s <- 2s + s^2);
//   log   one Newton step x + a exp(-x) - 1 from the double log;
//   atan  reduction to [0, 1] by atan(a) = pi/2 - atan(1/a), five halvings
//         atan(a) = 2 atan(a / (1 + sqrt(1 + a^2))), Taylor series;
//   asinh sign(t) log(|t| + sqrt(t^2 + 1)).
// Each is accurate to a few units of 2^-104 in absolute terms for the
// arguments of the Newell functions (relative for exp, sqrt and the
// reduced atan), which is what the tensor needs: its 27-point differences
// cancel up to R^6 ~ 5e10 (R = 60 cells) of the function values.  The
// constants below were computed to 60 digits (Python decimal: ln 2 from
// Decimal.ln, pi from Machin's formula) and split into hi + lo.
#pragma once
#include <cmath>

namespace mm {
namespace dd {

struct DD {
  double hi, lo;
};

__host__ __device__ inline DD mk(double a) { return DD{a, 0.0}; }

__host__ __device__ inline DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return DD{s, (a - (s - bb)) + (b - bb)};
}
__host__ __device__ inline DD quick_two_sum(double a, double b) {
  const double s = a + b;
  return DD{s, b - (s - a)};
}
__host__ __device__ inline DD two_prod(double a, double b) {
  const double p = a * b;
  return DD{p, fma(a, b, -p)};
}

__host__ __device__ inline DD add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
__host__ __device__ inline DD neg(DD a) { return DD{-a.hi, -a.lo}; }
__host__ __device__ inline DD sub(DD a, DD b) { return add(a, neg(b)); }
__host__ __device__ inline DD add(DD a, double b) {
  DD s = two_sum(a.hi, b);
  s.lo += a.lo;
  return quick_two_sum(s.hi, s.lo);
}

__host__ __device__ inline DD mul(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
__host__ __device__ inline DD mul(DD a, double b) {
  DD p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}
// exact scaling by a power of two
__host__ __device__ inline DD scale2(DD a, double p2) { return DD{a.hi * p2, a.lo * p2}; }

__host__ __device__ inline DD div(DD a, DD b) {
  const double q1 = a.hi / b.hi;
  DD r = sub(a, mul(b, q1));
  const double q2 = r.hi / b.hi;
  r = sub(r, mul(b, q2));
  const double q3 = r.hi / b.hi;
  return add(quick_two_sum(q1, q2), q3);
}
__host__ __device__ inline DD div(DD a, double b) { return div(a, mk(b)); }

__host__ __device__ inline DD sqrt(DD a) {
  if (a.hi <= 0.0) return mk(0.0);
  const double s = ::sqrt(a.hi);
  const DD r = sub(a, two_prod(s, s));
  return quick_two_sum(s, r.hi / (2.0 * s));
}

__host__ __device__ inline bool is_zero(DD a) { return a.hi == 0.0; }
__host__ __device__ inline bool positive(DD a) { return a.hi > 0.0; }
__host__ __device__ inline double to_double(DD a) { return a.hi + a.lo; }

// ln 2 and pi/2 as double-double constants (hi = the nearest double, lo =
// the nearest double to the remainder)
constexpr double kLn2Hi = 6.93147180559945286227e-01, kLn2Lo = 2.31904681384629955842e-17;
constexpr double kPi2Hi = 1.57079632679489655800e+00, kPi2Lo = 6.12323399573676603587e-17;
constexpr double kPiHi = 3.14159265358979311600e+00, kPiLo = 1.22464679914735320717e-16;

__host__ __device__ inline DD exp(DD x) {
  if (x.hi == 0.0) return mk(1.0);
  const double k = ::floor(x.hi / kLn2Hi + 0.5);
  DD r = sub(x, mul(DD{kLn2Hi, kLn2Lo}, k));
  r = scale2(r, 1.0 / 1024.0);
  // expm1(r) = r (1 + r/2 (1 + r/3 (... (1 + r/9))))
  DD u = mk(1.0);
  for (int i = 9; i >= 2; --i) u = add(div(mul(r, u), static_cast<double>(i)), 1.0);
  DD s = mul(r, u);
  for (int i = 0; i < 10; ++i) s = add(scale2(s, 2.0), mul(s, s));  // (1+s)^2 - 1
  const DD e = add(s, 1.0);
  const double p = ::ldexp(1.0, static_cast<int>(k));
  return DD{e.hi * p, e.lo * p};
}

// a > 0
__host__ __device__ inline DD log(DD a) {
  const double x = ::log(a.hi);
  const DD t = mul(a, exp(mk(-x)));
  return add(add(t, -1.0), x);
}

__host__ __device__ inline DD asinh(DD t) {
  if (is_zero(t)) return mk(0.0);
  const bool ng = t.hi < 0.0;
  const DD a = ng ? neg(t) : t;
  const DD v = log(add(a, sqrt(add(mul(a, a), 1.0))));
  return ng ? neg(v) : v;
}

__host__ __device__ inline DD atan(DD t) {
  if (is_zero(t)) return mk(0.0);
  const bool ng = t.hi < 0.0;
  DD a = ng ? neg(t) : t;
  const bool inv = a.hi > 1.0;
  if (inv) a = div(mk(1.0), a);
  for (int i = 0; i < 5; ++i) a = div(a, add(sqrt(add(mul(a, a), 1.0)), 1.0));
  // atan(a) = a (1 - a^2 (1/3 - a^2 (1/5 - ...))), |a| <= tan(pi/128)
  const DD a2 = mul(a, a);
  DD p = div(mk(1.0), 23.0);
  for (int k = 10; k >= 0; --k) p = sub(div(mk(1.0), static_cast<double>(2 * k + 1)), mul(a2, p));
  DD v = scale2(mul(a, p), 32.0);
  if (inv) v = sub(DD{kPi2Hi, kPi2Lo}, v);
  return ng ? neg(v) : v;
}

}  // namespace dd
}  // namespace mm
