// pgmath.h -- pow, exp and log in double-double arithmetic, identical on the
// host (g++, -ffp-contract=off) and the device (nvcc, --fmad=false).
//
// Why: the reference's conservative-to-primitive chain (recovery/scheme_*.h)
// is chaotic in floor-dominated cells -- whether a Newton solve converges in
// 30 iterations flips on one-ulp differences of its inputs -- so the engine
// and the CPU oracle must round every operation identically. Basic IEEE
// operations (+ - * / sqrt) already do; the C library's pow and CUDA's pow
// do not agree with each other. Both sides therefore call these routines.
//
// Method (textbook double-double arithmetic, own implementation):
//   * error-free transforms two_sum (Knuth) and two_prod via fused
//     multiply-add (Dekker's product with an exact fma);
//   * slow path: log x = e ln 2 + 2 atanh(s), s = (m - 1)/(m + 1), m in
//     [1/sqrt2, sqrt2), the atanh series summed to |s|^42 (first nine terms in
//     double-double); exp t = 2^k exp(r), r = (t - k ln 2)/64, Taylor series
//     of exp(r) - 1 to r^12 (first five terms in double-double), then six
//     squarings. Relative error before the final rounding below 2^-95.
//   * fast path of pow (table-driven, pgmath_tables.h): ln m = L_j +
//     log1p(m inv_j - 1) with |m inv_j - 1| < 2^-9.49 (363 intervals of width
//     1/512; the product m inv_j is formed exactly), the high parts summed by
//     exact two-sums and the low parts in double (error < 2^-80.5 +
//     2^-84 |ln x|); exp t = 2^(k/128) exp(r), |r| <= ln2/256, Cody-Waite
//     reduction, r + r^2/2 exact and the series to r^7 in double (relative
//     error < 2^-76.9). Horner steps use explicit fused multiply-adds, which
//     round identically on both sides. The result hi + lo is returned only if
//     every value within the error bound rounds to the same double (Ziv's
//     rounding test); otherwise the slow path decides, so both paths give
//     the same correctly rounded result except within 2^-95 of a rounding
//     boundary.
// tests/test_pgmath.py checks the results against 60-digit decimal
// arithmetic and the C library on many inputs.
#ifndef PANGU_PGMATH_H
#define PANGU_PGMATH_H

#include <cmath>
#include <cstring>

#include "pgmath_tables.h"

#if defined(__CUDACC__)
#define PGM_FN __host__ __device__ __forceinline__
#else
#define PGM_FN inline
#endif

namespace pgm {

struct dd {
  double hi, lo;
};

PGM_FN double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

PGM_FN long long as_bits(double x) {
#if defined(__CUDA_ARCH__)
  return __double_as_longlong(x);
#else
  long long b;
  std::memcpy(&b, &x, sizeof b);
  return b;
#endif
}
PGM_FN double from_bits(long long b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(b);
#else
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
#endif
}

PGM_FN dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
PGM_FN dd quick_two_sum(double a, double b) {  // |a| >= |b| (or a == 0)
  const double s = a + b;
  const double e = b - (s - a);
  return {s, e};
}
PGM_FN dd two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma_(a, b, -p)};
}
PGM_FN dd add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
PGM_FN dd sub(dd a, dd b) { return add(a, dd{-b.hi, -b.lo}); }
PGM_FN dd mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
PGM_FN dd mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}
PGM_FN dd div(dd a, dd b) {
  const double q1 = a.hi / b.hi;
  dd r = sub(a, mul_d(b, q1));
  const double q2 = r.hi / b.hi;
  r = sub(r, mul_d(b, q2));
  const double q3 = r.hi / b.hi;
  const dd q = quick_two_sum(q1, q2);
  return add(q, dd{q3, 0.0});
}

// ln 2 and 1/ln 2
#define PGM_LN2 (::pgm::dd{0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56})
#define PGM_INV_LN2 0x1.71547652b82fep+0

// 1/(2k+1), k = 1..9, as double-double
PGM_FN dd atanh_coef(int k) {
  switch (k) {
    case 1: return {0x1.5555555555555p-2, 0x1.5555555555555p-56};
    case 2: return {0x1.999999999999ap-3, -0x1.999999999999ap-57};
    case 3: return {0x1.2492492492492p-3, 0x1.2492492492492p-57};
    case 4: return {0x1.c71c71c71c71cp-4, 0x1.c71c71c71c71cp-58};
    case 5: return {0x1.745d1745d1746p-4, -0x1.745d1745d1746p-59};
    case 6: return {0x1.3b13b13b13b14p-4, -0x1.3b13b13b13b14p-58};
    case 7: return {0x1.1111111111111p-4, 0x1.1111111111111p-60};
    case 8: return {0x1.e1e1e1e1e1e1ep-5, 0x1.e1e1e1e1e1e1ep-61};
    default: return {0x1.af286bca1af28p-5, 0x1.af286bca1af28p-59};
  }
}

// log x as double-double for finite x > 0.
PGM_FN dd log_dd(double x) {
  int e;
  double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
  if (m < 0.70710678118654752) {
    m *= 2.0;
    e -= 1;
  }
  const double f = m - 1.0;  // exact
  const dd s = div(dd{f, 0.0}, two_sum(m, 1.0));
  const dd s2 = mul(s, s);
  // sum_{k=10}^{20} s2^(k-10) / (2k+1) in double
  double t = 0x1.8f9c18f9c18fap-6;                 // 1/41
  t = 0x1.a41a41a41a41ap-6 + s2.hi * t;           // 1/39
  t = 0x1.bacf914c1bad0p-6 + s2.hi * t;           // 1/37
  t = 0x1.d41d41d41d41dp-6 + s2.hi * t;           // 1/35
  t = 0x1.f07c1f07c1f08p-6 + s2.hi * t;           // 1/33
  t = 0x1.0842108421084p-5 + s2.hi * t;           // 1/31
  t = 0x1.1a7b9611a7b96p-5 + s2.hi * t;           // 1/29
  t = 0x1.2f684bda12f68p-5 + s2.hi * t;           // 1/27
  t = 0x1.47ae147ae147bp-5 + s2.hi * t;           // 1/25
  t = 0x1.642c8590b2164p-5 + s2.hi * t;           // 1/23
  t = 0x1.8618618618618p-5 + s2.hi * t;           // 1/21
  dd acc = {t, 0.0};
  for (int k = 9; k >= 1; --k) acc = add(mul(acc, s2), atanh_coef(k));
  acc = add(mul(acc, s2), dd{1.0, 0.0});
  const dd logm = mul(mul_d(s, 2.0), acc);
  return add(mul_d(PGM_LN2, (double)e), logm);
}

// exp t rounded to double, t a double-double.
PGM_FN double exp_round(dd t) {
  if (t.hi > 709.79) return HUGE_VAL;
  if (t.hi < -745.2) return 0.0;
  const double kd = rint(t.hi * PGM_INV_LN2);
  dd r = sub(t, mul_d(PGM_LN2, kd));
  r.hi *= 0.015625;  // 2^-6, exact
  r.lo *= 0.015625;
  // T6 = sum_{n=6}^{12} r^(n-6)/n! in double
  double tl = 0x1.1eed8eff8d898p-29;              // 1/12!
  tl = 0x1.ae64567f544e4p-26 + r.hi * tl;         // 1/11!
  tl = 0x1.27e4fb7789f5cp-22 + r.hi * tl;         // 1/10!
  tl = 0x1.71de3a556c734p-19 + r.hi * tl;         // 1/9!
  tl = 0x1.a01a01a01a01ap-16 + r.hi * tl;         // 1/8!
  tl = 0x1.a01a01a01a01ap-13 + r.hi * tl;         // 1/7!
  tl = 0x1.6c16c16c16c17p-10 + r.hi * tl;         // 1/6!
  dd acc = {tl, 0.0};
  acc = add(mul(acc, r), dd{0x1.1111111111111p-7, 0x1.1111111111111p-63});  // 1/5!
  acc = add(mul(acc, r), dd{0x1.5555555555555p-5, 0x1.5555555555555p-59});  // 1/4!
  acc = add(mul(acc, r), dd{0x1.5555555555555p-3, 0x1.5555555555555p-57});  // 1/3!
  acc = add(mul(acc, r), dd{0.5, 0.0});
  acc = add(mul(acc, r), dd{1.0, 0.0});
  dd q = mul(acc, r);  // exp(r) - 1
  for (int i = 0; i < 6; ++i) q = add(mul_d(q, 2.0), mul(q, q));  // (1+q)^2 - 1
  const dd E = add(dd{1.0, 0.0}, q);
  return ldexp(E.hi, (int)kd);
}

// Tables of the fast path, readable from host and device code.
static const double kLogTabH[] = PGM_LOG_TABLE_INIT;
static const double kExpTabH[] = PGM_EXP_TABLE_INIT;
#if defined(__CUDACC__)
static __device__ const double kLogTabD[] = PGM_LOG_TABLE_INIT;
static __device__ const double kExpTabD[] = PGM_EXP_TABLE_INIT;
#endif
PGM_FN double log_tab(int i) {
#if defined(__CUDA_ARCH__)
  return __ldg(kLogTabD + i);
#else
  return kLogTabH[i];
#endif
}
PGM_FN double exp_tab(int i) {
#if defined(__CUDA_ARCH__)
  return __ldg(kExpTabD + i);
#else
  return kExpTabH[i];
#endif
}

#if defined(__CUDACC__)
// Brings both tables into this SM's L1 (one 128-byte line per lane and
// step). For kernels where a few threads run long chains of pow calls, each
// of whose table loads would otherwise wait on L2 in turn.
__device__ __forceinline__ void prefetch_tables_l1() {
#if defined(__CUDA_ARCH__)
  const int lane = threadIdx.x & 31;
  const char *lt = reinterpret_cast<const char *>(kLogTabD);
  const char *et = reinterpret_cast<const char *>(kExpTabD);
  for (int o = lane * 128; o < (int)sizeof(kLogTabD); o += 32 * 128)
    asm volatile("prefetch.global.L1 [%0];" ::"l"(lt + o));
  for (int o = lane * 128; o < (int)sizeof(kExpTabD); o += 32 * 128)
    asm volatile("prefetch.global.L1 [%0];" ::"l"(et + o));
#endif
}
#endif

// x = 2^e m for finite x > 0, m in [1/sqrt2, sqrt2), by the bits of x.
PGM_FN double split_exponent(double x, int &e) {
  long long bits = as_bits(x);
  int shift = 0;
  if ((bits >> 52) == 0) {  // subnormal: scale by 2^54 first (exact)
    bits = as_bits(x * 0x1p54);
    shift = 54;
  }
  e = (int)(bits >> 52) - 1023 - shift;
  double m = from_bits((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);  // [1, 2)
  if (m > 1.4142135623730951) {
    m *= 0.5;
    e += 1;
  }
  return m;
}

// ln x = hi + lo for finite x > 0, error below 2^-80.5 + 2^-84 |ln x|.
//   ln x = e ln2 + L + log1p(r), r = m inv - 1 = rh + rl exactly (two_prod),
//   |rh| < 2^-9.49, |rl| <= 2^-53; L = 0 and rl = 0 in the interval centred
//   on 1. log1p(r) = r - r^2/2 + f(r), f(r) = r^3 Q(r) with Q to its r^6 term
//   (truncation below 2^-98); f(rh) carries about five roundings (below
//   2^-80.9 for |f| < 2^-30); f(rh + rl) = f(rh) + rh^2 (1 - rh) rl up to
//   2^-91; -r^2/2 is exact up to 2^-106. The high parts
//   L + rh - rh^2/2 + f + e ln2_hi are summed by exact two-sums, each ordered
//   by binade: |L| lies above every |rh| of its interval where L != 0 (a
//   property of the table), and |e ln2| >= 0.69 > |ln m|. The low parts add to
//   below 2^-51 + 2^-43.5 |ln x|, so their rounding is below 2^-95 |ln x|.
PGM_FN dd log_fast(double x) {
  int e;
  const double m = split_exponent(x, e);
  const int j = (int)((m - PGM_LOG_M0) * 512.0);
  const double inv = log_tab(3 * j);
  const double Lh = log_tab(3 * j + 1), Ll = log_tab(3 * j + 2);
  const double ph = m * inv;
  const double rl = fma_(m, inv, -ph);
  const double rh = ph - 1.0;  // exact (Sterbenz)
  const double sq = rh * rh;
  const double sh = -0.5 * sq;
  const double sl = -0.5 * fma_(rh, rh, -sq) - rh * rl;
  double q = 0x1.c71c71c71c71cp-4;          // 1/9
  q = fma_(rh, q, -0x1.0000000000000p-3);   // -1/8
  q = fma_(rh, q, 0x1.2492492492492p-3);    // 1/7
  q = fma_(rh, q, -0x1.5555555555555p-3);   // -1/6
  q = fma_(rh, q, 0x1.999999999999ap-3);    // 1/5
  q = fma_(rh, q, -0x1.0000000000000p-2);   // -1/4
  q = fma_(rh, q, 0x1.5555555555555p-2);    // 1/3
  const double f = (sq * rh) * q;
  const dd s = quick_two_sum(Lh, rh);
  const dd u = quick_two_sum(s.hi, sh);
  const dd w = quick_two_sum(u.hi, f);
  const dd z = quick_two_sum((double)e * PGM_LN2_HI, w.hi);
  const double lo = ((Ll + rl) + (sl + (sq * rl) * (1.0 - rh))) + (double)e * PGM_LN2_LO +
                    ((s.lo + u.lo) + (w.lo + z.lo));
  return {z.hi, lo};
}

// e^t for t = th + tl (|th| < 700, |tl| <= 2^-33) as hi + lo with the power of
// two k >> 7 still to apply, relative error below 2^-76.9.
//   k = rint(th 128/ln2), r = t - k ln2/128 with |r| <= 2^-8.52: th - k C1 is
//   exact (k C1 has at most 52 bits and lies within a factor of 2 of th, or
//   th - k C1 fits in 53 bits), k C2 - tl has one rounding below 2^-78, and
//   r = rh + rl by an exact two-sum (|rl| <= 2^-62).
//   e^r - 1 = rh + rh^2/2 + rest, rest = rl (1 + rh) + rh^3 P(rh), P to the
//   r^4 term (truncation below 2^-83); rh + rh^2/2 by an exact product and
//   two-sum, rest < 2^-28 in double (below 2^-79).
//   2^(k/128) e^r = Th + Th ph + (Th pl + Tl (1 + ph)): Th + Th ph exact, the
//   rest (below 2^-27) in one fused rounding (below 2^-80).
PGM_FN dd exp_fast(double th, double tl, int &scale) {
  const double kd = rint(th * PGM_INV_LN2_128);
  const int k = (int)kd;
  const double a = th - kd * PGM_LN2_128_C1;
  const double b = fma_(kd, PGM_LN2_128_C2, -tl);
  const dd r = two_sum(a, -b);
  const double rh = r.hi, rl = r.lo - kd * PGM_LN2_128_C3;
  double P = 0x1.a01a01a01a01ap-13;         // 1/7!
  P = fma_(rh, P, 0x1.6c16c16c16c17p-10);   // 1/6!
  P = fma_(rh, P, 0x1.1111111111111p-7);    // 1/5!
  P = fma_(rh, P, 0x1.5555555555555p-5);    // 1/4!
  P = fma_(rh, P, 0x1.5555555555555p-3);    // 1/3!
  const double sq = rh * rh;
  const double rest = (0.5 * fma_(rh, rh, -sq) + fma_(rh, rl, rl)) + (sq * rh) * P;
  const dd p = quick_two_sum(rh, 0.5 * sq);
  const double pl = p.lo + rest;
  const int jj = k & 127;
  scale = k >> 7;  // arithmetic shift: floor(k / 128)
  const double Th = exp_tab(2 * jj), Tl = exp_tab(2 * jj + 1);
  const dd h = two_prod(Th, p.hi);
  const dd v = quick_two_sum(Th, h.hi);
  return {v.hi, fma_(Th, pl, ((h.lo + v.lo) + Tl) + Tl * p.hi)};
}

// x^y for finite x > 0 when the fast path's error bound decides the rounding.
// t = y ln x = th + tl is within |y| 2^-80.4 + |t| 2^-83.9 of y ln x (the
// log's error times |y|, and the product's roundings), and e^t within a
// relative 2^-76.9 of 2^scale (hi + lo); the bound below doubles each term.
// The result is returned only if every value within it rounds to the same
// double (Ziv's rounding test). |th| < 700 keeps the result normal.
PGM_FN bool pow_fast(double x, double y, double &out) {
  const dd l = log_fast(x);
  const double th = l.hi * y;
  if (!(fabs(th) < 700.0)) return false;
  const double tl = fma_(l.hi, y, -th) + l.lo * y;
  int scale;
  const dd v0 = exp_fast(th, tl, scale);
  const dd v = quick_two_sum(v0.hi, v0.lo);
  const double err = v.hi * ((0x1p-76 + fabs(y) * 0x1p-79) + fabs(th) * 0x1p-83);
  const double a = v.hi + (v.lo + err), b = v.hi + (v.lo - err);
  if (a != b) return false;
  out = a * from_bits((long long)(scale + 1023) << 52);  // exact: |scale| <= 1010
  return true;
}

PGM_FN bool is_inf(double x) { return fabs(x) == HUGE_VAL; }
PGM_FN bool sign_bit(double x) { return copysign(1.0, x) < 0.0; }

PGM_FN bool is_odd_integer(double y) {
  if (floor(y) != y) return false;
  if (fabs(y) >= 9007199254740992.0) return false;  // 2^53: even
  return fmod(y, 2.0) != 0.0;
}

PGM_FN double pow(double x, double y) {
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  if (x != x || y != y) return x + y;
  if (is_inf(y)) {
    const double ax = fabs(x);
    if (ax == 1.0) return 1.0;
    if ((ax < 1.0) == (y > 0.0)) return 0.0;
    return HUGE_VAL;
  }
  bool negate = false;
  if (x < 0.0 || (x == 0.0 && sign_bit(x))) {
    if (x != 0.0 && floor(y) != y) return (x - x) / (x - x);  // NaN
    negate = is_odd_integer(y);
    x = -x;
  }
  double r;
  if (x == 0.0) {
    r = y < 0.0 ? HUGE_VAL : 0.0;
  } else if (is_inf(x)) {
    r = y < 0.0 ? 0.0 : HUGE_VAL;
  } else {
    const bool done = pow_fast(x, y, r);
    if (!done) r = exp_round(mul_d(log_dd(x), y));  // slow path
  }
  return negate ? -r : r;
}

PGM_FN double exp(double x) {
  if (x != x) return x;
  if (is_inf(x)) return x > 0.0 ? x : 0.0;
  return exp_round(dd{x, 0.0});
}

PGM_FN double log(double x) {
  if (x != x) return x;
  if (x < 0.0) return (x - x) / (x - x);
  if (x == 0.0) return -HUGE_VAL;
  if (is_inf(x)) return x;
  return log_dd(x).hi;
}

}  // namespace pgm
#endif  // PANGU_PGMATH_H
