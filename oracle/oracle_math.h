/*
 * oracle_math.h - TEST INFRASTRUCTURE (the oracle).  Never linked into the
 * product library.
 *
 * Deterministic FP64 elementary functions for the oracle, written from the
 * textbook methods named below using only IEEE +, -, *, /, sqrt and bit
 * manipulation, so that a device restatement of the same steps compiled
 * without FMA contraction gives bit-identical results:
 *   - natural log: exponent/mantissa split, mantissa folded into
 *     (sqrt(1/2), sqrt(2)], then log(m) = 2*atanh(f), f = (m-1)/(m+1), summed as
 *     the odd power series of atanh (Abramowitz & Stegun 4.1.27 / 4.6.22),
 *     terms up to f^23 (|f| <= 0.1716 so the truncation error is < 1e-19).
 *   - sin / cos of 2*pi*u for u in [0,1): octant reduction u*8 = k + r
 *     (exact), then Taylor series of sin and cos on [0, pi/4] (terms to
 *     t^21 / t^20, truncation error < 1e-20) and the octant symmetries.
 * Philox4x32-10 follows Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11 (multipliers 0xD2511F53 / 0xCD9E8D57, Weyl
 * key increments 0x9E3779B9 / 0xBB67AE85).
 */
#ifndef ORACLE_MATH_H
#define ORACLE_MATH_H

#include <stdint.h>
#include <string.h>

namespace orc {

struct Philox4 {
  uint32_t v[4];
};

static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds. */
static inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                    uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  Philox4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

/* Uniform double on the open interval (0,1) from two 32-bit words:
   k = top 52 bits, u = (k + 0.5) * 2^-52 (exact). */
static inline double u52(uint32_t a, uint32_t b) {
  uint64_t k = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
  return ((double)k + 0.5) * (1.0 / 4503599627370496.0);
}

static inline uint64_t dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static inline double bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* Natural logarithm of a positive normal double. */
static inline double log_pos(double x) {
  const double SQRT2 = 1.4142135623730951;
  const double LN2 = 0.69314718055994531;
  uint64_t b = dbits(x);
  int e = (int)((b >> 52) & 0x7FF) - 1023;
  double m = bitsd((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  if (m > SQRT2) { m = m * 0.5; e = e + 1; }
  double f = (m - 1.0) / (m + 1.0);
  double s = f * f;
  double p = 1.0 / 23.0;
  p = 1.0 / 21.0 + s * p;
  p = 1.0 / 19.0 + s * p;
  p = 1.0 / 17.0 + s * p;
  p = 1.0 / 15.0 + s * p;
  p = 1.0 / 13.0 + s * p;
  p = 1.0 / 11.0 + s * p;
  p = 1.0 / 9.0 + s * p;
  p = 1.0 / 7.0 + s * p;
  p = 1.0 / 5.0 + s * p;
  p = 1.0 / 3.0 + s * p;
  double f2 = f + f;
  double logm = f2 + f2 * (s * p);
  return (double)e * LN2 + logm;
}

/* sin and cos of t for t in [0, pi/4]. */
static inline void sincos_oct(double t, double* s, double* c) {
  double t2 = t * t;
  double ps = 1.0 / 51090942171709440000.0;      /* 1/21! */
  ps = -1.0 / 121645100408832000.0 + t2 * ps;   /* 1/19! */
  ps = 1.0 / 355687428096000.0 + t2 * ps;       /* 1/17! */
  ps = -1.0 / 1307674368000.0 + t2 * ps;        /* 1/15! */
  ps = 1.0 / 6227020800.0 + t2 * ps;            /* 1/13! */
  ps = -1.0 / 39916800.0 + t2 * ps;             /* 1/11! */
  ps = 1.0 / 362880.0 + t2 * ps;                /* 1/9!  */
  ps = -1.0 / 5040.0 + t2 * ps;                 /* 1/7!  */
  ps = 1.0 / 120.0 + t2 * ps;                   /* 1/5!  */
  ps = -1.0 / 6.0 + t2 * ps;                    /* 1/3!  */
  *s = t + t * (t2 * ps);
  double pc = 1.0 / 2432902008176640000.0;      /* 1/20! */
  pc = -1.0 / 6402373705728000.0 + t2 * pc;     /* 1/18! */
  pc = 1.0 / 20922789888000.0 + t2 * pc;        /* 1/16! */
  pc = -1.0 / 87178291200.0 + t2 * pc;          /* 1/14! */
  pc = 1.0 / 479001600.0 + t2 * pc;             /* 1/12! */
  pc = -1.0 / 3628800.0 + t2 * pc;              /* 1/10! */
  pc = 1.0 / 40320.0 + t2 * pc;                 /* 1/8!  */
  pc = -1.0 / 720.0 + t2 * pc;                  /* 1/6!  */
  pc = 1.0 / 24.0 + t2 * pc;                    /* 1/4!  */
  pc = -0.5 + t2 * pc;                          /* 1/2!  */
  *c = 1.0 + t2 * pc;
}

/* sin(2*pi*u), cos(2*pi*u) for u in [0,1). */
static inline void sincos_2pi(double u, double* sn, double* cs) {
  const double PI_4 = 0.78539816339744831;
  double x = u * 8.0;
  int k = (int)x;
  if (k > 7) k = 7;
  double r = x - (double)k;
  double s, c;
  int q;
  if ((k & 1) == 0) {
    sincos_oct(r * PI_4, &s, &c);
    q = (k >> 1) & 3;
    /* angle = q*pi/2 + t */
    switch (q) {
      case 0: *sn = s; *cs = c; break;
      case 1: *sn = c; *cs = -s; break;
      case 2: *sn = -s; *cs = -c; break;
      default: *sn = -c; *cs = s; break;
    }
  } else {
    sincos_oct((1.0 - r) * PI_4, &s, &c);
    q = ((k + 1) >> 1) & 3;
    /* angle = q*pi/2 - t */
    switch (q) {
      case 1: *sn = c; *cs = s; break;
      case 2: *sn = s; *cs = -c; break;
      case 3: *sn = -c; *cs = -s; break;
      default: *sn = -s; *cs = c; break;
    }
  }
}

}  // namespace orc

#endif
