/*
 * fp64_math.cuh - deterministic FP64 log and sin/cos(2*pi*u) for the plain
 * FP64 kernel, built from IEEE +, -, *, /, sqrt only (the translation unit is
 * compiled with --fmad=false), so a host restatement of the same steps gives
 * the same bits and FP64 trajectories can be replayed on the CPU.
 *   log: x = m*2^e with m folded into (sqrt(1/2), sqrt(2)]; log m = 2 atanh f,
 *        f = (m-1)/(m+1), odd series to f^23 (Abramowitz & Stegun 4.6.22).
 *   sin/cos(2*pi*u): u*8 = k + r exactly; Taylor series on [0, pi/4]
 *        (sin to t^21, cos to t^20) and the octant symmetries.
 */
#ifndef PTG_FP64_MATH_CUH
#define PTG_FP64_MATH_CUH

namespace ptg {

__device__ __forceinline__ double dlog_pos(double x) {
  const long long b = __double_as_longlong(x);
  int e = (int)((b >> 52) & 0x7FF) - 1023;
  double m = __longlong_as_double((b & 0x000FFFFFFFFFFFFFll) | 0x3FF0000000000000ll);
  if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
  const double f = (m - 1.0) / (m + 1.0);
  const double s = f * f;
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
  const double f2 = f + f;
  return (double)e * 0.69314718055994531 + (f2 + f2 * (s * p));
}

__device__ __forceinline__ void dsincos_oct(double t, double* s, double* c) {
  const double t2 = t * t;
  double ps = 1.0 / 51090942171709440000.0;
  ps = -1.0 / 121645100408832000.0 + t2 * ps;
  ps = 1.0 / 355687428096000.0 + t2 * ps;
  ps = -1.0 / 1307674368000.0 + t2 * ps;
  ps = 1.0 / 6227020800.0 + t2 * ps;
  ps = -1.0 / 39916800.0 + t2 * ps;
  ps = 1.0 / 362880.0 + t2 * ps;
  ps = -1.0 / 5040.0 + t2 * ps;
  ps = 1.0 / 120.0 + t2 * ps;
  ps = -1.0 / 6.0 + t2 * ps;
  *s = t + t * (t2 * ps);
  double pc = 1.0 / 2432902008176640000.0;
  pc = -1.0 / 6402373705728000.0 + t2 * pc;
  pc = 1.0 / 20922789888000.0 + t2 * pc;
  pc = -1.0 / 87178291200.0 + t2 * pc;
  pc = 1.0 / 479001600.0 + t2 * pc;
  pc = -1.0 / 3628800.0 + t2 * pc;
  pc = 1.0 / 40320.0 + t2 * pc;
  pc = -1.0 / 720.0 + t2 * pc;
  pc = 1.0 / 24.0 + t2 * pc;
  pc = -0.5 + t2 * pc;
  *c = 1.0 + t2 * pc;
}

/* sin(2*pi*u), cos(2*pi*u) for u in [0,1). */
__device__ __forceinline__ void dsincos_2pi(double u, double* sn, double* cs) {
  const double x = u * 8.0;
  int k = (int)x;
  if (k > 7) k = 7;
  const double r = x - (double)k;
  double s, c;
  if ((k & 1) == 0) {
    dsincos_oct(r * 0.78539816339744831, &s, &c);
    switch ((k >> 1) & 3) {
      case 0: *sn = s; *cs = c; break;
      case 1: *sn = c; *cs = -s; break;
      case 2: *sn = -s; *cs = -c; break;
      default: *sn = -c; *cs = s; break;
    }
  } else {
    dsincos_oct((1.0 - r) * 0.78539816339744831, &s, &c);
    switch (((k + 1) >> 1) & 3) {
      case 1: *sn = c; *cs = s; break;
      case 2: *sn = s; *cs = -c; break;
      case 3: *sn = -c; *cs = -s; break;
      default: *sn = -s; *cs = c; break;
    }
  }
}

}  // namespace ptg

#endif
