// hf_pow.h -- correctly rounded x^c for the two exponents of the step.
//
// The reference raises to two fixed powers: h.powf(4.0 / 3.0) in Manning
// friction (solver-2d/src/source.rs:161) and (..).powf(3.0 / 5.0) in the
// dry-inflow ghost depth (boundary.rs:209). Neither the platform libm pow
// nor the GPU's pow is correctly rounded (glibc misrounds ~0.1% of these
// calls), and on wet/dry runs a one-ulp difference in friction can flip a
// depth threshold and grow into a visible divergence. These functions
// return the double nearest to x^c (c = the double nearest 4/3 or 3/5)
// except when x^c lies within ~1e-14 ulp of a rounding midpoint, so the GPU
// kernels and the oracle (in its correctly-rounded mode) agree bit for bit.
//
// Method (from the mathematics; double-double arithmetic after Dekker 1971):
//   x^fl(4/3) = x * cbrt(x) * x^-(4/3 - fl(4/3)),  4/3 - fl(4/3) = 2^-52 / 3
//   x^fl(3/5) = (x^3)^(1/5) * x^-(3/5 - fl(3/5)),  3/5 - fl(3/5) = 2^-53 / 5
// The root is one Newton step from a libm guess (error < 4 ulp), evaluated
// with exact products (fma) and a Sterbenz-exact residual, which brings it
// to ~2^-100 relative; the exponent offset enters as the first-order factor
// 1 - eps*ln(x) (|eps*ln x| < 3e-15, so the neglected terms are < 1e-30).
// The final double addition rounds the double-double value once.
#pragma once

#include <cmath>

#include "hf_arith.h"

#if defined(__CUDACC__)
#define HF_POW_HD __host__ __device__ __forceinline__
#else
#define HF_POW_HD inline
#endif

namespace hfpow {

HF_POW_HD void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

// x^fl(4/3) for x > 0; 0 at 0; NaN for x < 0 or NaN; libm pow outside
// [1e-280, 1e280] (no refinement there: cubes would leave the double range).
HF_POW_HD double pow_4_3(double x) {
  if (!(x > 0.0)) return x == 0.0 ? 0.0 : (x - x) / (x - x);
  if (!(x >= 1.0e-280 && x <= 1.0e280)) return pow(x, 4.0 / 3.0);
  const double r0 = cbrt(x);
  double p, e, q, f;
  two_prod(r0, r0, p, e);  // r0^2 = p + e
  two_prod(p, r0, q, f);   // r0^3 = q + f + e*r0
  const double res = (x - q) - (f + e * r0);  // x - q is exact (q ~ x)
  const double corr = hfa::div_rn(res, 3.0 * p);  // Newton: cbrt(x) ~ r0 + corr
  double a_hi, a_lo;
  two_prod(x, r0, a_hi, a_lo);
  a_lo = a_lo + x * corr;
  const double eps = 7.4014868308343765e-17;  // 2^-52 / 3
  a_lo = a_lo - a_hi * (eps * log(x));
  return a_hi + a_lo;
}

// x^fl(3/5) for x > 0; 0 at 0; NaN for x < 0 or NaN; libm pow outside
// [1e-90, 1e90] (x^3 and r^5 must stay in range).
HF_POW_HD double pow_3_5(double x) {
  if (!(x > 0.0)) return x == 0.0 ? 0.0 : (x - x) / (x - x);
  if (!(x >= 1.0e-90 && x <= 1.0e90)) return pow(x, 3.0 / 5.0);
  const double r0 = pow(x, 3.0 / 5.0);
  double p2, e2, p3, e3;
  two_prod(x, x, p2, e2);
  two_prod(p2, x, p3, e3);  // x^3 = p3 + e3 + e2*x
  double s2, f2, s4, f4, s5, f5;
  two_prod(r0, r0, s2, f2);
  two_prod(s2, s2, s4, f4);
  f4 = f4 + 2.0 * s2 * f2;  // r0^4 = s4 + f4
  two_prod(s4, r0, s5, f5);
  f5 = f5 + f4 * r0;        // r0^5 = s5 + f5
  const double res = (p3 - s5) + ((e3 + e2 * x) - f5);  // p3 - s5 is exact
  const double corr = hfa::div_rn(res, 5.0 * s4);        // Newton on r^5 = x^3
  const double eps = 2.2204460492503131e-17;             // 2^-53 / 5
  return r0 + (corr - r0 * (eps * log(x)));
}

}  // namespace hfpow
