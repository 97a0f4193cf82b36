// hf_arith.h -- IEEE division and square root without the zero slow path.
//
// On the GPU, double division by a finite nonzero divisor runs ~3.4x slower
// when the numerator is zero (measured: 356 vs 1,214 G div/s on B200), and the
// shallow-water step divides zeros all the time: still water, zero tangential
// velocity, flat stretches in the slope limiter, zero momentum in friction.
// IEEE 754 fixes the result of those cases exactly: +-0 / b is the zero with
// sign(a) xor sign(b), and sqrt(+-0) is +-0. These helpers return that value
// directly and otherwise compute the correctly rounded a / b or sqrt(x), so
// they are bit-identical to `/` and `sqrt` for every input. The division
// itself never sees the zero numerator: it divides 1 / b on those lanes and
// discards the quotient, so predicated code avoids the slow path too. The
// substituted operand goes through an empty asm statement; without it the
// compiler may fold it back into `a` (the quotient is unused on exactly the
// lanes where they differ) and divide the zero after all, which measured
// 96 instead of 28 instructions per division.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define HF_ARITH_HD __host__ __device__ __forceinline__
#else
#define HF_ARITH_HD inline
#endif

namespace hfa {

// Division by a fixed divisor d (a grid spacing) through its reciprocal,
// correctly rounded like a / d (div_recip). Method: y = hi + lo is 1/d to
// ~2^-105 (hi = RN(1/d), lo = RN((1 - d*hi) * hi), the residual being exact);
// q0 = RN(a*hi + RN(a*lo)) is then within one ulp of a/d, so r = a - d*q0 is
// exact in one fma and RN(q0 + r*hi) is RN(a/d) (Markstein's theorem:
// P. Markstein, IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook
// of Floating-Point Arithmetic, "division with an FMA"). It holds without
// underflow or overflow in the intermediates, so it is used only for d with
// an exponent in [-100, 100] (ok) and a with one in [-700, 900]; everything
// else (zeros, subnormals, infinities, NaN, extreme values) takes the IEEE
// division. A default RecipD (ok = false) always divides. make_recip runs
// on the host (kernel arguments) or the device with the same result.
struct RecipD {
  double d = 0.0, hi = 0.0, lo = 0.0;
  bool ok = false;
};
HF_ARITH_HD int biased_exponent(double x) {
#if defined(__CUDA_ARCH__)
  const long long b = __double_as_longlong(x);
#else
  long long b;
  std::memcpy(&b, &x, sizeof b);
#endif
  return (int)((b >> 52) & 0x7ff);
}
HF_ARITH_HD RecipD make_recip(double d) {
  RecipD r;
  r.d = d;
  r.hi = 1.0 / d;
  r.lo = fma(-d, r.hi, 1.0) * r.hi;
  const int e = biased_exponent(d);
  r.ok = d > 0.0 && e >= 1023 - 100 && e <= 1023 + 100;
  return r;
}

#if defined(__CUDA_ARCH__)
HF_ARITH_HD double div_rn(double a, double b) {
  const long long ia = __double_as_longlong(a), ib = __double_as_longlong(b);
  const bool a_zero = (ia << 1) == 0;
  const bool b_regular = ((ib >> 52) & 0x7ff) != 0x7ff && (ib << 1) != 0;
  const bool shortcut = a_zero && b_regular;
  double num = shortcut ? 1.0 : a;
  asm volatile("" : "+d"(num));
  const double q = num / b;
  return shortcut ? __longlong_as_double((ia ^ ib) & (long long)0x8000000000000000ull) : q;
}
// a / b for a divisor known to be > 0 (compared greater than a positive
// threshold, or a positive grid spacing; +inf allowed): then a zero
// numerator's quotient is a itself, and the divisor needs no test.
HF_ARITH_HD double div_rn_pos(double a, double b) {
  const bool a_zero = (__double_as_longlong(a) << 1) == 0;
  double num = a_zero ? 1.0 : a;
  asm volatile("" : "+d"(num));
  const double q = num / b;
  return a_zero ? a : q;
}
HF_ARITH_HD double div_recip(double a, const RecipD& r) {
  const int e = biased_exponent(a);
  if (!r.ok || e < 1023 - 700 || e > 1023 + 900) return div_rn_pos(a, r.d);
  const double q0 = fma(a, r.hi, a * r.lo);
  const double res = fma(-r.d, q0, a);
  return fma(res, r.hi, q0);
}
HF_ARITH_HD double sqrt_rn(double x) {
  const bool zero = (__double_as_longlong(x) << 1) == 0;
  double y = zero ? 1.0 : x;
  asm volatile("" : "+d"(y));
  const double s = sqrt(y);
  return zero ? x : s;
}
// +-0 and finiteness from the bit pattern (integer pipe, not the FP64 pipe).
HF_ARITH_HD bool is_zero(double x) { return (__double_as_longlong(x) << 1) == 0; }
HF_ARITH_HD bool is_finite(double x) {
  return ((__double_as_longlong(x) >> 52) & 0x7ff) != 0x7ff;
}
#else
HF_ARITH_HD double div_rn(double a, double b) { return a / b; }
HF_ARITH_HD double div_rn_pos(double a, double b) { return a / b; }
HF_ARITH_HD double div_recip(double a, const RecipD& r) { return a / r.d; }
HF_ARITH_HD double sqrt_rn(double x) { return std::sqrt(x); }
HF_ARITH_HD bool is_zero(double x) { return x == 0.0; }
HF_ARITH_HD bool is_finite(double x) { return std::isfinite(x); }
#endif

}  // namespace hfa
