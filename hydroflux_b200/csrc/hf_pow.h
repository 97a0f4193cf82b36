// hf_pow.h -- x^y rounded exactly as the platform C library's pow rounds it.
//
// The reference raises to fixed powers with Rust's f64::powf, which is the C
// library's pow: h.powf(4.0 / 3.0) in Manning friction (solver-2d/src/
// source.rs:161) and (..).powf(3.0 / 5.0) in the dry-inflow ghost depth
// (boundary.rs:209); its forward-mode Dual adds n * x.powf(n - 1)
// (autograd/src/dual.rs:112-117). pow is not correctly rounded (glibc
// misrounds ~0.1% of these calls), and on wetting runs a one-ulp difference in
// friction flips depth thresholds and grows into a visible divergence. So the
// GPU evaluates pow with the algorithm of the host's glibc (>= 2.28, x86-64,
// the build selected on CPUs with FMA), step for step, and gets the same
// double on every input of the domain below.
//
// Method: the table-driven pow of Szabolcs Nagy (ARM optimized-routines,
// 2018; glibc sysdeps/ieee754/dbl-64/e_pow.c since 2.28):
//   1. log x = k ln2 + log c + log1p(z/c - 1) in double-double (hi + lo):
//      x = 2^k z, c from a 128-entry table with 1/c of few bits, so that
//      r = z/c - 1 is exact in one fma; log1p(r) = r - r^2/2 + r^3 q(r)
//      with a degree-6 q (relative error 2^-68).
//   2. y log x = ehi + elo (one exact product in fma).
//   3. exp(ehi + elo) = 2^(k/128) exp(r'): k = round(128 ehi / ln2),
//      r' = ehi - k ln2/128 + elo, 2^(j/128) = H (1 + T) from a 128-entry
//      table, exp(r') - 1 = r' + r'^2 (c2 + c3 r') + r'^4 (c4 + c5 r');
//      result = scale + scale * (T + exp(r') - 1) in one fma.
// The tables are regenerated from their published definitions by
// gen_pow_tables.py (hf_pow_tables.h); the polynomial coefficients and the
// reduction constants are the published ones. Which products are fused
// with the following addition is what the compiler did in glibc's FMA
// build (a product with a single use in an addition is fused); it was
// determined by comparing against the host libm, which this header matches
// bit for bit (oracle mode "port" against "libm", tests/test_oracle_kat.py).
//
// Domain: y finite, not an integer, 2^-65 <= |y| < 2^63 (the step's
// exponents 4/3, 3/5, 1/3 and -2/5 are), any x: x > 0 (normal or subnormal)
// takes the algorithm above incl. its overflow / underflow branches; +-0 and
// +-inf give x*x (y > 0) or 1/(x*x); finite x < 0 and NaN give NaN.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "hf_pow_tables.h"

#if defined(__CUDACC__)
#define HF_POW_HD __host__ __device__ __forceinline__
#else
#define HF_POW_HD inline
#endif

namespace hfpow {

struct LogEntry {
  double invc, logc, ctail;
};
struct ExpEntry {
  double h, t;
};

#if defined(__CUDACC__)
static __device__ const LogEntry kLogTableDev[128] = HF_POW_LOG_TABLE;
static __device__ const ExpEntry kExpTableDev[128] = HF_POW_EXP_TABLE;
#endif
static const LogEntry kLogTableHost[128] = HF_POW_LOG_TABLE;
static const ExpEntry kExpTableHost[128] = HF_POW_EXP_TABLE;

HF_POW_HD const LogEntry& log_entry(int i) {
#if defined(__CUDA_ARCH__)
  return kLogTableDev[i];
#else
  return kLogTableHost[i];
#endif
}
HF_POW_HD const ExpEntry& exp_entry(int j) {
#if defined(__CUDA_ARCH__)
  return kExpTableDev[j];
#else
  return kExpTableHost[j];
#endif
}

HF_POW_HD uint64_t to_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t b;
  std::memcpy(&b, &x, sizeof b);
  return b;
#endif
}
HF_POW_HD double from_bits(uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
#endif
}

// Reduction constants: ln2 = kLn2Hi + kLn2Lo with k * kLn2Hi exact for any
// exponent k; 128/ln2; ln2/128 = kLn2NHi + kLn2NLo; the round-to-integer
// shift 1.5 * 2^52.
constexpr double kLn2Hi = 0x1.62e42fefa3800p-1;
constexpr double kLn2Lo = 0x1.ef35793c76730p-45;
constexpr double kInvLn2N = 0x1.71547652b82fep7;
constexpr double kLn2NHi = 0x1.62e42fefa0000p-8;
constexpr double kLn2NLo = 0x1.cf79abc9e3b3ap-47;
constexpr double kShift = 0x1.8p52;
constexpr uint64_t kLogOff = 0x3fe6955500000000ull;
// log1p(r) - r + r^2/2 = (-r^3/2) * (a1 + a2 r + (-r^2/2) (a3 + a4 r +
// (-r^2/2) (a5 + a6 r))): the published coefficients, pre-scaled by the
// powers of -1/2 the evaluation multiplies in.
constexpr double kA1 = 0x1.555555555556p-2 * -2;
constexpr double kA2 = -0x1.0000000000006p-2 * -2;
constexpr double kA3 = 0x1.999999959554ep-3 * 4;
constexpr double kA4 = -0x1.555555529a47ap-3 * 4;
constexpr double kA5 = 0x1.2495b9b4845e9p-3 * -8;
constexpr double kA6 = -0x1.0002b8b263fc3p-3 * -8;
// exp(r) - 1 - r ~ r^2 (c2 + c3 r) + r^4 (c4 + c5 r) on |r| <= ln2/256.
constexpr double kC2 = 0x1.ffffffffffdbdp-2;
constexpr double kC3 = 0x1.555555555543cp-3;
constexpr double kC4 = 0x1.55555cf172b91p-5;
constexpr double kC5 = 0x1.1111167a4d017p-7;

// log(x) = hi + lo for the bit pattern ix of a positive normal double (a
// subnormal enters with its exponent already lowered by 52).
HF_POW_HD double log_hi_lo(uint64_t ix, double& lo) {
  const uint64_t t = ix - kLogOff;
  const int i = (int)((t >> 45) & 127);
  const double kd = (double)((int64_t)t >> 52);
  const double z = from_bits(ix - (t & (0xfffull << 52)));
  const LogEntry& e = log_entry(i);
  const double r = fma(z, e.invc, -1.0);
  const double t1 = fma(kd, kLn2Hi, e.logc);
  const double t2 = t1 + r;
  const double lo1 = fma(kd, kLn2Lo, e.ctail);
  const double lo2 = t1 - t2 + r;
  const double ar = -0.5 * r;
  const double ar2 = r * ar;
  const double ar3 = r * ar2;
  const double hi = t2 + ar2;
  const double lo3 = fma(ar, r, -ar2);
  const double lo4 = t2 - hi + ar2;
  const double q = fma(ar2, fma(ar2, fma(r, kA6, kA5), fma(r, kA4, kA3)), fma(r, kA2, kA1));
  const double l = fma(ar3, q, lo1 + lo2 + lo3 + lo4);
  const double y = hi + l;
  lo = hi - y + l;
  return y;
}

// exp(x + xt), |xt| tiny against x.
HF_POW_HD double exp_hi_lo(double x, double xt) {
  const uint32_t top = (uint32_t)(to_bits(x) >> 52) & 0x7ff;
  bool wide = false;  // 512 <= |x| < 1024: the scale's exponent needs care
  if (top - 0x3c9u >= 0x408u - 0x3c9u) {
    if (top < 0x3c9u) return 1.0 + x;                        // |x| < 2^-54
    if (top >= 0x409u) return (x < 0.0) ? 0.0 : HUGE_VAL;   // |x| >= 1024
    wide = true;
  }
  double kd = fma(kInvLn2N, x, kShift);
  const uint64_t ki = to_bits(kd);
  kd -= kShift;
  const double r = fma(kd, -kLn2NLo, fma(kd, -kLn2NHi, x)) + xt;
  const int j = (int)(ki & 127);
  const ExpEntry& e = exp_entry(j);
  uint64_t sbits = to_bits(e.h) + ((ki - (uint64_t)j) << 45);  // H * 2^(k div 128)
  const double r2 = r * r;
  const double tmp = fma(r2 * r2, fma(r, kC5, kC4), fma(r2, fma(r, kC3, kC2), e.t + r));
  if (wide) {
    if ((ki & 0x80000000u) == 0) {  // large positive: scale's exponent overflowed
      sbits -= 1009ull << 52;
      const double s = from_bits(sbits);
      return 0x1p1009 * fma(s, tmp, s);
    }
    // large negative: round once in the normal range, then scale down. Here
    // the library's build computes s * tmp once and adds it unfused (the
    // product has two uses).
    sbits += 1022ull << 52;
    const double s = from_bits(sbits);
    const double st = s * tmp;
    double y = s + st;
    if (fabs(y) < 1.0) {
      const double one = y < 0.0 ? -1.0 : 1.0;
      double lo = s - y + st;
      const double hi = one + y;
      lo = one - hi + y + lo;
      y = (hi + lo) - one;
      if (y == 0.0) y = from_bits(sbits & 0x8000000000000000ull);
    }
    return 0x1p-1022 * y;
  }
  const double s = from_bits(sbits);
  return fma(s, tmp, s);
}

// x^y for y in the domain stated at the top.
HF_POW_HD double pow_libm(double x, double y) {
  uint64_t ix = to_bits(x);
  const uint32_t topx = (uint32_t)(ix >> 52);
  if (topx - 1u >= 0x7ffu - 1u) {  // zero, subnormal, negative, inf or NaN
    if (2 * ix - 1 >= 2 * 0x7ff0000000000000ull - 1) {  // +-0, +-inf, NaN
      const double x2 = x * x;
      return y < 0.0 ? 1.0 / x2 : x2;
    }
    if (ix >> 63) return (x - x) / (x - x);  // finite x < 0, y not an integer
    ix = to_bits(x * 0x1p52) & 0x7fffffffffffffffull;  // subnormal: normalize
    ix -= 52ull << 52;
  }
  double lo;
  const double hi = log_hi_lo(ix, lo);
  const double ehi = y * hi;
  const double elo = fma(y, lo, fma(y, hi, -ehi));
  return exp_hi_lo(ehi, elo);
}

// The step's two powers (source.rs:161, boundary.rs:209).
HF_POW_HD double pow_4_3(double x) { return pow_libm(x, 4.0 / 3.0); }
HF_POW_HD double pow_3_5(double x) { return pow_libm(x, 3.0 / 5.0); }

}  // namespace hfpow
