// hf_scalar.cuh -- the scalar layer of the device arithmetic: f64 and Dual.
//
// The reference evaluates one generic step for `T: Real` (autograd/src/real.rs)
// with T = f64 for production and T = Dual for forward-mode derivatives. The
// device code is templated the same way: with T = double these helpers are the
// plain IEEE operations; with T = DualD they follow the reference's Dual
// rules (autograd/src/dual.rs): product / quotient rules, Dual-op-f64 forms,
// sqrt with derivative 0 where the root is 0, max / min that average the
// derivatives on a tie, powf's n * x^(n-1) derivative, and branches decided
// on values only (the step never takes abs of a state value outside a
// branch). The value part of a DualD computation equals the f64 one bit for
// bit.
#pragma once

#include "hf_arith.h"
#include "hf_pow.h"

namespace hf {

struct DualD {
  double v;  // value
  double d;  // derivative along the seeded direction
};

__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(DualD x) { return x.v; }

template <class T> __device__ __forceinline__ T cst(double x);
template <> __device__ __forceinline__ double cst<double>(double x) { return x; }
template <> __device__ __forceinline__ DualD cst<DualD>(double x) { return DualD{x, 0.0}; }

// dual.rs:166-230
__device__ __forceinline__ DualD operator+(DualD a, DualD b) { return DualD{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ DualD operator-(DualD a, DualD b) { return DualD{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ DualD operator*(DualD a, DualD b) {
  return DualD{a.v * b.v, a.d * b.v + a.v * b.d};
}
__device__ __forceinline__ DualD operator-(DualD a) { return DualD{-a.v, -a.d}; }
// dual.rs:233-299 (the f64 operand is a constant)
__device__ __forceinline__ DualD operator+(DualD a, double b) { return DualD{a.v + b, a.d}; }
__device__ __forceinline__ DualD operator+(double a, DualD b) { return DualD{a + b.v, b.d}; }
__device__ __forceinline__ DualD operator-(DualD a, double b) { return DualD{a.v - b, a.d}; }
__device__ __forceinline__ DualD operator-(double a, DualD b) { return DualD{a - b.v, -b.d}; }
__device__ __forceinline__ DualD operator*(DualD a, double b) { return DualD{a.v * b, a.d * b}; }
__device__ __forceinline__ DualD operator*(double a, DualD b) { return DualD{a * b.v, a * b.d}; }

// Division (the value part through the zero-safe IEEE division).
__device__ __forceinline__ double dv(double a, double b) { return hfa::div_rn(a, b); }
__device__ __forceinline__ DualD dv(DualD a, DualD b) {
  return DualD{hfa::div_rn(a.v, b.v), hfa::div_rn(a.d * b.v - a.v * b.d, b.v * b.v)};
}
__device__ __forceinline__ DualD dv(DualD a, double b) {
  return DualD{hfa::div_rn(a.v, b), hfa::div_rn(a.d, b)};
}
__device__ __forceinline__ DualD dv(double a, DualD b) {
  return DualD{hfa::div_rn(a, b.v), hfa::div_rn(-a * b.d, b.v * b.v)};
}

// Division by a divisor known to be > 0 (see hfa::div_rn_pos); the
// derivative parts whose divisor is b^2 (which can underflow to 0) keep the
// general division.
__device__ __forceinline__ double dvp(double a, double b) { return hfa::div_rn_pos(a, b); }
__device__ __forceinline__ DualD dvp(DualD a, DualD b) {
  return DualD{hfa::div_rn_pos(a.v, b.v), hfa::div_rn(a.d * b.v - a.v * b.d, b.v * b.v)};
}
__device__ __forceinline__ DualD dvp(DualD a, double b) {
  return DualD{hfa::div_rn_pos(a.v, b), hfa::div_rn_pos(a.d, b)};
}
__device__ __forceinline__ DualD dvp(double a, DualD b) {
  return DualD{hfa::div_rn_pos(a, b.v), hfa::div_rn(-a * b.d, b.v * b.v)};
}

// Two quotients a1 / b and a2 / b by one divisor b > 0: the same correctly
// rounded quotients as dvp. For f64 they share one division: the reciprocal
// of b (hfa::make_recip) and Markstein's correction per numerator
// (hfa::div_recip, which divides outright wherever that does not hold).
// DualD divides each value and tangent as dvp does.
__device__ __forceinline__ void dvp2(double a1, double a2, double b, double& q1, double& q2) {
  const hfa::RecipD r = hfa::make_recip(b);
  q1 = hfa::div_recip(a1, r);
  q2 = hfa::div_recip(a2, r);
}
__device__ __forceinline__ void dvp2(DualD a1, DualD a2, DualD b, DualD& q1, DualD& q2) {
  q1 = dvp(a1, b);
  q2 = dvp(a2, b);
}

// Division by a grid spacing through its precomputed reciprocal (the same
// correctly rounded quotient as dvp; hfa::div_recip).
__device__ __forceinline__ double dvr(double a, const hfa::RecipD& r) {
  return hfa::div_recip(a, r);
}
__device__ __forceinline__ DualD dvr(DualD a, const hfa::RecipD& r) {
  return DualD{hfa::div_recip(a.v, r), hfa::div_recip(a.d, r)};
}

// sqrt (dual.rs:46-50): derivative 0 where the root is 0.
__device__ __forceinline__ double r_sqrt(double x) { return hfa::sqrt_rn(x); }
__device__ __forceinline__ DualD r_sqrt(DualD x) {
  const double s = hfa::sqrt_rn(x.v);
  return DualD{s, s == 0.0 ? 0.0 : hfa::div_rn(x.d, 2.0 * s)};
}

// sqrt of an argument known to be positive (plain IEEE sqrt for double).
__device__ __forceinline__ double r_sqrt_pos(double x) { return sqrt(x); }
__device__ __forceinline__ DualD r_sqrt_pos(DualD x) { return r_sqrt(x); }

// max / min (dual.rs:130-155): ties average the derivatives.
__device__ __forceinline__ double r_max(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double r_min(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ DualD r_max(DualD a, DualD b) {
  if (a.v > b.v) return a;
  if (b.v > a.v) return b;
  return DualD{a.v, 0.5 * (a.d + b.d)};
}
__device__ __forceinline__ DualD r_min(DualD a, DualD b) {
  if (a.v < b.v) return a;
  if (b.v < a.v) return b;
  return DualD{a.v, 0.5 * (a.d + b.d)};
}

// x^fl(4/3), x^fl(3/5) (dual.rs:112-117: dval = n * val^(n-1) * dval), every
// power rounded as the host libm's pow rounds it (hf_pow.h).
__device__ __forceinline__ double r_pow43(double x) { return hfpow::pow_4_3(x); }
__device__ __forceinline__ double r_pow35(double x) { return hfpow::pow_3_5(x); }
__device__ __forceinline__ DualD r_pow43(DualD x) {
  const double n = 4.0 / 3.0;
  return DualD{hfpow::pow_4_3(x.v), n * hfpow::pow_libm(x.v, n - 1.0) * x.d};
}
__device__ __forceinline__ DualD r_pow35(DualD x) {
  const double n = 3.0 / 5.0;
  return DualD{hfpow::pow_3_5(x.v), n * hfpow::pow_libm(x.v, n - 1.0) * x.d};
}

// Loads / stores of a field held as value and (optional) tangent arrays.
template <class T> struct Field;
template <> struct Field<double> {
  __device__ static double ld(const double* v, const double*, int64_t g) { return v[g]; }
  __device__ static void st(double* v, double*, int64_t g, double x) { v[g] = x; }
};
template <> struct Field<DualD> {
  __device__ static DualD ld(const double* v, const double* d, int64_t g) {
    return DualD{v[g], d ? d[g] : 0.0};
  }
  // v == nullptr: a tangent lane other than the first, which leaves the
  // (shared) value arrays to lane 0.
  __device__ static void st(double* v, double* d, int64_t g, DualD x) {
    if (v) v[g] = x.v;
    d[g] = x.d;
  }
};

}  // namespace hf
