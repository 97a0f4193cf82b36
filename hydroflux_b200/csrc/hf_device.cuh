// hf_device.cuh -- per-face and per-cell device arithmetic of the explicit step.
//
// Every function keeps the operation order of the Rust reference
// (franciscoparrao/hydroflux, solver-2d) so that, compiled with
// --fmad=false and IEEE division / square root, it rounds like the
// reference's f64 code. Citations are file:line in that crate.
//
// The state arithmetic is generic over the scalar T (hf_scalar.cuh): double
// for the production step, DualD for the forward-mode tangent, like the
// reference's `T: Real` code. Bed elevations are never differentiated and
// stay double; branches read values only.
#pragma once

#include <cstdint>

#include "hf_arith.h"
#include "hf_internal.h"
#include "hf_pow.h"
#include "hf_scalar.cuh"

namespace hf {

// solver-2d/src/lib.rs:43, 63, 72; riemann.rs:74; boundary.rs:68, 76
constexpr double GRAVITY = 9.81;
constexpr double H_DRY = 1.0e-6;
constexpr double H_VEL = 1.0e-5;
constexpr double DRY_TOL = 1.0e-12;
constexpr double DRY_INFLOW_SLOPE_THRESHOLD = 5.0e-4;
constexpr double DRY_INFLOW_H_MAX = 10.0;

enum { BC_TRANSMISSIVE = 0, BC_WALL = 1, BC_DISCHARGE = 2, BC_DEPTH = 3 };
enum { SIDE_NORTH = 0, SIDE_SOUTH = 1, SIDE_WEST = 2, SIDE_EAST = 3 };

template <class T> struct GhostT {
  T h, hu, hv;
  double z;
};
using Ghost = GhostT<double>;

// ghost_cell (boundary.rs:193-219) with ghost_state (274-333) and ghost_bed
// (335-367). `c0` is the boundary cell, `c1` the next cell inward along the
// face normal (only read for Discharge / Depth, which need two cells). The
// Manning value (and, for DualD, its tangent `dnman`) is read only by the
// dry-inflow Discharge ghost.
template <class T>
__device__ __forceinline__ GhostT<T> ghost_cell(int side, const BcDev& bc, T h, T hu, T hv,
                                                const double* __restrict__ z,
                                                const double* __restrict__ nman,
                                                const double* __restrict__ dnman, int64_t c0,
                                                int64_t c1, double d_normal) {
  const int kind = bc.kind[side];
  const double bval = bc.val[side];
  const bool xf = side >= SIDE_WEST;
  GhostT<T> g{h, hu, hv, 0.0};
  if (kind == BC_WALL) {
    if (xf) g.hu = -hu; else g.hv = -hv;
  } else if (kind == BC_DISCHARGE) {
    if (xf) g.hu = cst<T>(bval); else g.hv = cst<T>(bval);
  } else if (kind == BC_DEPTH) {
    g.h = cst<T>(bval);
  }
  if (kind == BC_TRANSMISSIVE || kind == BC_WALL) {
    g.z = z[c0];
  } else {
    g.z = z[c0] * 2.0 - z[c1];
  }
  if (kind == BC_DISCHARGE && val(h) < H_DRY) {
    // |bed_slope| along the normal (boundary.rs:241-271); |a-b| is exact in
    // either order, so the side-specific operand order does not matter.
    const double slope_mag = fabs(hfa::div_rn(z[c0] - z[c1], d_normal));
    if (slope_mag > DRY_INFLOW_SLOPE_THRESHOLD) {
      const T n0 = Field<T>::ld(nman, dnman, c0);
      const T h_n = r_pow35(n0 * hfa::div_rn(fabs(bval), sqrt(slope_mag)));
      g.h = r_min(h_n, cst<T>(DRY_INFLOW_H_MAX));
    }
  }
  return g;
}

// hllc_normal_flux (riemann.rs:114-204). Only the side that the sampling
// picks has its tangential velocity and star depth evaluated; those are the
// only values the reference's result reads, so the result is identical.
template <class T>
__device__ __forceinline__ void hllc_normal(T h_l, T qn_l, T qt_l, T h_r, T qn_r, T qt_r,
                                            T& o_m, T& o_n, T& o_t) {
  const bool wl = val(h_l) > DRY_TOL;
  const bool wr = val(h_r) > DRY_TOL;
  const T Z = cst<T>(0.0);
  if (!wl && !wr) {
    o_m = Z; o_n = Z; o_t = Z;
    return;
  }
  const T cl = wl ? r_sqrt_pos(h_l * GRAVITY) : Z;
  const T cr = wr ? r_sqrt_pos(h_r * GRAVITY) : Z;
  const T un_l = wl ? dvp(qn_l, h_l) : Z;  // h > DRY_TOL > 0
  const T un_r = wr ? dvp(qn_r, h_r) : Z;
  T sl, sr;
  if (wl && wr) {
    sl = r_min(un_l - cl, un_r - cr);
    sr = r_max(un_l + cl, un_r + cr);
  } else if (!wl) {
    sl = un_r - cr * 2.0;
    sr = un_r + cr;
  } else {
    sl = un_l - cl;
    sr = un_l + cl * 2.0;
  }
  bool left, star;
  T s_star = Z;
  if (val(sl) >= 0.0) {
    left = true; star = false;
  } else if (val(sr) <= 0.0) {
    left = false; star = false;
  } else {
    const T denom = h_r * (un_r - sr) - h_l * (un_l - sl);
    s_star = fabs(val(denom)) > 1.0e-12
                 ? dv(h_r * (un_r - sr) * sl - h_l * (un_l - sl) * sr, denom)
                 : (sl + sr) * 0.5;
    left = val(s_star) >= 0.0;
    star = true;
  }
  const T h = left ? h_l : h_r;
  const T qn = left ? qn_l : qn_r;
  const T qt = left ? qt_l : qt_r;
  const T un = left ? un_l : un_r;
  const bool wet = left ? wl : wr;
  const T ut = wet ? dvp(qt, h) : Z;
  T fm = Z, fn = Z, ft = Z;
  if (wet) {
    fm = qn;
    fn = qn * un + h * h * (0.5 * GRAVITY);
    ft = qn * ut;
  }
  if (!star) {
    o_m = fm; o_n = fn; o_t = ft;
    return;
  }
  const T s = left ? sl : sr;
  const T hs = dv(h * (s - un), s - s_star);
  o_m = fm + (hs - h) * s;
  o_n = fn + (hs * s_star - qn) * s;
  o_t = ft + (hs * ut - qt) * s;
}

// well_balanced_x_face / _y_face (update.rs:256-353) with z_left = z_right =
// zf (every call site passes the shared face bed). States are oriented:
// (h, normal momentum, tangential momentum). Outputs: mass, the normal
// momentum flux seen by the minus (left/top) and plus (right/bottom) cell,
// and the tangential momentum flux.
template <class T>
__device__ __forceinline__ void wb_face(T hL, T qnL, T qtL, T hR, T qnR, T qtR, double zf,
                                        T& mass, T& n_minus, T& n_plus, T& tang) {
  const double z_max = fmax(zf, zf);
  const T Z = cst<T>(0.0);
  const T hsL = r_max(hL + zf - z_max, Z);
  const T hsR = r_max(hR + zf - z_max, Z);
  T unL = Z, utL = Z, unR = Z, utR = Z;
  if (val(hL) > H_VEL) dvp2(qnL, qtL, hL, unL, utL);  // hL > H_VEL
  if (val(hR) > H_VEL) dvp2(qnR, qtR, hR, unR, utR);
  T fm, fn, ft;
  hllc_normal<T>(hsL, hsL * unL, hsL * utL, hsR, hsR * unR, hsR * utR, fm, fn, ft);
  const T corrL = (hL * hL - hsL * hsL) * (0.5 * GRAVITY);
  const T corrR = (hR * hR - hsR * hsR) * (0.5 * GRAVITY);
  mass = fm;
  n_minus = fn + corrL;
  n_plus = fn + corrR;
  tang = ft;
}

// The reference's minmod(dl / d, dr / d) evaluated literally (update.rs:362-370).
template <class T> __device__ __noinline__ T minmod_literal(T dl, T dr, double d) {
  const T a = dvp(dl, d), b = dvp(dr, d);  // d = dx or dy > 0
  if (val(a) * val(b) <= 0.0) return cst<T>(0.0);
  return fabs(val(a)) < fabs(val(b)) ? a : b;
}

// minmod(dl / d, dr / d) with one division. Division by d > 0 keeps the sign
// and the weak order of the numerators, so the operand selected here has the
// quotient the reference returns (when the quotients tie, both are the same
// value). A zero difference makes the reference's product of quotients +-0,
// hence 0. Tiny or infinite operands, where the reference's product of
// quotients could underflow or be NaN, take the literal path out of line.
template <class T> __device__ __forceinline__ T minmod_div(T dl, T dr, const hfa::RecipD& rd) {
  const double l = val(dl), r = val(dr);
  const bool finite = hfa::is_finite(l) && hfa::is_finite(r);
  if ((hfa::is_zero(l) || hfa::is_zero(r)) && finite) return cst<T>(0.0);
  if (!finite || fabs(l) < 1.0e-140 || fabs(r) < 1.0e-140) return minmod_literal<T>(dl, dr, rd.d);
  if (l * r <= 0.0) return cst<T>(0.0);
  return dvr(fabs(l) < fabs(r) ? dl : dr, rd);
}

// Which operand minmod_div(dl, dr, d) returns: -1 for the constant zero, 0
// for dl / d, 1 for dr / d. Same branches as minmod_div / minmod_literal.
__device__ __forceinline__ int minmod_pick(double l, double r, double d) {
  const bool finite = hfa::is_finite(l) && hfa::is_finite(r);
  if ((hfa::is_zero(l) || hfa::is_zero(r)) && finite) return -1;
  if (!finite || fabs(l) < 1.0e-140 || fabs(r) < 1.0e-140) {
    const double a = hfa::div_rn(l, d), b = hfa::div_rn(r, d);
    if (a * b <= 0.0) return -1;
    return fabs(a) < fabs(b) ? 0 : 1;
  }
  if (l * r <= 0.0) return -1;
  return fabs(l) < fabs(r) ? 0 : 1;
}

// Manning friction on one cell (source.rs:150-164); h^(4/3) correctly rounded.
template <class T>
__device__ __forceinline__ void friction_cell(T h, T& hu, T& hv, T n, double dt, double dry_tol) {
  if (val(h) <= dry_tol) return;
  if (val(n) == 0.0) return;
  const double dt_g = dt * GRAVITY;
  const T speed = dv(r_sqrt(hu * hu + hv * hv), h);
  const T factor = dv(n * n * speed, r_pow43(h)) * dt_g + 1.0;
  hu = dv(hu, factor);
  hv = dv(hv, factor);
}

// Piecewise-linear series (same definition as the host forcing descriptor).
__device__ __forceinline__ double series_eval(const double* ts, const double* vs, int n, double t) {
  if (n <= 0) return 0.0;
  if (n == 1 || t <= ts[0]) return vs[0];
  if (t >= ts[n - 1]) return vs[n - 1];
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (ts[mid] <= t) lo = mid; else hi = mid;
  }
  const double w = hfa::div_rn(t - ts[lo], ts[lo + 1] - ts[lo]);
  return vs[lo] + (vs[lo + 1] - vs[lo]) * w;
}

// A series with units: sampled at t / t_div, value (v * v_mul) / v_div, the
// arithmetic of a caller that keeps its hydrograph in minutes and mm/h
// (solver-2d/examples/uk_ea_test8a_official.rs:119-134). The default units
// (1, 1, 1) give series_eval exactly.
__device__ __forceinline__ double series_eval_u(const double* ts, const double* vs, int n,
                                                double t, const SeriesUnits& u) {
  const double v = series_eval(ts, vs, n, hfa::div_rn(t, u.t_div));
  return hfa::div_rn(v * u.v_mul, u.v_div);
}

// Wave speeds of an interior cell for the CFL bound (update.rs:121-135).
__device__ __forceinline__ void cell_speeds(double h, double hu, double hv, double& sx,
                                            double& sy) {
  if (!(h <= H_DRY)) {
    // NaN depth: the reference's `h <= H_DRY` is false and sqrt(NaN) is
    // folded into f64::max, which ignores NaN; fmax does the same.
    const double c = sqrt(GRAVITY * h);
    double u = 0.0, v = 0.0;
    if (h > H_VEL) {
      u = hfa::div_rn(hu, h);
      v = hfa::div_rn(hv, h);
    }
    sx = fmax(sx, fabs(u) + c);
    sy = fmax(sy, fabs(v) + c);
  }
}

// Ghost-cell wave speeds (update.rs:177-188): no H_VEL cutoff there.
__device__ __forceinline__ void ghost_speeds(const Ghost& g, double& sx, double& sy) {
  const double h = g.h;
  if (h <= H_DRY) return;
  const double c = sqrt(GRAVITY * h);
  const double u = hfa::div_rn(g.hu, h);
  const double v = hfa::div_rn(g.hv, h);
  sx = fmax(sx, fabs(u) + c);
  sy = fmax(sy, fabs(v) + c);
}

}  // namespace hf
