// hf_device.cuh -- per-face and per-cell device arithmetic of the explicit step.
//
// Every function keeps the operation order of the Rust reference
// (franciscoparrao/hydroflux, solver-2d) so that, compiled with
// --fmad=false and IEEE division / square root, it rounds like the
// reference's f64 code. Citations are file:line in that crate.
#pragma once

#include <cstdint>

#include "hf_arith.h"
#include "hf_internal.h"
#include "hf_pow.h"

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

struct Ghost {
  double h, hu, hv, z;
};

// ghost_cell (boundary.rs:193-219) with ghost_state (274-333) and ghost_bed
// (335-367). `c0` is the boundary cell, `c1` the next cell inward along the
// face normal (only read for Discharge / Depth, which need two cells).
__device__ __forceinline__ Ghost ghost_cell(int side, const BcDev& bc, double h, double hu,
                                            double hv, const double* __restrict__ z,
                                            const double* __restrict__ nman, int64_t c0,
                                            int64_t c1, double d_normal) {
  const int kind = bc.kind[side];
  const double val = bc.val[side];
  const bool xf = side >= SIDE_WEST;
  Ghost g{h, hu, hv, 0.0};
  if (kind == BC_WALL) {
    if (xf) g.hu = -hu; else g.hv = -hv;
  } else if (kind == BC_DISCHARGE) {
    if (xf) g.hu = val; else g.hv = val;
  } else if (kind == BC_DEPTH) {
    g.h = val;
  }
  if (kind == BC_TRANSMISSIVE || kind == BC_WALL) {
    g.z = z[c0];
  } else {
    g.z = z[c0] * 2.0 - z[c1];
  }
  if (kind == BC_DISCHARGE && h < H_DRY) {
    // |bed_slope| along the normal (boundary.rs:241-271); |a-b| is exact in
    // either order, so the side-specific operand order does not matter.
    const double slope_mag = fabs(hfa::div_rn(z[c0] - z[c1], d_normal));
    if (slope_mag > DRY_INFLOW_SLOPE_THRESHOLD) {
      const double h_n = hfpow::pow_3_5(nman[c0] * hfa::div_rn(fabs(val), sqrt(slope_mag)));
      g.h = fmin(h_n, DRY_INFLOW_H_MAX);
    }
  }
  return g;
}

// hllc_normal_flux (riemann.rs:114-204). Only the side that the sampling
// picks has its tangential velocity and star depth evaluated; those are the
// only values the reference's result reads, so the result is identical.
__device__ __forceinline__ void hllc_normal(double h_l, double qn_l, double qt_l, double h_r,
                                            double qn_r, double qt_r, double& o_m, double& o_n,
                                            double& o_t) {
  const bool wl = h_l > DRY_TOL;
  const bool wr = h_r > DRY_TOL;
  if (!wl && !wr) {
    o_m = 0.0; o_n = 0.0; o_t = 0.0;
    return;
  }
  const double cl = wl ? sqrt(h_l * GRAVITY) : 0.0;
  const double cr = wr ? sqrt(h_r * GRAVITY) : 0.0;
  const double un_l = wl ? hfa::div_rn(qn_l, h_l) : 0.0;
  const double un_r = wr ? hfa::div_rn(qn_r, h_r) : 0.0;
  double sl, sr;
  if (wl && wr) {
    sl = fmin(un_l - cl, un_r - cr);
    sr = fmax(un_l + cl, un_r + cr);
  } else if (!wl) {
    sl = un_r - cr * 2.0;
    sr = un_r + cr;
  } else {
    sl = un_l - cl;
    sr = un_l + cl * 2.0;
  }
  bool left, star;
  double s_star = 0.0;
  if (sl >= 0.0) {
    left = true; star = false;
  } else if (sr <= 0.0) {
    left = false; star = false;
  } else {
    const double denom = h_r * (un_r - sr) - h_l * (un_l - sl);
    s_star = fabs(denom) > 1.0e-12
                 ? hfa::div_rn(h_r * (un_r - sr) * sl - h_l * (un_l - sl) * sr, denom)
                 : (sl + sr) * 0.5;
    left = s_star >= 0.0;
    star = true;
  }
  const double h = left ? h_l : h_r;
  const double qn = left ? qn_l : qn_r;
  const double qt = left ? qt_l : qt_r;
  const double un = left ? un_l : un_r;
  const bool wet = left ? wl : wr;
  const double ut = wet ? hfa::div_rn(qt, h) : 0.0;
  double fm = 0.0, fn = 0.0, ft = 0.0;
  if (wet) {
    fm = qn;
    fn = qn * un + h * h * (0.5 * GRAVITY);
    ft = qn * ut;
  }
  if (!star) {
    o_m = fm; o_n = fn; o_t = ft;
    return;
  }
  const double s = left ? sl : sr;
  const double hs = hfa::div_rn(h * (s - un), s - s_star);
  o_m = fm + (hs - h) * s;
  o_n = fn + (hs * s_star - qn) * s;
  o_t = ft + (hs * ut - qt) * s;
}

// well_balanced_x_face / _y_face (update.rs:256-353) with z_left = z_right =
// zf (every call site passes the shared face bed). States are oriented:
// (h, normal momentum, tangential momentum). Outputs: mass, the normal
// momentum flux seen by the minus (left/top) and plus (right/bottom) cell,
// and the tangential momentum flux.
__device__ __forceinline__ void wb_face(double hL, double qnL, double qtL, double hR, double qnR,
                                        double qtR, double zf, double& mass, double& n_minus,
                                        double& n_plus, double& tang) {
  const double z_max = fmax(zf, zf);
  const double hsL = fmax(hL + zf - z_max, 0.0);
  const double hsR = fmax(hR + zf - z_max, 0.0);
  double unL = 0.0, utL = 0.0, unR = 0.0, utR = 0.0;
  if (hL > H_VEL) {
    unL = hfa::div_rn(qnL, hL);
    utL = hfa::div_rn(qtL, hL);
  }
  if (hR > H_VEL) {
    unR = hfa::div_rn(qnR, hR);
    utR = hfa::div_rn(qtR, hR);
  }
  double fm, fn, ft;
  hllc_normal(hsL, hsL * unL, hsL * utL, hsR, hsR * unR, hsR * utR, fm, fn, ft);
  const double corrL = (hL * hL - hsL * hsL) * (0.5 * GRAVITY);
  const double corrR = (hR * hR - hsR * hsR) * (0.5 * GRAVITY);
  mass = fm;
  n_minus = fn + corrL;
  n_plus = fn + corrR;
  tang = ft;
}

// The reference's minmod(dl / d, dr / d) evaluated literally (update.rs:362-370).
__device__ __noinline__ double minmod_literal(double dl, double dr, double d) {
  const double a = hfa::div_rn(dl, d), b = hfa::div_rn(dr, d);
  if (a * b <= 0.0) return 0.0;
  return fabs(a) < fabs(b) ? a : b;
}

// minmod(dl / d, dr / d) with one division. Division by d > 0 keeps the sign
// and the weak order of the numerators, so the operand selected here has the
// quotient the reference returns (when the quotients tie, both are the same
// value). A zero difference makes the reference's product of quotients +-0,
// hence 0. Tiny or infinite operands, where the reference's product of
// quotients could underflow or be NaN, take the literal path out of line.
__device__ __forceinline__ double minmod_div(double dl, double dr, double d) {
  const bool finite = hfa::is_finite(dl) && hfa::is_finite(dr);
  if ((hfa::is_zero(dl) || hfa::is_zero(dr)) && finite) return 0.0;
  if (!finite || fabs(dl) < 1.0e-140 || fabs(dr) < 1.0e-140) return minmod_literal(dl, dr, d);
  if (dl * dr <= 0.0) return 0.0;
  return hfa::div_rn(fabs(dl) < fabs(dr) ? dl : dr, d);
}

// Manning friction on one cell (source.rs:150-164); h^(4/3) correctly rounded.
__device__ __forceinline__ void friction_cell(double h, double& hu, double& hv, double n,
                                              double dt, double dry_tol) {
  if (h <= dry_tol) return;
  if (n == 0.0) return;
  const double dt_g = dt * GRAVITY;
  const double speed = hfa::div_rn(hfa::sqrt_rn(hu * hu + hv * hv), h);
  const double factor = hfa::div_rn(n * n * speed, hfpow::pow_4_3(h)) * dt_g + 1.0;
  hu = hfa::div_rn(hu, factor);
  hv = hfa::div_rn(hv, factor);
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
