// hf_adjoint_math.cuh -- reverse-mode counterparts of the per-face and
// per-cell functions of hf_device.cuh (host and device).
//
// Each function takes the forward arguments (values), recomputes the
// forward intermediates and branches exactly as the forward code does, and
// maps the adjoint of the outputs to the adjoint of the arguments: the
// transpose of the derivative that the reference's Dual arithmetic
// (autograd/src/dual.rs) propagates through the same code. Values that
// decide a branch are recomputed with the forward's exact operations; values
// that only scale adjoints use one shared reciprocal per denominator (the
// adjoint is a derivative, not a bit-exact quantity). Ties of max/min
// split the adjoint in halves (dual.rs:130-155), sqrt at 0 passes none
// (dual.rs:46-50), powf contributes n x^(n-1) (dual.rs:112-117).
#pragma once

#include <cmath>
#include <cstdint>

#include "hf_arith.h"
#include "hf_device.cuh"
#include "hf_pow.h"

#define HF_ADJ_HD __host__ __device__ __forceinline__

namespace hf {

// d max(x, 0) / dx with the Dual tie rule (dual.rs:130-141).
HF_ADJ_HD double dmax0(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? 0.0 : 0.5); }

// Reverse of hllc_normal: inputs are the forward arguments (values) and the
// adjoint (Lm, Ln, Lt) of the outputs; the adjoint of the six arguments is
// added to the L* references.
HF_ADJ_HD void hllc_normal_rev(double h_l, double qn_l, double qt_l, double h_r,
                                                double qn_r, double qt_r, double Lm, double Ln,
                                                double Lt, double& L_hl, double& L_qnl,
                                                double& L_qtl, double& L_hr, double& L_qnr,
                                                double& L_qtr) {
  const bool wl = h_l > DRY_TOL;
  const bool wr = h_r > DRY_TOL;
  if (!wl && !wr) return;  // constant zero flux
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
  double s_star = 0.0, denom = 0.0;
  if (sl >= 0.0) {
    left = true; star = false;
  } else if (sr <= 0.0) {
    left = false; star = false;
  } else {
    denom = h_r * (un_r - sr) - h_l * (un_l - sl);
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
  const double inv_hl = wl ? 1.0 / h_l : 0.0;
  const double inv_hr = wr ? 1.0 / h_r : 0.0;
  const double inv_h = left ? inv_hl : inv_hr;
  const double ut = wet ? qt * inv_h : 0.0;

  double L_h = 0.0, L_qn = 0.0, L_qt = 0.0, L_un = 0.0, L_ut = 0.0;  // picked side
  double L_sl = 0.0, L_sr = 0.0, L_ss = 0.0;
  if (star) {
    // o = f + (hs - h) s, (hs s* - qn) s, (hs ut - qt) s; hs = h (s - un) / (s - s*)
    const double s = left ? sl : sr;
    const double D = s - s_star;
    const double inv_D = 1.0 / D;
    const double hs = h * (s - un) * inv_D;
    const double L_hs = Lm * s + Ln * s_star * s + Lt * ut * s;
    double L_s = Lm * (hs - h) + Ln * (hs * s_star - qn) + Lt * (hs * ut - qt);
    L_h -= Lm * s;
    L_ss += Ln * hs * s;
    L_qn -= Ln * s;
    L_ut += Lt * hs * s;
    L_qt -= Lt * s;
    const double L_N = L_hs * inv_D;
    const double L_D = -L_hs * hs * inv_D;
    L_h += L_N * (s - un);
    L_s += L_N * h;
    L_un -= L_N * h;
    L_s += L_D;
    L_ss -= L_D;
    if (left) L_sl += L_s; else L_sr += L_s;
  }
  if (wet) {
    // fm = qn, fn = qn un + h^2 g/2, ft = qn ut; ut = qt / h
    L_qn += Lm + Ln * un + Lt * ut;
    L_un += Ln * qn;
    L_h += Ln * (2.0 * h) * (0.5 * GRAVITY);
    L_ut += Lt * qn;
    L_qt += L_ut * inv_h;
    L_h -= L_ut * ut * inv_h;
  }
  double L_unl = 0.0, L_unr = 0.0;
  if (left) {
    L_hl += L_h; L_qnl += L_qn; L_qtl += L_qt; L_unl += L_un;
  } else {
    L_hr += L_h; L_qnr += L_qn; L_qtr += L_qt; L_unr += L_un;
  }
  if (star) {
    if (fabs(denom) > 1.0e-12) {
      // s* = (a1 sl - b1 sr) / (a1 - b1), a1 = h_r (un_r - sr), b1 = h_l (un_l - sl)
      const double a1 = h_r * (un_r - sr), b1 = h_l * (un_l - sl);
      const double inv_den = 1.0 / denom;
      const double L_num = L_ss * inv_den;
      const double L_den = -L_ss * s_star * inv_den;
      const double L_a1 = L_num * sl + L_den;
      const double L_b1 = -L_num * sr - L_den;
      L_sl += L_num * a1;
      L_sr -= L_num * b1;
      L_hr += L_a1 * (un_r - sr);
      L_unr += L_a1 * h_r;
      L_sr -= L_a1 * h_r;
      L_hl += L_b1 * (un_l - sl);
      L_unl += L_b1 * h_l;
      L_sl -= L_b1 * h_l;
    } else {
      L_sl += 0.5 * L_ss;
      L_sr += 0.5 * L_ss;
    }
  }
  double L_cl = 0.0, L_cr = 0.0;
  if (wl && wr) {
    const double a = un_l - cl, b = un_r - cr;
    const double wa = a < b ? 1.0 : (b < a ? 0.0 : 0.5);
    L_unl += L_sl * wa;
    L_cl -= L_sl * wa;
    L_unr += L_sl * (1.0 - wa);
    L_cr -= L_sl * (1.0 - wa);
    const double c1 = un_l + cl, c2 = un_r + cr;
    const double wc = c1 > c2 ? 1.0 : (c2 > c1 ? 0.0 : 0.5);
    L_unl += L_sr * wc;
    L_cl += L_sr * wc;
    L_unr += L_sr * (1.0 - wc);
    L_cr += L_sr * (1.0 - wc);
  } else if (!wl) {
    L_unr += L_sl + L_sr;
    L_cr += L_sr - 2.0 * L_sl;
  } else {
    L_unl += L_sl + L_sr;
    L_cl += 2.0 * L_sr - L_sl;
  }
  if (wl) {  // un_l = qn_l / h_l; cl = sqrt(g h_l), dcl/dh = g / (2 cl) = cl / (2 h_l)
    L_qnl += L_unl * inv_hl;
    L_hl += (L_cl * (0.5 * cl) - L_unl * un_l) * inv_hl;
  }
  if (wr) {
    L_qnr += L_unr * inv_hr;
    L_hr += (L_cr * (0.5 * cr) - L_unr * un_r) * inv_hr;
  }
}

// Reverse of wb_face: adjoint (L_mass, L_nm, L_np, L_t) of the outputs to the
// adjoint of the oriented states (added to the L* references).
HF_ADJ_HD void wb_face_rev(double hL, double qnL, double qtL, double hR,
                                            double qnR, double qtR, double zf, double L_mass,
                                            double L_nm, double L_np, double L_t, double& LhL,
                                            double& LqnL, double& LqtL, double& LhR,
                                            double& LqnR, double& LqtR) {
  const double z_max = fmax(zf, zf);
  const double xL = hL + zf - z_max, xR = hR + zf - z_max;
  const double hsL = fmax(xL, 0.0), hsR = fmax(xR, 0.0);
  double unL = 0.0, utL = 0.0, unR = 0.0, utR = 0.0;
  if (hL > H_VEL) {
    unL = hfa::div_rn(qnL, hL);
    utL = hfa::div_rn(qtL, hL);
  }
  if (hR > H_VEL) {
    unR = hfa::div_rn(qnR, hR);
    utR = hfa::div_rn(qtR, hR);
  }
  // corr = (h^2 - hs^2) g/2 enters n_minus (left) and n_plus (right)
  LhL += L_nm * (2.0 * hL) * (0.5 * GRAVITY);
  LhR += L_np * (2.0 * hR) * (0.5 * GRAVITY);
  double L_hsL = -L_nm * (2.0 * hsL) * (0.5 * GRAVITY);
  double L_hsR = -L_np * (2.0 * hsR) * (0.5 * GRAVITY);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
  hllc_normal_rev(hsL, hsL * unL, hsL * utL, hsR, hsR * unR, hsR * utR, L_mass, L_nm + L_np, L_t,
                  a0, a1, a2, b0, b1, b2);
  L_hsL += a0 + a1 * unL + a2 * utL;
  L_hsR += b0 + b1 * unR + b2 * utR;
  LhL += L_hsL * dmax0(xL);
  LhR += L_hsR * dmax0(xR);
  if (hL > H_VEL) {  // qns = hs * (qn / h)
    const double LunL = a1 * hsL, LutL = a2 * hsL, inv = 1.0 / hL;
    LqnL += LunL * inv;
    LqtL += LutL * inv;
    LhL -= (LunL * unL + LutL * utL) * inv;
  }
  if (hR > H_VEL) {
    const double LunR = b1 * hsR, LutR = b2 * hsR, inv = 1.0 / hR;
    LqnR += LunR * inv;
    LqtR += LutR * inv;
    LhR -= (LunR * unR + LutR * utR) * inv;
  }
}

// Reverse of ghost_cell for the state: the adjoint (LGh, LGn, LGt) of the
// ghost's oriented state goes to the boundary cell's (h, hu, hv) and, for the
// dry-inflow Discharge ghost (whose depth is the Manning normal depth), to
// its Manning value.
HF_ADJ_HD void ghost_rev(int side, const BcDev& bc, double h,
                                          const double* __restrict__ z,
                                          const double* __restrict__ nman, int64_t c0,
                                          int64_t c1, double d_normal, double LGh, double LGn,
                                          double LGt, double& Lh, double& Lhu, double& Lhv,
                                          double& Ln) {
  const int kind = bc.kind[side];
  const double bval = bc.val[side];
  const bool xf = side >= SIDE_WEST;
  const double LGhu = xf ? LGn : LGt, LGhv = xf ? LGt : LGn;
  bool h_from_cell = kind != BC_DEPTH;
  if (kind == BC_DISCHARGE && h < H_DRY) {
    const double slope_mag = fabs(hfa::div_rn(z[c0] - z[c1], d_normal));
    if (slope_mag > DRY_INFLOW_SLOPE_THRESHOLD) {
      h_from_cell = false;
      const double qs = hfa::div_rn(fabs(bval), sqrt(slope_mag));
      const double x = nman[c0] * qs;
      const double h_n = hfpow::pow_3_5(x);
      const double w = h_n < DRY_INFLOW_H_MAX ? 1.0 : (DRY_INFLOW_H_MAX < h_n ? 0.0 : 0.5);
      const double e = 3.0 / 5.0;
      Ln += LGh * w * (e * hfpow::pow_libm(x, e - 1.0)) * qs;
    }
  }
  if (h_from_cell) Lh += LGh;
  if (kind == BC_WALL) {
    if (xf) { Lhu -= LGhu; Lhv += LGhv; } else { Lhu += LGhu; Lhv -= LGhv; }
  } else if (kind == BC_DISCHARGE) {
    if (xf) Lhv += LGhv; else Lhu += LGhu;  // the normal discharge is a constant
  } else {
    Lhu += LGhu;
    Lhv += LGhv;
  }
}

// Reverse of friction_cell on the pre-friction values (h, hu, hv) and n: the
// adjoint (Lhu, Lhv) of the post-friction momentum is replaced by that of the
// pre-friction state; Lh and Ln are added to.
HF_ADJ_HD void friction_rev(double h, double hu, double hv, double n, double dt,
                             double dry_tol, double& Lh, double& Lhu, double& Lhv, double& Ln) {
  if (h <= dry_tol) return;
  if (n == 0.0) return;
  // Forward values (they only scale adjoints): speed = |q| / h,
  // A = n^2 speed / h^(4/3), factor = A dt g + 1, hu' = hu / factor.
  const double dt_g = dt * GRAVITY;
  const double inv_h = 1.0 / h;
  const double S = hfa::sqrt_rn(hu * hu + hv * hv);
  const double speed = S * inv_h;
  // d h^e / dh = e h^(e-1) (dual.rs:112-117) with e = fl(4/3); cbrt(h) is
  // h^(e-1) to within 1e-15 relative (e - 1 = 1/3 - 7.4e-17).
  const double e = 4.0 / 3.0;
  const double q = cbrt(h);
  const double inv_P = 1.0 / (h * q);
  const double A = n * n * speed * inv_P;
  const double inv_f = 1.0 / (A * dt_g + 1.0);
  const double L_factor = -(Lhu * hu + Lhv * hv) * inv_f * inv_f;
  const double nLhu = Lhu * inv_f, nLhv = Lhv * inv_f;
  const double L_A = L_factor * dt_g;
  const double L_N2S = L_A * inv_P;  // adjoint of n n speed
  const double L_P = -L_A * A * inv_P;
  Ln += L_N2S * (2.0 * n) * speed;
  const double L_speed = L_N2S * n * n;
  Lh += L_P * (e * q);
  const double L_S = L_speed * inv_h;
  Lh -= L_speed * speed * inv_h;
  Lhu = nLhu;
  Lhv = nLhv;
  if (S != 0.0) {  // sqrt(0) passes no derivative (dual.rs:46-50)
    const double L_Q = L_S * (0.5 / S);
    Lhu += L_Q * (2.0 * hu);
    Lhv += L_Q * (2.0 * hv);
  }
}

}  // namespace hf
