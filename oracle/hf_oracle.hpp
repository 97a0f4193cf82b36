// hf_oracle.hpp -- CPU restatement of hydroflux solver-2d's explicit step.
//
// TEST INFRASTRUCTURE ONLY. This header is the parity oracle for the
// B200 kernels: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it, and only as the checker (or as the timed
// CPU reference arm). The product path never calls it.
//
// It restates, pass by pass and in the same operation order, the Rust
// reference (franciscoparrao/hydroflux):
//   solver-2d/src/update.rs   (CFL, MUSCL slopes, face beds, Audusse+HLLC
//                              faces, alpha rescale, FV update, SSP-RK2)
//   solver-2d/src/riemann.rs  (HLLC normal flux)
//   solver-2d/src/boundary.rs (ghost cells)
//   solver-2d/src/source.rs   (Manning friction, rain, point sources)
//   solver-2d/src/sim.rs      (Simulation::step / run_until)
//   autograd/src/dual.rs      (forward-mode Dual arithmetic rules)
// It is templated on the scalar like the reference's `T: Real`, so the
// same code runs with T = double and T = Dual (tangent mode).
//
// Compile with -ffp-contract=off: Rust never contracts a*b+c into an FMA,
// and every op here must round exactly like the reference's.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

// Correctly rounded x^fl(4/3) and x^fl(3/5) (shared with the GPU kernels).
#include "../hydroflux_b200/csrc/hf_pow.h"

namespace hfo {

// solver-2d/src/lib.rs:43, 63, 72
constexpr double GRAVITY = 9.81;
constexpr double H_DRY = 1.0e-6;
constexpr double H_VEL = 1.0e-5;
// solver-2d/src/riemann.rs:74
constexpr double DRY_TOL = 1.0e-12;
// solver-2d/src/boundary.rs:68, 76
constexpr double DRY_INFLOW_SLOPE_THRESHOLD = 5.0e-4;
constexpr double DRY_INFLOW_H_MAX = 10.0;

// ---------------------------------------------------------------------------
// Scalar layer: autograd/src/real.rs:73-113 (f64) and autograd/src/dual.rs
// ---------------------------------------------------------------------------
inline double value(double x) { return x; }
inline double r_sqrt(double x) { return std::sqrt(x); }
inline double r_abs(double x) { return std::fabs(x); }
inline double r_max(double a, double b) { return std::fmax(a, b); }
inline double r_min(double a, double b) { return std::fmin(a, b); }
// pow mode: 0 = the platform libm (what the Rust reference's f64::powf
// calls); 1 = the restatement of that libm's algorithm in hf_pow.h, which
// the GPU kernels run. The two agree bit for bit on this host (pinned by
// tests/test_oracle_kat.py); mode 1 lets a test show it on whole runs.
inline int& pow_mode() {
  static int mode = 0;
  return mode;
}
inline double r_powf(double a, double n) {
  return pow_mode() == 1 ? hfpow::pow_libm(a, n) : std::pow(a, n);
}

template <class T> struct Scalar;
template <> struct Scalar<double> {
  static double zero() { return 0.0; }
  static double one() { return 1.0; }
  static double from_f64(double x) { return x; }
};

// Dual number val + dval*eps (autograd/src/dual.rs:12-18). No implicit
// conversion from double: mixed expressions use the Dual-op-f64 overloads
// (dual.rs:233-299), which is what the reference's generic code calls.
struct Dual {
  double val;
  double dval;
};
inline double value(Dual x) { return x.val; }
template <> struct Scalar<Dual> {
  static Dual zero() { return Dual{0.0, 0.0}; }
  static Dual one() { return Dual{1.0, 0.0}; }
  static Dual from_f64(double x) { return Dual{x, 0.0}; }
};
// dual.rs:166-230
inline Dual operator+(Dual a, Dual b) { return Dual{a.val + b.val, a.dval + b.dval}; }
inline Dual operator-(Dual a, Dual b) { return Dual{a.val - b.val, a.dval - b.dval}; }
inline Dual operator*(Dual a, Dual b) {
  return Dual{a.val * b.val, a.dval * b.val + a.val * b.dval};
}
inline Dual operator/(Dual a, Dual b) {
  return Dual{a.val / b.val, (a.dval * b.val - a.val * b.dval) / (b.val * b.val)};
}
inline Dual operator-(Dual a) { return Dual{-a.val, -a.dval}; }
// dual.rs:233-299
inline Dual operator+(Dual a, double b) { return Dual{a.val + b, a.dval}; }
inline Dual operator+(double a, Dual b) { return Dual{a + b.val, b.dval}; }
inline Dual operator-(Dual a, double b) { return Dual{a.val - b, a.dval}; }
inline Dual operator-(double a, Dual b) { return Dual{a - b.val, -b.dval}; }
inline Dual operator*(Dual a, double b) { return Dual{a.val * b, a.dval * b}; }
inline Dual operator*(double a, Dual b) { return Dual{a * b.val, a * b.dval}; }
inline Dual operator/(Dual a, double b) { return Dual{a.val / b, a.dval / b}; }
inline Dual operator/(double a, Dual b) {
  return Dual{a / b.val, -a * b.dval / (b.val * b.val)};
}
// dual.rs:46-50: derivative 0 where sqrt is 0.
inline Dual r_sqrt(Dual x) {
  double s = std::sqrt(x.val);
  double d = (s == 0.0) ? 0.0 : x.dval / (2.0 * s);
  return Dual{s, d};
}
// dual.rs:88-101
inline Dual r_abs(Dual x) {
  double sign = x.val > 0.0 ? 1.0 : (x.val < 0.0 ? -1.0 : 0.0);
  return Dual{std::fabs(x.val), x.dval * sign};
}
// dual.rs:112-117: dval = n * val^(n-1) * dval
inline Dual r_powf(Dual x, double n) {
  return Dual{r_powf(x.val, n), n * r_powf(x.val, n - 1.0) * x.dval};
}
// dual.rs:130-141: ties average the derivatives.
inline Dual r_max(Dual a, Dual b) {
  if (a.val > b.val) return a;
  if (b.val > a.val) return b;
  return Dual{a.val, 0.5 * (a.dval + b.dval)};
}
// dual.rs:144-155
inline Dual r_min(Dual a, Dual b) {
  if (a.val < b.val) return a;
  if (b.val < a.val) return b;
  return Dual{a.val, 0.5 * (a.dval + b.dval)};
}

// ---------------------------------------------------------------------------
// Types: state.rs:21, geometry.rs:31, flux.rs:28-47, boundary.rs:80-160
// ---------------------------------------------------------------------------
template <class T> struct Cons {
  T h, hu, hv;
};
template <class T> inline Cons<T> cons_dry() {
  return Cons<T>{Scalar<T>::zero(), Scalar<T>::zero(), Scalar<T>::zero()};
}

template <class T> struct Mesh {
  int64_t nr = 0, nc = 0;
  double dx = 1.0, dy = 1.0;
  std::vector<T> bed;      // (nr, nc) row-major; i along y, j along x
  std::vector<T> manning;  // same shape
  const T& z(int64_t i, int64_t j) const { return bed[i * nc + j]; }
  const T& n(int64_t i, int64_t j) const { return manning[i * nc + j]; }
  // geometry.rs:133, 142
  T bed_slope_x(int64_t i, int64_t j) const { return (z(i, j) - z(i, j + 1)) / dx; }
  T bed_slope_y(int64_t i, int64_t j) const { return (z(i, j) - z(i + 1, j)) / dy; }
};

enum BcKind { BC_TRANSMISSIVE = 0, BC_WALL = 1, BC_DISCHARGE = 2, BC_DEPTH = 3 };
struct Boundary {
  int kind;
  double value;  // q for Discharge, h for Depth
};
struct Boundaries {
  Boundary north, south, west, east;  // boundary.rs:131-140 field order
};
enum Side { NORTH = 0, SOUTH = 1, WEST = 2, EAST = 3 };
inline bool is_x_face(Side s) { return s == WEST || s == EAST; }

template <class T> struct Flux {
  T mass, xm, ym;  // FluxXG/FluxYG {mass, x_momentum, y_momentum}
};
template <class T> inline Flux<T> flux_zero() {
  return Flux<T>{Scalar<T>::zero(), Scalar<T>::zero(), Scalar<T>::zero()};
}
template <class T> struct Face {
  Flux<T> minus, plus;  // FaceFluxXG / FaceFluxYG (update.rs:216-250)
};

// ---------------------------------------------------------------------------
// Boundary ghosts: boundary.rs:193-367
// ---------------------------------------------------------------------------
template <class T>
Cons<T> ghost_state(Cons<T> inner, Boundary b, Side side) {  // boundary.rs:274
  switch (b.kind) {
    case BC_WALL:
      if (is_x_face(side)) return Cons<T>{inner.h, -inner.hu, inner.hv};
      return Cons<T>{inner.h, inner.hu, -inner.hv};
    case BC_DISCHARGE:
      if (is_x_face(side)) return Cons<T>{inner.h, Scalar<T>::from_f64(b.value), inner.hv};
      return Cons<T>{inner.h, inner.hu, Scalar<T>::from_f64(b.value)};
    case BC_DEPTH:
      return Cons<T>{Scalar<T>::from_f64(b.value), inner.hu, inner.hv};
    default:
      return inner;
  }
}

template <class T>
T ghost_bed(const Mesh<T>& m, Boundary b, Side side, int64_t idx) {  // boundary.rs:335
  const int64_t nr = m.nr, nc = m.nc;
  if (b.kind == BC_TRANSMISSIVE || b.kind == BC_WALL) {
    switch (side) {
      case NORTH: return m.z(0, idx);
      case SOUTH: return m.z(nr - 1, idx);
      case WEST: return m.z(idx, 0);
      default: return m.z(idx, nc - 1);
    }
  }
  switch (side) {  // linear extrapolation (needs >= 2 cells along the normal)
    case NORTH: return m.z(0, idx) * 2.0 - m.z(1, idx);
    case SOUTH: return m.z(nr - 1, idx) * 2.0 - m.z(nr - 2, idx);
    case WEST: return m.z(idx, 0) * 2.0 - m.z(idx, 1);
    default: return m.z(idx, nc - 1) * 2.0 - m.z(idx, nc - 2);
  }
}

template <class T>
double streamwise_bed_slope_magnitude(const Mesh<T>& m, Side side, int64_t idx) {  // boundary.rs:241
  switch (side) {
    case WEST: return m.nc < 2 ? 0.0 : std::fabs(value(m.bed_slope_x(idx, 0)));
    case EAST: return m.nc < 2 ? 0.0 : std::fabs(value(m.bed_slope_x(idx, m.nc - 2)));
    case NORTH: return m.nr < 2 ? 0.0 : std::fabs(value(m.bed_slope_y(0, idx)));
    default: return m.nr < 2 ? 0.0 : std::fabs(value(m.bed_slope_y(m.nr - 2, idx)));
  }
}

template <class T>
void ghost_cell(const Mesh<T>& m, Cons<T> inner, Boundary b, Side side, int64_t idx,
                Cons<T>* g_out, T* z_out) {  // boundary.rs:193-219
  Cons<T> state = ghost_state<T>(inner, b, side);
  T bed = ghost_bed<T>(m, b, side, idx);
  if (b.kind == BC_DISCHARGE && value(inner.h) < H_DRY) {
    double slope_mag = streamwise_bed_slope_magnitude<T>(m, side, idx);
    if (slope_mag > DRY_INFLOW_SLOPE_THRESHOLD) {
      int64_t ci, cj;  // boundary.rs:224 boundary_cell_index
      switch (side) {
        case WEST: ci = idx; cj = 0; break;
        case EAST: ci = idx; cj = m.nc - 1; break;
        case NORTH: ci = 0; cj = idx; break;
        default: ci = m.nr - 1; cj = idx; break;
      }
      T n = m.n(ci, cj);
      T h_n = r_powf(n * (std::fabs(b.value) / std::sqrt(slope_mag)), 3.0 / 5.0);
      state.h = r_min(h_n, Scalar<T>::from_f64(DRY_INFLOW_H_MAX));
    }
  }
  *g_out = state;
  *z_out = bed;
}

// ---------------------------------------------------------------------------
// HLLC: riemann.rs:80-204
// ---------------------------------------------------------------------------
template <class T>
void hllc_normal_flux(T h_l, T qn_l, T qt_l, T h_r, T qn_r, T qt_r, T* o_mass, T* o_n,
                      T* o_t) {
  const T Z = Scalar<T>::zero();
  const bool h_l_wet = value(h_l) > DRY_TOL;
  const bool h_r_wet = value(h_r) > DRY_TOL;
  if (!h_l_wet && !h_r_wet) {
    *o_mass = Z; *o_n = Z; *o_t = Z;
    return;
  }
  T cl = h_l_wet ? r_sqrt(h_l * GRAVITY) : Z;
  T cr = h_r_wet ? r_sqrt(h_r * GRAVITY) : Z;
  T un_l = h_l_wet ? qn_l / h_l : Z;
  T un_r = h_r_wet ? qn_r / h_r : Z;
  T ut_l = h_l_wet ? qt_l / h_l : Z;
  T ut_r = h_r_wet ? qt_r / h_r : Z;
  T sl, sr;
  if (h_l_wet && h_r_wet) {
    sl = r_min(un_l - cl, un_r - cr);
    sr = r_max(un_l + cl, un_r + cr);
  } else if (!h_l_wet) {
    sl = un_r - cr * 2.0;
    sr = un_r + cr;
  } else {
    sl = un_l - cl;
    sr = un_l + cl * 2.0;
  }
  T fm_l = Z, fn_l = Z, ft_l = Z, fm_r = Z, fn_r = Z, ft_r = Z;
  if (h_l_wet) {
    fm_l = qn_l;
    fn_l = qn_l * un_l + h_l * h_l * (0.5 * GRAVITY);
    ft_l = qn_l * ut_l;
  }
  if (h_r_wet) {
    fm_r = qn_r;
    fn_r = qn_r * un_r + h_r * h_r * (0.5 * GRAVITY);
    ft_r = qn_r * ut_r;
  }
  if (value(sl) >= 0.0) {
    *o_mass = fm_l; *o_n = fn_l; *o_t = ft_l;
    return;
  }
  if (value(sr) <= 0.0) {
    *o_mass = fm_r; *o_n = fn_r; *o_t = ft_r;
    return;
  }
  T denom = h_r * (un_r - sr) - h_l * (un_l - sl);
  T s_star = std::fabs(value(denom)) > 1.0e-12
                 ? (h_r * (un_r - sr) * sl - h_l * (un_l - sl) * sr) / denom
                 : (sl + sr) * 0.5;
  T h_star_l = h_l * (sl - un_l) / (sl - s_star);
  T h_star_r = h_r * (sr - un_r) / (sr - s_star);
  if (value(s_star) >= 0.0) {
    *o_mass = fm_l + (h_star_l - h_l) * sl;
    *o_n = fn_l + (h_star_l * s_star - qn_l) * sl;
    *o_t = ft_l + (h_star_l * ut_l - qt_l) * sl;
  } else {
    *o_mass = fm_r + (h_star_r - h_r) * sr;
    *o_n = fn_r + (h_star_r * s_star - qn_r) * sr;
    *o_t = ft_r + (h_star_r * ut_r - qt_r) * sr;
  }
}

template <class T> Flux<T> hllc_flux_x(Cons<T> ul, Cons<T> ur) {  // riemann.rs:80
  Flux<T> f;
  hllc_normal_flux(ul.h, ul.hu, ul.hv, ur.h, ur.hu, ur.hv, &f.mass, &f.xm, &f.ym);
  return f;
}
template <class T> Flux<T> hllc_flux_y(Cons<T> ul, Cons<T> ur) {  // riemann.rs:97
  Flux<T> f;
  hllc_normal_flux(ul.h, ul.hv, ul.hu, ur.h, ur.hv, ur.hu, &f.mass, &f.ym, &f.xm);
  return f;
}

// ---------------------------------------------------------------------------
// Well-balanced faces: update.rs:256-353
// ---------------------------------------------------------------------------
template <class T>
Face<T> well_balanced_face(bool x_dir, Cons<T> left, T z_left, Cons<T> right, T z_right) {
  const T Z = Scalar<T>::zero();
  T z_max = r_max(z_left, z_right);
  T h_star_left = r_max(left.h + z_left - z_max, Z);
  T h_star_right = r_max(right.h + z_right - z_max, Z);
  T u_left = Z, v_left = Z, u_right = Z, v_right = Z;
  if (value(left.h) > H_VEL) {
    u_left = left.hu / left.h;
    v_left = left.hv / left.h;
  }
  if (value(right.h) > H_VEL) {
    u_right = right.hu / right.h;
    v_right = right.hv / right.h;
  }
  Cons<T> rl{h_star_left, h_star_left * u_left, h_star_left * v_left};
  Cons<T> rr{h_star_right, h_star_right * u_right, h_star_right * v_right};
  Flux<T> f = x_dir ? hllc_flux_x(rl, rr) : hllc_flux_y(rl, rr);
  T corr_left = (left.h * left.h - h_star_left * h_star_left) * (0.5 * GRAVITY);
  T corr_right = (right.h * right.h - h_star_right * h_star_right) * (0.5 * GRAVITY);
  Face<T> out;
  out.minus = f;
  out.plus = f;
  if (x_dir) {
    out.minus.xm = f.xm + corr_left;
    out.plus.xm = f.xm + corr_right;
  } else {
    out.minus.ym = f.ym + corr_left;
    out.plus.ym = f.ym + corr_right;
  }
  return out;
}

// update.rs:362-370
template <class T> T minmod(T a, T b) {
  if (value(a) * value(b) <= 0.0) return Scalar<T>::zero();
  if (std::fabs(value(a)) < std::fabs(value(b))) return a;
  return b;
}

template <class T> struct Tri {
  T eta, u, v;  // PrimG / CellSlopesG (update.rs:384-400)
};

// update.rs:650-656
template <class T> T interior_z_face(bool l_dry, T z_l, bool r_dry, T z_r) {
  if (l_dry != r_dry) return r_max(z_l, z_r);
  return (z_l + z_r) * 0.5;
}

// StepWorkspace2D (update.rs:743-777)
template <class T> struct Workspace {
  int64_t nr = 0, nc = 0;
  std::vector<Tri<T>> prim, slopes_x, slopes_y;
  std::vector<T> z_face_x, z_face_y, alpha;
  std::vector<Face<T>> faces_x, faces_y;
  std::vector<uint8_t> was_dry;
  std::vector<Cons<T>> u_n;
  Workspace() = default;
  Workspace(int64_t r, int64_t c) { resize(r, c); }
  void resize(int64_t r, int64_t c) {
    nr = r; nc = c;
    prim.assign(r * c, Tri<T>{});
    slopes_x.assign(r * c, Tri<T>{});
    slopes_y.assign(r * c, Tri<T>{});
    z_face_x.assign(r * (c + 1), Scalar<T>::zero());
    z_face_y.assign((r + 1) * c, Scalar<T>::zero());
    faces_x.assign(r * (c + 1), Face<T>{});
    faces_y.assign((r + 1) * c, Face<T>{});
    alpha.assign(r * c, Scalar<T>::one());
    was_dry.assign(r * c, 0);
    u_n.assign(r * c, cons_dry<T>());
  }
};

inline int omp_threads_for(int64_t rows) {
#ifdef _OPENMP
  return rows > 8 ? omp_get_max_threads() : 1;
#else
  (void)rows;
  return 1;
#endif
}

// ---------------------------------------------------------------------------
// CFL: update.rs:113-208
// ---------------------------------------------------------------------------
template <class T>
void max_wave_speeds(const std::vector<Cons<T>>& s, int64_t nr, int64_t nc, double* sx_out,
                     double* sy_out) {
  double s_x = 0.0, s_y = 0.0;
  const int64_t ncell = nr * nc;
#ifdef _OPENMP
#pragma omp parallel for reduction(max : s_x, s_y) num_threads(omp_threads_for(nr)) schedule(static)
#endif
  for (int64_t k = 0; k < ncell; ++k) {
    double h = value(s[k].h);
    if (h <= H_DRY) continue;
    double c = std::sqrt(GRAVITY * h);
    double u = 0.0, v = 0.0;
    if (h > H_VEL) {
      u = value(s[k].hu) / h;
      v = value(s[k].hv) / h;
    }
    s_x = std::fmax(s_x, std::fabs(u) + c);
    s_y = std::fmax(s_y, std::fabs(v) + c);
  }
  *sx_out = s_x;
  *sy_out = s_y;
}

template <class T>
double cfl_time_step(const std::vector<Cons<T>>& s, const Mesh<T>& m, double cfl) {
  double s_x, s_y;
  max_wave_speeds(s, m.nr, m.nc, &s_x, &s_y);
  double denom = s_x / m.dx + s_y / m.dy;
  return denom > 0.0 ? cfl / denom : std::numeric_limits<double>::infinity();
}

template <class T>
double cfl_time_step_with_bcs(const std::vector<Cons<T>>& s, const Mesh<T>& m,
                              const Boundaries& bcs, double cfl) {
  double s_x, s_y;
  max_wave_speeds(s, m.nr, m.nc, &s_x, &s_y);
  const int64_t nr = m.nr, nc = m.nc;
  auto upd = [&](Cons<T> g) {
    double h = value(g.h);
    if (h <= H_DRY) return;
    double c = std::sqrt(GRAVITY * h);
    double u = value(g.hu) / h;
    double v = value(g.hv) / h;
    s_x = std::fmax(s_x, std::fabs(u) + c);
    s_y = std::fmax(s_y, std::fabs(v) + c);
  };
  Cons<T> g;
  T zg;
  for (int64_t i = 0; i < nr; ++i) {
    ghost_cell(m, s[i * nc + 0], bcs.west, WEST, i, &g, &zg);
    upd(g);
    ghost_cell(m, s[i * nc + nc - 1], bcs.east, EAST, i, &g, &zg);
    upd(g);
  }
  for (int64_t j = 0; j < nc; ++j) {
    ghost_cell(m, s[j], bcs.north, NORTH, j, &g, &zg);
    upd(g);
    ghost_cell(m, s[(nr - 1) * nc + j], bcs.south, SOUTH, j, &g, &zg);
    upd(g);
  }
  double denom = s_x / m.dx + s_y / m.dy;
  return denom > 0.0 ? cfl / denom : std::numeric_limits<double>::infinity();
}

// ---------------------------------------------------------------------------
// Forward Euler: update.rs:805-1211 (pass by pass)
// ---------------------------------------------------------------------------
template <class T>
void forward_euler_step_with(std::vector<Cons<T>>& st, const Mesh<T>& m, const Boundaries& bcs,
                             double dt, Workspace<T>& ws) {
  const int64_t nr = m.nr, nc = m.nc;
  if (nr == 0 || nc == 0) return;
  if (ws.nr != nr || ws.nc != nc) ws.resize(nr, nc);
  const T Z = Scalar<T>::zero();
  const int nthr = omp_threads_for(nr);
  (void)nthr;
  auto S = [&](int64_t i, int64_t j) -> Cons<T>& { return st[i * nc + j]; };
  auto DRY = [&](int64_t i, int64_t j) -> bool { return ws.was_dry[i * nc + j] != 0; };
  auto P = [&](int64_t i, int64_t j) -> const Tri<T>& { return ws.prim[i * nc + j]; };

  // was_dry snapshot (update.rs:853-855)
  for (int64_t k = 0; k < nr * nc; ++k) ws.was_dry[k] = value(st[k].h) <= H_DRY;

  // fill_primitives (update.rs:405-426)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      const Cons<T>& s = S(i, j);
      Tri<T>& p = ws.prim[i * nc + j];
      p.eta = s.h + m.z(i, j);
      if (value(s.h) > H_VEL) {
        p.u = s.hu / s.h;
        p.v = s.hv / s.h;
      } else {
        p.u = Z;
        p.v = Z;
      }
    }

  // fill_slopes_x (update.rs:459-500) and fill_slopes_y (503-540)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      Tri<T>& sl = ws.slopes_x[i * nc + j];
      bool anyd = false;
      if (nc >= 2) {
        int64_t lo = j >= 2 ? j - 2 : 0, hi = std::min<int64_t>(j + 2, nc - 1);
        for (int64_t jj = lo; jj <= hi; ++jj) anyd = anyd || DRY(i, jj);
      }
      if (nc < 2 || anyd) {
        sl = Tri<T>{Z, Z, Z};
      } else if (j == 0) {
        const Tri<T>& c = P(i, 0);
        const Tri<T>& r = P(i, 1);
        sl = Tri<T>{(r.eta - c.eta) / m.dx, (r.u - c.u) / m.dx, (r.v - c.v) / m.dx};
      } else if (j + 1 == nc) {
        const Tri<T>& l = P(i, j - 1);
        const Tri<T>& c = P(i, j);
        sl = Tri<T>{(c.eta - l.eta) / m.dx, (c.u - l.u) / m.dx, (c.v - l.v) / m.dx};
      } else {
        const Tri<T>& l = P(i, j - 1);
        const Tri<T>& c = P(i, j);
        const Tri<T>& r = P(i, j + 1);
        sl = Tri<T>{minmod((c.eta - l.eta) / m.dx, (r.eta - c.eta) / m.dx),
                    minmod((c.u - l.u) / m.dx, (r.u - c.u) / m.dx),
                    minmod((c.v - l.v) / m.dx, (r.v - c.v) / m.dx)};
      }
    }
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      Tri<T>& sl = ws.slopes_y[i * nc + j];
      bool anyd = false;
      if (nr >= 2) {
        int64_t lo = i >= 2 ? i - 2 : 0, hi = std::min<int64_t>(i + 2, nr - 1);
        for (int64_t ii = lo; ii <= hi; ++ii) anyd = anyd || DRY(ii, j);
      }
      if (nr < 2 || anyd) {
        sl = Tri<T>{Z, Z, Z};
      } else if (i == 0) {
        const Tri<T>& c = P(0, j);
        const Tri<T>& b = P(1, j);
        sl = Tri<T>{(b.eta - c.eta) / m.dy, (b.u - c.u) / m.dy, (b.v - c.v) / m.dy};
      } else if (i + 1 == nr) {
        const Tri<T>& t = P(i - 1, j);
        const Tri<T>& c = P(i, j);
        sl = Tri<T>{(c.eta - t.eta) / m.dy, (c.u - t.u) / m.dy, (c.v - t.v) / m.dy};
      } else {
        const Tri<T>& t = P(i - 1, j);
        const Tri<T>& c = P(i, j);
        const Tri<T>& b = P(i + 1, j);
        sl = Tri<T>{minmod((c.eta - t.eta) / m.dy, (b.eta - c.eta) / m.dy),
                    minmod((c.u - t.u) / m.dy, (b.u - c.u) / m.dy),
                    minmod((c.v - t.v) / m.dy, (b.v - c.v) / m.dy)};
      }
    }

  // fill_z_face_x / fill_z_face_y (update.rs:676-728)
  Cons<T> g;
  T zg;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) private(g, zg)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j <= nc; ++j) {
      T& zf = ws.z_face_x[i * (nc + 1) + j];
      if (j == 0) {
        ghost_cell(m, S(i, 0), bcs.west, WEST, i, &g, &zg);
        zf = (zg + m.z(i, 0)) * 0.5;
      } else if (j == nc) {
        ghost_cell(m, S(i, nc - 1), bcs.east, EAST, i, &g, &zg);
        zf = (m.z(i, nc - 1) + zg) * 0.5;
      } else {
        zf = interior_z_face(DRY(i, j - 1), m.z(i, j - 1), DRY(i, j), m.z(i, j));
      }
    }
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) private(g, zg)
#endif
  for (int64_t i = 0; i <= nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      T& zf = ws.z_face_y[i * nc + j];
      if (i == 0) {
        ghost_cell(m, S(0, j), bcs.north, NORTH, j, &g, &zg);
        zf = (zg + m.z(0, j)) * 0.5;
      } else if (i == nr) {
        ghost_cell(m, S(nr - 1, j), bcs.south, SOUTH, j, &g, &zg);
        zf = (m.z(nr - 1, j) + zg) * 0.5;
      } else {
        zf = interior_z_face(DRY(i - 1, j), m.z(i - 1, j), DRY(i, j), m.z(i, j));
      }
    }

  // faces_x (update.rs:890-907) with reconstruct_x_face_states (560-592)
  const double half_dx = 0.5 * m.dx;
  const double half_dy = 0.5 * m.dy;
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) private(g, zg)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j <= nc; ++j) {
      const T zf = ws.z_face_x[i * (nc + 1) + j];
      Face<T>& face = ws.faces_x[i * (nc + 1) + j];
      if (j == 0) {
        ghost_cell(m, S(i, 0), bcs.west, WEST, i, &g, &zg);
        face = well_balanced_face<T>(true, g, zf, S(i, 0), zf);
      } else if (j == nc) {
        ghost_cell(m, S(i, nc - 1), bcs.east, EAST, i, &g, &zg);
        face = well_balanced_face<T>(true, S(i, nc - 1), zf, g, zf);
      } else if (DRY(i, j - 1) && DRY(i, j)) {
        face = Face<T>{flux_zero<T>(), flux_zero<T>()};
      } else {
        const Tri<T>& l = P(i, j - 1);
        const Tri<T>& sl = ws.slopes_x[i * nc + j - 1];
        T eta_minus = l.eta + sl.eta * half_dx;
        T u_minus = l.u + sl.u * half_dx;
        T v_minus = l.v + sl.v * half_dx;
        const Tri<T>& r = P(i, j);
        const Tri<T>& sr = ws.slopes_x[i * nc + j];
        T eta_plus = r.eta - sr.eta * half_dx;
        T u_plus = r.u - sr.u * half_dx;
        T v_plus = r.v - sr.v * half_dx;
        T h_minus = r_max(eta_minus - zf, Z);
        T h_plus = r_max(eta_plus - zf, Z);
        Cons<T> rl{h_minus, h_minus * u_minus, h_minus * v_minus};
        Cons<T> rr{h_plus, h_plus * u_plus, h_plus * v_plus};
        face = well_balanced_face<T>(true, rl, zf, rr, zf);
      }
    }
  // faces_y (update.rs:909-926) with reconstruct_y_face_states (595-623)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static) private(g, zg)
#endif
  for (int64_t i = 0; i <= nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      const T zf = ws.z_face_y[i * nc + j];
      Face<T>& face = ws.faces_y[i * nc + j];
      if (i == 0) {
        ghost_cell(m, S(0, j), bcs.north, NORTH, j, &g, &zg);
        face = well_balanced_face<T>(false, g, zf, S(0, j), zf);
      } else if (i == nr) {
        ghost_cell(m, S(nr - 1, j), bcs.south, SOUTH, j, &g, &zg);
        face = well_balanced_face<T>(false, S(nr - 1, j), zf, g, zf);
      } else if (DRY(i - 1, j) && DRY(i, j)) {
        face = Face<T>{flux_zero<T>(), flux_zero<T>()};
      } else {
        const Tri<T>& t = P(i - 1, j);
        const Tri<T>& st_ = ws.slopes_y[(i - 1) * nc + j];
        T eta_minus = t.eta + st_.eta * half_dy;
        T u_minus = t.u + st_.u * half_dy;
        T v_minus = t.v + st_.v * half_dy;
        const Tri<T>& b = P(i, j);
        const Tri<T>& sb = ws.slopes_y[i * nc + j];
        T eta_plus = b.eta - sb.eta * half_dy;
        T u_plus = b.u - sb.u * half_dy;
        T v_plus = b.v - sb.v * half_dy;
        T h_minus = r_max(eta_minus - zf, Z);
        T h_plus = r_max(eta_plus - zf, Z);
        Cons<T> rt{h_minus, h_minus * u_minus, h_minus * v_minus};
        Cons<T> rb{h_plus, h_plus * u_plus, h_plus * v_plus};
        face = well_balanced_face<T>(false, rt, zf, rb, zf);
      }
    }

  const double dt_dx = dt / m.dx;  // update.rs:930
  const double dt_dy = dt / m.dy;
  auto FX = [&](int64_t i, int64_t j) -> Face<T>& { return ws.faces_x[i * (nc + 1) + j]; };
  auto FY = [&](int64_t i, int64_t j) -> Face<T>& { return ws.faces_y[i * nc + j]; };

  // alpha (update.rs:953-982)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      T fx_right = FX(i, j + 1).minus.mass;
      T fx_left = FX(i, j).plus.mass;
      T fy_bottom = FY(i + 1, j).minus.mass;
      T fy_top = FY(i, j).plus.mass;
      T out_mass = Z;
      if (value(fx_right) > 0.0) out_mass = out_mass + fx_right * dt_dx;
      if (value(fx_left) < 0.0) out_mass = out_mass + (-fx_left) * dt_dx;
      if (value(fy_bottom) > 0.0) out_mass = out_mass + fy_bottom * dt_dy;
      if (value(fy_top) < 0.0) out_mass = out_mass + (-fy_top) * dt_dy;
      T available = r_max(S(i, j).h - H_DRY, Z);
      ws.alpha[i * nc + j] = (value(out_mass) > value(available) && value(out_mass) > 0.0)
                                 ? available / out_mass
                                 : Scalar<T>::one();
    }
  auto A = [&](int64_t i, int64_t j) -> T { return ws.alpha[i * nc + j]; };
  auto scale = [](Face<T>& f, T a) {
    f.minus.mass = f.minus.mass * a;
    f.minus.xm = f.minus.xm * a;
    f.minus.ym = f.minus.ym * a;
    f.plus.mass = f.plus.mass * a;
    f.plus.xm = f.plus.xm * a;
    f.plus.ym = f.plus.ym * a;
  };
  // face rescale x (update.rs:992-1022)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j <= nc; ++j) {
      if (j > 0 && j < nc && DRY(i, j - 1) && DRY(i, j)) continue;
      Face<T>& f = FX(i, j);
      T a;
      if (j == 0)
        a = value(f.minus.mass) < 0.0 ? A(i, 0) : Scalar<T>::one();
      else if (j == nc)
        a = value(f.minus.mass) > 0.0 ? A(i, nc - 1) : Scalar<T>::one();
      else if (value(f.minus.mass) > 0.0)
        a = A(i, j - 1);
      else
        a = A(i, j);
      scale(f, a);
    }
  // face rescale y (update.rs:1023-1053)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i <= nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      if (i > 0 && i < nr && DRY(i - 1, j) && DRY(i, j)) continue;
      Face<T>& f = FY(i, j);
      T a;
      if (i == 0)
        a = value(f.minus.mass) < 0.0 ? A(0, j) : Scalar<T>::one();
      else if (i == nr)
        a = value(f.minus.mass) > 0.0 ? A(nr - 1, j) : Scalar<T>::one();
      else if (value(f.minus.mass) > 0.0)
        a = A(i - 1, j);
      else
        a = A(i, j);
      scale(f, a);
    }

  // FV update + bed source + moisture floor (update.rs:1071-1210)
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthr) schedule(static)
#endif
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) {
      Cons<T>& cell = S(i, j);
      if (DRY(i, j) && i > 0 && i + 1 < nr && j > 0 && j + 1 < nc && DRY(i - 1, j) &&
          DRY(i + 1, j) && DRY(i, j - 1) && DRY(i, j + 1)) {
        cell.hu = Z;
        cell.hv = Z;
        continue;
      }
      const Flux<T> fx_right = FX(i, j + 1).minus;
      const Flux<T> fx_left = FX(i, j).plus;
      const Flux<T> fy_bottom = FY(i + 1, j).minus;
      const Flux<T> fy_top = FY(i, j).plus;
      T dh = (fx_right.mass - fx_left.mass) * dt_dx + (fy_bottom.mass - fy_top.mass) * dt_dy;
      T new_h = cell.h - dh;
      T dhu = (fx_right.xm - fx_left.xm) * dt_dx + (fy_bottom.xm - fy_top.xm) * dt_dy;
      T dhv = (fx_right.ym - fx_left.ym) * dt_dx + (fy_bottom.ym - fy_top.ym) * dt_dy;

      T h_old = cell.h;
      T eta_cell = h_old + m.z(i, j);
      T slope_eta_x = ws.slopes_x[i * nc + j].eta;
      T eta_left = j > 0 ? eta_cell - slope_eta_x * (0.5 * m.dx) : eta_cell;
      T eta_right = j + 1 < nc ? eta_cell + slope_eta_x * (0.5 * m.dx) : eta_cell;
      T h_face_left = r_max(eta_left - ws.z_face_x[i * (nc + 1) + j], Z);
      T h_face_right = r_max(eta_right - ws.z_face_x[i * (nc + 1) + j + 1], Z);
      T z_eff_left = eta_left - h_face_left;
      T z_eff_right = eta_right - h_face_right;
      T s_hu = (h_face_left + h_face_right) * (z_eff_left - z_eff_right) * (0.5 * GRAVITY) / m.dx;

      T slope_eta_y = ws.slopes_y[i * nc + j].eta;
      T eta_top = i > 0 ? eta_cell - slope_eta_y * (0.5 * m.dy) : eta_cell;
      T eta_bottom = i + 1 < nr ? eta_cell + slope_eta_y * (0.5 * m.dy) : eta_cell;
      T h_face_top = r_max(eta_top - ws.z_face_y[i * nc + j], Z);
      T h_face_bottom = r_max(eta_bottom - ws.z_face_y[(i + 1) * nc + j], Z);
      T z_eff_top = eta_top - h_face_top;
      T z_eff_bottom = eta_bottom - h_face_bottom;
      T s_hv = (h_face_top + h_face_bottom) * (z_eff_top - z_eff_bottom) * (0.5 * GRAVITY) / m.dy;

      if (value(new_h) <= H_VEL) {
        cell = Cons<T>{r_max(new_h, Z), Z, Z};
      } else {
        T hu_old = Z, hv_old = Z;
        if (value(h_old) > H_VEL) {
          hu_old = cell.hu;
          hv_old = cell.hv;
        }
        cell.h = new_h;
        cell.hu = hu_old - dhu + s_hu * dt;
        cell.hv = hv_old - dhv + s_hv * dt;
      }
    }
}

// SSP-RK2 (update.rs:1255-1287)
template <class T>
void ssprk2_step_with(std::vector<Cons<T>>& st, const Mesh<T>& m, const Boundaries& bcs,
                      double dt, Workspace<T>& ws) {
  if (ws.nr != m.nr || ws.nc != m.nc) ws.resize(m.nr, m.nc);
  ws.u_n = st;
  forward_euler_step_with(st, m, bcs, dt, ws);
  forward_euler_step_with(st, m, bcs, dt, ws);
  const int64_t ncell = m.nr * m.nc;
  const T Z = Scalar<T>::zero();
#ifdef _OPENMP
#pragma omp parallel for num_threads(omp_threads_for(m.nr)) schedule(static)
#endif
  for (int64_t k = 0; k < ncell; ++k) {
    const Cons<T> prev = ws.u_n[k];
    Cons<T>& s = st[k];
    s.h = (prev.h + s.h) * 0.5;
    s.hu = (prev.hu + s.hu) * 0.5;
    s.hv = (prev.hv + s.hv) * 0.5;
    if (value(s.h) <= H_VEL) {
      s.h = r_max(s.h, Z);
      s.hu = Z;
      s.hv = Z;
    }
  }
}

// Manning friction (source.rs:130-165)
template <class T>
void manning_friction_step(std::vector<Cons<T>>& st, const Mesh<T>& m, double dt,
                           double dry_tol) {
  const double dt_g = dt * GRAVITY;
  const int64_t ncell = m.nr * m.nc;
#ifdef _OPENMP
#pragma omp parallel for num_threads(omp_threads_for(m.nr)) schedule(static)
#endif
  for (int64_t k = 0; k < ncell; ++k) {
    Cons<T>& s = st[k];
    const T n = m.manning[k];
    if (value(s.h) <= dry_tol) continue;
    if (value(n) == 0.0) continue;
    T speed = r_sqrt(s.hu * s.hu + s.hv * s.hv) / s.h;
    T factor = n * n * speed / r_powf(s.h, 4.0 / 3.0) * dt_g + 1.0;
    s.hu = s.hu / factor;
    s.hv = s.hv / factor;
  }
}

// Rain (source.rs:88-101); f64 only in the reference. For T = Dual the
// forcing is a constant: only the value is changed, the derivative of the
// added depth is zero (rate and dt are not seeds).
template <class T> void apply_rain(std::vector<Cons<T>>& st, double rate, double dt) {
  if (rate == 0.0) return;
  const double dh = rate * dt;
  const int64_t ncell = (int64_t)st.size();
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (ncell > 65536)
#endif
  for (int64_t k = 0; k < ncell; ++k) {
    Cons<T>& c = st[k];
    T new_h = c.h + dh;
    if (value(new_h) <= 0.0)
      c = cons_dry<T>();
    else
      c.h = new_h;
  }
}

struct PointSource {
  int64_t row, col;
  double q_mass;
};
// Point sources (source.rs:52-69)
template <class T>
void apply_point_sources(std::vector<Cons<T>>& st, int64_t nc, const PointSource* src, int64_t n,
                         double dt, double dx, double dy) {
  const double cell_area = dx * dy;
  for (int64_t k = 0; k < n; ++k) {
    const double dh = src[k].q_mass * dt / cell_area;
    Cons<T>& c = st[src[k].row * nc + src[k].col];
    c.h = r_max(c.h + dh, Scalar<T>::zero());
    if (value(c.h) == 0.0) {
      c.hu = Scalar<T>::zero();
      c.hv = Scalar<T>::zero();
    }
  }
}

// Piecewise-linear time series used for the hydrograph / hyetograph forcing
// (this build's forcing descriptor; the reference's callers evaluate their own
// closures at t_new, e.g. solver-2d/examples/uk_ea_test8a_official.rs:203-217).
// Holds the first value before t[0] and the last after t[n-1]; equal time
// stamps make a step.
inline double series_eval(const double* ts, const double* vs, int64_t n, double t) {
  if (n <= 0) return 0.0;
  if (n == 1 || t <= ts[0]) return vs[0];
  if (t >= ts[n - 1]) return vs[n - 1];
  int64_t lo = 0, hi = n - 1;  // find k with ts[k] <= t < ts[k+1]
  while (hi - lo > 1) {
    int64_t mid = (lo + hi) / 2;
    if (ts[mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  const double w = (t - ts[lo]) / (ts[lo + 1] - ts[lo]);
  return vs[lo] + (vs[lo + 1] - vs[lo]) * w;
}

}  // namespace hfo
