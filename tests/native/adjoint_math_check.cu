// Host-side check of the hand-written reverse functions (hf_adjoint_math.cuh)
// against the oracle's forward-mode Dual evaluation of the same functions
// (oracle/hf_oracle.hpp, T = Dual). For inputs x, an input direction v and an
// output adjoint lam, the forward side gives lam . (J v) from the Dual
// tangents of the outputs, the reverse side gives v . (J^T lam); the two must
// agree to rounding; out[2] is the sum of |terms| of the reverse side, the
// scale of that rounding. Test code: built by tests/test_adjoint_math.py with nvcc
// (host code only) and called through ctypes.
#include <cmath>
#include <cstring>
#include <vector>

#include "hf_adjoint_math.cuh"
#include "hf_oracle.hpp"

using hfo::Dual;

namespace {
Dual D(double v, double d) { return Dual{v, d}; }
}  // namespace

extern "C" {

// x = (h_l, qn_l, qt_l, h_r, qn_r, qt_r); lam: 3 output adjoints (mass,
// normal, tangential); out = (forward, reverse).
int chk_hllc(const double* x, const double* v, const double* lam, double* out) {
  Dual m, n, t;
  hfo::hllc_normal_flux<Dual>(D(x[0], v[0]), D(x[1], v[1]), D(x[2], v[2]), D(x[3], v[3]),
                              D(x[4], v[4]), D(x[5], v[5]), &m, &n, &t);
  out[0] = lam[0] * m.dval + lam[1] * n.dval + lam[2] * t.dval;
  double L[6] = {0, 0, 0, 0, 0, 0};
  hf::hllc_normal_rev(x[0], x[1], x[2], x[3], x[4], x[5], lam[0], lam[1], lam[2], L[0], L[1],
                      L[2], L[3], L[4], L[5]);
  double r = 0.0, a = 0.0;
  for (int k = 0; k < 6; ++k) {
    r += L[k] * v[k];
    a += std::fabs(L[k] * v[k]);
  }
  out[1] = r;
  out[2] = a;
  return 0;
}

// Well-balanced x face with the shared bed zf; lam: (mass, n_minus, n_plus,
// tangential).
int chk_wb(const double* x, double zf, const double* v, const double* lam, double* out) {
  hfo::Cons<Dual> l{D(x[0], v[0]), D(x[1], v[1]), D(x[2], v[2])};
  hfo::Cons<Dual> r{D(x[3], v[3]), D(x[4], v[4]), D(x[5], v[5])};
  const hfo::Face<Dual> f = hfo::well_balanced_face<Dual>(true, l, D(zf, 0.0), r, D(zf, 0.0));
  out[0] = lam[0] * f.minus.mass.dval + lam[1] * f.minus.xm.dval + lam[2] * f.plus.xm.dval +
           lam[3] * f.minus.ym.dval;
  double L[6] = {0, 0, 0, 0, 0, 0};
  hf::wb_face_rev(x[0], x[1], x[2], x[3], x[4], x[5], zf, lam[0], lam[1], lam[2], lam[3], L[0],
                  L[1], L[2], L[3], L[4], L[5]);
  double s = 0.0, a = 0.0;
  for (int k = 0; k < 6; ++k) {
    s += L[k] * v[k];
    a += std::fabs(L[k] * v[k]);
  }
  out[1] = s;
  out[2] = a;
  return 0;
}

// Manning friction on one cell: x = (h, hu, hv, n), v its direction, lam the
// adjoint of the post-friction (h, hu, hv).
int chk_friction(const double* x, const double* v, double dt, double dry_tol, const double* lam,
                 double* out) {
  hfo::Mesh<Dual> m;
  m.nr = 1;
  m.nc = 1;
  m.bed.assign(1, D(0.0, 0.0));
  m.manning.assign(1, D(x[3], v[3]));
  std::vector<hfo::Cons<Dual>> st(1, hfo::Cons<Dual>{D(x[0], v[0]), D(x[1], v[1]), D(x[2], v[2])});
  hfo::manning_friction_step(st, m, dt, dry_tol);
  out[0] = lam[0] * st[0].h.dval + lam[1] * st[0].hu.dval + lam[2] * st[0].hv.dval;
  double Lh = lam[0], Lhu = lam[1], Lhv = lam[2], Ln = 0.0;
  hf::friction_rev(x[0], x[1], x[2], x[3], dt, dry_tol, Lh, Lhu, Lhv, Ln);
  out[1] = Lh * v[0] + Lhu * v[1] + Lhv * v[2] + Ln * v[3];
  out[2] = std::fabs(Lh * v[0]) + std::fabs(Lhu * v[1]) + std::fabs(Lhv * v[2]) +
           std::fabs(Ln * v[3]);
  return 0;
}

// Ghost cell of a 3 x 3 mesh (beds z[9], Manning n[9] with direction vn[9])
// for `side` at boundary index idx = 1 of boundary kind / value; the inner
// state x = (h, hu, hv) with direction v. lam: adjoint of the ghost state
// (h, hu, hv). The reverse maps it to the inner state and the Manning field.
int chk_ghost(int side, int kind, double value, const double* z, const double* n,
              const double* vn, const double* x, const double* v, const double* lam,
              double* out) {
  hfo::Mesh<Dual> m;
  m.nr = 3;
  m.nc = 3;
  m.dx = 2.0;
  m.dy = 3.0;
  m.bed.resize(9);
  m.manning.resize(9);
  for (int k = 0; k < 9; ++k) {
    m.bed[k] = D(z[k], 0.0);
    m.manning[k] = D(n[k], vn[k]);
  }
  hfo::Boundary b{kind, value};
  hfo::Cons<Dual> inner{D(x[0], v[0]), D(x[1], v[1]), D(x[2], v[2])};
  hfo::Cons<Dual> g;
  Dual zg;
  hfo::ghost_cell<Dual>(m, inner, b, (hfo::Side)side, 1, &g, &zg);
  out[0] = lam[0] * g.h.dval + lam[1] * g.hu.dval + lam[2] * g.hv.dval;
  // boundary cell and its inward neighbour (row-major 3 x 3, idx = 1)
  int c0, c1;
  double dn;
  switch (side) {
    case 0: c0 = 1; c1 = 4; dn = m.dy; break;   // north: row 0
    case 1: c0 = 7; c1 = 4; dn = m.dy; break;   // south: row 2
    case 2: c0 = 3; c1 = 4; dn = m.dx; break;   // west: col 0
    default: c0 = 5; c1 = 4; dn = m.dx; break;  // east: col 2
  }
  hf::BcDev bc;
  for (int k = 0; k < 4; ++k) {
    bc.kind[k] = kind;
    bc.val[k] = value;
  }
  const bool xf = side >= 2;
  const double Lgn = xf ? lam[1] : lam[2], Lgt = xf ? lam[2] : lam[1];
  double Lh = 0.0, Lhu = 0.0, Lhv = 0.0, Ln = 0.0;
  hf::ghost_rev(side, bc, x[0], z, n, c0, c1, dn, lam[0], Lgn, Lgt, Lh, Lhu, Lhv, Ln);
  out[1] = Lh * v[0] + Lhu * v[1] + Lhv * v[2] + Ln * vn[c0];
  out[2] = std::fabs(Lh * v[0]) + std::fabs(Lhu * v[1]) + std::fabs(Lhv * v[2]) +
           std::fabs(Ln * vn[c0]);
  return 0;
}

void chk_set_pow_mode(int mode) { hfo::pow_mode() = mode; }

}  // extern "C"
