// hf_oracle_capi.cpp -- extern "C" entry points of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (see hf_oracle.hpp): loaded by tests/, by
// __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline /
// reference arm. State arrays are SoA (h, hu, hv) row-major; internally the
// oracle keeps the reference's AoS Conserved2D layout.
#include <cstdio>
#include <cstring>
#include <string>

#include "../include/hydroflux_gpu.h"
#include "hf_oracle.hpp"

using namespace hfo;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

Boundary to_b(const hf_boundary& b) { return Boundary{b.kind, b.value}; }
Boundaries to_bcs(const hf_boundaries* b) {
  if (!b) {
    Boundary t{BC_TRANSMISSIVE, 0.0};
    return Boundaries{t, t, t, t};
  }
  return Boundaries{to_b(b->north), to_b(b->south), to_b(b->west), to_b(b->east)};
}

template <class T>
Mesh<T> make_mesh(int64_t nr, int64_t nc, double dx, double dy, const double* z, const double* n) {
  Mesh<T> m;
  m.nr = nr;
  m.nc = nc;
  m.dx = dx;
  m.dy = dy;
  m.bed.resize(nr * nc);
  m.manning.resize(nr * nc);
  for (int64_t k = 0; k < nr * nc; ++k) {
    m.bed[k] = Scalar<T>::from_f64(z[k]);
    m.manning[k] = Scalar<T>::from_f64(n ? n[k] : 0.0);
  }
  return m;
}

std::vector<Cons<double>> load(int64_t ncell, const double* h, const double* hu, const double* hv) {
  std::vector<Cons<double>> s(ncell);
  for (int64_t k = 0; k < ncell; ++k) s[k] = Cons<double>{h[k], hu[k], hv[k]};
  return s;
}
void store(const std::vector<Cons<double>>& s, double* h, double* hu, double* hv) {
  for (size_t k = 0; k < s.size(); ++k) {
    h[k] = s[k].h;
    hu[k] = s[k].hu;
    hv[k] = s[k].hv;
  }
}

int check_bcs(const Boundaries& b, int64_t nr, int64_t nc) {
  const Boundary* all[4] = {&b.north, &b.south, &b.west, &b.east};
  for (int s = 0; s < 4; ++s) {
    int k = all[s]->kind;
    if (k < 0 || k > 3) return fail(HF_ERR_INVALID_CONFIG, "unknown boundary kind");
    if (k == BC_DISCHARGE || k == BC_DEPTH) {
      int64_t along = (s < 2) ? nr : nc;
      if (along < 2)
        return fail(HF_ERR_INVALID_CONFIG,
                    "linear bed extrapolation requires >= 2 cells normal to the boundary");
    }
  }
  return HF_OK;
}

// Units of the forcing series (hf_sim_set_rain_units /
// hf_sim_set_point_source_units): sampled at t / t_div, value
// (v * v_mul) / v_div, the order of the reference example's
// `interp_min(table, t_s) * 1e-3 / 3600.0` (t_s / 60 inside interp_min;
// solver-2d/examples/uk_ea_test8a_official.rs:119-134).
struct Units {
  double t_div = 1.0, v_mul = 1.0, v_div = 1.0;
};
Units g_rain_units, g_src_units;  // set by hfo_set_series_units

double series_eval_u(const double* ts, const double* vs, int64_t n, double t, const Units& u) {
  return series_eval(ts, vs, n, t / u.t_div) * u.v_mul / u.v_div;
}

// Control-point recorder of hfo_sim_run (hf_sim_set_gauges): after every
// step, peak = fold(0.0, f64::max) and last = h at each gauge cell
// (uk_ea_test8a_official.rs:219-246). Set by hfo_set_gauges, the buffers
// are the caller's; n = 0 disables it.
struct GaugeRec {
  int64_t n = 0;
  const int64_t* cells = nullptr;
  double* peak = nullptr;
  double* last = nullptr;
};
GaugeRec g_gauges;

// Forcing descriptor (see hf_sim_set_rain / hf_sim_set_point_sources).
struct Forcing {
  int64_t n_rain = 0;
  const double* rain_t = nullptr;
  const double* rain_v = nullptr;
  int64_t n_src = 0;
  const int64_t* rows = nullptr;
  const int64_t* cols = nullptr;
  const int64_t* offs = nullptr;
  const double* src_t = nullptr;
  const double* src_q = nullptr;
  Units rain_u = g_rain_units;
  Units src_u = g_src_units;
};

// Simulation::step (sim.rs:204-228) followed by the forcings at t_new.
template <class T>
int sim_step(std::vector<Cons<T>>& st, const Mesh<T>& m, const hf_config& cfg,
             const Boundaries& bcs, Workspace<T>& ws, const Forcing& f, double dt_cap,
             double* t, uint64_t* steps, double* dt_out) {
  double dt = cfl_time_step_with_bcs(st, m, bcs, cfg.cfl);
  dt = std::fmin(dt, cfg.max_dt);
  dt = std::fmin(dt, dt_cap);
  if (!(std::isfinite(dt) && dt > 0.0)) {
    *dt_out = dt;
    char buf[160];
    std::snprintf(buf, sizeof buf, "degenerate time step dt = %g at t = %g (step %llu)", dt, *t,
                  (unsigned long long)*steps);
    return fail(HF_ERR_DEGENERATE_DT, buf);
  }
  if (cfg.integrator == HF_FORWARD_EULER)
    forward_euler_step_with(st, m, bcs, dt, ws);
  else
    ssprk2_step_with(st, m, bcs, dt, ws);
  manning_friction_step(st, m, dt, cfg.friction_dry_tol);
  *t += dt;
  *steps += 1;
  const double t_new = *t;
  if (f.n_rain > 0)
    apply_rain(st, series_eval_u(f.rain_t, f.rain_v, f.n_rain, t_new, f.rain_u), dt);
  if (f.n_src > 0) {
    std::vector<PointSource> ps(f.n_src);
    for (int64_t k = 0; k < f.n_src; ++k) {
      int64_t a = f.offs[k], b = f.offs[k + 1];
      ps[k] = PointSource{f.rows[k], f.cols[k],
                          series_eval_u(f.src_t + a, f.src_q + a, b - a, t_new, f.src_u)};
    }
    apply_point_sources(st, m.nc, ps.data(), f.n_src, dt, m.dx, m.dy);
  }
  *dt_out = dt;
  return HF_OK;
}

int validate_cfg(const hf_config* cfg) {
  if (!cfg) return fail(HF_ERR_INVALID_ARG, "null config");
  if (!(cfg->cfl > 0.0 && cfg->cfl <= 1.0))
    return fail(HF_ERR_INVALID_CONFIG, "cfl must be in (0, 1]");
  if (!(cfg->max_dt > 0.0)) return fail(HF_ERR_INVALID_CONFIG, "max_dt must be positive");
  return HF_OK;
}

}  // namespace

extern "C" {

const char* hfo_last_error(void) { return g_err.c_str(); }

int hfo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// 0: libm pow (the reference's platform behaviour); 1: its restatement
// (hf_pow.h, the GPU's pow).
int hfo_set_pow_mode(int mode) {
  pow_mode() = mode ? 1 : 0;
  return pow_mode();
}

double hfo_pow_port(double x, double y) { return hfpow::pow_libm(x, y); }

// Counts the x[k] (k < n) whose x^y differs, bit for bit, between the
// restatement and the host libm; the first few go to first_bad (up to 8).
int64_t hfo_pow_mismatches(int64_t n, const double* x, double y, double* first_bad) {
  int64_t bad = 0;
  for (int64_t k = 0; k < n; ++k) {
    const double a = hfpow::pow_libm(x[k], y), b = std::pow(x[k], y);
    uint64_t ba, bb;
    std::memcpy(&ba, &a, 8);
    std::memcpy(&bb, &b, 8);
    if (ba != bb && !(a != a && b != b)) {
      if (first_bad && bad < 8) first_bad[bad] = x[k];
      ++bad;
    }
  }
  return bad;
}

int hfo_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int hfo_hllc_flux(int x_dir, const double* ul, const double* ur, double* out) {
  Cons<double> l{ul[0], ul[1], ul[2]}, r{ur[0], ur[1], ur[2]};
  Flux<double> f = x_dir ? hllc_flux_x(l, r) : hllc_flux_y(l, r);
  out[0] = f.mass;
  out[1] = f.xm;
  out[2] = f.ym;
  return HF_OK;
}

int hfo_ghost_cell(int64_t nr, int64_t nc, double dx, double dy, const double* z, const double* n,
                   const hf_boundary* b, int side, int64_t idx, const double* inner,
                   double* out_state, double* out_bed) {
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  Cons<double> g;
  double zg;
  ghost_cell(m, Cons<double>{inner[0], inner[1], inner[2]}, to_b(*b), (Side)side, idx, &g, &zg);
  out_state[0] = g.h;
  out_state[1] = g.hu;
  out_state[2] = g.hv;
  *out_bed = zg;
  return HF_OK;
}

int hfo_max_wave_speeds(int64_t nr, int64_t nc, const double* h, const double* hu,
                        const double* hv, double* sx, double* sy) {
  auto s = load(nr * nc, h, hu, hv);
  max_wave_speeds(s, nr, nc, sx, sy);
  return HF_OK;
}

int hfo_cfl_time_step(int64_t nr, int64_t nc, double dx, double dy, const double* z,
                      const double* n, const double* h, const double* hu, const double* hv,
                      const hf_boundaries* bcs, double cfl, double* dt_out) {
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  auto s = load(nr * nc, h, hu, hv);
  if (bcs) {
    Boundaries b = to_bcs(bcs);
    int rc = check_bcs(b, nr, nc);
    if (rc) return rc;
    *dt_out = cfl_time_step_with_bcs(s, m, b, cfl);
  } else {
    *dt_out = cfl_time_step(s, m, cfl);
  }
  return HF_OK;
}

int hfo_forward_euler_step(int64_t nr, int64_t nc, double dx, double dy, const double* z,
                           const double* n, double* h, double* hu, double* hv,
                           const hf_boundaries* bcs, double dt) {
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  Boundaries b = to_bcs(bcs);
  int rc = check_bcs(b, nr, nc);
  if (rc) return rc;
  auto s = load(nr * nc, h, hu, hv);
  Workspace<double> ws(nr, nc);
  forward_euler_step_with(s, m, b, dt, ws);
  store(s, h, hu, hv);
  return HF_OK;
}

int hfo_ssprk2_step(int64_t nr, int64_t nc, double dx, double dy, const double* z,
                    const double* n, double* h, double* hu, double* hv, const hf_boundaries* bcs,
                    double dt) {
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  Boundaries b = to_bcs(bcs);
  int rc = check_bcs(b, nr, nc);
  if (rc) return rc;
  auto s = load(nr * nc, h, hu, hv);
  Workspace<double> ws(nr, nc);
  ssprk2_step_with(s, m, b, dt, ws);
  store(s, h, hu, hv);
  return HF_OK;
}

int hfo_manning_friction_step(int64_t nr, int64_t nc, const double* n, double* h, double* hu,
                              double* hv, double dt, double dry_tol) {
  Mesh<double> m;
  m.nr = nr;
  m.nc = nc;
  m.manning.assign(n, n + nr * nc);
  auto s = load(nr * nc, h, hu, hv);
  manning_friction_step(s, m, dt, dry_tol);
  store(s, h, hu, hv);
  return HF_OK;
}

int hfo_apply_rain(int64_t ncell, double* h, double* hu, double* hv, double rate, double dt) {
  auto s = load(ncell, h, hu, hv);
  apply_rain(s, rate, dt);
  store(s, h, hu, hv);
  return HF_OK;
}

int hfo_apply_point_sources(int64_t nr, int64_t nc, double* h, double* hu, double* hv,
                            int64_t nsrc, const int64_t* rows, const int64_t* cols,
                            const double* q, double dt, double dx, double dy) {
  std::vector<PointSource> ps(nsrc);
  for (int64_t k = 0; k < nsrc; ++k) {
    if (rows[k] < 0 || rows[k] >= nr || cols[k] < 0 || cols[k] >= nc)
      return fail(HF_ERR_INVALID_ARG, "point source outside the mesh");
    ps[k] = PointSource{rows[k], cols[k], q[k]};
  }
  auto s = load(nr * nc, h, hu, hv);
  apply_point_sources(s, nc, ps.data(), nsrc, dt, dx, dy);
  store(s, h, hu, hv);
  return HF_OK;
}

double hfo_series_eval(const double* t, const double* v, int64_t n, double x) {
  return series_eval(t, v, n, x);
}

void hfo_set_series_units(double rain_t_div, double rain_v_mul, double rain_v_div,
                          double src_t_div, double src_v_mul, double src_v_div) {
  g_rain_units = Units{rain_t_div, rain_v_mul, rain_v_div};
  g_src_units = Units{src_t_div, src_v_mul, src_v_div};
}

// Simulation driver: Simulation::new checks (sim.rs:130-165), then
// run_until (sim.rs:231-245) with the forcings after each step. Runs until
// t_target, an error, or `stop_after` steps in this call (stop_after < 0:
// no limit; reaching it is not an error). t/steps are in-out (resume).
// dt_log (optional) receives each step's dt.
int hfo_sim_run(int64_t nr, int64_t nc, double dx, double dy, const double* z, const double* n,
                double* h, double* hu, double* hv, const hf_config* cfg, int64_t n_rain,
                const double* rain_t, const double* rain_v, int64_t n_src, const int64_t* rows,
                const int64_t* cols, const int64_t* offs, const double* src_t,
                const double* src_q, double t_target, int64_t stop_after, double* t_io,
                uint64_t* steps_io, double* dt_log, int64_t dt_log_cap, double* err_dt) {
  int rc = validate_cfg(cfg);
  if (rc) return rc;
  if (nr <= 0 || nc <= 0) return fail(HF_ERR_SHAPE_MISMATCH, "empty mesh");
  Boundaries b = to_bcs(&cfg->boundaries);
  rc = check_bcs(b, nr, nc);
  if (rc) return rc;
  for (int64_t k = 0; k < n_src; ++k)
    if (rows[k] < 0 || rows[k] >= nr || cols[k] < 0 || cols[k] >= nc)
      return fail(HF_ERR_INVALID_ARG, "point source outside the mesh");
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  auto s = load(nr * nc, h, hu, hv);
  Workspace<double> ws(nr, nc);
  Forcing f{n_rain, rain_t, rain_v, n_src, rows, cols, offs, src_t, src_q};
  uint64_t budget = cfg->max_steps;
  int64_t taken = 0;
  const GaugeRec gr = g_gauges;
  for (int64_t k = 0; k < gr.n; ++k) {
    gr.peak[k] = std::fmax(0.0, s[gr.cells[k]].h);
    gr.last[k] = s[gr.cells[k]].h;
  }
  rc = HF_OK;
  while (*t_io < t_target) {
    if (stop_after >= 0 && taken >= stop_after) break;
    if (budget == 0) {
      char buf[160];
      std::snprintf(buf, sizeof buf, "step budget exhausted: %llu steps, t = %g of %g s",
                    (unsigned long long)*steps_io, *t_io, t_target);
      rc = fail(HF_ERR_STEP_BUDGET, buf);
      break;
    }
    double dt = 0.0;
    rc = sim_step(s, m, *cfg, b, ws, f, t_target - *t_io, t_io, steps_io, &dt);
    if (rc) {
      if (err_dt) *err_dt = dt;
      break;
    }
    if (dt_log && taken < dt_log_cap) dt_log[taken] = dt;
    for (int64_t k = 0; k < gr.n; ++k) {
      const double v = s[gr.cells[k]].h;
      gr.peak[k] = std::fmax(gr.peak[k], v);
      gr.last[k] = v;
    }
    ++taken;
    --budget;
  }
  store(s, h, hu, hv);
  return rc;
}

void hfo_set_gauges(int64_t n, const int64_t* cells, double* peak, double* last) {
  g_gauges = GaugeRec{n, cells, peak, last};
}

// One Simulation::step(dt_cap) (+ forcings); t/steps in-out.
int hfo_sim_step(int64_t nr, int64_t nc, double dx, double dy, const double* z, const double* n,
                 double* h, double* hu, double* hv, const hf_config* cfg, int64_t n_rain,
                 const double* rain_t, const double* rain_v, int64_t n_src, const int64_t* rows,
                 const int64_t* cols, const int64_t* offs, const double* src_t,
                 const double* src_q, double dt_cap, double* t_io, uint64_t* steps_io,
                 double* dt_out) {
  int rc = validate_cfg(cfg);
  if (rc) return rc;
  Boundaries b = to_bcs(&cfg->boundaries);
  rc = check_bcs(b, nr, nc);
  if (rc) return rc;
  Mesh<double> m = make_mesh<double>(nr, nc, dx, dy, z, n);
  auto s = load(nr * nc, h, hu, hv);
  Workspace<double> ws(nr, nc);
  Forcing f{n_rain, rain_t, rain_v, n_src, rows, cols, offs, src_t, src_q};
  rc = sim_step(s, m, *cfg, b, ws, f, dt_cap, t_io, steps_io, dt_out);
  store(s, h, hu, hv);
  return rc;
}

// Forward-mode tangent run with T = Dual (the reference's generic code at
// T = Dual: autograd/src/dual.rs). The Manning field carries the tangent
// direction `dn`; the state carries (dh, dhu, dhv) in-out. Time steps come
// from the primal values (cfl_time_step reads .value(), update.rs:113-136),
// so dt is the primal run's dt. Follows the free-function loop of the
// reference's calibration demos: dt = min(cfl_time_step_with_bcs, max_dt,
// t_end - t); ssprk2_step; manning_friction_step(dry_tol); forcings.
// Optionally accumulates the gauge misfit J = sum over steps 1..n and
// gauges of (h - h_obs[step][g])^2 and its directional derivative dJ.
int hfo_tangent_run(int64_t nr, int64_t nc, double dx, double dy, const double* z,
                    const double* n, const double* dn, double* h, double* hu, double* hv,
                    double* dh, double* dhu, double* dhv, const hf_config* cfg, int64_t n_rain,
                    const double* rain_t, const double* rain_v, int64_t n_src,
                    const int64_t* rows, const int64_t* cols, const int64_t* offs,
                    const double* src_t, const double* src_q, int64_t n_steps,
                    const double* dts, int64_t n_gauges, const int64_t* gauge_cells,
                    const double* h_obs, double* J_out, double* dJ_out) {
  int rc = validate_cfg(cfg);
  if (rc) return rc;
  Boundaries b = to_bcs(&cfg->boundaries);
  rc = check_bcs(b, nr, nc);
  if (rc) return rc;
  Mesh<Dual> m = make_mesh<Dual>(nr, nc, dx, dy, z, n);
  for (int64_t k = 0; k < nr * nc; ++k) m.manning[k].dval = dn ? dn[k] : 0.0;
  std::vector<Cons<Dual>> s(nr * nc);
  for (int64_t k = 0; k < nr * nc; ++k)
    s[k] = Cons<Dual>{Dual{h[k], dh ? dh[k] : 0.0}, Dual{hu[k], dhu ? dhu[k] : 0.0},
                      Dual{hv[k], dhv ? dhv[k] : 0.0}};
  Workspace<Dual> ws(nr, nc);
  double t = 0.0;
  double J = 0.0, dJ = 0.0;
  for (int64_t step = 0; step < n_steps; ++step) {
    const double dt = dts[step];
    if (cfg->integrator == HF_FORWARD_EULER)
      forward_euler_step_with(s, m, b, dt, ws);
    else
      ssprk2_step_with(s, m, b, dt, ws);
    manning_friction_step(s, m, dt, cfg->friction_dry_tol);
    t += dt;
    if (n_rain > 0) apply_rain(s, series_eval(rain_t, rain_v, n_rain, t), dt);
    if (n_src > 0) {
      std::vector<PointSource> ps(n_src);
      for (int64_t k = 0; k < n_src; ++k) {
        int64_t a = offs[k], bb = offs[k + 1];
        ps[k] = PointSource{rows[k], cols[k], series_eval(src_t + a, src_q + a, bb - a, t)};
      }
      apply_point_sources(s, nc, ps.data(), n_src, dt, dx, dy);
    }
    for (int64_t g = 0; g < n_gauges; ++g) {
      const Dual hh = s[gauge_cells[g]].h;
      const double r = hh.val - h_obs[step * n_gauges + g];
      J += r * r;
      dJ += 2.0 * r * hh.dval;
    }
  }
  for (int64_t k = 0; k < nr * nc; ++k) {
    h[k] = s[k].h.val;
    hu[k] = s[k].hu.val;
    hv[k] = s[k].hv.val;
    if (dh) dh[k] = s[k].h.dval;
    if (dhu) dhu[k] = s[k].hu.dval;
    if (dhv) dhv[k] = s[k].hv.dval;
  }
  if (J_out) *J_out = J;
  if (dJ_out) *dJ_out = dJ;
  return HF_OK;
}

// Generic Dual evaluation of one forward-Euler or SSP-RK2 step with a single
// scalar seed applied to every cell's depth (update.rs:1954-1992) or to a
// uniform bed shift (update.rs:1995-2038). Returns (mass, d mass).
int hfo_dual_mass_step(int64_t nr, int64_t nc, double dx, double dy, int seed_bed, double seed,
                       double eta_or_h, int ssprk2, int bc_kind, double dt, double* mass,
                       double* dmass) {
  Mesh<Dual> m;
  m.nr = nr;
  m.nc = nc;
  m.dx = dx;
  m.dy = dy;
  Dual zval = seed_bed ? Dual{seed, 1.0} : Dual{0.0, 0.0};
  m.bed.assign(nr * nc, zval);
  m.manning.assign(nr * nc, Dual{0.0, 0.0});
  Dual hval = seed_bed ? (eta_or_h - zval) : Dual{seed, 1.0};
  std::vector<Cons<Dual>> s(nr * nc, Cons<Dual>{hval, Dual{0, 0}, Dual{0, 0}});
  Boundary bb{bc_kind, 0.0};
  Boundaries b{bb, bb, bb, bb};
  Workspace<Dual> ws(nr, nc);
  if (ssprk2)
    ssprk2_step_with(s, m, b, dt, ws);
  else
    forward_euler_step_with(s, m, b, dt, ws);
  Dual acc{0.0, 0.0};
  for (auto& c : s) acc = acc + c.h * (dx * dy);
  *mass = acc.val;
  *dmass = acc.dval;
  return HF_OK;
}

// Dual HLLC mass flux with h_l (or h_r) seeded (riemann.rs:428-471).
int hfo_dual_hllc_mass(int seed_right, const double* ul, const double* ur, double* val,
                       double* dval) {
  Cons<Dual> l{Dual{ul[0], seed_right ? 0.0 : 1.0}, Dual{ul[1], 0}, Dual{ul[2], 0}};
  Cons<Dual> r{Dual{ur[0], seed_right ? 1.0 : 0.0}, Dual{ur[1], 0}, Dual{ur[2], 0}};
  Flux<Dual> f = hllc_flux_x(l, r);
  *val = f.mass.val;
  *dval = f.mass.dval;
  return HF_OK;
}

// Dual Manning friction on one cell, seeding n (source.rs:420-446) or h
// with hu = h*u, hv = h*v (source.rs:448-473). Returns hu after one step.
int hfo_dual_friction_hu(int seed_h, double h, double u_or_hu, double v_or_hv, double n, double dt,
                         double dry_tol, double* val, double* dval) {
  Mesh<Dual> m;
  m.nr = 1;
  m.nc = 1;
  m.bed.assign(1, Dual{0, 0});
  m.manning.assign(1, seed_h ? Dual{n, 0.0} : Dual{n, 1.0});
  std::vector<Cons<Dual>> s(1);
  if (seed_h) {
    Dual hd{h, 1.0};
    s[0] = Cons<Dual>{hd, hd * u_or_hu, hd * v_or_hv};
  } else {
    s[0] = Cons<Dual>{Dual{h, 0}, Dual{u_or_hu, 0}, Dual{v_or_hv, 0}};
  }
  manning_friction_step(s, m, dt, dry_tol);
  *val = s[0].hu.val;
  *dval = s[0].hu.dval;
  return HF_OK;
}

}  // extern "C"
