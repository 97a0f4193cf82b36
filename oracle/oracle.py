"""ctypes wrapper of the CPU oracle (oracle/libhf_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the B200 kernels, and the timed
CPU reference arm of bench.py. Never part of the product path.

All arrays are numpy float64, row-major (n_rows, n_cols); the state is SoA
(h, hu, hv). Functions return new arrays and leave their inputs untouched.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from hydroflux_b200 import abi  # noqa: E402  (struct declarations only)

_LIB = None
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


def lib():
    global _LIB
    if _LIB is None:
        from oracle import build_oracle
        path = build_oracle.OUT
        if not os.path.exists(path):
            build_oracle.build()
        _LIB = C.CDLL(path)
        _LIB.hfo_last_error.restype = C.c_char_p
        _LIB.hfo_series_eval.restype = C.c_double
        _LIB.hfo_pow_port.restype = C.c_double
        _LIB.hfo_pow_port.argtypes = [C.c_double, C.c_double]
        _LIB.hfo_pow_mismatches.restype = C.c_int64
        _LIB.hfo_pow_mismatches.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_void_p]
        _LIB.hfo_set_series_units.restype = None
        _LIB.hfo_set_series_units.argtypes = [C.c_double] * 6
        _LIB.hfo_set_gauges.restype = None
        _LIB.hfo_set_gauges.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    return _LIB


def set_pow_mode(mode: str) -> None:
    """'libm' (the host C library's pow, which the Rust reference's
    f64::powf calls; default) or 'port' (the restatement of that library's
    algorithm in hydroflux_b200/csrc/hf_pow.h, which the GPU runs)."""
    if mode not in ("libm", "port"):
        raise ValueError(f"unknown pow mode {mode!r}")
    lib().hfo_set_pow_mode(1 if mode == "port" else 0)


def pow_port(x: float, y: float) -> float:
    """x^y by the restatement in hf_pow.h (host build)."""
    return lib().hfo_pow_port(float(x), float(y))


def pow_mismatches(x, y: float):
    """(count, first few x) of the x whose x^y differs bit for bit between
    the restatement and the host libm."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    first = np.full(8, np.nan)
    n = lib().hfo_pow_mismatches(x.size, x.ctypes.data, float(y), first.ctypes.data)
    return int(n), first[:min(int(n), 8)]


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle status {code}: {msg}")
        self.code = code


def _chk(rc):
    if rc != 0:
        raise OracleError(rc, lib().hfo_last_error().decode())
    return rc


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def _pi(a):
    if a is None:
        return None
    return a.ctypes.data_as(_I64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> int:
    return lib().hfo_set_threads(int(n))


def get_threads() -> int:
    return lib().hfo_get_threads()


def hllc_flux(x_dir: bool, ul, ur):
    out = np.zeros(3)
    _chk(lib().hfo_hllc_flux(int(bool(x_dir)), _p(_f64(ul)), _p(_f64(ur)), _p(out)))
    return out


def ghost_cell(z, n, dx, dy, kind, value, side, idx, inner):
    z = _f64(z)
    n = _f64(n) if n is not None else np.zeros_like(z)
    b = abi.hf_boundary(int(kind), 0, float(value))
    out = np.zeros(3)
    zb = C.c_double()
    _chk(lib().hfo_ghost_cell(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx),
                              C.c_double(dy), _p(z), _p(n), C.byref(b), int(side),
                              C.c_int64(idx), _p(_f64(inner)), _p(out), C.byref(zb)))
    return out, zb.value


SIDE = {"north": 0, "south": 1, "west": 2, "east": 3}


def max_wave_speeds(h, hu, hv):
    h, hu, hv = _f64(h), _f64(hu), _f64(hv)
    sx, sy = C.c_double(), C.c_double()
    _chk(lib().hfo_max_wave_speeds(C.c_int64(h.shape[0]), C.c_int64(h.shape[1]), _p(h), _p(hu),
                                   _p(hv), C.byref(sx), C.byref(sy)))
    return sx.value, sy.value


def cfl_time_step(z, dx, dy, h, hu, hv, cfl, bcs=None, n=None):
    z, h, hu, hv = _f64(z), _f64(h), _f64(hu), _f64(hv)
    n = _f64(n) if n is not None else np.zeros_like(z)
    out = C.c_double()
    _chk(lib().hfo_cfl_time_step(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx),
                                 C.c_double(dy), _p(z), _p(n), _p(h), _p(hu), _p(hv),
                                 C.byref(bcs) if bcs is not None else None, C.c_double(cfl),
                                 C.byref(out)))
    return out.value


def _step(fn, z, dx, dy, h, hu, hv, bcs, dt, n=None):
    z = _f64(z)
    n = _f64(n) if n is not None else np.zeros_like(z)
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    _chk(fn(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx), C.c_double(dy), _p(z),
            _p(n), _p(h), _p(hu), _p(hv), C.byref(bcs), C.c_double(dt)))
    return h, hu, hv


def forward_euler_step(z, dx, dy, h, hu, hv, bcs, dt, n=None):
    return _step(lib().hfo_forward_euler_step, z, dx, dy, h, hu, hv, bcs, dt, n)


def ssprk2_step(z, dx, dy, h, hu, hv, bcs, dt, n=None):
    return _step(lib().hfo_ssprk2_step, z, dx, dy, h, hu, hv, bcs, dt, n)


def manning_friction_step(n, h, hu, hv, dt, dry_tol):
    n = _f64(n)
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    _chk(lib().hfo_manning_friction_step(C.c_int64(h.shape[0]), C.c_int64(h.shape[1]), _p(n),
                                         _p(h), _p(hu), _p(hv), C.c_double(dt),
                                         C.c_double(dry_tol)))
    return h, hu, hv


def apply_rain(h, hu, hv, rate, dt):
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    _chk(lib().hfo_apply_rain(C.c_int64(h.size), _p(h), _p(hu), _p(hv), C.c_double(rate),
                              C.c_double(dt)))
    return h, hu, hv


def apply_point_sources(h, hu, hv, sources, dt, dx, dy):
    """sources: list of (row, col, q_mass)."""
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    rows = np.array([s[0] for s in sources], dtype=np.int64)
    cols = np.array([s[1] for s in sources], dtype=np.int64)
    q = np.array([s[2] for s in sources], dtype=np.float64)
    _chk(lib().hfo_apply_point_sources(C.c_int64(h.shape[0]), C.c_int64(h.shape[1]), _p(h),
                                       _p(hu), _p(hv), C.c_int64(len(sources)), _pi(rows),
                                       _pi(cols), _p(q), C.c_double(dt), C.c_double(dx),
                                       C.c_double(dy)))
    return h, hu, hv


def max_depth_exceeds_relief(h, z, factor):
    """max_depth_exceeds_relief (solver-2d/src/sim.rs:262-271), restated:
    the depth max folds from 0.0 and the bed's max/min from -inf/+inf with
    f64::max/min, which skip NaN (np.fmax/np.fmin do the same); the relief
    is floored at 1 m with f64::max (NaN gives 1)."""
    max_depth = float(np.fmax.reduce(np.ravel(h), initial=0.0))
    bed_max = float(np.fmax.reduce(np.ravel(z), initial=-np.inf))
    bed_min = float(np.fmin.reduce(np.ravel(z), initial=np.inf))
    relief = float(np.fmax(bed_max - bed_min, 1.0))
    return max_depth > factor * relief


def series_eval(t, v, x):
    t, v = _f64(t), _f64(v)
    return lib().hfo_series_eval(_p(t), _p(v), C.c_int64(len(t)), C.c_double(x))


class Forcing:
    """Rain series and point-source series (host side of hf_sim_set_rain /
    hf_sim_set_point_sources)."""

    def __init__(self, rain=None, sources=None, rain_units=(1.0, 1.0, 1.0),
                 src_units=(1.0, 1.0, 1.0)):
        # rain: (t array, rate array) or None; sources: list of (row, col, t array, q array);
        # units: (t_div, v_mul, v_div) of each series (hf_sim_set_rain_units)
        self.rain_units = tuple(float(u) for u in rain_units)
        self.src_units = tuple(float(u) for u in src_units)
        self.rain_t = _f64(rain[0]) if rain is not None else np.zeros(0)
        self.rain_v = _f64(rain[1]) if rain is not None else np.zeros(0)
        sources = sources or []
        self.rows = np.array([s[0] for s in sources], dtype=np.int64)
        self.cols = np.array([s[1] for s in sources], dtype=np.int64)
        offs = [0]
        ts, qs = [], []
        for s in sources:
            ts.append(_f64(s[2]))
            qs.append(_f64(s[3]))
            offs.append(offs[-1] + len(s[2]))
        self.offs = np.array(offs, dtype=np.int64)
        self.src_t = np.concatenate(ts) if ts else np.zeros(0)
        self.src_q = np.concatenate(qs) if qs else np.zeros(0)

    def args(self):
        # the units travel through a setter read when the oracle call starts
        lib().hfo_set_series_units(*self.rain_units, *self.src_units)
        return (C.c_int64(len(self.rain_t)), _p(self.rain_t), _p(self.rain_v),
                C.c_int64(len(self.rows)), _pi(self.rows), _pi(self.cols), _pi(self.offs),
                _p(self.src_t), _p(self.src_q))


def sim_run(z, n, dx, dy, h, hu, hv, cfg, t_target, forcing=None, stop_after=-1, t0=0.0,
            steps0=0, dt_log_cap=0, gauges=None):
    """Simulation::run_until semantics (+ forcings). Returns dict with state,
    t, steps, status, dts (first dt_log_cap step sizes) and err_dt; with
    gauges (flat cell indices), also their peaks (fold(0.0, max) over the
    initial and every stepped depth) and last depths."""
    z = _f64(z)
    n = _f64(n) if n is not None else np.zeros_like(z)
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    forcing = forcing or Forcing()
    t = C.c_double(t0)
    steps = C.c_uint64(steps0)
    dts = np.zeros(max(dt_log_cap, 1))
    err_dt = C.c_double(0.0)
    g_cells = np.ascontiguousarray(gauges if gauges is not None else [], dtype=np.int64)
    g_peak, g_last = np.zeros(max(len(g_cells), 1)), np.zeros(max(len(g_cells), 1))
    lib().hfo_set_gauges(len(g_cells), g_cells.ctypes.data, g_peak.ctypes.data,
                         g_last.ctypes.data)
    try:
        rc = _sim_run_call(z, n, dx, dy, h, hu, hv, cfg, t_target, forcing, stop_after, t, steps,
                           dts, dt_log_cap, err_dt)
    finally:
        lib().hfo_set_gauges(0, None, None, None)
    msg = lib().hfo_last_error().decode() if rc else ""
    out = dict(h=h, hu=hu, hv=hv, t=t.value, steps=steps.value, status=rc, message=msg,
               dts=dts[:min(dt_log_cap, steps.value - steps0)], err_dt=err_dt.value)
    if gauges is not None:
        out["gauge_peak"], out["gauge_last"] = g_peak[:len(g_cells)], g_last[:len(g_cells)]
    return out


def _sim_run_call(z, n, dx, dy, h, hu, hv, cfg, t_target, forcing, stop_after, t, steps, dts,
                  dt_log_cap, err_dt):
    return lib().hfo_sim_run(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx),
                           C.c_double(dy), _p(z), _p(n), _p(h), _p(hu), _p(hv), C.byref(cfg),
                           *forcing.args(), C.c_double(t_target), C.c_int64(stop_after),
                           C.byref(t), C.byref(steps), _p(dts), C.c_int64(dt_log_cap),
                           C.byref(err_dt))


def sim_step(z, n, dx, dy, h, hu, hv, cfg, dt_cap, forcing=None, t0=0.0, steps0=0):
    z = _f64(z)
    n = _f64(n) if n is not None else np.zeros_like(z)
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    forcing = forcing or Forcing()
    t = C.c_double(t0)
    steps = C.c_uint64(steps0)
    dt = C.c_double(0.0)
    rc = lib().hfo_sim_step(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx),
                            C.c_double(dy), _p(z), _p(n), _p(h), _p(hu), _p(hv), C.byref(cfg),
                            *forcing.args(), C.c_double(dt_cap), C.byref(t), C.byref(steps),
                            C.byref(dt))
    msg = lib().hfo_last_error().decode() if rc else ""
    return dict(h=h, hu=hu, hv=hv, t=t.value, steps=steps.value, status=rc, message=msg,
                dt=dt.value)


def tangent_run(z, n, dn, dx, dy, h, hu, hv, cfg, dts, forcing=None, dh=None, dhu=None,
                dhv=None, gauges=None, h_obs=None):
    """Forward-mode (Dual) run over the given dt schedule. Returns primal
    state, tangent state, J and dJ (gauge misfit, if gauges given)."""
    z, n = _f64(z), _f64(n)
    dn = _f64(dn) if dn is not None else np.zeros_like(z)
    h, hu, hv = _f64(h).copy(), _f64(hu).copy(), _f64(hv).copy()
    dh = _f64(dh).copy() if dh is not None else np.zeros_like(h)
    dhu = _f64(dhu).copy() if dhu is not None else np.zeros_like(h)
    dhv = _f64(dhv).copy() if dhv is not None else np.zeros_like(h)
    dts = _f64(dts)
    forcing = forcing or Forcing()
    gauges = np.zeros(0, dtype=np.int64) if gauges is None else np.ascontiguousarray(gauges, np.int64)
    h_obs = np.zeros(0) if h_obs is None else _f64(h_obs)
    J, dJ = C.c_double(0.0), C.c_double(0.0)
    _chk(lib().hfo_tangent_run(C.c_int64(z.shape[0]), C.c_int64(z.shape[1]), C.c_double(dx),
                               C.c_double(dy), _p(z), _p(n), _p(dn), _p(h), _p(hu), _p(hv),
                               _p(dh), _p(dhu), _p(dhv), C.byref(cfg), *forcing.args(),
                               C.c_int64(len(dts)), _p(dts), C.c_int64(len(gauges)), _pi(gauges),
                               _p(h_obs), C.byref(J), C.byref(dJ)))
    return dict(h=h, hu=hu, hv=hv, dh=dh, dhu=dhu, dhv=dhv, J=J.value, dJ=dJ.value)


def dual_mass_step(nr, nc, dx, dy, seed_bed, seed, eta_or_h, ssprk2, bc_kind, dt):
    m, dm = C.c_double(), C.c_double()
    _chk(lib().hfo_dual_mass_step(C.c_int64(nr), C.c_int64(nc), C.c_double(dx), C.c_double(dy),
                                  int(seed_bed), C.c_double(seed), C.c_double(eta_or_h),
                                  int(ssprk2), int(bc_kind), C.c_double(dt), C.byref(m),
                                  C.byref(dm)))
    return m.value, dm.value


def dual_hllc_mass(seed_right, ul, ur):
    v, d = C.c_double(), C.c_double()
    _chk(lib().hfo_dual_hllc_mass(int(seed_right), _p(_f64(ul)), _p(_f64(ur)), C.byref(v),
                                  C.byref(d)))
    return v.value, d.value


def dual_friction_hu(seed_h, h, a, b, n, dt, dry_tol):
    v, d = C.c_double(), C.c_double()
    _chk(lib().hfo_dual_friction_hu(int(seed_h), C.c_double(h), C.c_double(a), C.c_double(b),
                                    C.c_double(n), C.c_double(dt), C.c_double(dry_tol),
                                    C.byref(v), C.byref(d)))
    return v.value, d.value
