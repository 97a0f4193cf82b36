"""Gauge-misfit calibration of the Manning field: forward runs, the
forward-mode (Dual) tangent and the reverse-mode (adjoint) gradient on the GPU
(hf_calib_*, hf_tangent, hf_grad_manning in include/hydroflux_gpu.h).

The reference differentiates by running its generic step with T = Dual
(solver-2d/examples/m1_inverse_manning_demo.rs:84-110); `Calibration.tangent`
is that, and `Calibration.gradient` gives dJ/dn for every cell at once, the
transpose of the same tangent map (dt frozen to the primal run, branches on
values), with checkpointed recomputation.

    J = sum over steps k = 1..K and gauges g of (h_k[cell_g] - h_obs[k-1, g])^2
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from ._lib import lib
from .ensemble import _Desc
from .sim import raise_for
from .workloads import Scenario

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _f64(a, n=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class Calibration:
    """A misfit problem: scenario + gauges, up to `n_steps` steps (or t_end)."""

    def __init__(self, scenario: Scenario, n_steps: int, gauges: Sequence[int] = (),
                 checkpoint_every: int = 45, device: int = 0):
        self.shape = scenario.shape
        self.ncell = scenario.n_cells
        self.n_steps = int(n_steps)
        self.gauges = np.ascontiguousarray(gauges, dtype=np.int64).reshape(-1)
        self._desc = _Desc(scenario, 10_000_000)
        h = C.c_void_p()
        raise_for(lib().hf_calib_create(C.byref(self._desc.c), self.n_steps, len(self.gauges),
                                        self.gauges.ctypes.data_as(_I64) if self.gauges.size
                                        else None, int(checkpoint_every), int(device),
                                        C.byref(h)))
        self._h = h

    def set_observations(self, h_obs: np.ndarray) -> None:
        obs = _f64(h_obs, self.n_steps * len(self.gauges))
        raise_for(lib().hf_calib_set_observations(self._h, _dp(obs)))

    def run(self, manning, replay_dt: bool = False):
        """(J, gauge depths [K, G], K). replay_dt: frozen dt of the last run."""
        n = _f64(manning, self.ncell)
        gh = np.zeros(max(self.n_steps * len(self.gauges), 1))
        J, k = C.c_double(), C.c_int64()
        raise_for(lib().hf_calib_run(self._h, _dp(n), int(bool(replay_dt)), C.byref(J), _dp(gh),
                                     C.byref(k)))
        G = len(self.gauges)
        return J.value, gh[:k.value * G].reshape(k.value, G), k.value

    def tangent(self, manning, dn=None, dh0=None, dhu0=None, dhv0=None):
        """(J, dJ) along the direction (dn, dh0, dhu0, dhv0)."""
        arrs = [_f64(a, self.ncell) for a in (manning, dn, dh0, dhu0, dhv0)]
        J, dJ = C.c_double(), C.c_double()
        raise_for(lib().hf_tangent(self._h, *[_dp(a) for a in arrs], C.byref(J), C.byref(dJ)))
        return J.value, dJ.value

    def tangent_lanes(self, manning, dn=None, dh0=None, dhu0=None, dhv0=None):
        """Vector mode (DualN, autograd/src/dual_n.rs): (J, dJ[lanes]) for
        `lanes` directions in one run. Each direction argument is None or an
        array of shape (lanes, rows, cols); the lane count is their first
        dimension. Every lane equals `tangent` along its direction bitwise."""
        dirs = [a for a in (dn, dh0, dhu0, dhv0) if a is not None]
        if not dirs:
            raise ValueError("give at least one direction array of shape (lanes, rows, cols)")
        lanes = int(np.shape(dirs[0])[0])
        n = _f64(manning, self.ncell)
        arrs = [None if a is None else _f64(a, lanes * self.ncell) for a in (dn, dh0, dhu0, dhv0)]
        J = C.c_double()
        dJ = np.zeros(lanes)
        raise_for(lib().hf_tangent_lanes(self._h, _dp(n), lanes, *[_dp(a) for a in arrs],
                                         C.byref(J), _dp(dJ)))
        self._lanes = lanes
        return J.value, dJ

    def lane_state(self, lane: int) -> dict:
        """Final tangent (dh, dhu, dhv) of one lane of the last tangent_lanes."""
        out = {k: np.zeros(self.shape) for k in ("dh", "dhu", "dhv")}
        raise_for(lib().hf_calib_lane_state(self._h, int(lane), *[_dp(out[k]) for k in
                                                                  ("dh", "dhu", "dhv")]))
        return out

    def gradient(self, manning, initial_state: bool = False):
        """(J, dJ/dn) or, with initial_state, (J, dJ/dn, (dJ/dh0, dJ/dhu0, dJ/dhv0))."""
        n = _f64(manning, self.ncell)
        g = np.zeros(self.ncell)
        g0 = [np.zeros(self.ncell) for _ in range(3)] if initial_state else [None] * 3
        J = C.c_double()
        raise_for(lib().hf_grad_manning(self._h, _dp(n), C.byref(J), _dp(g), *[_dp(a) for a in g0]))
        shape = self.shape
        if initial_state:
            return J.value, g.reshape(shape), tuple(a.reshape(shape) for a in g0)
        return J.value, g.reshape(shape)

    def final_state(self) -> dict:
        out = {k: np.zeros(self.shape) for k in ("h", "hu", "hv", "dh", "dhu", "dhv")}
        raise_for(lib().hf_calib_final_state(self._h, *[_dp(out[k]) for k in
                                                        ("h", "hu", "hv", "dh", "dhu", "dhv")]))
        return out

    def dts(self) -> np.ndarray:
        n = C.c_int64()
        raise_for(lib().hf_calib_dt(self._h, None, C.byref(n)))
        out = np.zeros(max(n.value, 1))
        raise_for(lib().hf_calib_dt(self._h, _dp(out), C.byref(n)))
        return out[:n.value]

    def close(self):
        if getattr(self, "_h", None):
            lib().hf_calib_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
