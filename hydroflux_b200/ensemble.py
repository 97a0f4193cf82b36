"""Ensembles of independent flood scenarios advanced together on one GPU.

Each scenario behaves like its own `Simulation` run to its horizon
(Simulation::run_until, solver-2d/src/sim.rs:231-245): own grid size, bed,
roughness, forcings, CFL dt, clock, step budget and errors. One batch step
advances every unfinished scenario by one of its own steps with a single
persistent launch per stage over the tiles of all scenarios (hf_batch_* in
include/hydroflux_gpu.h); a scenario large enough to fill the GPU by itself
(512 or more tiles of 32 x 32) runs its stages as its own launches in the
same step. Results are bit-identical to separate solves.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import abi
from ._lib import lib
from .sim import raise_for
from .workloads import Scenario

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None and a.size else None


def _ip(a):
    return a.ctypes.data_as(_I64) if a is not None and a.size else None


def scenario_config(s: Scenario, max_steps: int = 10_000_000) -> abi.hf_config:
    return abi.make_config(cfl=s.cfl, boundaries=abi.make_boundaries(*s.bcs), max_dt=s.max_dt,
                           max_steps=max_steps, integrator=s.integrator)


class _Desc:
    """hf_scenario_desc plus the arrays it points to (kept alive)."""

    def __init__(self, s: Scenario, max_steps: int):
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        self.bed, self.man = f64(s.bed), f64(s.manning)
        self.h, self.hu, self.hv = f64(s.h), f64(s.hu), f64(s.hv)
        self.rain_t = f64(s.rain[0]) if s.rain is not None else np.zeros(0)
        self.rain_v = f64(s.rain[1]) if s.rain is not None else np.zeros(0)
        self.rows = np.array([x[0] for x in s.sources], dtype=np.int64)
        self.cols = np.array([x[1] for x in s.sources], dtype=np.int64)
        offs = [0]
        for x in s.sources:
            offs.append(offs[-1] + len(x[2]))
        self.offs = np.array(offs, dtype=np.int64)
        self.st = np.concatenate([f64(x[2]) for x in s.sources]) if s.sources else np.zeros(0)
        self.sq = np.concatenate([f64(x[3]) for x in s.sources]) if s.sources else np.zeros(0)
        nr, nc = self.bed.shape
        mesh = abi.hf_mesh_desc(nr, nc, s.dx, s.dy, _dp(self.bed), _dp(self.man), 0.0)
        self.c = abi.hf_scenario_desc(
            mesh, _dp(self.h), _dp(self.hu), _dp(self.hv), scenario_config(s, max_steps),
            float(s.t_end), len(self.rain_t), _dp(self.rain_t), _dp(self.rain_v),
            len(self.rows), _ip(self.rows), _ip(self.cols), _ip(self.offs), _dp(self.st),
            _dp(self.sq))


class Ensemble:
    def __init__(self, scenarios: Sequence[Scenario], device: int = 0,
                 max_steps: int = 10_000_000):
        self._shapes = [s.shape for s in scenarios]
        descs = [_Desc(s, max_steps) for s in scenarios]
        arr = (abi.hf_scenario_desc * len(descs))(*[d.c for d in descs])
        h = C.c_void_p()
        raise_for(lib().hf_batch_create(len(descs), arr, int(device), C.byref(h)))
        self._h = h

    def __len__(self):
        return len(self._shapes)

    def run(self, max_batch_steps: int = 1 << 62) -> int:
        """Advance; returns the number of scenarios still running."""
        left = C.c_int64()
        raise_for(lib().hf_batch_run(self._h, int(max_batch_steps), C.byref(left)))
        return left.value

    SCHEDULES = {0: "static, scenario order", 1: "dynamic, scenario order",
                 2: "static, largest first", 3: "dynamic, largest first"}

    def set_schedule(self, schedule: int = -1) -> None:
        """Tile schedule of the batched kernel (-1: autotune on the first
        run of >= 64 steps); no schedule changes any result."""
        raise_for(lib().hf_batch_set_schedule(self._h, int(schedule)))

    def schedule(self):
        """(schedule in use, -1 before tuning; per-candidate tuning ms)."""
        sc = C.c_int()
        ms = np.zeros(4)
        raise_for(lib().hf_batch_schedule(self._h, C.byref(sc), ms.ctypes.data_as(
            C.POINTER(C.c_double))))
        return sc.value, ms

    def info(self, k: int):
        t, st, status = C.c_double(), C.c_uint64(), C.c_int()
        raise_for(lib().hf_batch_scenario_info(self._h, int(k), C.byref(t), C.byref(st),
                                               C.byref(status)))
        return {"t": t.value, "steps": st.value, "status": status.value}

    def states(self, k: int):
        shape = self._shapes[k]
        out = [np.empty(shape) for _ in range(3)]
        raise_for(lib().hf_batch_get_state(self._h, int(k), *[o.ctypes.data for o in out]))
        return tuple(out)

    def close(self):
        if getattr(self, "_h", None):
            lib().hf_batch_destroy(self._h)
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


def ensemble_scenarios(count: int = 512, seed: int = 0, side_lo: int = 64, side_hi: int = 1024,
                       horizon: float = 1800.0, dx: float = 5.0) -> List[Scenario]:
    """The ensemble workload: sides log-uniform in [side_lo, side_hi] (square,
    not padded), the valley generator with a per-scenario seed, a uniform
    Manning n ~ U[0.02, 0.08] per scenario, inflow peak 500 m^3/s scaled by
    U[0.5, 2], horizon `horizon` seconds each."""
    from .workloads import uniform, valley
    u_side = uniform(seed, 100, count)
    u_n = uniform(seed, 101, count, 0.02, 0.08)
    u_peak = uniform(seed, 102, count, 0.5, 2.0)
    out = []
    for k in range(count):
        side = int(round(float(np.exp(np.log(side_lo) + u_side[k] * (np.log(side_hi)
                                                                      - np.log(side_lo))))))
        s = valley(n=side, dx=dx, seed=seed * 100003 + k + 1, peak=500.0 * float(u_peak[k]),
                   t_end=horizon, manning=np.full((side, side), float(u_n[k])))
        s.name = f"ens{k}_{side}"
        out.append(s)
    return out
