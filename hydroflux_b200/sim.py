"""Host mirror of the reference crate's driver API over the C ABI.

Same names, argument meaning and error behaviour as hydroflux-solver-2d
(franciscoparrao/hydroflux): `Simulation` (solver-2d/src/sim.rs:119-245),
`SimulationConfig` (sim.rs:49-77), `Integrator` (sim.rs:38-46), `SimError`
(sim.rs:81-115), `Boundary` / `Boundaries2D` (boundary.rs:80-160),
`Mesh2D` (geometry.rs:31-47) and `PointSource` (source.rs:36-44). The state
lives on the GPU; `states()` returns host copies.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import threading
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import abi
from ._lib import last_error, lib

GRAVITY = abi.GRAVITY
H_DRY = abi.H_DRY
H_VEL = abi.H_VEL


class SimError(Exception):
    """Errors surfaced by the simulation driver (sim.rs:81-115)."""
    code = None


class ShapeMismatch(SimError):
    code = abi.HF_ERR_SHAPE_MISMATCH


class InvalidConfig(SimError):
    code = abi.HF_ERR_INVALID_CONFIG


class DegenerateDt(SimError):
    code = abi.HF_ERR_DEGENERATE_DT

    def __init__(self, msg, dt=None, t=None, step=None):
        super().__init__(msg)
        self.dt, self.t, self.step = dt, t, step


class StepBudgetExhausted(SimError):
    code = abi.HF_ERR_STEP_BUDGET

    def __init__(self, msg, steps=None, t=None, target=None):
        super().__init__(msg)
        self.steps, self.t, self.target = steps, t, target


class NonFinite(SimError):
    code = abi.HF_ERR_NONFINITE


class GpuError(SimError):
    code = abi.HF_ERR_CUDA


_BY_CODE = {c.code: c for c in (ShapeMismatch, InvalidConfig, DegenerateDt, StepBudgetExhausted,
                                NonFinite)}


def raise_for(rc: int, sim_handle=None, target=None):
    if rc == 0:
        return
    msg = last_error()
    cls = _BY_CODE.get(rc)
    if cls is DegenerateDt or cls is StepBudgetExhausted:
        dt, t, step = C.c_double(), C.c_double(), C.c_uint64()
        if sim_handle is not None:
            lib().hf_sim_error_detail(sim_handle, C.byref(dt), C.byref(t), C.byref(step))
        if cls is DegenerateDt:
            raise DegenerateDt(msg, dt.value, t.value, step.value)
        raise StepBudgetExhausted(msg, step.value, t.value, target)
    if cls is not None:
        raise cls(msg)
    if rc == abi.HF_ERR_INVALID_ARG:
        raise ValueError(msg)
    if rc == abi.HF_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise GpuError(f"status {rc}: {msg}")


class Integrator(enum.IntEnum):
    ForwardEuler = abi.HF_FORWARD_EULER
    SspRk2 = abi.HF_SSPRK2


class Side(enum.IntEnum):
    North = 0
    South = 1
    West = 2
    East = 3


@dataclass(frozen=True)
class Boundary:
    kind: int
    value: float = 0.0

    @staticmethod
    def transmissive():
        return Boundary(abi.HF_BC_TRANSMISSIVE)

    @staticmethod
    def wall():
        return Boundary(abi.HF_BC_WALL)

    @staticmethod
    def discharge(q: float):
        return Boundary(abi.HF_BC_DISCHARGE, float(q))

    @staticmethod
    def depth(h: float):
        return Boundary(abi.HF_BC_DEPTH, float(h))


@dataclass(frozen=True)
class Boundaries2D:
    north: Boundary
    south: Boundary
    west: Boundary
    east: Boundary

    def to_c(self) -> abi.hf_boundaries:
        return abi.make_boundaries(*[(b.kind, b.value) for b in
                                     (self.north, self.south, self.west, self.east)])


Boundaries2D.TRANSMISSIVE = Boundaries2D(*(Boundary.transmissive(),) * 4)
Boundaries2D.WALLS = Boundaries2D(*(Boundary.wall(),) * 4)


@dataclass
class SimulationConfig:
    cfl: float = 0.4
    integrator: Integrator = Integrator.SspRk2
    boundaries: Boundaries2D = field(default_factory=lambda: Boundaries2D.WALLS)
    max_steps: int = 10_000_000
    max_dt: float = 60.0
    friction_dry_tol: float = H_DRY
    check_finite: bool = False

    def to_c(self) -> abi.hf_config:
        return abi.hf_config(float(self.cfl), int(self.integrator), int(bool(self.check_finite)),
                             self.boundaries.to_c(), int(self.max_steps), float(self.max_dt),
                             float(self.friction_dry_tol))


_CHECK_POOL = None
_CHECK_LOCK = threading.Lock()
_CHECK_WORKERS = max(1, min(8, os.cpu_count() or 1))


def _all_nonnegative(a: np.ndarray) -> bool:
    """a.min() >= 0.0 over the whole field (a NaN fails). Large fields are
    reduced in contiguous chunks on a few threads (numpy releases the GIL in
    reductions); each chunk's minimum is tested on its own, so a NaN chunk
    fails whatever the order."""
    flat = a.reshape(-1)
    n = flat.size
    if n < (1 << 22) or _CHECK_WORKERS == 1:
        return bool(flat.min() >= 0.0)
    global _CHECK_POOL
    with _CHECK_LOCK:
        if _CHECK_POOL is None:
            from concurrent.futures import ThreadPoolExecutor
            _CHECK_POOL = ThreadPoolExecutor(max_workers=_CHECK_WORKERS)
    k = _CHECK_WORKERS
    cuts = [n * i // k for i in range(k + 1)]
    mins = list(_CHECK_POOL.map(lambda i: flat[cuts[i]:cuts[i + 1]].min(), range(k)))
    return all(bool(m >= 0.0) for m in mins)


class Mesh2D:
    """Mesh2D (geometry.rs:31-147). `manning` is a scalar (Mesh2D::new) or a
    field of the bed's shape (Mesh2D::with_manning_field)."""

    def __init__(self, bed, dx: float, dy: float, manning=0.0):
        bed = np.ascontiguousarray(bed, dtype=np.float64)
        if not dx > 0.0:
            raise ValueError(f"dx must be strictly positive (got {dx})")
        if not dy > 0.0:
            raise ValueError(f"dy must be strictly positive (got {dy})")
        if bed.ndim != 2 or bed.size == 0:
            raise ValueError("mesh must have at least one cell")
        if np.ndim(manning) == 0:
            if not float(manning) >= 0.0:
                raise ValueError(f"Manning n must be non-negative (got {manning})")
            manning = np.full(bed.shape, float(manning))
        else:
            manning = np.ascontiguousarray(manning, dtype=np.float64)
            if manning.shape != bed.shape:
                raise ValueError(f"manning field shape {manning.shape} must match bed shape "
                                 f"{bed.shape}")
            if not _all_nonnegative(manning):  # a NaN fails too
                raise ValueError("Manning n must be non-negative at every cell")
        self.bed, self.dx, self.dy, self.manning = bed, float(dx), float(dy), manning

    @classmethod
    def with_manning_field(cls, bed, dx, dy, manning):
        return cls(bed, dx, dy, np.asarray(manning, dtype=np.float64))

    def n_rows(self):
        return self.bed.shape[0]

    def n_cols(self):
        return self.bed.shape[1]

    def n_cells(self):
        return self.bed.size


@dataclass
class PointSource:
    """PointSource (source.rs:36-44) with a time series: q_mass may be a
    constant or a piecewise-linear series ((t0, q0), (t1, q1), ...)."""
    row: int
    col: int
    q_mass: object

    def series(self):
        if np.ndim(self.q_mass) == 0:
            return np.array([0.0]), np.array([float(self.q_mass)])
        pts = np.asarray(self.q_mass, dtype=np.float64).reshape(-1, 2)
        return pts[:, 0].copy(), pts[:, 1].copy()


class _CudaArray:
    """__cuda_array_interface__ view of device memory owned by a handle."""

    def __init__(self, ptr, shape, owner):
        self._owner = owner
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def _f64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _split_states(states, shape):
    if isinstance(states, (tuple, list)) and len(states) == 3:
        h, hu, hv = (np.ascontiguousarray(s, dtype=np.float64) for s in states)
    else:
        arr = np.ascontiguousarray(states, dtype=np.float64)
        if arr.ndim != 3 or arr.shape[2] != 3:
            raise ShapeMismatch(f"states shape {arr.shape} must be (rows, cols, 3) or (h, hu, hv)")
        h, hu, hv = (np.ascontiguousarray(arr[..., k]) for k in range(3))
    for s in (h, hu, hv):
        if s.shape != shape:
            raise ShapeMismatch(f"states shape {s.shape} must match mesh {shape}")
    return h, hu, hv


class Simulation:
    """Simulation (sim.rs:119-245) on a B200. One CUDA stream per handle."""

    def __init__(self, mesh: Mesh2D, states, config: Optional[SimulationConfig] = None,
                 device: int = 0):
        config = config or SimulationConfig()
        shape = mesh.bed.shape
        h, hu, hv = _split_states(states, shape)
        self._mesh = mesh
        self._config = config
        desc = abi.hf_mesh_desc(shape[0], shape[1], mesh.dx, mesh.dy, _f64p(mesh.bed),
                                _f64p(mesh.manning), 0.0)
        cfg = config.to_c()
        handle = C.c_void_p()
        rc = lib().hf_sim_create(C.byref(desc), _f64p(h), _f64p(hu), _f64p(hv), C.byref(cfg),
                                 int(device), C.byref(handle))
        raise_for(rc)
        self._h = handle
        self._shape = shape

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            lib().hf_sim_destroy(self._h)
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

    # -- driver
    def step(self, dt_cap: float = float("inf")) -> float:
        dt = C.c_double()
        raise_for(lib().hf_sim_step(self._h, float(dt_cap), C.byref(dt)), self._h)
        return dt.value

    def run_until(self, t_target: float) -> None:
        raise_for(lib().hf_sim_run_until(self._h, float(t_target)), self._h, t_target)

    def run_steps(self, n_steps: int, t_target: float = float("inf")) -> None:
        """Exactly n_steps steps (fewer if t_target is reached), no host
        round trip between them."""
        raise_for(lib().hf_sim_run_steps(self._h, int(n_steps), float(t_target)), self._h,
                  t_target)

    def run_steps_timed(self, n_steps: int, t_target: float = float("inf")):
        """run_steps with CUDA events around every stage kernel. Returns
        (summed stage-kernel ms, stage launches, region ms)."""
        st, tot = C.c_double(), C.c_double()
        nl = C.c_uint64()
        raise_for(lib().hf_sim_run_steps_timed(self._h, int(n_steps), float(t_target),
                                               C.byref(st), C.byref(nl), C.byref(tot)), self._h,
                  t_target)
        return st.value, nl.value, tot.value

    def time(self) -> float:
        t = C.c_double()
        raise_for(lib().hf_sim_time(self._h, C.byref(t)))
        return t.value

    def steps(self) -> int:
        s = C.c_uint64()
        raise_for(lib().hf_sim_steps(self._h, C.byref(s)))
        return s.value

    def mesh(self) -> Mesh2D:
        return self._mesh

    def states(self):
        """Host copies (h, hu, hv)."""
        h = np.empty(self._shape)
        hu = np.empty(self._shape)
        hv = np.empty(self._shape)
        raise_for(lib().hf_sim_get_state(self._h, h.ctypes.data, hu.ctypes.data, hv.ctypes.data))
        return h, hu, hv

    STAGE_KERNELS = {"auto": 0, "tile": 1, "strip": 2, "tile32": 3}

    def set_stage_kernel(self, kind: str) -> None:
        """'tile' (32 x 8 tiles), 'tile32' (32 x 32 tiles), 'strip' or 'auto'
        (hf_sim_set_stage_kernel): which kernel runs the stages; auto takes
        tile32 on grids of at least 100 tiles of 32 x 32, else tile. Results
        are bit-identical."""
        raise_for(lib().hf_sim_set_stage_kernel(self._h, self.STAGE_KERNELS[kind]))

    def stage_kernel(self) -> str:
        k = C.c_int()
        raise_for(lib().hf_sim_stage_kernel(self._h, C.byref(k)))
        return {v: n for n, v in self.STAGE_KERNELS.items()}[k.value]

    def max_depth_exceeds_relief(self, factor: float) -> bool:
        """max_depth_exceeds_relief(sim.states(), sim.mesh(), factor)
        (sim.rs:248-271): whether the largest depth exceeds `factor` times
        the bed's relief (floored at 1 m), reduced on the device."""
        out = C.c_int()
        raise_for(lib().hf_sim_max_depth_exceeds_relief(self._h, float(factor), C.byref(out)))
        return bool(out.value)

    def set_states(self, states) -> None:
        h, hu, hv = _split_states(states, self._shape)
        raise_for(lib().hf_sim_set_state(self._h, h.ctypes.data, hu.ctypes.data, hv.ctypes.data))

    def set_boundaries(self, bcs: Boundaries2D) -> None:
        c = bcs.to_c()
        raise_for(lib().hf_sim_set_boundaries(self._h, C.byref(c)))
        self._config.boundaries = bcs

    def set_rain(self, series) -> None:
        """series: constant rate [m/s], or ((t0, r0), (t1, r1), ...), or None."""
        if series is None:
            raise_for(lib().hf_sim_set_rain(self._h, 0, None, None))
            return
        if np.ndim(series) == 0:
            t, r = np.array([0.0]), np.array([float(series)])
        else:
            pts = np.asarray(series, dtype=np.float64).reshape(-1, 2)
            t, r = pts[:, 0].copy(), pts[:, 1].copy()
        raise_for(lib().hf_sim_set_rain(self._h, len(t), _f64p(t), _f64p(r)))

    def set_point_sources(self, sources: Sequence[PointSource]) -> None:
        rows = np.array([s.row for s in sources], dtype=np.int64)
        cols = np.array([s.col for s in sources], dtype=np.int64)
        ts, qs, offs = [], [], [0]
        for s in sources:
            t, q = s.series()
            ts.append(t)
            qs.append(q)
            offs.append(offs[-1] + len(t))
        t = np.concatenate(ts) if ts else np.zeros(1)
        q = np.concatenate(qs) if qs else np.zeros(1)
        offs = np.array(offs, dtype=np.int64)
        i64 = C.POINTER(C.c_int64)
        raise_for(lib().hf_sim_set_point_sources(
            self._h, len(sources), rows.ctypes.data_as(i64), cols.ctypes.data_as(i64),
            offs.ctypes.data_as(i64), _f64p(t), _f64p(q)))

    def set_rain_units(self, t_div: float = 1.0, v_mul: float = 1.0, v_div: float = 1.0) -> None:
        """The rain series is sampled at t / t_div and its value converted
        as (v * v_mul) / v_div: (60, 1e-3, 3600) for a hyetograph in minutes
        and mm/h, with the arithmetic of the reference's urban example
        (solver-2d/examples/uk_ea_test8a_official.rs:119-129)."""
        raise_for(lib().hf_sim_set_rain_units(self._h, float(t_div), float(v_mul), float(v_div)))

    def set_point_source_units(self, t_div: float = 1.0, v_mul: float = 1.0,
                               v_div: float = 1.0) -> None:
        """Units of every point-source series, as set_rain_units (the
        example's inflow: t_div = 60, v_mul = cellsize, ibid. 131-134)."""
        raise_for(lib().hf_sim_set_point_source_units(self._h, float(t_div), float(v_mul),
                                                      float(v_div)))

    def set_gauges(self, cells: Sequence[Tuple[int, int]], capacity: int = 1 << 20) -> None:
        """Record the depth at these (row, col) cells after every step, on
        the device: the control-point series and peaks the reference's
        urban example keeps (uk_ea_test8a_official.rs:187-246). Row 0 is the
        current state; at most `capacity` rows are stored."""
        cells = list(cells)
        rows = np.array([c[0] for c in cells] or [0], dtype=np.int64)
        cols = np.array([c[1] for c in cells] or [0], dtype=np.int64)
        i64 = C.POINTER(C.c_int64)
        raise_for(lib().hf_sim_set_gauges(self._h, len(cells), rows.ctypes.data_as(i64),
                                          cols.ctypes.data_as(i64), int(capacity)))
        self._n_gauges = len(cells)

    def gauge_peaks(self):
        """(peak, last) depth per gauge; peak = fold(0.0, f64::max) over
        every recorded depth."""
        n = getattr(self, "_n_gauges", 0)
        peak, last = np.empty(max(n, 1)), np.empty(max(n, 1))
        raise_for(lib().hf_sim_gauge_peaks(self._h, _f64p(peak), _f64p(last)))
        return peak[:n], last[:n]

    def gauge_series(self):
        """(t[rows], h[rows, gauges], rows seen): the stored rows."""
        n = getattr(self, "_n_gauges", 0)
        stored, seen = C.c_int64(), C.c_int64()
        raise_for(lib().hf_sim_gauge_series(self._h, None, None, C.byref(stored), C.byref(seen)))
        t = np.empty(max(stored.value, 1))
        h = np.empty((max(stored.value, 1), max(n, 1)))
        raise_for(lib().hf_sim_gauge_series(self._h, _f64p(t), _f64p(h), C.byref(stored),
                                            C.byref(seen)))
        return t[:stored.value], h[:stored.value, :n], seen.value

    def device_state(self):
        """Zero-copy torch views (h, hu, hv) of the resident state and the
        handle's CUDA stream pointer."""
        import torch
        ptrs = [C.c_void_p() for _ in range(4)]
        raise_for(lib().hf_sim_device_state(self._h, *[C.byref(p) for p in ptrs]))
        views = tuple(torch.as_tensor(_CudaArray(p.value, self._shape, self), device="cuda")
                      for p in ptrs[:3])
        return views + (ptrs[3].value,)
