"""The reference's free functions over device-resident torch tensors.

Mirrors solver-2d's re-exports (lib.rs:74-91): `cfl_time_step`,
`cfl_time_step_with_bcs`, `forward_euler_step(_with)`, `ssprk2_step(_with)`,
`manning_friction_step`, `apply_rain`, `apply_point_sources`,
`max_depth_exceeds_relief` (sim.rs:262), and the `StepWorkspace2D` scratch
object. Arrays are float64 CUDA tensors of shape
(n_rows, n_cols); steps mutate h/hu/hv in place on torch's current stream.
Shape mismatches raise ValueError where the reference panics.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import abi
from ._lib import lib
from .sim import Boundaries2D, raise_for


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(t, shape=None, name="tensor"):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64:
        raise TypeError(f"{name} must be a float64 CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"states shape {tuple(t.shape)} must match mesh {tuple(shape)}")
    return C.c_void_p(t.data_ptr())


class DeviceMesh:
    """Mesh2D with bed and Manning field resident on the GPU."""

    def __init__(self, bed, dx: float, dy: float, manning=0.0, device=None):
        import torch
        device = device or torch.device("cuda")
        bed = torch.as_tensor(np.asarray(bed, dtype=np.float64) if not isinstance(bed, torch.Tensor)
                              else bed, dtype=torch.float64, device=device).contiguous()
        if np.ndim(manning) == 0 and not isinstance(manning, torch.Tensor):
            man = torch.full_like(bed, float(manning))
        else:
            man = torch.as_tensor(manning, dtype=torch.float64, device=device).contiguous()
        if man.shape != bed.shape:
            raise ValueError(f"manning field shape {tuple(man.shape)} must match bed shape "
                             f"{tuple(bed.shape)}")
        if not (dx > 0 and dy > 0):
            raise ValueError("dx and dy must be strictly positive")
        self.bed, self.manning, self.dx, self.dy = bed, man, float(dx), float(dy)
        self.shape = tuple(bed.shape)

    def grid(self) -> abi.hf_grid:
        return abi.hf_grid(self.shape[0], self.shape[1], self.dx, self.dy,
                           C.c_void_p(self.bed.data_ptr()), C.c_void_p(self.manning.data_ptr()))


class StepWorkspace2D:
    """StepWorkspace2D (update.rs:743-777): stage buffer + reduction scratch."""

    def __init__(self, n_rows: int, n_cols: int, device: int = None):
        import torch
        if device is None:
            device = torch.cuda.current_device()
        h = C.c_void_p()
        raise_for(lib().hf_workspace_create(int(n_rows), int(n_cols), int(device), C.byref(h)))
        self._h = h
        self.shape = (n_rows, n_cols)

    @classmethod
    def for_mesh(cls, mesh: DeviceMesh):
        return cls(*mesh.shape)

    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().hf_workspace_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _bcs(bcs: Optional[Boundaries2D]):
    return C.byref(bcs.to_c()) if bcs is not None else None


def cfl_time_step_with_bcs(h, hu, hv, mesh: DeviceMesh, bcs: Optional[Boundaries2D], cfl: float,
                           ws: Optional[StepWorkspace2D] = None) -> float:
    g = mesh.grid()
    ws = ws or StepWorkspace2D(*mesh.shape)
    out = C.c_double()
    raise_for(lib().hf_cfl_time_step(C.byref(g), _check(h, mesh.shape, "h"),
                                     _check(hu, mesh.shape, "hu"), _check(hv, mesh.shape, "hv"),
                                     _bcs(bcs), float(cfl), ws.handle(), _stream(), C.byref(out)))
    return out.value


def cfl_time_step(h, hu, hv, mesh: DeviceMesh, cfl: float, ws=None) -> float:
    return cfl_time_step_with_bcs(h, hu, hv, mesh, None, cfl, ws)


def forward_euler_step(h, hu, hv, mesh: DeviceMesh, bcs: Boundaries2D, dt: float,
                       ws: Optional[StepWorkspace2D] = None):
    ws = ws or StepWorkspace2D(*mesh.shape)
    g = mesh.grid()
    raise_for(lib().hf_forward_euler_step(C.byref(g), _check(h, mesh.shape, "h"),
                                          _check(hu, mesh.shape, "hu"),
                                          _check(hv, mesh.shape, "hv"), _bcs(bcs), float(dt),
                                          ws.handle(), _stream()))


forward_euler_step_with = forward_euler_step


def ssprk2_step(h, hu, hv, mesh: DeviceMesh, bcs: Boundaries2D, dt: float,
                ws: Optional[StepWorkspace2D] = None):
    ws = ws or StepWorkspace2D(*mesh.shape)
    g = mesh.grid()
    raise_for(lib().hf_ssprk2_step(C.byref(g), _check(h, mesh.shape, "h"),
                                   _check(hu, mesh.shape, "hu"), _check(hv, mesh.shape, "hv"),
                                   _bcs(bcs), float(dt), ws.handle(), _stream()))


ssprk2_step_with = ssprk2_step


def manning_friction_step(h, hu, hv, mesh: DeviceMesh, dt: float, dry_tol: float):
    g = mesh.grid()
    raise_for(lib().hf_manning_friction_step(C.byref(g), _check(h, mesh.shape, "h"),
                                             _check(hu, mesh.shape, "hu"),
                                             _check(hv, mesh.shape, "hv"), float(dt),
                                             float(dry_tol), _stream()))


def max_depth_exceeds_relief(h, mesh: DeviceMesh, factor: float,
                             ws: Optional[StepWorkspace2D] = None) -> bool:
    """max_depth_exceeds_relief (sim.rs:248-271) on a device depth field."""
    ws = ws or StepWorkspace2D(*mesh.shape)
    g = mesh.grid()
    out = C.c_int()
    raise_for(lib().hf_max_depth_exceeds_relief(C.byref(g), _check(h, mesh.shape, "h"),
                                                float(factor), ws.handle(), _stream(),
                                                C.byref(out)))
    return bool(out.value)


def apply_rain(h, hu, hv, rate: float, dt: float):
    n = h.numel()
    raise_for(lib().hf_apply_rain(n, _check(h, None, "h"), _check(hu, h.shape, "hu"),
                                  _check(hv, h.shape, "hv"), float(rate), float(dt), _stream()))


def apply_point_sources(h, hu, hv, sources: Sequence, dt: float, dx: float, dy: float):
    """sources: PointSource objects or (row, col, q_mass) tuples."""
    rows = np.array([getattr(s, "row", s[0] if isinstance(s, tuple) else None) for s in sources],
                    dtype=np.int64)
    cols = np.array([getattr(s, "col", s[1] if isinstance(s, tuple) else None) for s in sources],
                    dtype=np.int64)
    q = np.array([float(getattr(s, "q_mass", s[2] if isinstance(s, tuple) else 0.0))
                  for s in sources], dtype=np.float64)
    g = abi.hf_grid(h.shape[0], h.shape[1], float(dx), float(dy), None, None)
    i64 = C.POINTER(C.c_int64)
    raise_for(lib().hf_apply_point_sources(
        C.byref(g), _check(h, None, "h"), _check(hu, h.shape, "hu"), _check(hv, h.shape, "hv"),
        len(rows), rows.ctypes.data_as(i64), cols.ctypes.data_as(i64),
        q.ctypes.data_as(C.POINTER(C.c_double)), float(dt), _stream()))


def hllc_flux(x_dir: bool, ul, ur):
    """hllc_flux_x / hllc_flux_y over n faces: ul, ur are (n, 3) CUDA tensors."""
    import torch
    n = ul.shape[0]
    out = torch.empty((n, 3), dtype=torch.float64, device=ul.device)
    raise_for(lib().hf_hllc_flux(int(bool(x_dir)), n, _check(ul, (n, 3), "ul"),
                                 _check(ur, (n, 3), "ur"), _check(out, (n, 3), "out"), _stream()))
    return out
