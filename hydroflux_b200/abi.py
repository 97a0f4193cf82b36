"""ctypes mirrors of the structs and constants in include/hydroflux_gpu.h.

Pure declarations: importing this module loads no shared library.
"""
from __future__ import annotations

import ctypes as C

HF_ABI_VERSION = 1

HF_OK = 0
HF_ERR_SHAPE_MISMATCH = -1
HF_ERR_INVALID_CONFIG = -2
HF_ERR_DEGENERATE_DT = -3
HF_ERR_STEP_BUDGET = -4
HF_ERR_NONFINITE = -5
HF_ERR_TIMEOUT = -6
HF_ERR_CUDA = -7
HF_ERR_INVALID_ARG = -8
HF_ERR_OUT_OF_MEMORY = -9
HF_ERR_UNSUPPORTED = -10
HF_ERR_CAPACITY = -11

HF_BC_TRANSMISSIVE = 0
HF_BC_WALL = 1
HF_BC_DISCHARGE = 2
HF_BC_DEPTH = 3

HF_FORWARD_EULER = 0
HF_SSPRK2 = 1

# Physical constants of the reference (solver-2d/src/lib.rs:43, 63, 72).
GRAVITY = 9.81
H_DRY = 1.0e-6
H_VEL = 1.0e-5


class hf_boundary(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("value", C.c_double)]


class hf_boundaries(C.Structure):
    _fields_ = [("north", hf_boundary), ("south", hf_boundary),
                ("west", hf_boundary), ("east", hf_boundary)]


class hf_config(C.Structure):
    _fields_ = [("cfl", C.c_double), ("integrator", C.c_int32), ("check_finite", C.c_int32),
                ("boundaries", hf_boundaries), ("max_steps", C.c_uint64),
                ("max_dt", C.c_double), ("friction_dry_tol", C.c_double)]


class hf_mesh_desc(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("n_cols", C.c_int64), ("dx", C.c_double),
                ("dy", C.c_double), ("bed", C.POINTER(C.c_double)),
                ("manning", C.POINTER(C.c_double)), ("manning_uniform", C.c_double)]


class hf_scenario_desc(C.Structure):
    _fields_ = [("mesh", hf_mesh_desc), ("h", C.POINTER(C.c_double)),
                ("hu", C.POINTER(C.c_double)), ("hv", C.POINTER(C.c_double)),
                ("cfg", hf_config), ("t_end", C.c_double), ("n_rain", C.c_int64),
                ("rain_t", C.POINTER(C.c_double)), ("rain_rate", C.POINTER(C.c_double)),
                ("n_sources", C.c_int64), ("src_rows", C.POINTER(C.c_int64)),
                ("src_cols", C.POINTER(C.c_int64)), ("src_offsets", C.POINTER(C.c_int64)),
                ("src_t", C.POINTER(C.c_double)), ("src_q", C.POINTER(C.c_double))]


class hf_grid(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("n_cols", C.c_int64), ("dx", C.c_double),
                ("dy", C.c_double), ("bed", C.c_void_p), ("manning", C.c_void_p)]


def make_boundaries(north, south, west, east) -> hf_boundaries:
    """Each side is (kind, value)."""
    def one(b):
        kind, val = b
        return hf_boundary(int(kind), 0, float(val))
    return hf_boundaries(one(north), one(south), one(west), one(east))


def make_config(cfl=0.4, integrator=HF_SSPRK2, boundaries=None, max_steps=10_000_000,
                max_dt=60.0, friction_dry_tol=H_DRY, check_finite=0) -> hf_config:
    if boundaries is None:
        w = (HF_BC_WALL, 0.0)
        boundaries = make_boundaries(w, w, w, w)
    return hf_config(float(cfl), int(integrator), int(check_finite), boundaries,
                     int(max_steps), float(max_dt), float(friction_dry_tol))


class hf_ascii_grid_header(C.Structure):
    _fields_ = [("ncols", C.c_int64), ("nrows", C.c_int64), ("xllcorner", C.c_double),
                ("yllcorner", C.c_double), ("cellsize", C.c_double), ("nodata_value", C.c_double)]
