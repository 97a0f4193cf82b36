"""Loader of the sm_100a library (libhydroflux_gpu.so) with ctypes prototypes.

There is no CPU fallback: if the library is missing or no CUDA device is
present, every compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhydroflux_gpu.so")

_LIB = None

_D = C.POINTER(C.c_double)
_VP = C.c_void_p
_I64P = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol declared in include/hydroflux_gpu.h
PROTOTYPES = {
    "hf_last_error": (C.c_char_p, []),
    "hf_abi_version": (C.c_int, []),
    "hf_config_default": (None, [C.POINTER(abi.hf_config)]),
    "hf_kernel_launches": (C.c_int, [C.POINTER(C.c_uint64)]),
    "hf_sim_create": (C.c_int, [C.POINTER(abi.hf_mesh_desc), _D, _D, _D,
                                C.POINTER(abi.hf_config), C.c_int, C.POINTER(_VP)]),
    "hf_sim_create_aos": (C.c_int, [C.POINTER(abi.hf_mesh_desc), _D, C.POINTER(abi.hf_config),
                                    C.c_int, C.POINTER(_VP)]),
    "hf_sim_destroy": (C.c_int, [_VP]),
    "hf_sim_step": (C.c_int, [_VP, C.c_double, _D]),
    "hf_sim_run_until": (C.c_int, [_VP, C.c_double]),
    "hf_sim_run_steps": (C.c_int, [_VP, C.c_uint64, C.c_double]),
    "hf_sim_run_steps_timed": (C.c_int, [_VP, C.c_uint64, C.c_double, _D,
                                         C.POINTER(C.c_uint64), _D]),
    "hf_sim_time": (C.c_int, [_VP, _D]),
    "hf_sim_steps": (C.c_int, [_VP, C.POINTER(C.c_uint64)]),
    "hf_sim_get_state": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hf_sim_set_state": (C.c_int, [_VP, _VP, _VP, _VP]),
    "hf_sim_get_state_aos": (C.c_int, [_VP, _VP]),
    "hf_sim_max_depth_exceeds_relief": (C.c_int, [_VP, C.c_double, C.POINTER(C.c_int)]),
    "hf_sim_set_state_aos": (C.c_int, [_VP, _VP]),
    "hf_sim_set_boundaries": (C.c_int, [_VP, C.POINTER(abi.hf_boundaries)]),
    "hf_sim_set_stage_kernel": (C.c_int, [_VP, C.c_int]),
    "hf_sim_stage_kernel": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "hf_release_cached_memory": (C.c_int, [C.c_int]),
    "hf_sim_error_detail": (C.c_int, [_VP, _D, _D, C.POINTER(C.c_uint64)]),
    "hf_sim_device_state": (C.c_int, [_VP, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                      C.POINTER(_VP)]),
    "hf_sim_set_rain": (C.c_int, [_VP, C.c_int64, _D, _D]),
    "hf_sim_set_point_sources": (C.c_int, [_VP, C.c_int64, _I64P, _I64P, _I64P, _D, _D]),
    "hf_sim_set_rain_units": (C.c_int, [_VP, C.c_double, C.c_double, C.c_double]),
    "hf_sim_set_point_source_units": (C.c_int, [_VP, C.c_double, C.c_double, C.c_double]),
    "hf_sim_set_gauges": (C.c_int, [_VP, C.c_int64, _I64P, _I64P, C.c_int64]),
    "hf_sim_gauge_peaks": (C.c_int, [_VP, _D, _D]),
    "hf_sim_gauge_series": (C.c_int, [_VP, _D, _D, _I64P, _I64P]),
    "hf_batch_create": (C.c_int, [C.c_int64, C.POINTER(abi.hf_scenario_desc), C.c_int,
                                  C.POINTER(_VP)]),
    "hf_batch_destroy": (C.c_int, [_VP]),
    "hf_batch_run": (C.c_int, [_VP, C.c_uint64, C.POINTER(C.c_int64)]),
    "hf_batch_scenario_info": (C.c_int, [_VP, C.c_int64, _D, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_int)]),
    "hf_batch_get_state": (C.c_int, [_VP, C.c_int64, _VP, _VP, _VP]),
    "hf_batch_set_schedule": (C.c_int, [_VP, C.c_int]),
    "hf_batch_schedule": (C.c_int, [_VP, C.POINTER(C.c_int), _D]),
    "hf_server_create": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.POINTER(_VP)]),
    "hf_server_destroy": (C.c_int, [_VP]),
    "hf_server_admit": (C.c_int, [_VP, C.POINTER(abi.hf_scenario_desc), C.POINTER(C.c_int)]),
    "hf_server_advance": (C.c_int, [_VP, C.c_uint64, C.POINTER(C.c_int)]),
    "hf_server_finished": (C.c_int, [_VP, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
    "hf_server_collect": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, _D, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_int)]),
    "hf_server_usage": (C.c_int, [_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]),
    "hf_calib_create": (C.c_int, [C.POINTER(abi.hf_scenario_desc), C.c_int64, C.c_int64, _I64P,
                                  C.c_int64, C.c_int, C.POINTER(_VP)]),
    "hf_calib_destroy": (C.c_int, [_VP]),
    "hf_calib_set_observations": (C.c_int, [_VP, _D]),
    "hf_calib_run": (C.c_int, [_VP, _D, C.c_int, _D, _D, C.POINTER(C.c_int64)]),
    "hf_tangent": (C.c_int, [_VP, _D, _D, _D, _D, _D, _D, _D]),
    "hf_tangent_lanes": (C.c_int, [_VP, _D, C.c_int64, _D, _D, _D, _D, _D, _D]),
    "hf_calib_lane_state": (C.c_int, [_VP, C.c_int64, _D, _D, _D]),
    "hf_grad_manning": (C.c_int, [_VP, _D, _D, _D, _D, _D, _D]),
    "hf_calib_final_state": (C.c_int, [_VP, _D, _D, _D, _D, _D, _D]),
    "hf_calib_dt": (C.c_int, [_VP, _D, C.POINTER(C.c_int64)]),
    "hf_read_ascii_grid": (C.c_int, [C.c_char_p, C.POINTER(abi.hf_ascii_grid_header),
                                     C.POINTER(_D)]),
    "hf_free_buffer": (None, [_VP]),
    "hf_write_ascii_grid": (C.c_int, [C.c_char_p, C.POINTER(abi.hf_ascii_grid_header), _D]),
    "hf_depth_raster": (C.c_int, [C.c_int64, _D, C.c_int, C.c_double, _D]),
    "hf_worldcover_manning": (C.c_double, [C.c_int]),
    "hf_workspace_create": (C.c_int, [C.c_int64, C.c_int64, C.c_int, C.POINTER(_VP)]),
    "hf_workspace_destroy": (C.c_int, [_VP]),
    "hf_cfl_time_step": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP,
                                   C.POINTER(abi.hf_boundaries), C.c_double, _VP, _VP, _D]),
    "hf_forward_euler_step": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP,
                                        C.POINTER(abi.hf_boundaries), C.c_double, _VP, _VP]),
    "hf_ssprk2_step": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP,
                                 C.POINTER(abi.hf_boundaries), C.c_double, _VP, _VP]),
    "hf_manning_friction_step": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP, C.c_double,
                                           C.c_double, _VP]),
    "hf_apply_rain": (C.c_int, [C.c_int64, _VP, _VP, _VP, C.c_double, C.c_double, _VP]),
    "hf_apply_point_sources": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP, C.c_int64,
                                         _I64P, _I64P, _D, C.c_double, _VP]),
    "hf_hllc_flux": (C.c_int, [C.c_int, C.c_int64, _VP, _VP, _VP, _VP]),
    "hf_max_depth_exceeds_relief": (C.c_int, [C.POINTER(abi.hf_grid), _VP, C.c_double, _VP, _VP,
                                              C.POINTER(C.c_int)]),
    "hf_ssprk2_step_noalloc": (C.c_int, [C.POINTER(abi.hf_grid), _VP, _VP, _VP,
                                         C.POINTER(abi.hf_boundaries), C.c_double, C.c_int,
                                         _VP]),
}


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded library. Raises if it was not built (no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is missing: build it with `python -m hydroflux_b200.build` "
                "(the B200 path has no CPU fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def last_error() -> str:
    return lib().hf_last_error().decode()


def kernel_launches() -> int:
    """Kernels the library has launched in this process (hf_kernel_launches)."""
    n = C.c_uint64()
    lib().hf_kernel_launches(C.byref(n))
    return n.value
