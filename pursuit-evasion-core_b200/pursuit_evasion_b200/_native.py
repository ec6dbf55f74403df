"""ctypes binding of libpe_b200.so (the C ABI declared in include/pe_b200.h).

The library is the product path: importing this module fails loudly when the
shared library is missing (build it with pursuit-evasion-core_b200/build.py);
there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().with_name("libpe_b200.so")

PE_OK = 0
PE_EINVAL = -1
PE_ENOMEM = -2
PE_ENONFINITE = -3
PE_ETIMEOUT = -4
PE_ECUDA = -5
PE_ESTATE = -6

PE_LOCAL_F32 = 0
PE_LOCAL_F64 = 1
PE_SCHEME_ENO_LF = 0


class NativeError(RuntimeError):
    """A libpe_b200 call failed; `code` is the negative PE_* code."""

    def __init__(self, code, message):
        super().__init__(f"{message} (code {code})")
        self.code = code


class NonFiniteError(NativeError, FloatingPointError):
    pass


class RelativeParams(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_int32),
        ("headings", ctypes.c_int32),
        ("p_speeds", ctypes.c_int32),
        ("e_speeds", ctypes.c_int32),
        ("extent", ctypes.c_double),
        ("capture_radius", ctypes.c_double),
        ("p_speed_min", ctypes.c_double),
        ("p_speed_max", ctypes.c_double),
        ("p_acceleration", ctypes.c_double),
        ("p_curvature", ctypes.c_double),
        ("e_speed_min", ctypes.c_double),
        ("e_speed_max", ctypes.c_double),
        ("e_acceleration", ctypes.c_double),
        ("e_curvature", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("order", ctypes.c_int32),
        ("scheme", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class WorldParams(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_int32),
        ("headings", ctypes.c_int32),
        ("p_speeds", ctypes.c_int32),
        ("e_speeds", ctypes.c_int32),
        ("extent", ctypes.c_double),
        ("arena", ctypes.c_double),
        ("capture_radius", ctypes.c_double),
        ("p_speed_min", ctypes.c_double),
        ("p_speed_max", ctypes.c_double),
        ("p_acceleration", ctypes.c_double),
        ("p_curvature", ctypes.c_double),
        ("e_speed_min", ctypes.c_double),
        ("e_speed_max", ctypes.c_double),
        ("e_acceleration", ctypes.c_double),
        ("e_curvature", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("order", ctypes.c_int32),
        ("linear_speed_boundary", ctypes.c_int32),
        ("avoid_mode", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("fast", ctypes.c_int32),
    ]


class SemiLagParams(ctypes.Structure):
    _fields_ = [
        ("positions", ctypes.c_int32),
        ("headings", ctypes.c_int32),
        ("p_speeds", ctypes.c_int32),
        ("e_speeds", ctypes.c_int32),
        ("extent", ctypes.c_double),
        ("capture_radius", ctypes.c_double),
        ("p_speed_min", ctypes.c_double),
        ("p_speed_max", ctypes.c_double),
        ("p_acceleration", ctypes.c_double),
        ("p_curvature", ctypes.c_double),
        ("e_speed_min", ctypes.c_double),
        ("e_speed_max", ctypes.c_double),
        ("e_acceleration", ctypes.c_double),
        ("e_curvature", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("mode", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class VehicleGridArrays(ctypes.Structure):
    """pe_vehicle_grid: one car's legal states and held-control stencils."""
    _fields_ = [
        ("states", ctypes.c_int32),
        ("actions", ctypes.c_int32),
        ("pose", ctypes.c_void_p),
        ("ids", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("allowed", ctypes.c_void_p),
    ]


class PairDomainArrays(ctypes.Structure):
    """pe_pair_domain: the pairs within the exit radius."""
    _fields_ = [
        ("positions", ctypes.c_int32),
        ("max_count", ctypes.c_int32),
        ("p_position", ctypes.c_void_p),
        ("lookup", ctypes.c_void_p),
        ("e_indices", ctypes.c_void_p),
        ("counts", ctypes.c_void_p),
        ("offsets", ctypes.c_void_p),
    ]


class SquareParams(ctypes.Structure):
    """pe_square_params: the options of native_square.cpp."""
    _fields_ = [
        ("positions", ctypes.c_int32),
        ("headings", ctypes.c_int32),
        ("extent", ctypes.c_double),
        ("arena", ctypes.c_double),
        ("capture_radius", ctypes.c_double),
        ("p_speed", ctypes.c_double),
        ("e_speed", ctypes.c_double),
        ("p_turn_rate", ctypes.c_double),
        ("e_turn_rate", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("order", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


PE_SL_KERNEL_AUTO, PE_SL_KERNEL_GENERIC, PE_SL_KERNEL_TILED = 0, 1, 2
PE_SL_TUBE = 0
PE_SL_MINTIME = 1

_P = ctypes.c_void_p
_I64P = ctypes.POINTER(ctypes.c_int64)
_DP = ctypes.POINTER(ctypes.c_double)

class VehicleModel(ctypes.Structure):
    """pe_vehicle_model: one car's limits, rectangle and control period."""
    _fields_ = [(name, ctypes.c_double) for name in (
        "speed_min", "speed_max", "acceleration", "max_curvature", "length", "width",
        "control_dt")]


# name -> (restype, argtypes)
SIGNATURES = {
    "pe_version": (ctypes.c_int, []),
    "pe_last_error": (ctypes.c_char_p, []),
    "pe_launch_count": (ctypes.c_int64, []),
    "pe_relative_cells": (ctypes.c_int, [ctypes.POINTER(RelativeParams), _I64P]),
    "pe_relative_cfl_limit": (ctypes.c_int, [ctypes.POINTER(RelativeParams), _DP]),
    "pe_relative_create": (
        ctypes.c_int,
        [ctypes.POINTER(RelativeParams), ctypes.POINTER(ctypes.c_void_p)],
    ),
    "pe_relative_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_relative_init": (ctypes.c_int, [_P, _P, _P, ctypes.c_double]),
    "pe_relative_advance": (ctypes.c_int, [_P, ctypes.c_double, _I64P]),
    "pe_relative_step": (ctypes.c_int, [_P, ctypes.c_double]),
    "pe_relative_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_relative_synchronize": (ctypes.c_int, [_P]),
    "pe_relative_copy_field": (ctypes.c_int, [_P, _P]),
    "pe_relative_copy_arrival": (ctypes.c_int, [_P, _P]),
    "pe_relative_device_field": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_relative_row_pitch": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "pe_relative_set_tile": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "pe_relative_get_tile": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int32)]),
    "pe_relative_kernel_info": (ctypes.c_int, [_P] + [ctypes.POINTER(ctypes.c_int32)] * 3),
    "pe_relative_stats": (ctypes.c_int, [_P, _DP, _DP]),
    "pe_relative_profile": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_relative_kernel_time": (ctypes.c_int, [_P, ctypes.c_int, _DP, _I64P]),
    "pe_relative_destroy": (ctypes.c_int, [_P]),
    "pe_relative_step_noalloc": (ctypes.c_int, [ctypes.POINTER(RelativeParams), _P, _P,
                                                _P, ctypes.c_double, ctypes.c_double,
                                                _P, _DP]),
    "pe_geometry_clearance": (ctypes.c_int, [ctypes.POINTER(VehicleModel), _P,
                                             ctypes.c_int64, _P, ctypes.c_int32,
                                             ctypes.c_double, _P, ctypes.c_int32]),
    "pe_geometry_backup_safe": (ctypes.c_int, [ctypes.POINTER(VehicleModel), _P,
                                               ctypes.c_int64, _P, ctypes.c_int32,
                                               ctypes.c_double, _P, ctypes.c_int32]),
    "pe_geometry_actions": (ctypes.c_int, [ctypes.POINTER(VehicleModel), _P, ctypes.c_int64,
                                           _P, ctypes.c_int32, ctypes.c_double, _P,
                                           ctypes.c_int32, ctypes.c_double, _P, _P,
                                           ctypes.c_int32]),
    "pe_geometry_connections": (ctypes.c_int, [ctypes.POINTER(VehicleModel), _P, _P,
                                               ctypes.c_int64, _P, ctypes.c_int32,
                                               ctypes.c_double, _P, ctypes.c_int32]),
    "pe_relative_f64_create": (
        ctypes.c_int,
        [ctypes.POINTER(RelativeParams), ctypes.POINTER(ctypes.c_void_p)],
    ),
    "pe_relative_f64_destroy": (ctypes.c_int, [_P]),
    "pe_relative_f64_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_relative_f64_initialize": (ctypes.c_int, [_P]),
    "pe_relative_f64_step": (ctypes.c_int, [_P, ctypes.c_double]),
    "pe_relative_f64_advance": (ctypes.c_int, [_P, ctypes.c_double, _I64P]),
    "pe_relative_f64_time": (ctypes.c_int, [_P, _DP, _I64P, _DP]),
    "pe_relative_f64_stats": (ctypes.c_int, [_P, _DP]),
    "pe_relative_f64_copy_field": (ctypes.c_int, [_P, _P]),
    "pe_batch_create": (ctypes.c_int, [ctypes.POINTER(RelativeParams), _DP, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_batch_set_tile": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "pe_batch_get_tile": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "pe_batch_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_batch_init": (ctypes.c_int, [_P]),
    "pe_batch_run": (ctypes.c_int, [_P]),
    "pe_batch_synchronize": (ctypes.c_int, [_P]),
    "pe_batch_solve_info": (ctypes.c_int, [_P, ctypes.c_int32, _I64P, _I64P, _DP]),
    "pe_batch_copy_field": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "pe_batch_copy_arrival": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "pe_batch_stats": (ctypes.c_int, [_P, ctypes.c_int32, _DP, _DP]),
    "pe_batch_launch_info": (ctypes.c_int, [_P] + [ctypes.POINTER(ctypes.c_int32)] * 3
                             + [_I64P]),
    "pe_batch_profile": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_batch_kernel_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_batch_destroy": (ctypes.c_int, [_P]),
    "pe_table_create": (ctypes.c_int, [_P, ctypes.c_int32, _DP, ctypes.POINTER(ctypes.c_int32),
                                       _DP, _DP, _DP, ctypes.c_double, _DP, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "pe_table_value": (ctypes.c_int, [_P, _DP, ctypes.c_int64, _DP]),
    "pe_table_field": (ctypes.c_int, [_P, _DP, _DP, ctypes.c_int64, _DP]),
    "pe_table_destroy": (ctypes.c_int, [_P]),
    "pe_relative_init_plane": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_double]),
    "pe_relative_set_exit": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double]),
    "pe_relative_probe": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, _P]),
    "pe_relative_snapshot": (ctypes.c_int, [_P, ctypes.c_int32]),
    "pe_relative_copy_snapshot": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "pe_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_host_free": (ctypes.c_int, [_P]),
    "pe_square_cells": (ctypes.c_int, [ctypes.POINTER(SquareParams), _I64P]),
    "pe_square_dt_limit": (ctypes.c_int, [ctypes.POINTER(SquareParams), _DP]),
    "pe_square_create": (ctypes.c_int, [ctypes.POINTER(SquareParams),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "pe_square_init": (ctypes.c_int, [_P]),
    "pe_square_advance": (ctypes.c_int, [_P, ctypes.c_double, _I64P]),
    "pe_square_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_square_synchronize": (ctypes.c_int, [_P]),
    "pe_square_copy_field": (ctypes.c_int, [_P, _P]),
    "pe_square_copy_arrival": (ctypes.c_int, [_P, _P]),
    "pe_square_residual": (ctypes.c_int, [_P, _DP]),
    "pe_square_profile": (ctypes.c_int, [_P, ctypes.c_int32]),
    "pe_square_kernel_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_square_destroy": (ctypes.c_int, [_P]),
    "pe_compact_create": (ctypes.c_int, [ctypes.POINTER(VehicleGridArrays),
                                         ctypes.POINTER(VehicleGridArrays),
                                         ctypes.POINTER(PairDomainArrays), ctypes.c_double,
                                         ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_compact_cells": (ctypes.c_int, [_P, _I64P]),
    "pe_compact_init": (ctypes.c_int, [_P] + [ctypes.c_double] * 4),
    "pe_compact_set_field": (ctypes.c_int, [_P, _P, ctypes.c_int64]),
    "pe_compact_backup": (ctypes.c_int, [_P, ctypes.c_int32]),
    "pe_compact_copy_field": (ctypes.c_int, [_P, _P, ctypes.c_int64]),
    "pe_compact_field_device": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_compact_query": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, _P, _P]),
    "pe_compact_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_compact_synchronize": (ctypes.c_int, [_P]),
    "pe_compact_profile": (ctypes.c_int, [_P, ctypes.c_int32]),
    "pe_compact_kernel_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_compact_destroy": (ctypes.c_int, [_P]),
    "pe_world_cells": (ctypes.c_int, [ctypes.POINTER(WorldParams), _I64P]),
    "pe_world_dt_limit": (ctypes.c_int, [ctypes.POINTER(WorldParams), _DP]),
    "pe_world_create": (ctypes.c_int, [ctypes.POINTER(WorldParams),
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "pe_world_init_contact": (ctypes.c_int, [_P] + [ctypes.c_double] * 4),
    "pe_world_set_clearance": (ctypes.c_int, [_P, _P, _P]),
    "pe_world_init_map": (ctypes.c_int, [_P]),
    "pe_world_init_square": (ctypes.c_int, [_P]),
    "pe_world_init_field": (ctypes.c_int, [_P, _P, _P, ctypes.c_double]),
    "pe_world_advance": (ctypes.c_int, [_P, ctypes.c_double, _I64P]),
    "pe_world_step": (ctypes.c_int, [_P, ctypes.c_double]),
    "pe_world_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_world_synchronize": (ctypes.c_int, [_P]),
    "pe_world_copy_field": (ctypes.c_int, [_P, _P]),
    "pe_world_copy_arrival": (ctypes.c_int, [_P, _P]),
    "pe_world_residual": (ctypes.c_int, [_P, _DP]),
    "pe_world_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_world_profile": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_world_kernel_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_world_destroy": (ctypes.c_int, [_P]),
    "pe_semilag_dt": (ctypes.c_int, [ctypes.POINTER(SemiLagParams), _DP]),
    "pe_semilag_create": (ctypes.c_int, [ctypes.POINTER(SemiLagParams),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "pe_semilag_init": (ctypes.c_int, [_P, _P]),
    "pe_semilag_init_device": (ctypes.c_int, [_P, _P]),
    "pe_semilag_backup": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_semilag_iterate": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_double,
                                          ctypes.c_int32, _I64P, _DP,
                                          ctypes.POINTER(ctypes.c_int32)]),
    "pe_semilag_residual": (ctypes.c_int, [_P, _DP]),
    "pe_semilag_evaluations": (ctypes.c_int, [_P, _I64P]),
    "pe_semilag_set_skip": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_semilag_items_computed": (ctypes.c_int, [_P, _I64P]),
    "pe_semilag_copy_value": (ctypes.c_int, [_P, _P]),
    "pe_semilag_copy_value_device": (ctypes.c_int, [_P, _P]),
    "pe_semilag_copy_policy": (ctypes.c_int, [_P, _P, _P]),
    "pe_semilag_device_value": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_void_p)]),
    "pe_semilag_iterations": (ctypes.c_int, [_P, _I64P]),
    "pe_semilag_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_semilag_set_kernel": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_semilag_kernel": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "pe_semilag_set_tile": (ctypes.c_int, [_P, ctypes.c_int32]),
    "pe_semilag_get_tile": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32), _I64P]),
    "pe_semilag_profile": (ctypes.c_int, [_P, ctypes.c_int]),
    "pe_semilag_kernel_time": (ctypes.c_int, [_P, _DP, _I64P]),
    "pe_relative_shard_create": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P]),
    "pe_relative_shard_layout": (ctypes.c_int, [_P, _P, _P]),
    "pe_relative_shard_set_stream": (ctypes.c_int, [_P, _P]),
    "pe_relative_shard_init": (ctypes.c_int, [_P, _P, ctypes.c_double]),
    "pe_relative_shard_stage": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double]),
    "pe_relative_shard_buffer": (ctypes.c_int, [_P, _P]),
    "pe_relative_shard_copy_field": (ctypes.c_int, [_P, _P]),
    "pe_relative_shard_copy_arrival": (ctypes.c_int, [_P, _P]),
    "pe_relative_shard_stats": (ctypes.c_int, [_P, _P, _P]),
    "pe_relative_shard_synchronize": (ctypes.c_int, [_P]),
    "pe_relative_shard_destroy": (ctypes.c_int, [_P]),
    "pe_semilag_track_arrival": (ctypes.c_int, [_P, _P, ctypes.c_double]),
    "pe_semilag_copy_arrival": (ctypes.c_int, [_P, _P]),
    "pe_semilag_destroy": (ctypes.c_int, [_P]),
    "pe_mlp_gemm": (ctypes.c_int, [_P, _P] + [ctypes.c_int] * 9 + [_P, _P, ctypes.c_int,
                                                                   _P, _P, _P]),
    "pe_mlp_gemm_tc": (ctypes.c_int, [_P, _P] + [ctypes.c_int] * 6 + [_P, _P, ctypes.c_int,
                                                                     _P, _P, _P]),
    "pe_mlp_gemm_tc_splitk": (ctypes.c_int, [_P, _P] + [ctypes.c_int] * 6 + [_P, ctypes.c_int,
                                                                            _P]),
    "pe_mlp_gemm_tc_timeouts": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "pe_mlp_adam": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, _P,
                                   ctypes.c_float, _P]),
    "pe_mlp_head_forward": (ctypes.c_int, [_P] * 7 + [ctypes.c_int, ctypes.c_int, _P]),
    "pe_mlp_head_backward": (ctypes.c_int, [_P] * 7 + [ctypes.c_int, ctypes.c_int, _P]),
    "pe_mlp_transpose": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _P]),
    "pe_mlp_colsum": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _P]),
    "pe_mlp_encode_relative_nodes": (ctypes.c_int, [_P, _P] + [ctypes.c_int] * 5
                                     + [ctypes.c_double] * 5 + [_P, ctypes.c_int, _P, _P]),
    "pe_mlp_encode_relative_states": (ctypes.c_int, [_P, ctypes.c_int] + [ctypes.c_double] * 5
                                      + [_P, ctypes.c_int, _P]),
    "pe_mlp_encode_world_nodes": (ctypes.c_int, [_P, _P] + [ctypes.c_int] * 5
                                  + [ctypes.c_double] * 5 + [_P, ctypes.c_int, _P, _P]),
}

_lib = None


def library():
    """Load libpe_b200.so once; raise if it is absent."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with "
                "pursuit-evasion-core_b200/build.py (no CPU fallback exists)"
            )
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def check(code):
    """Raise the exception matching a PE_* return code."""
    if code == PE_OK:
        return
    message = library().pe_last_error().decode(errors="replace")
    if code == PE_EINVAL:
        raise ValueError(message)
    if code == PE_ENOMEM:
        raise MemoryError(message)
    if code == PE_ENONFINITE:
        raise NonFiniteError(code, message)
    raise NativeError(code, message)


def launch_count():
    return int(library().pe_launch_count())
