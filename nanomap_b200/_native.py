"""ctypes bindings of include/nanomap_b200.h (the test and benchmark harness's view of the C ABI).

The library is loaded from the package directory.  There is no fallback: when the shared
library is missing or a call fails, a ``NanomapError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libnanomap_b200.so"
HEADER = PKG.parent / "include" / "nanomap_b200.h"

NM_OK = 0
NM_ERR_ARG = 1
NM_ERR_CAPACITY = 2
NM_ERR_CUDA = 3
NM_ERR_TIMEOUT = 4
NM_ERR_STATE = 5
NM_ERR_IO = 6
NM_ERR_UNSUPPORTED = 7

NM_SENSOR_FRUSTUM = 0
NM_SENSOR_LASER = 1
NM_UPDATE_LABEL = 0
NM_UPDATE_ACCUMULATE = 1
NM_CLAMP_ALWAYS = 0
NM_CLAMP_ON_CROSSING = 1
NM_ROUND_NEAREST = 0
NM_ROUND_DOWN = 1

NM_INPUT_HOST = 0x1
NM_DEFER_INTEGRATE = 0x2
NM_SYNC = 0x4
NM_OUTPUT_HOST = 0x8
NM_FILTER_MEAN = 0x10
NM_FILTER_CENTRE = 0x20
NM_CAVE_2D = 0x1
NM_CAVE_COUNTER_RNG = 0x2


class NanomapError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"nanomap_b200 error {code}: {message}")
        self.code = code


class NmPose(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("orientation", C.c_float * 4)]


class NmSensorDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("id", C.c_int32), ("hres", C.c_int32), ("vres", C.c_int32),
        ("hfov_deg", C.c_float), ("vfov_deg", C.c_float),
        ("min_range", C.c_float), ("max_range", C.c_float),
        ("prob_hit", C.c_float), ("prob_miss", C.c_float),
        ("log_odds_hit", C.c_float), ("log_odds_miss", C.c_float),
        ("explicit_log_odds", C.c_int32), ("rate", C.c_int32),
        ("frame_transform", C.c_float * 9),
    ]


class NmMapDesc(C.Structure):
    _fields_ = [
        ("res", C.c_float), ("leaf_edge", C.c_int32),
        ("thres_hit", C.c_float), ("thres_miss", C.c_float),
        ("clamp_min", C.c_float), ("clamp_max", C.c_float),
        ("clamp_mode", C.c_int32), ("update_mode", C.c_int32), ("rounding", C.c_int32),
        ("initial_leaf_capacity", C.c_uint32), ("max_agents", C.c_int32),
    ]


class NmStats(C.Structure):
    _fields_ = [
        ("frames", C.c_uint64), ("rays", C.c_uint64), ("visits", C.c_uint64),
        ("unique_voxels", C.c_uint64), ("touched_leaves", C.c_uint64),
        ("leaf_count", C.c_uint64), ("leaf_capacity", C.c_uint64),
        ("error_flags", C.c_uint32), ("grow_count", C.c_uint32),
        ("depth_visits", C.c_uint64),
    ]


class NmConfigInfo(C.Structure):
    _fields_ = [
        ("mapping_res", C.c_float), ("grid_res", C.c_float),
        ("prob_hit_thres", C.c_float), ("prob_miss_thres", C.c_float),
        ("frustum_allocation_factor", C.c_float),
        ("clamp_min", C.c_float), ("clamp_max", C.c_float),
        ("leaf_edge", C.c_int32), ("filter_type", C.c_int32), ("update_type", C.c_int32),
        ("precision_type", C.c_int32), ("publish_sensor", C.c_int32), ("process_type", C.c_int32),
        ("update_mode", C.c_int32), ("clamp_mode", C.c_int32), ("rounding", C.c_int32),
        ("n_sensors", C.c_int32), ("n_agents", C.c_int32),
        ("sim_grid", C.c_char * 512),
    ]


class NmAgentInfo(C.Structure):
    _fields_ = [
        ("spawn_random", C.c_int32), ("position", C.c_float * 3), ("num_obs", C.c_int32),
        ("len_obs", C.c_float), ("collision_dist", C.c_float), ("n_sensors", C.c_int32),
    ]


class NmRayPose(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("rotation", C.c_double * 9)]


class NmRefineDesc(C.Structure):
    _fields_ = [("scale", C.c_float), ("bias", C.c_float), ("max_residual", C.c_float),
                ("steps", C.c_int32), ("lr_position", C.c_float), ("lr_rotation", C.c_float),
                ("surface_offset", C.c_float), ("edge_threshold", C.c_float)]


class NmCaveDesc(C.Structure):
    _fields_ = [
        ("map_size", C.c_double * 3), ("grid_res", C.c_double), ("fill_percentage", C.c_int32),
        ("smoothing_count", C.c_int32), ("active_max", C.c_int32), ("active_min", C.c_int32),
        ("time_seed", C.c_int32), ("seed", C.c_uint32), ("file_out", C.c_char * 256),
    ]


class NmFrame(C.Structure):
    _fields_ = [
        ("sensor", C.c_void_p), ("pose", NmPose), ("ranges", C.c_void_p),
        ("agent", C.c_int32), ("pad", C.c_int32),
    ]


_P = C.c_void_p
_I32 = C.c_int32
_U32 = C.c_uint32
_I64 = C.c_int64
_U64 = C.c_uint64
_F = C.c_float
_PF = C.POINTER(C.c_float)
_PD = C.POINTER(C.c_double)
_PI32 = C.POINTER(C.c_int32)
_PU32 = C.POINTER(C.c_uint32)
_PU64 = C.POINTER(C.c_uint64)

# name -> (restype, argtypes); every int-returning entry returns a status code.
_SIGS = {
    "nm_abi_version": (C.c_int, []),
    "nm_last_error": (C.c_char_p, []),
    "nm_context_create": (C.c_int, [_I32, C.POINTER(_P)]),
    "nm_context_destroy": (C.c_int, [_P]),
    "nm_context_sync": (C.c_int, [_P]),
    "nm_alloc_device": (C.c_int, [_P, C.c_size_t, C.POINTER(_P)]),
    "nm_free_device": (C.c_int, [_P]),
    "nm_config_load": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "nm_config_destroy": (C.c_int, [_P]),
    "nm_config_get_info": (C.c_int, [_P, _P]),
    "nm_config_sensor": (C.c_int, [_P, _I32, C.POINTER(NmSensorDesc), C.c_char_p, _I32]),
    "nm_config_agent": (C.c_int, [_P, _I32, _P]),
    "nm_config_agent_sensor": (C.c_int, [_P, _I32, _I32, C.c_char_p, _I32, C.POINTER(NmPose)]),
    "nm_config_map_desc": (C.c_int, [_P, C.POINTER(NmMapDesc)]),
    "nm_simmap_load": (C.c_int, [_P, C.c_char_p, C.POINTER(_P)]),
    "nm_vdb_active_voxels": (C.c_int, [C.c_char_p, C.c_char_p, _PD, _PD, _P, _I64,
                                       C.POINTER(_I64)]),
    "nm_vdb_write_active_voxels": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, _P, _I64]),
    "nm_sensor_create": (C.c_int, [_P, C.POINTER(NmSensorDesc), C.POINTER(_P)]),
    "nm_sensor_destroy": (C.c_int, [_P]),
    "nm_sensor_params": (C.c_int, [_P, _PF]),
    "nm_map_create": (C.c_int, [_P, C.POINTER(NmMapDesc), C.POINTER(_P)]),
    "nm_map_destroy": (C.c_int, [_P]),
    "nm_map_reset": (C.c_int, [_P]),
    "nm_map_stats": (C.c_int, [_P, C.POINTER(NmStats)]),
    "nm_map_status_async": (C.c_int, [_P, _P, _P]),
    "nm_map_insert_points": (C.c_int, [_P, _P, C.POINTER(NmPose), _P, _I32, _I32, _I32, _U32, _P]),
    "nm_sim_render_noisy": (C.c_int, [_P, _P, C.POINTER(NmPose), _P, _F, _F, _U64, _U32, _P]),
    "nm_sim_cast_rays": (C.c_int, [_P, _P, _P, _I64, _F, _P, _U32, _P]),
    "nm_sim_insert": (C.c_int, [_P, _P, _P, C.POINTER(NmPose), _F, _F, _U64, _P, _U32, _P]),
    "nm_observation_sphere": (C.c_int, [_I32, _PF]),
    "nm_ray_pose_from_pose": (C.c_int, [_P, C.POINTER(NmPose), C.POINTER(NmRayPose)]),
    "nm_map_values_copy": (C.c_int, [_P, _P, _U64, _PU64, _P]),
    "nm_map_slot_origins": (C.c_int, [_P, _PI32, _U64, _PU64]),
    "nm_depth_render": (C.c_int, [_P, _P, C.POINTER(NmRayPose), _P, _U64, _F, _F, _P, _P]),
    "nm_depth_backward": (C.c_int, [_P, _P, C.POINTER(NmRayPose), _P, _U64, _F, _F, _P, _P, _P,
                                    _PD, _P]),
    "nm_pose_refine": (C.c_int, [_P, _P, C.POINTER(NmRayPose), _P, _F, _F, _F, _I32, _F, _F,
                                 _PF]),
    "nm_pose_refine_desc": (C.c_int, [_P, _P, C.POINTER(NmRayPose), _P, C.POINTER(NmRefineDesc),
                                      _PF]),
    "nm_map_filter_points": (C.c_int, [_P, _P, C.POINTER(NmPose), _P, _I32, _I32, _I32, _U32,
                                       _PF, _PU32, _U64, _PU64]),
    "nm_map_insert_ranges": (C.c_int, [_P, _P, C.POINTER(NmPose), _P, _U32, _P]),
    "nm_map_integrate": (C.c_int, [_P, _P]),
    "nm_map_set_launch": (C.c_int, [_P, _I32, _I32, _I32]),
    "nm_map_tick": (C.c_int, [_P, C.POINTER(NmFrame), _I32, _U32, _P]),
    "nm_tick_plan_create": (C.c_int, [_P, _P, C.POINTER(NmFrame), _I32, C.POINTER(_P)]),
    "nm_tick_plan_destroy": (C.c_int, [_P]),
    "nm_tick_plan_set_pose": (C.c_int, [_P, _I32, C.POINTER(NmPose)]),
    "nm_tick_plan_set_noise": (C.c_int, [_P, _F, _F, _U64]),
    "nm_tick_plan_set_launch": (C.c_int, [_P, _I32, _I32, _I32]),
    "nm_tick_plan_run": (C.c_int, [_P, _U32, _P]),
    "nm_tick_plan_autotune": (C.c_int, [_P, C.c_char_p, _PI32, _PF]),
    "nm_map_export": (C.c_int, [_P, _PI32, _PF, _PU32, _U64, _PU64]),
    "nm_map_export_labels": (C.c_int, [_P, _I32, _PI32, _PU32, _U64, _PU64]),
    "nm_map_frame_params": (C.c_int, [_P, _P, C.POINTER(NmPose), _PF, _PD, _PF]),
    "nm_frame_params": (C.c_int, [C.POINTER(NmSensorDesc), C.POINTER(NmPose), _F, _I32, _PF, _PD, _PF, _PF]),
    "nm_label_frame_static": (C.c_int, [_P, C.POINTER(NmPose), _P, _F, _I32, _P, _P, _U32, _P, _U32, _P]),
    "nm_simmap_create_primitives": (C.c_int, [_P, _F, _PI32, _PI32, _PD, _I32, _PD, _I32, C.POINTER(_P)]),
    "nm_simmap_create_voxels": (C.c_int, [_P, _F, _PI32, _I64, C.POINTER(_P)]),
    "nm_simmap_destroy": (C.c_int, [_P]),
    "nm_simmap_info": (C.c_int, [_P, _PI32, _PU64, _PU64]),
    "nm_simmap_export": (C.c_int, [_P, _PI32, _PU32, _U64, _PU64]),
    "nm_sim_render": (C.c_int, [_P, _P, C.POINTER(NmPose), _P, _U32, _P]),
    "nm_ranges_add_noise": (C.c_int, [_P, _P, _I64, _F, _F, _U64, _P]),
    "nm_cave_config_load": (C.c_int, [C.c_char_p, C.POINTER(NmCaveDesc)]),
    "nm_cave_create": (C.c_int, [_P, C.POINTER(NmCaveDesc), C.POINTER(_P)]),
    "nm_cave_destroy": (C.c_int, [_P]),
    "nm_cave_dims": (C.c_int, [_P, _PI32, _PI32]),
    "nm_cave_populate": (C.c_int, [_P, _U32]),
    "nm_cave_smooth": (C.c_int, [_P, _U32]),
    "nm_cave_floor_ceil": (C.c_int, [_P]),
    "nm_cave_regions": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I64)]),
    "nm_cave_keep_largest": (C.c_int, [_P]),
    "nm_cave_cells": (C.c_int, [_P, _PI32, _I64, C.POINTER(_I64)]),
    "nm_cave_simmap": (C.c_int, [_P, _I32, _I32, _I32, C.POINTER(_P)]),
    "nm_cave_save": (C.c_int, [_P, _I32, _I32, _I32, C.c_char_p, C.c_char_p]),
}

_lib = None


def declared_symbols() -> list[str]:
    """Function names declared in include/nanomap_b200.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(nm_\w+)\s*\(", text, re.M)))


def lib() -> C.CDLL:
    """Load libnanomap_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NanomapError(NM_ERR_STATE, f"{LIB_PATH} is missing; run python -m nanomap_b200.build")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != NM_OK:
        raise NanomapError(rc, lib().nm_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
