"""ctypes binding of the C ABI declared in include/ctsim_b200.h.

The library is the in-tree build ``ctsim_b200/_lib/libctsim_b200.so``.  There is
no fallback: if it is missing and cannot be built, importing the projector API
raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_f, _i, _p, _d = C.c_float, C.c_int, C.c_void_p, C.c_double
GEOM_ARGS = [_i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _f, _f, _f, _f, _f, _f, _f, _i, _p, _p, _i]

CTSIM_OK = 0
STATUS = {0: "OK", 1: "ERR_ARGUMENT", 2: "ERR_CUDA", 3: "ERR_ALLOC", 4: "ERR_UNSUPPORTED", 5: "ERR_NO_DEVICE"}
METHODS = {"proj,dd": 0, "proj,tf": 1, "back,dd": 2, "back,tf": 3, "back,pd": 4, "back,hpd": 5}

# symbols declared in include/ctsim_b200.h
INPUT_SCALED = 0x100  # CTSIM_INPUT_SCALED
EXPORTED = ["ctsim_last_error", "ctsim_version", "ctsim_proj_dd", "ctsim_back_dd", "ctsim_proj_tf", "ctsim_back_tf",
            "ctsim_back_pd", "ctsim_cbct_geom", "ctsim_plan_create", "ctsim_plan_destroy", "ctsim_plan_device_bytes",
            "ctsim_plan_project", "ctsim_plan_backproject", "ctsim_plan_check", "ctsim_back_dd_noalloc",
            "ctsim_fdk_create", "ctsim_fdk_destroy", "ctsim_fdk_filter", "ctsim_fdk_run", "ctsim_fdk_dbeta",
            "ctsim_fdk_design_filter", "ctsim_pwls_weights", "ctsim_pwls_residual", "ctsim_sqdiff",
            "ctsim_penalty", "ctsim_sqs_update", "ctsim_plan_project_ex", "ctsim_plan_backproject_ex",
            "ctsim_pwls_residual_ex", "ctsim_pwls_residual_scaled", "ctsim_fdk_filter_ex", "ctsim_fdk_run_ex",
            "ctsim_plan_create_async", "ctsim_pool_trim", "ctsim_nesterov_update",
            "ctsim_simulate_counts", "ctsim_log_attenuation", "ctsim_fbct_geom", "ctsim_fan_plan_create",
            "ctsim_fan_plan_destroy", "ctsim_fan_project", "ctsim_fan_backproject",
            "ctsim_plan_get_tuning", "ctsim_plan_set_tuning", "ctsim_plan_autotune", "ctsim_autotune_clear",
            "ctsim_batch_project", "ctsim_batch_backproject", "ctsim_host_cache_release",
            "ctsim_host_cache_enable"]


class CtsimGeom(C.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("nz", _i), ("dx", _f), ("dy", _f), ("dz", _f),
                ("offset_x", _f), ("offset_y", _f), ("offset_z", _f), ("nu", _i), ("nv", _i),
                ("du", _f), ("dv", _f), ("offset_u", _f), ("offset_v", _f),
                ("sad", _f), ("add", _f), ("sdd", _f), ("noviews", _i), ("detector_type", _i)]


class CtsimFanGeom(C.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("dx", _f), ("dy", _f), ("offset_x", _f), ("offset_y", _f), ("nu", _i),
                ("du", _f), ("offset_u", _f), ("sad", _f), ("add", _f), ("sdd", _f), ("noviews", _i),
                ("detector_type", _i)]


class CtsimTuning(C.Structure):
    _fields_ = [("proj_groups", _i), ("back_mz", _i), ("pd_mz", _i), ("back_mz_tf", _i), ("proj_rows", _i),
                ("proj_layout", _i), ("proj_slots", _i)]


class CtsimBatchItem(C.Structure):
    _fields_ = [("plan", _p), ("in_", _p), ("out", _p), ("view_begin", _i), ("view_stride", _i),
                ("view_count", _i), ("scale", _f), ("in_dtype", _i), ("out_dtype", _i)]


class CtsimError(RuntimeError):
    pass


_lib = None


def lib_path() -> str:
    return _build.LIB


def load():
    """Load (building first if needed) the projector library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path) or _build.needs_rebuild():
        try:
            _build.build()
        except Exception as exc:  # no nvcc on this machine and no prebuilt library
            if not os.path.exists(path):
                raise ImportError(f"libctsim_b200.so is missing and could not be built: {exc}") from exc
    L = C.CDLL(path)
    L.ctsim_last_error.restype = C.c_char_p
    L.ctsim_version.restype = C.c_char_p
    for name in ("ctsim_proj_dd", "ctsim_proj_tf"):
        fn = getattr(L, name)
        fn.argtypes = GEOM_ARGS + [_p, _p, _p]
        fn.restype = C.c_bool
    for name in ("ctsim_back_dd", "ctsim_back_tf"):
        fn = getattr(L, name)
        fn.argtypes = GEOM_ARGS + [_p, _p, _p]
        fn.restype = C.c_bool
    L.ctsim_back_pd.argtypes = GEOM_ARGS + [_p, _p, _p, C.c_bool]
    L.ctsim_back_pd.restype = C.c_bool
    L.ctsim_cbct_geom.argtypes = [C.c_char_p] + GEOM_ARGS + [_p, _p, _p]
    L.ctsim_cbct_geom.restype = C.c_bool
    L.ctsim_host_cache_release.argtypes = []
    L.ctsim_host_cache_release.restype = _i
    L.ctsim_host_cache_enable.argtypes = [_i]
    L.ctsim_host_cache_enable.restype = _i
    L.ctsim_plan_create.argtypes = [C.POINTER(CtsimGeom), _p, _p, _p, C.POINTER(_p)]
    L.ctsim_plan_create.restype = _i
    L.ctsim_plan_create_async.argtypes = [C.POINTER(CtsimGeom), _p, _p, _p, _p, C.POINTER(_p)]
    L.ctsim_plan_create_async.restype = _i
    L.ctsim_nesterov_update.argtypes = [_i, _f, _f, _i, _i, _i, _p, _p, _p, _p, _p, C.c_double, C.c_double, _p,
                                        _p, _p]
    L.ctsim_nesterov_update.restype = _i
    L.ctsim_plan_get_tuning.argtypes = [_p, C.POINTER(CtsimTuning)]
    L.ctsim_plan_get_tuning.restype = _i
    L.ctsim_plan_set_tuning.argtypes = [_p, C.POINTER(CtsimTuning)]
    L.ctsim_plan_set_tuning.restype = _i
    L.ctsim_plan_autotune.argtypes = [_p, _i, _i, _p, C.POINTER(CtsimTuning)]
    L.ctsim_plan_autotune.restype = _i
    L.ctsim_autotune_clear.argtypes = []
    L.ctsim_autotune_clear.restype = _i
    L.ctsim_batch_project.argtypes = [_i, C.POINTER(CtsimBatchItem), _i, _p]
    L.ctsim_batch_project.restype = _i
    L.ctsim_batch_backproject.argtypes = [_i, C.POINTER(CtsimBatchItem), _i, _p]
    L.ctsim_batch_backproject.restype = _i
    L.ctsim_fbct_geom.argtypes = [C.c_char_p, _i, _i, _f, _f, _f, _f, _i, _f, _f, _f, _f, _f, _i, _p, _i, _p, _p]
    L.ctsim_fbct_geom.restype = C.c_bool
    L.ctsim_fan_plan_create.argtypes = [C.POINTER(CtsimFanGeom), _p, C.POINTER(_p)]
    L.ctsim_fan_plan_create.restype = _i
    L.ctsim_fan_plan_destroy.argtypes = [_p]
    L.ctsim_fan_plan_destroy.restype = _i
    L.ctsim_fan_project.argtypes = [_p, _i, _p, _p, _i, _i, _i, _p]
    L.ctsim_fan_project.restype = _i
    L.ctsim_fan_backproject.argtypes = [_p, _i, _p, _p, _i, _i, _i, _f, _p]
    L.ctsim_fan_backproject.restype = _i
    L.ctsim_simulate_counts.argtypes = [_p, C.c_size_t, _f, _f, C.c_uint64, _i, _p, _p, _p]
    L.ctsim_simulate_counts.restype = _i
    L.ctsim_log_attenuation.argtypes = [_p, C.c_size_t, _f, _p, C.c_size_t, _p, _p]
    L.ctsim_log_attenuation.restype = _i
    L.ctsim_pool_trim.argtypes = [C.c_size_t]
    L.ctsim_pool_trim.restype = _i
    L.ctsim_plan_destroy.argtypes = [_p]
    L.ctsim_plan_destroy.restype = _i
    L.ctsim_plan_device_bytes.argtypes = [_p]
    L.ctsim_plan_device_bytes.restype = C.c_size_t
    L.ctsim_plan_project.argtypes = [_p, _i, _p, _p, _i, _i, _i, _p]
    L.ctsim_plan_project.restype = _i
    L.ctsim_plan_backproject.argtypes = [_p, _i, _p, _p, _i, _i, _i, _f, _p]
    L.ctsim_plan_backproject.restype = _i
    L.ctsim_plan_project_ex.argtypes = [_p, _i, _p, _i, _p, _i, _i, _i, _i, _p]
    L.ctsim_plan_project_ex.restype = _i
    L.ctsim_plan_backproject_ex.argtypes = [_p, _i, _p, _i, _p, _i, _i, _i, _i, _f, _p]
    L.ctsim_plan_backproject_ex.restype = _i
    L.ctsim_plan_check.argtypes = [_p]
    L.ctsim_plan_check.restype = _i
    L.ctsim_back_dd_noalloc.argtypes = [C.POINTER(CtsimGeom), _p, _p, _p, _p, _p, _p]
    L.ctsim_back_dd_noalloc.restype = _i
    L.ctsim_fdk_create.argtypes = [_p, C.c_char_p, _f, _i, C.POINTER(_p)]
    L.ctsim_fdk_create.restype = _i
    L.ctsim_fdk_destroy.argtypes = [_p]
    L.ctsim_fdk_destroy.restype = _i
    L.ctsim_fdk_filter.argtypes = [_p, _p, _p, _p]
    L.ctsim_fdk_filter.restype = _i
    L.ctsim_fdk_run.argtypes = [_p, _p, _p, _p]
    L.ctsim_fdk_run.restype = _i
    L.ctsim_fdk_filter_ex.argtypes = [_p, _p, _i, _p, _p]
    L.ctsim_fdk_filter_ex.restype = _i
    L.ctsim_fdk_run_ex.argtypes = [_p, _p, _i, _p, _p]
    L.ctsim_fdk_run_ex.restype = _i
    L.ctsim_fdk_dbeta.argtypes = [_p]
    L.ctsim_fdk_dbeta.restype = _f
    L.ctsim_fdk_design_filter.argtypes = [_i, _f, _f, _i, C.c_char_p, _f, _p, C.POINTER(_i)]
    L.ctsim_fdk_design_filter.restype = _i
    _sz = C.c_size_t
    L.ctsim_pwls_weights.argtypes = [_p, _f, _f, _p, _sz, _p]
    L.ctsim_pwls_weights.restype = _i
    L.ctsim_pwls_residual.argtypes = [_p, _p, _p, _p, _sz, _p, _p]
    L.ctsim_pwls_residual.restype = _i
    L.ctsim_pwls_residual_ex.argtypes = [_p, _p, _p, _i, _f, _p, _sz, _p, _p]
    L.ctsim_pwls_residual_ex.restype = _i
    L.ctsim_pwls_residual_scaled.argtypes = [_p, _p, _p, _p, _i, _f, _p, _i, _p, _p]
    L.ctsim_pwls_residual_scaled.restype = _i
    L.ctsim_sqdiff.argtypes = [_p, _p, _sz, _p, _p]
    L.ctsim_sqdiff.restype = _i
    L.ctsim_penalty.argtypes = [_i, _i, _f, _i, _i, _i, _p, _p, _p, _p]
    L.ctsim_penalty.restype = _i
    L.ctsim_sqs_update.argtypes = [_i, _f, _f, _i, _i, _i, _p, _p, _p, _p, _p]
    L.ctsim_sqs_update.restype = _i
    _lib = L
    return L


def check(status: int, what: str = "ctsim"):
    if status != CTSIM_OK:
        msg = load().ctsim_last_error().decode(errors="replace")
        raise CtsimError(f"{what}: {STATUS.get(status, status)}: {msg}")


def last_error() -> str:
    return load().ctsim_last_error().decode(errors="replace")
