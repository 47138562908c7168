"""ctypes binding of libseispstm.so (the C ABI declared in include/seispstm.h).

The library is built in-tree by ``seisproc_b200.build``.  There is no fallback:
if the shared library cannot be loaded, or no CUDA device is present, the
migration entry points raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# SEISPSTM_LIBRARY=checked loads the checked test build (bounds checks, short
# device wait limit, fault injection) instead of the product library.
CHECKED = os.environ.get("SEISPSTM_LIBRARY", "") == "checked"
LIB_PATH = os.path.join(HERE, "libseispstm_checked.so" if CHECKED else "libseispstm.so")

PSTM_OK, PSTM_EINVAL, PSTM_ENOMEM, PSTM_ETIMEOUT, PSTM_EBOUNDS, PSTM_ECUDA, PSTM_ENOTSUP = range(7)
PSTM_F32, PSTM_BF16, PSTM_F16, PSTM_F64 = range(4)
WEIGHT_OBLIQUITY_SPREADING, WEIGHT_SPREADING, WEIGHT_OBLIQUITY, WEIGHT_NONE = range(4)
CLAMP_FULL, CLAMP_MIGRATOR = range(2)

STATUS_NAMES = {0: "PSTM_OK", 1: "PSTM_EINVAL", 2: "PSTM_ENOMEM", 3: "PSTM_ETIMEOUT",
                4: "PSTM_EBOUNDS", 5: "PSTM_ECUDA", 6: "PSTM_ENOTSUP"}


class Grid(C.Structure):
    _fields_ = [("n_il", C.c_int32), ("n_xl", C.c_int32), ("n_times", C.c_int32),
                ("origin_x", C.c_double), ("origin_y", C.c_double),
                ("il_dx", C.c_double), ("il_dy", C.c_double),
                ("xl_dx", C.c_double), ("xl_dy", C.c_double),
                ("t0_ms", C.c_double), ("dt_ms", C.c_double)]


class Params(C.Structure):
    _fields_ = [("n_samples", C.c_int32), ("in_t0_ms", C.c_double), ("in_dt_ms", C.c_double),
                ("max_aperture_m", C.c_double), ("max_angle_deg", C.c_double),
                ("time_dependent_aperture", C.c_int32), ("weight", C.c_int32),
                ("clamp", C.c_int32), ("storage", C.c_int32), ("antialias", C.c_int32),
                ("aa_dx", C.c_double), ("aa_dy", C.c_double), ("aa_max_halfwidth", C.c_double),
                ("variant", C.c_int32), ("forward_only", C.c_int32),
                ("taper_width", C.c_double), ("ray_gradient", C.c_double)]


class Geometry(C.Structure):
    _fields_ = [("n_traces", C.c_int64), ("coord_dtype", C.c_int32),
                ("source_x", C.c_void_p), ("source_y", C.c_void_p),
                ("receiver_x", C.c_void_p), ("receiver_y", C.c_void_p)]


class PlanStats(C.Structure):
    _fields_ = [("n_traces", C.c_int64), ("n_tiles", C.c_int64), ("list_entries", C.c_int64),
                ("device_bytes", C.c_int64), ("tile_il", C.c_int32), ("tile_xl", C.c_int32),
                ("t_window", C.c_int32), ("variant", C.c_int32)]


class TimeRmsParams(C.Structure):
    _fields_ = [("n_samples", C.c_int64), ("n_traces", C.c_int64), ("n_points", C.c_int64),
                ("n_times", C.c_int32), ("tile", C.c_int32),
                ("dt_ms", C.c_double), ("t_min_ms", C.c_double),
                ("max_aperture_m", C.c_double), ("max_angle_deg", C.c_double),
                ("time_dependent_aperture", C.c_int32)]


class PSTMError(RuntimeError):
    """A non-OK status from libseispstm."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class PSTMTimeout(PSTMError):
    pass


_lock = threading.Lock()
_lib = None

_P = C.c_void_p
_SIGNATURES = {
    "pstm_abi_version": (C.c_int32, []),
    "pstm_last_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "pstm_launch_count": (C.c_int64, []),
    "pstm_plan_create": (C.c_int, [C.POINTER(_P), C.POINTER(Grid), C.POINTER(Params),
                                   C.POINTER(Geometry), _P]),
    "pstm_plan_destroy": (C.c_int, [_P]),
    "pstm_plan_get_stats": (C.c_int, [_P, C.POINTER(PlanStats)]),
    "pstm_trim_memory": (C.c_int, [C.c_int64]),
    "pstm_copy_trace_columns": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                          _P]),
    "pstm_load_traces": (C.c_int, [_P, _P, C.c_int32, _P]),
    "pstm_migrate_loaded": (C.c_int, [_P, _P, C.c_int64, C.c_int64, _P, _P, _P]),
    "pstm_migrate": (C.c_int, [_P, _P, C.c_int32, _P, C.c_int64, C.c_int64, _P, _P, _P]),
    "pstm_fold": (C.c_int, [_P, _P, C.c_int64, C.c_int64, _P, _P]),
    "pstm_demigrate": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, _P, C.c_int32, _P]),
    "pstm_velocity_gradient": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, _P, _P]),
    "pstm_check": (C.c_int, [_P, _P]),
    "pstm_normalize_by_fold": (C.c_int, [_P, _P, _P, C.c_int64, C.c_float, _P]),
    "pstm_normalize_mute": (C.c_int, [_P, _P, _P, C.c_int64, C.c_float, _P]),
    "pstm_batch_create": (C.c_int, [C.POINTER(_P), C.POINTER(_P), C.c_int32, C.POINTER(_P),
                                    C.POINTER(_P), _P, C.c_int64, C.c_int64, _P]),
    "pstm_batch_migrate": (C.c_int, [_P, _P]),
    "pstm_batch_destroy": (C.c_int, [_P]),
    "pstm_batch_size": (C.c_int32, [_P]),
    "pstm_velocity_grid": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, C.c_int32,
                                     _P, _P, _P, _P, C.c_int64, _P, _P]),
    "pstm_migrate_noalloc": (C.c_int, [C.POINTER(Grid), C.POINTER(Params), C.POINTER(Geometry),
                                       _P, _P, C.c_int64, C.c_int64, _P, _P, _P]),
    "pstm_time_rms_migrate": (C.c_int, [C.POINTER(TimeRmsParams), _P, _P, _P, _P, _P, _P, _P,
                                        _P, _P, C.c_int64, _P, _P, C.c_int64, _P, _P, _P]),
}


def lib():
    """Load libseispstm.so once (building it first if it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build(checked=CHECKED)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if CHECKED:
            L.pstm_test_set_injection.restype = C.c_int
            L.pstm_test_set_injection.argtypes = [C.c_int32]
        _lib = L
        return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().pstm_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    """Raise the Python exception matching a pstm_status (ValueError for invalid
    configuration, as the reference does)."""
    if status == PSTM_OK:
        return
    msg = last_error()
    if status == PSTM_EINVAL:
        raise ValueError(msg)
    if status == PSTM_ENOMEM:
        raise MemoryError(msg)
    if status == PSTM_ETIMEOUT:
        raise PSTMTimeout(status, msg)
    if status == PSTM_ENOTSUP:
        raise NotImplementedError(msg)
    raise PSTMError(status, msg)
