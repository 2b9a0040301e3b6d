"""ctypes binding of the in-tree native library (include/tlno_gpu.h).

The library is the only compute path: importing this module loads
origo_tlno_b200/_lib/libtlno_gpu.so and raises if it is missing; there is no
Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# TLNO_GPU_LIB selects another build of the same library (same C ABI)
LIB_PATH = os.environ.get("TLNO_GPU_LIB") or os.path.join(_HERE, "_lib", "libtlno_gpu.so")

OK = 0
E_INVALID = -1
E_CUDA = -2
E_STATE = -3
E_DEVICE = -4

DEVICE_PTRS = 0x1
WANT_J = 0x2
WANT_K = 0x4
WANT_G = 0x8
MIXED = 0x10
NO_VALIDATE = 0x20


class TlnoError(RuntimeError):
    """Raised for a negative status; .code holds the status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class Screening(C.Structure):
    _fields_ = [("integral_threshold", C.c_double),
                ("primitive_fastschwarz_threshold", C.c_double),
                ("decay_threshold", C.c_double),
                ("density_threshold", C.c_double),
                ("mixed_threshold", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("M", C.c_int), ("n_shells", C.c_int), ("shell_pairs", C.c_longlong),
                ("kept_pairs", C.c_longlong), ("quartets", C.c_longlong),
                ("primitive_quartets", C.c_longlong), ("flops", C.c_double),
                ("n_class_launches", C.c_int)]


class IncrementalOptions(C.Structure):
    _fields_ = [("base_options", Screening), ("exact_rebuild_interval", C.c_ulonglong),
                ("delta_density_threshold", C.c_double), ("use_first_delta_density_threshold", C.c_int),
                ("first_delta_density_threshold", C.c_double)]


class IncrementalInfo(C.Structure):
    _fields_ = [("updates", C.c_ulonglong), ("exact_rebuilds", C.c_ulonglong),
                ("incremental_updates", C.c_ulonglong), ("skipped_updates", C.c_ulonglong),
                ("last_status", C.c_int), ("initialized", C.c_int),
                ("last_max_abs_density_delta", C.c_double), ("last_effective_density_threshold", C.c_double),
                ("updates_since_exact_rebuild", C.c_ulonglong)]


class Tuning(C.Structure):
    _fields_ = [("generic_bk", C.c_int), ("generic_warps", C.c_int), ("grid_mult", C.c_int), ("streams", C.c_int)]


_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m origo_tlno_b200.build` "
                          "(the CUDA library is the only compute path)")
    L = C.CDLL(LIB_PATH)
    sig = {
        "tlno_gpu_last_error": (C.c_char_p, []),
        "tlno_gpu_version": (C.c_int, []),
        "tlno_gpu_device_count": (C.c_int, [_ip]),
        "tlno_gpu_create": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.c_int, C.POINTER(_vp)]),
        "tlno_gpu_create_from_components": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.c_int,
                                                      C.POINTER(_vp)]),
        "tlno_gpu_destroy": (None, [_vp]),
        "tlno_gpu_n_sph": (C.c_int, [_vp]),
        "tlno_gpu_n_shells": (C.c_int, [_vp]),
        "tlno_gpu_plan": (C.c_int, [_vp, C.POINTER(Screening)]),
        "tlno_gpu_plan_profile": (C.c_int, [_vp, C.POINTER(Profile)]),
        "tlno_gpu_jk": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int]),
        "tlno_gpu_jk_with_options": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.POINTER(Screening)]),
        "tlno_gpu_eri_checksum": (C.c_int, [_vp, _dp, _dp]),
        "tlno_gpu_incremental_create": (C.c_int, [_vp, C.POINTER(IncrementalOptions), C.POINTER(_vp)]),
        "tlno_gpu_incremental_destroy": (None, [_vp]),
        "tlno_gpu_incremental_update": (C.c_int, [_vp, _vp, C.c_int, C.c_int]),
        "tlno_gpu_incremental_g": (C.c_int, [_vp, _vp, C.c_int]),
        "tlno_gpu_incremental_density": (C.c_int, [_vp, _vp, C.c_int]),
        "tlno_gpu_incremental_info_get": (C.c_int, [_vp, C.POINTER(IncrementalInfo)]),
        "tlno_gpu_incremental_reset": (C.c_int, [_vp]),
        "tlno_gpu_incremental_fail_next_update": (C.c_int, [_vp, C.c_int]),
        "tlno_gpu_onee": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int]),
        "tlno_gpu_set_onee_thresholds": (C.c_int, [_vp, C.c_double, C.c_double]),
        "tlno_gpu_set_mixed_threshold": (C.c_int, [_vp, C.c_double]),
        "tlno_gpu_eri_blocks": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
        "tlno_gpu_eri_blocks_noalloc": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
        "tlno_gpu_schwarz": (C.c_int, [_vp, _vp]),
        "tlno_gpu_boys": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp]),
        "tlno_gpu_rys": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int]),
        "tlno_gpu_fma_peak": (C.c_int, [C.c_int, C.c_int, _dp]),
        "tlno_gpu_jk_graph_capture": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int]),
        "tlno_gpu_jk_graph_launch": (C.c_int, [_vp]),
        "tlno_gpu_synchronize": (C.c_int, [_vp]),
        "tlno_gpu_stream": (_vp, [_vp]),
        "tlno_gpu_batch_create": (C.c_int, [C.c_int, _vp, C.POINTER(Screening), C.POINTER(_vp)]),
        "tlno_gpu_batch_destroy": (None, [_vp]),
        "tlno_gpu_batch_total_elements": (C.c_longlong, [_vp]),
        "tlno_gpu_batch_offsets": (C.c_int, [_vp, _vp]),
        "tlno_gpu_batch_profile": (C.c_int, [_vp, C.POINTER(Profile)]),
        "tlno_gpu_batch_jk": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int]),
        "tlno_gpu_batch_graph_capture": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int]),
        "tlno_gpu_batch_graph_launch": (C.c_int, [_vp]),
        "tlno_gpu_batch_synchronize": (C.c_int, [_vp]),
        "tlno_gpu_batch_stream": (_vp, [_vp]),
        "tlno_gpu_set_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
        "tlno_gpu_set_combo_generic": (C.c_int, [_vp, C.c_int, C.c_int]),
        "tlno_gpu_plan_combos": (C.c_int, [_vp, C.c_int, _vp, _vp]),
        "tlno_gpu_time_combo": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp]),
        "tlno_gpu_set_class_tuning": (C.c_int, [_vp, C.c_int, C.c_double, C.c_int]),
        "tlno_gpu_batch_set_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
        "tlno_gpu_class_jk": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_int, _dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc: int) -> int:
    if rc < 0:
        msg = lib().tlno_gpu_last_error().decode(errors="replace")
        raise TlnoError(rc, msg)
    return rc


def ptr(a) -> int:
    """Address of a contiguous numpy array (or None -> 0)."""
    if a is None:
        return None
    return a.ctypes.data


EXPORTED = [
    "tlno_gpu_last_error", "tlno_gpu_version", "tlno_gpu_device_count", "tlno_gpu_create",
    "tlno_gpu_create_from_components", "tlno_gpu_destroy", "tlno_gpu_n_sph", "tlno_gpu_n_shells",
    "tlno_gpu_plan", "tlno_gpu_plan_profile", "tlno_gpu_jk", "tlno_gpu_jk_with_options", "tlno_gpu_eri_checksum",
    "tlno_gpu_incremental_create", "tlno_gpu_incremental_destroy", "tlno_gpu_incremental_update",
    "tlno_gpu_incremental_g", "tlno_gpu_incremental_density", "tlno_gpu_incremental_info_get",
    "tlno_gpu_incremental_reset", "tlno_gpu_incremental_fail_next_update",
    "tlno_gpu_onee", "tlno_gpu_set_onee_thresholds",
    "tlno_gpu_set_mixed_threshold",
    "tlno_gpu_eri_blocks", "tlno_gpu_eri_blocks_noalloc", "tlno_gpu_schwarz", "tlno_gpu_boys", "tlno_gpu_rys", "tlno_gpu_fma_peak",
    "tlno_gpu_jk_graph_capture",
    "tlno_gpu_jk_graph_launch", "tlno_gpu_synchronize", "tlno_gpu_stream", "tlno_gpu_batch_create",
    "tlno_gpu_batch_destroy", "tlno_gpu_batch_total_elements", "tlno_gpu_batch_offsets",
    "tlno_gpu_batch_profile", "tlno_gpu_batch_jk", "tlno_gpu_batch_graph_capture",
    "tlno_gpu_batch_graph_launch", "tlno_gpu_batch_synchronize", "tlno_gpu_batch_stream",
    "tlno_gpu_set_tuning", "tlno_gpu_set_combo_generic", "tlno_gpu_plan_combos", "tlno_gpu_time_combo",
    "tlno_gpu_set_class_tuning", "tlno_gpu_class_jk", "tlno_gpu_batch_set_tuning",
]
