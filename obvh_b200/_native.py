"""ctypes binding of libobvh_b200.so (the C ABI declared in include/*.h).

The library is the only compute path: if it cannot be found or built, every
entry point raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os
import re
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libobvh_b200.so")
INCLUDE = os.path.join(ROOT, "include")

_lock = threading.Lock()
_lib = None


class ObvhError(RuntimeError):
    """A non-NULL kr_error returned by the native library."""


class Obb3(ctypes.Structure):
    _fields_ = [("v", ctypes.c_float * 15)]


class DitoBatchTuning(ctypes.Structure):
    """obvh_dito_batch_tuning (include/obvh_batch.h)."""
    _fields_ = [(name, ctypes.c_uint32) for name in
                ("points_per_thread", "chunk_points", "warp_max_points", "cta_max_points", "lag_tasks",
                 "ctas_per_sm")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _declare(lib: ctypes.CDLL) -> None:
    c = ctypes
    vp = c.c_void_p
    err = c.c_void_p  # kr_error: NULL or a static C string
    sig = {
        "obvh_version": (c.c_char_p, []),
        "obvh_last_error": (err, []),
        "kr_cuda_points_obb": (Obb3, [vp, c.c_uint64, c.POINTER(c.c_float)]),
        "obvh_points_obb": (err, [vp, c.c_uint64, c.c_uint32, vp, c.POINTER(c.c_float)]),
        "obvh_dito_workspace_bytes": (c.c_uint64, []),
        "obvh_dito_workspace_init": (err, [vp, vp]),
        "obvh_dito_fit_async": (err, [vp, c.c_uint64, c.c_uint32, vp, vp, vp]),
        "obvh_dito_fit_pass_async": (err, [vp, c.c_uint64, c.c_uint32, vp, vp, vp, c.c_int]),
        "obvh_points_obb_noalloc": (err, [vp, c.c_uint64, c.c_uint32, vp, vp]),
        "kr_cuda_bvh_persistent": (err, [vp, vp, c.c_uint32]),
        "kr_cuda_obvh_persistent": (err, [vp, vp, vp, vp, c.c_uint32]),
        "kr_cuda_soa_obvh": (err, [vp, vp, c.POINTER(c.c_void_p), c.c_uint32, c.c_uint32]),
        "obvh_soa_obvh_free": (err, [vp]),
        "obvh_obvh_pack_async": (err, [vp, vp, vp, vp, vp, vp, vp, c.c_uint32, c.c_uint32, vp, vp]),
        "kr_cuda_soa_obvh_intersect": (err, [vp, vp, vp, vp, vp, vp, c.c_uint32, c.c_uint32, c.c_uint32, vp]),
        "obvh_soa_obvh_intersect_async": (err, [vp, vp, vp, c.c_uint32, c.c_uint32, vp, vp, c.c_uint32, vp,
                                                c.c_uint32, vp, vp, c.c_uint32, vp, vp]),
        "kr_bvh_sah": (c.c_float, [vp, c.c_int32, c.c_float, c.c_float, vp, c.c_char_p]),
        "obvh_bvh_sah_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_bvh_sah_async": (err, [vp, vp, vp, c.c_uint32, c.c_float, c.c_float, vp, vp, vp]),
        "kr_cuda_bbox_calculate": (err, [vp, vp, c.c_uint32, vp]),
        "kr_cuda_centroid_bbox_calculate": (err, [vp, vp, c.c_uint32, vp]),
        "obvh_lbvh_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_lbvh_workspace_init": (err, [vp, c.c_uint32, vp]),
        "obvh_lbvh_build_async": (err, [vp, vp, c.c_uint32, vp, vp, vp, vp, vp, vp, vp]),
        "kr_cuda_bvh_obb_tree": (err, [vp, vp, vp, vp, vp, vp, vp, vp, vp, c.c_float, c.c_float, c.c_float,
                                       c.c_uint32, c.c_uint32, c.c_uint32]),
        "obvh_obb_tree_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_bvh_obb_tree_async": (err, [vp, vp, vp, vp, vp, vp, c.c_uint32, c.c_uint32, vp, vp]),
        "obvh_obb_tree_error": (err, [vp, vp, c.POINTER(c.c_uint32)]),
        "kr_cuda_bvh_collapse": (err, [vp, vp, vp, vp, vp, vp, c.c_float, c.c_float, c.c_uint32, c.c_uint32, vp]),
        "obvh_collapse_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_bvh_collapse_async": (err, [vp, vp, vp, vp, vp, vp, c.c_float, c.c_float, c.c_uint32, c.c_uint32,
                                          vp, vp]),
        "obvh_profile_enable": (err, [c.c_int]),
        "obvh_check_bounded_wait": (err, [c.c_uint32, c.POINTER(c.c_uint32)]),
        "obvh_profile_summary": (err, [c.c_char_p, c.c_uint64]),
        "obvh_build_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_build_workspace_init": (err, [vp, c.c_uint32, vp]),
        "obvh_build_async": (err, [vp, vp, c.c_uint32, c.c_uint32, c.c_float, c.c_float] + [vp] * 11),
        "obvh_build_status": (err, [vp, c.c_uint32, vp, c.POINTER(c.c_uint32), c.POINTER(c.c_uint32)]),
        "obvh_build_graph_create": (err, [vp, vp, c.c_uint32, c.c_uint32, c.c_float, c.c_float] + [vp] * 10
                                    + [c.POINTER(vp)]),
        "obvh_build_graph_launch": (err, [vp, vp]),
        "obvh_build_graph_destroy": (err, [vp]),
        "obvh_atrbvh_workspace_bytes": (c.c_uint64, [c.c_uint32]),
        "obvh_atrbvh_workspace_init": (err, [vp, c.c_uint32, vp]),
        "obvh_atrbvh_build_async": (err, [vp, vp, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float, c.c_float]
                                    + [vp] * 7),
        "obvh_build_atrbvh_async": (err, [vp, vp, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                          c.c_float] + [vp] * 11),
        "obvh_atrbvh_status": (err, [vp, c.c_uint32, vp, c.POINTER(c.c_uint32), c.POINTER(c.c_uint32)]),
        "obvh_build_atrbvh_graph_create": (err, [vp, vp, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32, c.c_float,
                                                 c.c_float] + [vp] * 10 + [c.POINTER(vp)]),
        "obvh_dito_batch_create": (err, [vp, c.c_uint64, c.c_uint32, vp, c.POINTER(vp)]),
        "obvh_dito_batch_destroy": (err, [vp]),
        "obvh_dito_batch_get_tuning": (err, [vp, c.POINTER(DitoBatchTuning)]),
        "obvh_dito_batch_set_tuning": (err, [vp, c.POINTER(DitoBatchTuning)]),
        "obvh_dito_batch_enqueue": (err, [vp, vp, vp, vp]),
        "obvh_dito_batch_capture": (err, [vp, vp, vp]),
        "obvh_dito_batch_launch": (err, [vp, vp]),
        "obvh_dito_batch_autotune": (err, [vp, vp, vp, vp, c.c_uint32, c.POINTER(DitoBatchTuning),
                                           c.POINTER(c.c_float)]),
        "obvh_dito_batch_status": (err, [vp, vp, c.POINTER(c.c_uint32)]),
        "obvh_dito_batch_info": (err, [vp] + [c.POINTER(c.c_uint32)] * 4),
        "obvh_points_obb_batch": (err, [vp, vp, c.c_uint64, c.c_uint32, vp, c.POINTER(c.c_float)]),
        "obvh_dito_workspace_report": (err, [vp, vp, c.POINTER(c.c_uint32), c.POINTER(c.c_float),
                                             c.POINTER(c.c_uint32)]),
        "kr_cuda_soa_compressed_obvh": (err, [vp, vp, c.POINTER(c.c_void_p), c.c_uint32, c.c_uint32]),
        "obvh_soa_obvh_compressed_free": (err, [vp]),
        "obvh_soa_compressed_obvh_async": (err, [vp] * 5 + [c.c_uint32, c.c_uint32, vp]),
        "kr_cuda_obvh_compressed_persistent_intersect": (err, [vp] * 6 + [c.c_uint32] * 3 + [vp]),
        "obvh_soa_compressed_obvh_intersect_async": (err, [vp, vp, vp, c.c_uint32, c.c_uint32, vp, vp, c.c_uint32,
                                                           vp, c.c_uint32, vp, vp, c.c_uint32, vp, vp]),
        "obvh_build_batch_create": (err, [vp, vp, c.c_uint64, c.c_uint32, c.c_uint32, c.POINTER(vp)]),
        "obvh_build_batch_destroy": (err, [vp]),
        "obvh_build_batch_enqueue": (err, [vp, vp, vp, c.c_float, c.c_float] + [vp] * 10),
        "obvh_build_batch_capture": (err, [vp, vp, vp, c.c_float, c.c_float] + [vp] * 9),
        "obvh_build_batch_launch": (err, [vp, vp]),
        "obvh_build_batch_status": (err, [vp, vp, c.POINTER(c.c_uint32), vp]),
        "obvh_build_batch_info": (err, [vp] + [c.POINTER(c.c_uint32)] * 3),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def declared_symbols() -> list[str]:
    """Every OBVH_EXPORT function named in include/*.h."""
    names = []
    pat = re.compile(r"OBVH_EXPORT\s+[\w\s\*]+?\b(\w+)\s*\(")
    for f in sorted(os.listdir(INCLUDE)):
        if f.endswith(".h"):
            with open(os.path.join(INCLUDE, f)) as fh:
                names += pat.findall(fh.read())
    return names


def lib(build_if_missing: bool = True) -> ctypes.CDLL:
    """Loads the native library (building it from csrc/ if it is out of date)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing:
            from . import build as _build
            try:
                _build.build_core()
            except Exception as e:  # pragma: no cover - no toolchain and no prebuilt library
                if not os.path.exists(LIB_PATH):
                    raise ObvhError(f"libobvh_b200.so is missing and could not be built: {e}") from e
        if not os.path.exists(LIB_PATH):
            raise ObvhError(f"native library not found: {LIB_PATH}")
        l = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        _declare(l)
        _lib = l
        return l


def check(e) -> None:
    """Raises ObvhError for a non-NULL kr_error."""
    if e:
        raise ObvhError(ctypes.string_at(e).decode(errors="replace"))
