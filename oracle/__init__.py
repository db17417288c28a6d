"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  It loads

* ``liboracle.so`` - the scalar C restatements in this directory, and
* ``_ref/libref_dito.so`` - the reference's own CPU DiTO compiled from its
  sources (present where the reference tree was available at build time).

Both are (re)built with ``make`` on first use if missing.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libref_dito.so")

DITO_CPU = 0
DITO_GPU = 1

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build(force: bool = False, ref_tree: str | None = None) -> None:
    """Compile liboracle.so, and _ref from the reference source tree
    ``ref_tree`` (or the ``REF`` environment variable) when one is given."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_tree:
        cmd.append(f"REF={ref_tree}")
    if force or ref_tree or not os.path.exists(_LIB) or _stale():
        subprocess.run(cmd, check=True)


def _stale() -> bool:
    lib_t = os.path.getmtime(_LIB)
    for f in os.listdir(HERE):
        if f.endswith((".c", ".h")) and os.path.getmtime(os.path.join(HERE, f)) > lib_t:
            return True
    return False


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_dito14.argtypes = [_f32p, ctypes.c_int64, ctypes.c_int, _f32p, _f32p]
        _lib.oracle_dito14.restype = ctypes.c_int
        _lib.oracle_dito_extremal7.argtypes = [_f32p, ctypes.c_int64, _f32p, _f32p, _i64p, _i64p]
        _lib.oracle_dito_extremal7.restype = None
        _bind_bvh(_lib)
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref() -> ctypes.CDLL:
    """The reference's own DiTO_14<float> + kr_points_obb clamp."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            build()
        if not os.path.exists(_REF):
            raise FileNotFoundError("oracle/_ref/libref_dito.so was never built (no reference tree)")
        _ref = ctypes.CDLL(_REF)
        _ref.ref_dito14.argtypes = [_f32p, ctypes.c_int64, _f32p]
        _ref.ref_dito14.restype = None
        _ref.ref_dito14_batch.argtypes = [_f32p, _i64p, ctypes.c_int64, _f32p, ctypes.c_int]
        _ref.ref_dito14_batch.restype = None
    return _ref


def _pts(points) -> np.ndarray:
    p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    return p


def dito14(points, mode: int = DITO_CPU):
    """Returns (obb[15] = mid, v0, v1, v2, ext; axes[9]; path kind)."""
    p = _pts(points)
    out = np.zeros(15, np.float32)
    axes = np.zeros(9, np.float32)
    kind = lib().oracle_dito14(p.reshape(-1), p.shape[0], mode, out, axes)
    return out, axes, kind


def extremal7(points):
    p = _pts(points)
    mn = np.zeros(7, np.float32)
    mx = np.zeros(7, np.float32)
    amn = np.zeros(7, np.int64)
    amx = np.zeros(7, np.int64)
    lib().oracle_dito_extremal7(p.reshape(-1), p.shape[0], mn, mx, amn, amx)
    return mn, mx, amn, amx


def ref_dito14(points) -> np.ndarray:
    p = _pts(points)
    out = np.zeros(15, np.float32)
    ref().ref_dito14(p.reshape(-1), p.shape[0], out)
    return out


def ref_dito14_batch(points, offsets, threads: int) -> np.ndarray:
    p = _pts(points)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    out = np.zeros((len(off) - 1, 15), np.float32)
    ref().ref_dito14_batch(p.reshape(-1), off, len(off) - 1, out.reshape(-1), int(threads))
    return out


def _bind_bvh(l: ctypes.CDLL) -> None:
    """Bindings for the tree restatements (bvh_oracle.c), when compiled in."""
    if not hasattr(l, "oracle_lbvh_build"):
        return
    from . import bvh  # noqa: F401  (binds lazily on import)
