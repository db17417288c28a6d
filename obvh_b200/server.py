"""The request server through the C ABI (include/obvh_server.h).

``Server`` admits DiTO fits and LBVH + OBB-tree + collapse builds as they
arrive, under a device-memory budget, batches the fits continuously and runs
builds concurrently.  Inputs are numpy arrays (host; copied in on admission) or
CUDA tensors (read in place); the server keeps a reference to them until the
request is released.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .bvh import BUILD_COLLAPSE, BUILD_OBBS, NODE, as_faces4


class Config(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("build_lanes", ctypes.c_uint32),
                ("max_batch_sets", ctypes.c_uint32), ("fit_flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "completed", "failed", "fits", "builds", "fit_batches")] + \
               [(n, ctypes.c_float) for n in ("p50_ms", "p99_ms", "mean_ms", "max_ms")] + \
               [(n, ctypes.c_uint64) for n in ("arena_bytes", "peak_bytes", "in_use_bytes")] + \
               [("span_s", ctypes.c_float), ("build_batches", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class BuildView(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("nodes", "parents", "primitive_counts", "costs", "bounds", "obbs",
                                               "transforms", "collapsed", "primitives")] + \
               [("face_count", ctypes.c_uint32), ("primitive_slots", ctypes.c_uint32)]


def _bind(lib):
    c = ctypes
    vp, err, u64p = c.c_void_p, c.c_void_p, c.POINTER(c.c_uint64)
    for name, (res, args) in {
        "obvh_server_create": (err, [c.POINTER(Config), c.POINTER(vp)]),
        "obvh_server_destroy": (err, [vp]),
        "obvh_server_submit_fit": (err, [vp, vp, c.c_uint64, u64p]),
        "obvh_server_submit_fit_device": (err, [vp, vp, c.c_uint64, u64p]),
        "obvh_server_submit_build": (err, [vp, vp, c.c_uint64, vp, c.c_uint32, c.c_uint32, c.c_float, c.c_float,
                                           u64p]),
        "obvh_server_submit_build_device": (err, [vp, vp, c.c_uint64, vp, c.c_uint32, c.c_uint32, c.c_float,
                                                  c.c_float, u64p]),
        "obvh_server_wait": (err, [vp, c.c_uint64, c.c_uint32, c.POINTER(c.c_uint32)]),
        "obvh_server_drain": (err, [vp, c.c_uint32, c.POINTER(c.c_uint32)]),
        "obvh_server_fit_result": (err, [vp, c.c_uint64, vp]),
        "obvh_server_build_result": (err, [vp, c.c_uint64, c.POINTER(BuildView)]),
        "obvh_server_latency": (err, [vp, c.c_uint64, c.POINTER(c.c_float)]),
        "obvh_server_release": (err, [vp, c.c_uint64]),
        "obvh_server_get_stats": (err, [vp, c.POINTER(Stats)]),
    }.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


class Server:
    def __init__(self, budget_bytes: int = 0, build_lanes: int = 0, max_batch_sets: int = 0, fit_flags: int = 0):
        self.lib = _native.lib()
        _bind(self.lib)
        cfg = Config(budget_bytes, build_lanes, max_batch_sets, fit_flags, 0)
        h = ctypes.c_void_p()
        _native.check(self.lib.obvh_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def close(self):
        if self.h:
            self.lib.obvh_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- submission ---------------------------------------------------------
    def submit_fit(self, points) -> int:
        rid = ctypes.c_uint64()
        if hasattr(points, "is_cuda") and points.is_cuda:
            p = points.contiguous()
            _native.check(self.lib.obvh_server_submit_fit_device(self.h, ctypes.c_void_p(p.data_ptr()),
                                                                 p.numel() // 3, ctypes.byref(rid)))
        else:
            p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
            _native.check(self.lib.obvh_server_submit_fit(self.h, p.ctypes.data if p.size else None, p.shape[0],
                                                          ctypes.byref(rid)))
        self._keep[rid.value] = p
        return rid.value

    def submit_build(self, verts, faces, flags: int = BUILD_OBBS | BUILD_COLLAPSE, ci: float = 1.2,
                     ct: float = 1.0) -> int:
        rid = ctypes.c_uint64()
        if hasattr(verts, "is_cuda") and verts.is_cuda:
            v, f = verts.contiguous(), faces.contiguous()
            _native.check(self.lib.obvh_server_submit_build_device(
                self.h, ctypes.c_void_p(v.data_ptr()), v.numel() // 3, ctypes.c_void_p(f.data_ptr()),
                f.numel() // 4, flags, ci, ct, ctypes.byref(rid)))
        else:
            v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
            f = as_faces4(faces)
            _native.check(self.lib.obvh_server_submit_build(self.h, v.ctypes.data, v.shape[0], f.ctypes.data,
                                                            f.shape[0], flags, ci, ct, ctypes.byref(rid)))
        self._keep[rid.value] = (v, f)
        return rid.value

    # -- completion -----------------------------------------------------------
    def wait(self, rid: int, timeout_ms: int = 60_000) -> bool:
        done = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_server_wait(self.h, rid, timeout_ms, ctypes.byref(done)))
        return bool(done.value)

    def drain(self, timeout_ms: int = 300_000):
        done = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_server_drain(self.h, timeout_ms, ctypes.byref(done)))
        if not done.value:
            raise _native.ObvhError(f"obvh_server_drain: requests still in flight after {timeout_ms} ms")

    def fit_result(self, rid: int) -> np.ndarray:
        out = np.zeros(15, np.float32)
        _native.check(self.lib.obvh_server_fit_result(self.h, rid, out.ctypes.data))
        return out

    def build_view(self, rid: int) -> BuildView:
        v = BuildView()
        _native.check(self.lib.obvh_server_build_result(self.h, rid, ctypes.byref(v)))
        return v

    def build_result(self, rid: int) -> dict:
        """Copies a completed build's device-resident outputs to numpy arrays."""
        import torch  # noqa: F401  (the CUDA runtime)
        v = self.build_view(rid)
        rt = ctypes.CDLL("libcudart.so.12")
        n = v.face_count
        nn = 2 * n - 1

        def d2h(ptr, dtype, count):
            out = np.empty(count, dtype)
            if ptr and count:
                e = rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr),
                                  ctypes.c_size_t(out.nbytes), 2)
                if e != 0:
                    raise _native.ObvhError(f"cudaMemcpy failed ({e})")
            return out if ptr else None

        return {"nodes": d2h(v.nodes, NODE, nn), "parents": d2h(v.parents, np.uint32, nn),
                "counts": d2h(v.primitive_counts, np.uint32, nn), "costs": d2h(v.costs, np.float32, nn),
                "bounds": d2h(v.bounds, np.float32, 12),
                "obbs": None if not v.obbs else d2h(v.obbs, np.float32, 15 * nn).reshape(-1, 15),
                "transforms": None if not v.transforms else d2h(v.transforms, np.float32, 16 * nn).reshape(-1, 16),
                "collapsed": d2h(v.collapsed, NODE, nn), "primitives": d2h(v.primitives, np.uint32, n),
                "slots": v.primitive_slots}

    def latency_ms(self, rid: int) -> float:
        ms = ctypes.c_float(0)
        _native.check(self.lib.obvh_server_latency(self.h, rid, ctypes.byref(ms)))
        return ms.value

    def release(self, rid: int):
        _native.check(self.lib.obvh_server_release(self.h, rid))
        self._keep.pop(rid, None)

    def stats(self) -> dict:
        s = Stats()
        _native.check(self.lib.obvh_server_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()
