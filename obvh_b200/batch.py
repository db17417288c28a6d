"""Batched DiTO-14 fits through the C ABI (include/obvh_batch.h).

Thousands of point sets of uneven sizes, stored as one packed point array
with CSR offsets, are fitted by one persistent work-stealing kernel (optionally
replayed from a CUDA graph).  Each box equals the single-set fit of
``dito.points_obb`` on that set, bit for bit.

* ``points_obb_batch(points, offsets)`` - host arrays in, boxes out
  (``obvh_points_obb_batch``).
* ``DitoBatch`` - a planned batch on device buffers: ``run``, ``capture`` /
  ``launch`` (CUDA graph) and ``autotune``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


def _offsets(offsets) -> np.ndarray:
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    if o.ndim != 1 or o.size < 1:
        raise ValueError("offsets must be a 1-D array of sets + 1 values")
    return o


def points_obb_batch(points, offsets, flags: int = 0, return_time: bool = False):
    """Boxes [sets x 15] of the sets points[offsets[s]:offsets[s+1]] (host arrays)."""
    lib = _native.lib()
    p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    o = _offsets(offsets)
    sets = o.size - 1
    if int(o[-1]) != p.shape[0]:
        raise ValueError("offsets[-1] must equal the number of points")
    out = np.zeros((max(sets, 1), 15), np.float32)
    ms = ctypes.c_float(0.0)
    _native.check(lib.obvh_points_obb_batch(p.ctypes.data if p.size else None, o.ctypes.data, sets, flags,
                                            out.ctypes.data, ctypes.byref(ms)))
    out = out[:sets]
    return (out, ms.value) if return_time else out


class DitoBatch:
    """A planned batch bound to the current CUDA device.  ``points`` and
    ``obbs`` passed to the methods are CUDA tensors (float32 [N, 3] and float32
    [sets, 15]); torch only holds the memory and names the stream."""

    def __init__(self, offsets, flags: int = 0, tuning: dict | None = None):
        self.lib = _native.lib()
        self.offsets = _offsets(offsets)
        self.sets = self.offsets.size - 1
        h = ctypes.c_void_p()
        t = None
        if tuning is not None:
            t = _native.DitoBatchTuning(**tuning)
        _native.check(self.lib.obvh_dito_batch_create(self.offsets.ctypes.data, self.sets, flags,
                                                      ctypes.byref(t) if t is not None else None, ctypes.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            self.lib.obvh_dito_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stream(stream):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream)

    @property
    def tuning(self) -> dict:
        t = _native.DitoBatchTuning()
        _native.check(self.lib.obvh_dito_batch_get_tuning(self.handle, ctypes.byref(t)))
        return t.as_dict()

    @tuning.setter
    def tuning(self, value: dict):
        t = _native.DitoBatchTuning(**value)
        _native.check(self.lib.obvh_dito_batch_set_tuning(self.handle, ctypes.byref(t)))

    def info(self) -> dict:
        v = [ctypes.c_uint32() for _ in range(4)]
        _native.check(self.lib.obvh_dito_batch_info(self.handle, *[ctypes.byref(x) for x in v]))
        return dict(zip(("tasks", "large_sets", "chunks", "grid"), (x.value for x in v)))

    def run(self, points, obbs, stream=None):
        """Enqueues the fits on `stream` (default: torch's current stream)."""
        _native.check(self.lib.obvh_dito_batch_enqueue(self.handle, ctypes.c_void_p(points.data_ptr()),
                                                       ctypes.c_void_p(obbs.data_ptr()), self._stream(stream)))

    def capture(self, points, obbs):
        """Captures run() for these tensors into a CUDA graph kept by the batch."""
        _native.check(self.lib.obvh_dito_batch_capture(self.handle, ctypes.c_void_p(points.data_ptr()),
                                                       ctypes.c_void_p(obbs.data_ptr())))

    def launch(self, stream=None):
        """Replays the captured graph."""
        _native.check(self.lib.obvh_dito_batch_launch(self.handle, self._stream(stream)))

    def autotune(self, points, obbs, repeats: int = 5, stream=None):
        """Picks the fastest knobs on these tensors; returns (tuning, median ms)."""
        t = _native.DitoBatchTuning()
        ms = ctypes.c_float(0.0)
        _native.check(self.lib.obvh_dito_batch_autotune(self.handle, ctypes.c_void_p(points.data_ptr()),
                                                        ctypes.c_void_p(obbs.data_ptr()), self._stream(stream),
                                                        repeats, ctypes.byref(t), ctypes.byref(ms)))
        return t.as_dict(), ms.value

    def status(self, stream=None) -> int:
        """Device error word of the last run (0 = none); synchronises."""
        e = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_dito_batch_status(self.handle, self._stream(stream), ctypes.byref(e)))
        return e.value
