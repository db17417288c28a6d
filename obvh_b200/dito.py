"""DiTO-14 OBB fits through the C ABI (include/obvh_dito.h).

Mirrors the reference's two ways in:

* ``points_obb(points)`` - ``kr_cuda_points_obb`` (host array in, synchronous,
  box by value; src/common/algorithm/dito/dito.cuh:12-13).
* ``DitoFitter`` - the device-resident form (``obvh_dito_fit_async``) that
  keeps its workspace on the GPU and enqueues on a CUDA stream.

Boxes are returned as float32 arrays of 15 values: mid, v0, v1, v2, ext.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

REFERENCE_GPU = 0x1  # OBVH_DITO_REFERENCE_GPU


def _host_points(points) -> np.ndarray:
    p = np.ascontiguousarray(points, dtype=np.float32)
    if p.ndim != 2 or p.shape[1] != 3:
        p = p.reshape(-1, 3)
    return p


def points_obb(points, flags: int = 0, return_time: bool = False):
    """OBB of a host point array (N x 3 float32).  Raises ObvhError on failure."""
    lib = _native.lib()
    p = _host_points(points)
    out = np.zeros(15, np.float32)
    ms = ctypes.c_float(0.0)
    e = lib.obvh_points_obb(p.ctypes.data if p.size else None, p.shape[0], flags,
                            out.ctypes.data, ctypes.byref(ms))
    _native.check(e)
    return (out, ms.value) if return_time else out


def kr_cuda_points_obb(points):
    """The reference-signature call (no error channel): returns (obb[15], elapsed_ms)."""
    lib = _native.lib()
    p = _host_points(points)
    ms = ctypes.c_float(0.0)
    r = lib.kr_cuda_points_obb(p.ctypes.data if p.size else None, p.shape[0], ctypes.byref(ms))
    return np.frombuffer(bytes(r.v), dtype=np.float32).copy(), ms.value


class DitoFitter:
    """Device-resident fits: points and boxes are CUDA tensors (torch is used
    only to hold device memory and name the stream)."""

    def __init__(self, device=None):
        import torch
        self.torch = torch
        self.lib = _native.lib()
        self.device = torch.device(device or "cuda")
        nbytes = int(self.lib.obvh_dito_workspace_bytes())
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        _native.check(self.lib.obvh_dito_workspace_init(self.workspace.data_ptr(), self._stream()))

    def _stream(self, stream=None):
        s = stream if stream is not None else self.torch.cuda.current_stream(self.device)
        return ctypes.c_void_p(s.cuda_stream)

    def fit(self, points, out=None, flags: int = 0, stream=None):
        """Enqueues the fit of `points` (CUDA float32, N x 3, contiguous); returns
        the (CUDA) 15-float box without synchronising."""
        t = self.torch
        if points.dtype != t.float32 or not points.is_cuda or not points.is_contiguous():
            raise ValueError("points must be a contiguous CUDA float32 tensor")
        n = points.numel() // 3
        if out is None:
            out = t.empty(15, dtype=t.float32, device=points.device)
        e = self.lib.obvh_dito_fit_async(points.data_ptr() if n else None, n, flags, out.data_ptr(),
                                         self.workspace.data_ptr(), self._stream(stream))
        _native.check(e)
        return out

    def fit_pass(self, points, out, pass_no: int, flags: int = 0, stream=None):
        """Enqueues only pass 1 or pass 2 of a fit (for per-kernel timing)."""
        n = points.numel() // 3
        e = self.lib.obvh_dito_fit_pass_async(points.data_ptr() if n else None, n, flags, out.data_ptr(),
                                              self.workspace.data_ptr(), self._stream(stream), pass_no)
        _native.check(e)
        return out

    def report(self, stream=None):
        """(path, axes[9], device_error) of the last fit (synchronises)."""
        path = ctypes.c_uint32(0)
        err = ctypes.c_uint32(0)
        axes = (ctypes.c_float * 9)()
        _native.check(self.lib.obvh_dito_workspace_report(self.workspace.data_ptr(), self._stream(stream),
                                                          ctypes.byref(path), axes, ctypes.byref(err)))
        return path.value, np.array(axes[:], np.float32), err.value
