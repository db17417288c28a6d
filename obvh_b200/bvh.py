"""BVH builds and transforms through the C ABI (include/obvh_lbvh.h,
include/obvh_transforms.h).  Device buffers are torch tensors (raw bytes for
the 36-byte kr_bvh_node records); numpy views use the NODE dtype.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

NODE = np.dtype([("b", "<f4", (6,)), ("left", "<u4"), ("right", "<u4"), ("n_prims", "<u2"),
                 ("axis", "u1"), ("pad", "u1")])
NODE_BYTES = 36
assert NODE.itemsize == NODE_BYTES


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(torch, stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def nodes_numpy(t) -> np.ndarray:
    """A device node buffer (uint8 [k*36]) as a numpy NODE array."""
    return t.cpu().numpy().view(NODE).reshape(-1)


def as_faces4(faces) -> np.ndarray:
    f = np.ascontiguousarray(faces, dtype=np.uint32)
    if f.shape[1] == 3:
        f = np.concatenate([f, np.zeros((f.shape[0], 1), np.uint32)], axis=1)
    return np.ascontiguousarray(f)


class Mesh:
    """A triangle mesh resident on the device (vertices float32 [V,3], faces
    uint32 [F,4] stored in an int32 tensor)."""

    def __init__(self, verts, faces, device="cuda"):
        import torch
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        f = as_faces4(faces)
        self.n_vertices = v.shape[0]
        self.n_faces = f.shape[0]
        self.verts = torch.from_numpy(v).to(device)
        self.faces = torch.from_numpy(f.view(np.int32)).to(device)

    @classmethod
    def from_device(cls, verts, faces):
        """Wraps CUDA tensors already on the device (float32 [V,3], int32/uint32 [F,4])."""
        m = cls.__new__(cls)
        m.verts = verts.contiguous()
        m.faces = faces.contiguous()
        m.n_vertices = m.verts.shape[0]
        m.n_faces = m.faces.shape[0]
        return m


class LbvhBuilder:
    """obvh_lbvh_build_async with a workspace kept between builds."""

    def __init__(self, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.lib = _native.lib()
        self.ws = None
        self.ws_prims = -1

    def _workspace(self, n, stream):
        if self.ws is None or n > self.ws_prims:
            nbytes = int(self.lib.obvh_lbvh_workspace_bytes(n))
            self.ws = self.torch.empty(nbytes, dtype=self.torch.uint8, device=self.device)
            self.ws_prims = n
            _native.check(self.lib.obvh_lbvh_workspace_init(_ptr(self.ws), n, stream))
        return self.ws

    def build(self, mesh: Mesh, stream=None, out=None):
        """Enqueues the build; returns dict(nodes, parents, counts, costs, bounds) of device tensors."""
        t = self.torch
        n = mesh.n_faces
        nn = 2 * n - 1
        s = _stream(t, stream)
        ws = self._workspace(n, s)
        if out is None:
            out = {
                "nodes": t.empty(nn * NODE_BYTES, dtype=t.uint8, device=self.device),
                "parents": t.empty(nn, dtype=t.int32, device=self.device),
                "counts": t.empty(nn, dtype=t.int32, device=self.device),
                "costs": t.empty(nn, dtype=t.float32, device=self.device),
                "bounds": t.empty(12, dtype=t.float32, device=self.device),
            }
        e = self.lib.obvh_lbvh_build_async(_ptr(mesh.verts), _ptr(mesh.faces), n, _ptr(out["nodes"]),
                                           _ptr(out["parents"]), _ptr(out["counts"]), _ptr(out["costs"]),
                                           _ptr(out["bounds"]), _ptr(ws), s)
        _native.check(e)
        return out


def bbox_calculate(mesh: Mesh, centroid: bool = False, prefill=None):
    """kr_cuda_bbox_calculate / kr_cuda_centroid_bbox_calculate on a device mesh;
    returns the 6 floats of the (pre-filled, default empty) box after the call."""
    import torch
    lib = _native.lib()
    big = np.float32(3.402823466e+38)
    init = np.array([big, big, big, -big, -big, -big], np.float32) if prefill is None else np.asarray(prefill,
                                                                                                       np.float32)
    box = torch.from_numpy(init.copy()).cuda()
    f = lib.kr_cuda_centroid_bbox_calculate if centroid else lib.kr_cuda_bbox_calculate
    _native.check(f(_ptr(mesh.faces), _ptr(mesh.verts), mesh.n_faces, _ptr(box)))
    return box.cpu().numpy()


def obb_tree(mesh: Mesh, tree: dict, obbs=None, transforms=None):
    """kr_cuda_bvh_obb_tree (synchronous) on a device tree; returns (obbs [nn,15], transforms [nn,16])."""
    import torch
    lib = _native.lib()
    nn = tree["parents"].numel()
    n = (nn + 1) // 2
    if obbs is None:
        obbs = torch.empty((nn, 15), dtype=torch.float32, device=tree["parents"].device)
    if transforms is None:
        transforms = torch.empty((nn, 16), dtype=torch.float32, device=tree["parents"].device)
    e = lib.kr_cuda_bvh_obb_tree(_ptr(tree["nodes"]), _ptr(tree["parents"]), _ptr(tree.get("counts")),
                                 _ptr(tree.get("costs")), _ptr(mesh.verts), _ptr(mesh.faces), None, _ptr(obbs),
                                 _ptr(transforms), 1.2, 1.0, 1.0, n, n - 1, 0xFFFFFFFF)
    _native.check(e)
    return obbs, transforms


class ObbTreeTransformer:
    """obvh_bvh_obb_tree_async with a workspace kept between calls."""

    def __init__(self, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.lib = _native.lib()
        self.ws = None
        self.ws_prims = -1

    def __call__(self, mesh: Mesh, tree: dict, obbs, transforms, stream=None):
        t = self.torch
        nn = tree["parents"].numel()
        n = (nn + 1) // 2
        if self.ws is None or n > self.ws_prims:
            self.ws = t.empty(int(self.lib.obvh_obb_tree_workspace_bytes(n)), dtype=t.uint8, device=self.device)
            self.ws_prims = n
        e = self.lib.obvh_bvh_obb_tree_async(_ptr(tree["nodes"]), _ptr(tree["parents"]), _ptr(mesh.verts),
                                             _ptr(mesh.faces), _ptr(obbs), _ptr(transforms), n, n - 1, _ptr(self.ws),
                                             _stream(t, stream))
        _native.check(e)

    def device_error(self, stream=None):
        v = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_obb_tree_error(_ptr(self.ws), _stream(self.torch, stream), ctypes.byref(v)))
        return v.value


def collapse(tree: dict, ci: float = 1.2, ct: float = 1.0, metrics: bool = False):
    """kr_cuda_bvh_collapse (synchronous).  Rewrites tree['counts'] and tree['costs'] in
    place like the reference; returns dict(collapsed, primitives[, metrics])."""
    import torch
    lib = _native.lib()
    nn = tree["parents"].numel()
    n = (nn + 1) // 2
    dev = tree["parents"].device
    out = {"collapsed": torch.empty(nn * NODE_BYTES, dtype=torch.uint8, device=dev),
           "primitives": torch.zeros(n, dtype=torch.int32, device=dev)}
    m = (ctypes.c_float * 2)(0.0, 0.0)
    e = lib.kr_cuda_bvh_collapse(_ptr(tree["nodes"]), _ptr(tree["parents"]), _ptr(out["collapsed"]),
                                 _ptr(tree["counts"]), _ptr(out["primitives"]), _ptr(tree["costs"]), ci, ct, n,
                                 n - 1, ctypes.cast(m, ctypes.c_void_p) if metrics else None)
    _native.check(e)
    if metrics:
        out["metrics"] = (m[0], m[1])
    return out


BUILD_OBBS = 0x1
BUILD_COLLAPSE = 0x2


class ObvhBuilder:
    """obvh_build_async: LBVH + OBB tree + collapse in one chain of kernels,
    with the workspace kept between builds."""

    def __init__(self, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.lib = _native.lib()
        self.ws = None
        self.ws_faces = -1

    def _workspace(self, n, s):
        if self.ws is None or n > self.ws_faces:
            self.ws = self.torch.empty(int(self.lib.obvh_build_workspace_bytes(n)), dtype=self.torch.uint8,
                                       device=self.device)
            self.ws_faces = n
            _native.check(self.lib.obvh_build_workspace_init(_ptr(self.ws), n, s))
        return self.ws

    def outputs(self, n):
        t = self.torch
        nn = 2 * n - 1
        d = self.device
        return {"nodes": t.empty(nn * NODE_BYTES, dtype=t.uint8, device=d),
                "parents": t.empty(nn, dtype=t.int32, device=d), "counts": t.empty(nn, dtype=t.int32, device=d),
                "costs": t.empty(nn, dtype=t.float32, device=d), "bounds": t.empty(12, dtype=t.float32, device=d),
                "obbs": t.empty((nn, 15), dtype=t.float32, device=d),
                "transforms": t.empty((nn, 16), dtype=t.float32, device=d),
                "collapsed": t.empty(nn * NODE_BYTES, dtype=t.uint8, device=d),
                "primitives": t.zeros(n, dtype=t.int32, device=d)}

    def build(self, mesh: Mesh, flags=BUILD_OBBS | BUILD_COLLAPSE, ci=1.2, ct=1.0, stream=None, out=None):
        n = mesh.n_faces
        s = _stream(self.torch, stream)
        ws = self._workspace(n, s)
        o = out if out is not None else self.outputs(n)
        e = self.lib.obvh_build_async(_ptr(mesh.verts), _ptr(mesh.faces), n, flags, ci, ct, _ptr(o["nodes"]),
                                      _ptr(o["parents"]), _ptr(o["counts"]), _ptr(o["costs"]), _ptr(o["bounds"]),
                                      _ptr(o["obbs"]), _ptr(o["transforms"]), _ptr(o["collapsed"]),
                                      _ptr(o["primitives"]), _ptr(ws), s)
        _native.check(e)
        return o

    def status(self, n, stream=None):
        err = ctypes.c_uint32(0)
        slots = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_build_status(_ptr(self.ws), n, _stream(self.torch, stream), ctypes.byref(err),
                                                 ctypes.byref(slots)))
        return err.value, slots.value


ATRBVH_TREELET_SIZE = 9  # OBVH_ATRBVH_TREELET_SIZE: the reference intersector's treelet size
ATRBVH_ITERATIONS = 2


class AtrbvhBuilder(ObvhBuilder):
    """obvh_build_atrbvh_async: ATRBVH (LBVH-63 + agglomerative treelets), then
    the OBB tree and the collapse, with the workspace kept between builds."""

    def _workspace(self, n, s):
        if self.ws is None or n > self.ws_faces:
            self.ws = self.torch.empty(int(self.lib.obvh_atrbvh_workspace_bytes(n)), dtype=self.torch.uint8,
                                       device=self.device)
            self.ws_faces = n
            _native.check(self.lib.obvh_atrbvh_workspace_init(_ptr(self.ws), n, s))
        return self.ws

    def outputs(self, n):
        o = super().outputs(n)
        o["bounds"] = self.torch.empty(6, dtype=self.torch.float32, device=self.device)  # scene box only
        return o

    def build(self, mesh: Mesh, flags=BUILD_OBBS | BUILD_COLLAPSE, ci=1.2, ct=1.0, stream=None, out=None,
              treelet_size=ATRBVH_TREELET_SIZE, iterations=ATRBVH_ITERATIONS):
        n = mesh.n_faces
        s = _stream(self.torch, stream)
        ws = self._workspace(n, s)
        o = out if out is not None else self.outputs(n)
        e = self.lib.obvh_build_atrbvh_async(_ptr(mesh.verts), _ptr(mesh.faces), n, flags, treelet_size, iterations,
                                             ci, ct, _ptr(o["nodes"]), _ptr(o["parents"]), _ptr(o["counts"]),
                                             _ptr(o["costs"]), _ptr(o["bounds"]), _ptr(o["obbs"]),
                                             _ptr(o["transforms"]), _ptr(o["collapsed"]), _ptr(o["primitives"]),
                                             _ptr(ws), s)
        _native.check(e)
        return o

    def status(self, n, stream=None):
        err = ctypes.c_uint32(0)
        slots = ctypes.c_uint32(0)
        _native.check(self.lib.obvh_atrbvh_status(_ptr(self.ws), n, _stream(self.torch, stream), ctypes.byref(err),
                                                  ctypes.byref(slots)))
        return err.value, slots.value
