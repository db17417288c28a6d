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

    def capture(self, mesh: Mesh, out, flags=BUILD_OBBS | BUILD_COLLAPSE, ci=1.2, ct=1.0):
        """obvh_build_graph_create: the build of this mesh's buffers into `out`
        as a CUDA graph (BuildGraph), replayed by its launch()."""
        n = mesh.n_faces
        ws = self._workspace(n, _stream(self.torch, None))
        h = ctypes.c_void_p()
        _native.check(self.lib.obvh_build_graph_create(
            _ptr(mesh.verts), _ptr(mesh.faces), n, flags, ci, ct, _ptr(out["nodes"]), _ptr(out["parents"]),
            _ptr(out["counts"]), _ptr(out["costs"]), _ptr(out["bounds"]), _ptr(out["obbs"]), _ptr(out["transforms"]),
            _ptr(out["collapsed"]), _ptr(out["primitives"]), _ptr(ws), ctypes.byref(h)))
        return BuildGraph(self, h, (ws, mesh, out))


class BuildGraph:
    """A captured obvh_build_async chain (obvh_build_graph_*).  It holds the
    workspace, mesh and output tensors whose addresses the graph baked in, so
    that none of them is freed while the graph exists (the builder may move
    on to a larger workspace)."""

    def __init__(self, builder: ObvhBuilder, handle, buffers):
        self.builder = builder
        self.lib = builder.lib
        self.handle = handle
        self.buffers = buffers

    def launch(self, stream=None):
        _native.check(self.lib.obvh_build_graph_launch(self.handle, _stream(self.builder.torch, stream)))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.obvh_build_graph_destroy(h)
            self.handle = None


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

    def capture(self, mesh: Mesh, out, flags=BUILD_OBBS | BUILD_COLLAPSE, ci=1.2, ct=1.0,
                treelet_size=ATRBVH_TREELET_SIZE, iterations=ATRBVH_ITERATIONS):
        """obvh_build_atrbvh_graph_create: this build as a CUDA graph (BuildGraph)."""
        n = mesh.n_faces
        ws = self._workspace(n, _stream(self.torch, None))
        h = ctypes.c_void_p()
        _native.check(self.lib.obvh_build_atrbvh_graph_create(
            _ptr(mesh.verts), _ptr(mesh.faces), n, flags, treelet_size, iterations, ci, ct, _ptr(out["nodes"]),
            _ptr(out["parents"]), _ptr(out["counts"]), _ptr(out["costs"]), _ptr(out["bounds"]), _ptr(out["obbs"]),
            _ptr(out["transforms"]), _ptr(out["collapsed"]), _ptr(out["primitives"]), _ptr(ws), ctypes.byref(h)))
        return BuildGraph(self, h, (ws, mesh, out))


# ---- traversal packing (include/obvh_transforms.h) -------------------------
PACKED = np.dtype([("lb", "<f4", (6,)), ("rb", "<f4", (6,)), ("meta", "<i4", (4,))])
assert PACKED.itemsize == 64


def persistent(nodes, node_count: int, transforms=None, packed=None, pairs=None):
    """kr_cuda_bvh_persistent (transforms=None) or kr_cuda_obvh_persistent on
    device tensors; packed / pairs are updated in place (zeroed when not given).
    Returns dict(packed, pairs)."""
    import torch
    lib = _native.lib()
    dev = nodes.device
    ni = (node_count - 1) // 2
    if packed is None:
        packed = torch.zeros(node_count * 64, dtype=torch.uint8, device=dev)
    if transforms is None:
        _native.check(lib.kr_cuda_bvh_persistent(_ptr(nodes), _ptr(packed), node_count))
        return {"packed": packed, "pairs": None}
    if pairs is None:
        pairs = torch.zeros(max(ni, 1) * 32, dtype=torch.float32, device=dev)
    _native.check(lib.kr_cuda_obvh_persistent(_ptr(nodes), _ptr(transforms), _ptr(packed), _ptr(pairs), node_count))
    return {"packed": packed, "pairs": pairs}


def _cudart():
    import ctypes.util
    for name in ("libcudart.so", "libcudart.so.12", ctypes.util.find_library("cudart") or ""):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    raise _native.ObvhError("the CUDA runtime library is needed to read a kr_SoA_OBVH back")


def soa_obvh(packed, pairs, internal_count: int, node_count: int, out=None):
    """kr_cuda_soa_obvh: the library allocates the SoA arrays on the device; this
    reads them back and frees them with obvh_soa_obvh_free.  Returns numpy
    left_T [ni x 12], right_T [ni x 12], metadata [nodes x 4]; with `out`
    (dict of host tensors or arrays of those sizes, e.g. pinned) the arrays
    are copied into it instead."""
    lib = _native.lib()
    d_soa = ctypes.c_void_p(0)
    _native.check(lib.kr_cuda_soa_obvh(_ptr(packed), _ptr(pairs), ctypes.byref(d_soa), internal_count, node_count))
    rt = _cudart()
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    try:
        ptrs = (ctypes.c_void_p * 3)()
        if rt.cudaMemcpy(ctypes.cast(ptrs, ctypes.c_void_p), d_soa, 24, 2) != 0:
            raise _native.ObvhError("reading the kr_SoA_OBVH struct back failed")
        if out is None:
            out = {"left_T": np.zeros((internal_count, 12), np.float32),
                   "right_T": np.zeros((internal_count, 12), np.float32),
                   "metadata": np.zeros((node_count, 4), np.int32)}
        sizes = {"left_T": 48 * internal_count, "right_T": 48 * internal_count, "metadata": 16 * node_count}
        for k, key in enumerate(("left_T", "right_T", "metadata")):
            a = out[key]
            dst = a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
            if sizes[key] and rt.cudaMemcpy(ctypes.c_void_p(dst), ptrs[k], sizes[key], 2) != 0:
                raise _native.ObvhError("reading the SoA arrays back failed")
        return out
    finally:
        _native.check(lib.obvh_soa_obvh_free(d_soa))


def obvh_pack(nodes, node_count: int, internal_count: int, transforms=None, packed=None, pairs=None, soa=True,
              stream=None):
    """obvh_obvh_pack_async: packed records, pairs and (soa=True) the SoA
    arrays in one pass on `stream`.  Returns dict(packed, pairs, left_T,
    right_T, metadata, error) of device tensors (error: int32 [1])."""
    import torch
    lib = _native.lib()
    dev = nodes.device
    if packed is None:
        packed = torch.zeros(node_count * 64, dtype=torch.uint8, device=dev)
    out = {"packed": packed, "pairs": None, "left_T": None, "right_T": None, "metadata": None,
           "error": torch.zeros(1, dtype=torch.int32, device=dev)}
    if transforms is not None:
        out["pairs"] = pairs if pairs is not None else torch.zeros(max(internal_count, 1) * 32, dtype=torch.float32,
                                                                   device=dev)
        if soa:
            out["left_T"] = torch.empty(max(internal_count, 1) * 12, dtype=torch.float32, device=dev)
            out["right_T"] = torch.empty(max(internal_count, 1) * 12, dtype=torch.float32, device=dev)
            out["metadata"] = torch.empty(max(node_count, 1) * 4, dtype=torch.int32, device=dev)
    _native.check(lib.obvh_obvh_pack_async(_ptr(nodes), _ptr(transforms), _ptr(packed), _ptr(out["pairs"]),
                                           _ptr(out["left_T"]), _ptr(out["right_T"]), _ptr(out["metadata"]),
                                           node_count, internal_count, _ptr(out["error"]),
                                           _stream(torch, stream)))
    return out


# ---- SoA OBVH ray traversal ---------------------------------------------------
def soa_obvh_intersect(soa: dict, mesh: "Mesh", primitives, rays, node_count: int, internal_count: int,
                       isects=None, stream=None):
    """obvh_soa_obvh_intersect_async: closest hits of `rays` (a device uint8
    tensor of kr_ray records) against the SoA arrays of obvh_pack (soa:
    left_T, right_T, metadata).  Returns (isects uint8 tensor of 28-byte
    records, error int32 [1])."""
    import torch
    lib = _native.lib()
    n = rays.numel() // 32
    if isects is None:
        isects = torch.empty(max(n, 1) * 28, dtype=torch.uint8, device=rays.device)
    err = torch.zeros(1, dtype=torch.int32, device=rays.device)
    slots = 0 if primitives is None else primitives.numel()
    _native.check(lib.obvh_soa_obvh_intersect_async(
        _ptr(soa["left_T"]), _ptr(soa["right_T"]), _ptr(soa["metadata"]), internal_count, node_count,
        _ptr(mesh.verts), _ptr(mesh.faces), mesh.n_faces, _ptr(primitives), slots, _ptr(rays), _ptr(isects), n,
        _ptr(err), _stream(torch, stream)))
    return isects, err


# ---- compressed SoA OBVH --------------------------------------------------------
def soa_compressed_obvh(packed, pairs, internal_count: int, node_count: int, out=None, stream=None):
    """obvh_soa_compressed_obvh_async: the compressed SoA arrays (lbounds,
    rbounds: float32 [ni, 6], metadata: int32 [nodes, 4]) of packed records
    and pairs (device tensors), on `stream`."""
    import torch
    lib = _native.lib()
    dev = packed.device
    if out is None:
        out = {"lbounds": torch.empty((max(internal_count, 1), 6), dtype=torch.float32, device=dev),
               "rbounds": torch.empty((max(internal_count, 1), 6), dtype=torch.float32, device=dev),
               "metadata": torch.empty((max(node_count, 1), 4), dtype=torch.int32, device=dev)}
    _native.check(lib.obvh_soa_compressed_obvh_async(_ptr(packed), _ptr(pairs), _ptr(out["lbounds"]),
                                                     _ptr(out["rbounds"]), _ptr(out["metadata"]), internal_count,
                                                     node_count, _stream(torch, stream)))
    return out


def soa_compressed_obvh_sync(packed, pairs, internal_count: int, node_count: int):
    """kr_cuda_soa_compressed_obvh (the reference-signature, allocating form):
    numpy lbounds [ni, 6], rbounds [ni, 6], metadata [nodes, 4], read back and
    freed with obvh_soa_obvh_compressed_free."""
    lib = _native.lib()
    d_soa = ctypes.c_void_p(0)
    _native.check(lib.kr_cuda_soa_compressed_obvh(_ptr(packed), _ptr(pairs), ctypes.byref(d_soa), internal_count,
                                                  node_count))
    rt = _cudart()
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    try:
        ptrs = (ctypes.c_void_p * 3)()
        if rt.cudaMemcpy(ctypes.cast(ptrs, ctypes.c_void_p), d_soa, 24, 2) != 0:
            raise _native.ObvhError("reading the kr_SoA_OBVH_Compressed struct back failed")
        out = {"lbounds": np.zeros((internal_count, 6), np.float32), "rbounds": np.zeros((internal_count, 6), np.float32),
               "metadata": np.zeros((node_count, 4), np.int32)}
        for k, key in enumerate(("lbounds", "rbounds", "metadata")):
            if out[key].nbytes and rt.cudaMemcpy(ctypes.c_void_p(out[key].ctypes.data), ptrs[k], out[key].nbytes,
                                                 2) != 0:
                raise _native.ObvhError("reading the compressed SoA arrays back failed")
        return out
    finally:
        _native.check(lib.obvh_soa_obvh_compressed_free(d_soa))


def compressed_pairs_from_obbs(nodes: np.ndarray, obbs: np.ndarray) -> np.ndarray:
    """Transformation pairs in the form the compressed OBVH reads, one per
    internal node and child (float32 [internal, 32]: left pair, then right):
    column 0 the axis and angle / pi of the child box's rotation (box to
    world; kr_cuda_soa_compressed_obvh negates the axis, so the traversal
    applies world to box), column 1 the box centre, column 2 the box's full
    size along its unit axes.  The reference has no producer of this form
    (kr_cuda_soa_compressed_obvh, src/ads/common/cuda/transforms.cu:1452-1535,
    has no caller); this one derives it from an OBB tree (NODE records and
    kr_obb3 rows).  A left-handed frame is made right-handed by reversing its
    third axis, which leaves the symmetric box unchanged; rotations by about
    pi take their axis from R + I, where the skew part vanishes."""
    nodes = np.ascontiguousarray(nodes)
    ni = (nodes.shape[0] - 1) // 2
    o_all = np.asarray(obbs, np.float64).reshape(-1, 15)
    pairs = np.zeros((max(ni, 0), 32), np.float32)
    for side, key in ((0, "left"), (1, "right")):
        o = o_all[nodes[key][:ni].astype(np.int64)]
        axes = o[:, 3:12].reshape(-1, 3, 3)                  # rows a0, a1, a2
        length = np.linalg.norm(axes, axis=2)
        unit = axes / np.where(length > 0, length, 1.0)[..., None]
        unit[np.linalg.det(unit) < 0, 2] *= -1.0
        r = np.transpose(unit, (0, 2, 1))                      # columns: the box axes in world coordinates
        cos = np.clip((np.trace(r, axis1=1, axis2=2) - 1.0) * 0.5, -1.0, 1.0)
        angle = np.arccos(cos)
        axis = np.stack([r[:, 2, 1] - r[:, 1, 2], r[:, 0, 2] - r[:, 2, 0], r[:, 1, 0] - r[:, 0, 1]], 1)
        skew = np.linalg.norm(axis, axis=1)
        near_pi = skew < 1e-6
        if near_pi.any():
            sym = r[near_pi] + np.eye(3)                        # columns ~ 2 (axis . x) axis
            pick = np.argmax(np.linalg.norm(sym, axis=1), axis=1)
            axis[near_pi] = sym[np.arange(sym.shape[0]), :, pick]
            skew = np.linalg.norm(axis, axis=1)
        axis = np.where(skew[:, None] > 0, axis / np.where(skew > 0, skew, 1.0)[:, None], [1.0, 0.0, 0.0])
        m = pairs[:, 16 * side:16 * side + 16]
        m[:, 0:3] = axis
        m[:, 3] = angle / np.pi
        m[:, 4:7] = o[:, 0:3]
        m[:, 8:11] = 2.0 * o[:, 12:15] * length
    return pairs


def soa_compressed_obvh_intersect(soa: dict, mesh: "Mesh", primitives, rays, node_count: int, internal_count: int,
                                  isects=None, stream=None):
    """obvh_soa_compressed_obvh_intersect_async: closest hits of `rays`
    against the compressed arrays (soa: lbounds, rbounds, metadata).  Returns
    (isects uint8 tensor of 28-byte records, error int32 [1])."""
    import torch
    lib = _native.lib()
    n = rays.numel() // 32
    if isects is None:
        isects = torch.empty(max(n, 1) * 28, dtype=torch.uint8, device=rays.device)
    err = torch.zeros(1, dtype=torch.int32, device=rays.device)
    slots = 0 if primitives is None else primitives.numel()
    _native.check(lib.obvh_soa_compressed_obvh_intersect_async(
        _ptr(soa["lbounds"]), _ptr(soa["rbounds"]), _ptr(soa["metadata"]), internal_count, node_count,
        _ptr(mesh.verts), _ptr(mesh.faces), mesh.n_faces, _ptr(primitives), slots, _ptr(rays), _ptr(isects), n,
        _ptr(err), _stream(torch, stream)))
    return isects, err


# ---- SAH cost ----------------------------------------------------------------
def bvh_sah_host(nodes: np.ndarray, ci: float = 1.2, ct: float = 1.0, obbs: np.ndarray = None,
                 root: int = 0) -> float:
    """kr_bvh_sah on host arrays (NODE records, obbs [nodes x 15] or None)."""
    lib = _native.lib()
    n = np.ascontiguousarray(nodes)
    o = None if obbs is None else np.ascontiguousarray(obbs, np.float32)
    return float(lib.kr_bvh_sah(n.ctypes.data, root, ci, ct, None if o is None else o.ctypes.data, None))


def bvh_sah(nodes, parents, obbs=None, ci: float = 1.2, ct: float = 1.0, stream=None):
    """obvh_bvh_sah_async on device tensors: (SAH sum, SAH / root area), as
    a device float64 tensor [2]."""
    import torch
    lib = _native.lib()
    nn = parents.numel()
    ws = torch.empty(int(lib.obvh_bvh_sah_workspace_bytes(nn)), dtype=torch.uint8, device=parents.device)
    out = torch.empty(2, dtype=torch.float64, device=parents.device)
    _native.check(lib.obvh_bvh_sah_async(_ptr(nodes), _ptr(parents), _ptr(obbs), nn, ci, ct, _ptr(out), _ptr(ws),
                                         _stream(torch, stream)))
    return out


class BuildBatch:
    """obvh_build_batch_*: LBVH + OBB tree + collapse builds of many meshes
    in one launch sequence (include/obvh_build_batch.h).  `vertex_offsets`
    and `face_offsets` are CSR arrays (meshes + 1 values); faces index their
    own mesh's vertices.  Outputs: node arrays of 2F - M entries (mesh m at
    2 face_offsets[m] - m), primitives of F entries (mesh m at
    face_offsets[m]), bounds 2 boxes per mesh."""

    def __init__(self, vertex_offsets, face_offsets, flags=BUILD_OBBS | BUILD_COLLAPSE, cta_max_faces=0,
                 device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.lib = _native.lib()
        self.voff = np.ascontiguousarray(vertex_offsets, dtype=np.uint64)
        self.foff = np.ascontiguousarray(face_offsets, dtype=np.uint64)
        self.meshes = self.foff.shape[0] - 1
        self.flags = flags
        h = ctypes.c_void_p()
        _native.check(self.lib.obvh_build_batch_create(self.voff.ctypes.data, self.foff.ctypes.data, self.meshes,
                                                       flags, cta_max_faces, ctypes.byref(h)))
        self.handle = h
        self.faces = int(self.foff[-1])
        self.nodes = 2 * self.faces - self.meshes

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.obvh_build_batch_destroy(h)
            self.handle = None

    def node_offset(self, m: int) -> int:
        return 2 * int(self.foff[m]) - m

    def outputs(self):
        t, d, nn, f = self.torch, self.device, self.nodes, self.faces
        o = {"nodes": t.empty(nn * NODE_BYTES, dtype=t.uint8, device=d), "parents": t.empty(nn, dtype=t.int32, device=d),
             "counts": t.empty(nn, dtype=t.int32, device=d), "costs": t.empty(nn, dtype=t.float32, device=d),
             "bounds": t.empty((self.meshes, 12), dtype=t.float32, device=d)}
        if self.flags & BUILD_OBBS:
            o["obbs"] = t.empty((nn, 15), dtype=t.float32, device=d)
            o["transforms"] = t.empty((nn, 16), dtype=t.float32, device=d)
        if self.flags & BUILD_COLLAPSE:
            o["collapsed"] = t.empty(nn * NODE_BYTES, dtype=t.uint8, device=d)
            o["primitives"] = t.zeros(f, dtype=t.int32, device=d)
        return o

    def _args(self, verts, faces, o, ci, ct):
        return [_ptr(verts), _ptr(faces), ci, ct, _ptr(o["nodes"]), _ptr(o["parents"]), _ptr(o["counts"]),
                _ptr(o["costs"]), _ptr(o.get("bounds")), _ptr(o.get("obbs")), _ptr(o.get("transforms")),
                _ptr(o.get("collapsed")), _ptr(o.get("primitives"))]

    def enqueue(self, verts, faces, out=None, ci=1.2, ct=1.0, stream=None):
        """verts: float32 [V, 3], faces: int32/uint32 [F, 4] device tensors."""
        o = out if out is not None else self.outputs()
        _native.check(self.lib.obvh_build_batch_enqueue(self.handle, *self._args(verts, faces, o, ci, ct),
                                                        _stream(self.torch, stream)))
        return o

    def capture(self, verts, faces, out, ci=1.2, ct=1.0):
        _native.check(self.lib.obvh_build_batch_capture(self.handle, *self._args(verts, faces, out, ci, ct)))

    def launch(self, stream=None):
        _native.check(self.lib.obvh_build_batch_launch(self.handle, _stream(self.torch, stream)))

    def status(self, stream=None):
        """(device error word, per-mesh primitive slots)."""
        err = ctypes.c_uint32(0)
        slots = np.zeros(self.meshes, np.uint32)
        _native.check(self.lib.obvh_build_batch_status(self.handle, _stream(self.torch, stream), ctypes.byref(err),
                                                       slots.ctypes.data))
        return err.value, slots

    def info(self):
        a, b, g = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _native.check(self.lib.obvh_build_batch_info(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(g)))
        return {"cta_meshes": a.value, "chain_meshes": b.value, "grid": g.value}
