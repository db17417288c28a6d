"""TEST INFRASTRUCTURE ONLY: numpy access to the tree restatement (bvh_oracle.c)
and to the reference's host-callable vecmath helpers (oracle/_ref)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import HERE, lib

NODE = np.dtype([("b", "<f4", (6,)), ("left", "<u4"), ("right", "<u4"), ("n_prims", "<u2"),
                 ("axis", "u1"), ("pad", "u1")])
assert NODE.itemsize == 36

_f32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_node = np.ctypeslib.ndpointer(dtype=NODE, flags="C_CONTIGUOUS")
_u64 = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    l = lib()
    c = ctypes
    sig = {
        "oracle_morton30": (c.c_uint32, [c.c_float, c.c_float, c.c_float]),
        "oracle_minverse4": (None, [_f32, _f32]),
        "oracle_mmul4": (None, [_f32, _f32, _f32]),
        "oracle_aabb_area": (c.c_float, [_f32]),
        "oracle_scene_bounds": (None, [_f32, _u32, c.c_uint32, _f32, _f32]),
        "oracle_lbvh_codes": (None, [_f32, _u32, c.c_uint32, _f32, _u32]),
        "oracle_stable_order": (None, [_u32, c.c_uint32, _u32]),
        "oracle_karras": (None, [_u32, c.c_uint32, _node, _u32]),
        "oracle_lbvh_build": (None, [_f32, _u32, c.c_uint32, _node, _u32, _u32, _u32, _f32, _f32, _f32]),
        "oracle_leaf_obb": (None, [_f32, _f32, _f32]),
        "oracle_obb_tree": (c.c_int, [_node, _u32, _f32, _u32, c.c_uint32, c.c_uint32, _f32, _f32, _f32]),
        "oracle_obb_summaries": (c.c_int, [_node, _f32, _u32, c.c_uint32, c.c_uint32, _f32, _f32, _f32]),
        "oracle_pack": (None, [_node, c.c_void_p, c.c_uint32, c.c_int, c.c_void_p, c.c_void_p]),
        "oracle_soa_obvh": (None, [c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32, _f32, _f32, _i32]),
        "oracle_soa_obvh_intersect": (c.c_int64, [c.c_void_p, c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32,
                                                  c.c_void_p, c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32,
                                                  c.c_void_p, c.c_uint64, c.c_uint64, c.c_void_p]),
        "oracle_soa_obvh_intersect_counts": (c.c_int64, [c.c_void_p, c.c_void_p, c.c_void_p, c.c_uint32,
                                                         c.c_uint32, c.c_void_p, c.c_void_p, c.c_uint32, c.c_void_p,
                                                         c.c_uint32, c.c_void_p, c.c_uint64, c.c_uint64, c.c_void_p,
                                                         c.c_void_p]),
        "oracle_collapse": (c.c_int, [_node, _u32, _node, _u32, _u32, _f32, c.c_float, c.c_float, c.c_uint32,
                                      c.c_uint32]),
        "oracle_aabb_refit": (c.c_int, [_node, c.c_uint32, _u32, _f32]),
        "oracle_morton63": (c.c_uint64, [_f32, _f32]),
        "oracle_morton63_unit": (c.c_uint64, [c.c_float, c.c_float, c.c_float]),
        "oracle_atrbvh_box_area": (c.c_float, [_f32, _f32]),
        "oracle_atrbvh_union_area": (c.c_float, [_f32, _f32, _f32, _f32]),
        "oracle_trm_row": (c.c_int, [c.c_int]),
        "oracle_trm_col": (c.c_int, [c.c_int]),
        "oracle_stable_order64": (None, [_u64, c.c_uint32, _u32]),
        "oracle_karras63": (None, [_u64, _u32, c.c_uint32, _i32, _i32, _i32, _i32]),
        "oracle_atrbvh_build": (c.c_int, [_f32, _u32, c.c_uint32, c.c_int, c.c_int, c.c_float, c.c_float, _node,
                                          _u32, _u32, _f32, _u64, _f32]),
        "oracle_soa_compressed_obvh": (None, [c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32, c.c_void_p,
                                              c.c_void_p, c.c_void_p]),
        "oracle_atrbvh_seed": (c.c_int, [_f32, _u32, c.c_uint32, _i32, _i32, _i32, _i32, _f32, _f32, _f32, _u64]),
        "oracle_atrbvh_optimize": (c.c_int, [c.c_uint32, c.c_int, c.c_int, c.c_float, c.c_float, _i32, _i32, _i32,
                                             _i32, _f32, _f32, _f32, _f32]),
        "oracle_atrbvh_emit": (c.c_int, [c.c_uint32, _i32, _i32, _i32, _i32, _f32, _f32, _f32, _node, _u32, _u32,
                                         _f32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(l, name)
        f.restype = res
        f.argtypes = args
    _bound = True
    return l


def _mesh(verts, faces):
    v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1)
    f = np.ascontiguousarray(faces, dtype=np.uint32)
    if f.ndim == 2 and f.shape[1] == 3:
        f = np.concatenate([f, np.zeros((f.shape[0], 1), np.uint32)], axis=1)
    return v, np.ascontiguousarray(f.reshape(-1), dtype=np.uint32), f.reshape(-1, 4).shape[0]


def scene_bounds(verts, faces):
    l = _bind()
    v, f, n = _mesh(verts, faces)
    s = np.zeros(6, np.float32)
    c = np.zeros(6, np.float32)
    l.oracle_scene_bounds(v, f, n, s, c)
    return s, c


def lbvh_codes(verts, faces, centroid_box):
    l = _bind()
    v, f, n = _mesh(verts, faces)
    codes = np.zeros(n, np.uint32)
    l.oracle_lbvh_codes(v, f, n, np.ascontiguousarray(centroid_box, np.float32), codes)
    return codes


def lbvh_build(verts, faces):
    """The full LBVH build: dict of nodes, parents, sorted codes, counts, costs, scene, centroid."""
    l = _bind()
    v, f, n = _mesh(verts, faces)
    nn = 2 * n - 1
    nodes = np.zeros(nn, NODE)
    parents = np.zeros(nn, np.uint32)
    codes = np.zeros(n, np.uint32)
    counts = np.zeros(nn, np.uint32)
    costs = np.zeros(nn, np.float32)
    s = np.zeros(6, np.float32)
    c = np.zeros(6, np.float32)
    l.oracle_lbvh_build(v, f, n, nodes, parents, codes, counts, costs, s, c)
    return {"nodes": nodes, "parents": parents, "codes": codes, "counts": counts, "costs": costs,
            "scene": s, "centroid": c}


def karras(codes_sorted):
    l = _bind()
    codes = np.ascontiguousarray(codes_sorted, np.uint32)
    n = codes.shape[0]
    nodes = np.zeros(2 * n - 1, NODE)
    parents = np.zeros(2 * n - 1, np.uint32)
    l.oracle_karras(codes, n, nodes, parents)
    return nodes, parents


def obb_tree(nodes, parents, verts, faces):
    """(obbs [nodes x 15], transforms [nodes x 16], internal axes [internal x 9])."""
    l = _bind()
    v, f, _ = _mesh(verts, faces)
    nn = nodes.shape[0]
    n = (nn + 1) // 2
    ni = n - 1
    obbs = np.zeros((nn, 15), np.float32)
    xfs = np.zeros((nn, 16), np.float32)
    axes = np.zeros((max(ni, 1), 9), np.float32)
    rc = l.oracle_obb_tree(np.ascontiguousarray(nodes), np.ascontiguousarray(parents, np.uint32), v, f, n, ni,
                           obbs.reshape(-1), xfs.reshape(-1), axes.reshape(-1))
    if rc != 0:
        raise ValueError("malformed tree")
    return obbs, xfs, axes[:ni]


def obb_summaries(nodes, verts, faces):
    """The subtree summaries in the reference's arrays: (min_proj [nodes x 7],
    max_proj [nodes x 7], minmax pairs [nodes x 7 x 6])."""
    l = _bind()
    v, f, _ = _mesh(verts, faces)
    nn = nodes.shape[0]
    n = (nn + 1) // 2
    mn = np.zeros((nn, 7), np.float32)
    mx = np.zeros((nn, 7), np.float32)
    pairs = np.zeros((nn, 7, 6), np.float32)
    if l.oracle_obb_summaries(np.ascontiguousarray(nodes), v, f, n, n - 1, mn.reshape(-1), mx.reshape(-1),
                              pairs.reshape(-1)) != 0:
        raise ValueError("malformed tree")
    return mn, mx, pairs


def collapse(nodes, parents, counts, costs, ci=1.2, ct=1.0):
    """(collapsed nodes, counts, primitives, costs, used primitive slots)."""
    l = _bind()
    nn = nodes.shape[0]
    n = (nn + 1) // 2
    out = np.zeros(nn, NODE)
    cnt = np.ascontiguousarray(counts, np.uint32).copy()
    cst = np.ascontiguousarray(costs, np.float32).copy()
    prims = np.zeros(n, np.uint32)
    used = l.oracle_collapse(np.ascontiguousarray(nodes), np.ascontiguousarray(parents, np.uint32), out, cnt, prims,
                             cst, ci, ct, n, n - 1)
    if used < 0:
        raise ValueError("malformed tree")
    return out, cnt, prims, cst, used


def leaf_obb(tri9):
    l = _bind()
    o = np.zeros(15, np.float32)
    x = np.zeros(16, np.float32)
    l.oracle_leaf_obb(np.ascontiguousarray(tri9, np.float32).reshape(-1), o, x)
    return o, x


# ---- the reference's own helpers (oracle/_ref/libref_vecmath.so) ----------
_vm = None


def ref_vecmath():
    global _vm
    if _vm is None:
        p = os.path.join(HERE, "_ref", "libref_vecmath.so")
        if not os.path.exists(p):
            raise FileNotFoundError(p)
        l = ctypes.CDLL(p)
        l.ref_v32morton3.restype = ctypes.c_uint32
        l.ref_v32morton3.argtypes = [ctypes.c_float] * 3
        l.ref_minverse4.argtypes = [_f32, _f32]
        l.ref_mmul4.argtypes = [_f32, _f32, _f32]
        l.ref_aabb_area.restype = ctypes.c_float
        l.ref_aabb_area.argtypes = [_f32]
        _vm = l
    return _vm


def ref_vecmath_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_vecmath.so"))


def morton63(tri9, scene):
    """63-bit Morton code of one triangle (9 floats) in the scene box (6 floats)."""
    l = _bind()
    return int(l.oracle_morton63(np.ascontiguousarray(tri9, np.float32), np.ascontiguousarray(scene, np.float32)))


def karras63(sorted_codes, order):
    """SoA tree of the 63-bit Karras build: (left, right, parent, data) int32 arrays."""
    l = _bind()
    k = np.ascontiguousarray(sorted_codes, np.uint64)
    o = np.ascontiguousarray(order, np.uint32)
    n = k.shape[0]
    arrs = [np.full(2 * n - 1, -1, np.int32) for _ in range(4)]
    l.oracle_karras63(k, o, n, *arrs)
    return tuple(arrs)


def atrbvh_build(verts, faces, treelet_size=9, iterations=2, ci=1.2, ct=1.0):
    """LBVH-63 + agglomerative treelet optimisation, as kr_bvh_node records:
    dict of nodes, parents, counts, costs, sorted codes, and the optimiser's
    root SAH after each iteration."""
    l = _bind()
    v, f, n = _mesh(verts, faces)
    nn = 2 * n - 1
    out = {"nodes": np.zeros(nn, NODE), "parents": np.zeros(nn, np.uint32), "counts": np.zeros(nn, np.uint32),
           "costs": np.zeros(nn, np.float32), "codes": np.zeros(n, np.uint64),
           "sah": np.zeros(max(iterations, 1), np.float32)}
    rc = l.oracle_atrbvh_build(v, f, n, treelet_size, iterations, ci, ct, out["nodes"], out["parents"],
                               out["counts"], out["costs"], out["codes"], out["sah"])
    if rc != 0:
        raise ValueError("oracle_atrbvh_build failed")
    return out


SOA_FIELDS = ("parent", "left", "right", "data", "lo", "hi", "area")


def atrbvh_seed(verts, faces):
    """The ATRBVH seed tree (LBVH-63 with node boxes) in the reference's SoA
    layout (SoABVHTree.h:19-44): dict of int32 parent/left/right/data,
    float32 (nodes, 4) lo/hi boxes and float32 area, plus the sorted codes."""
    l = _bind()
    v, f, n = _mesh(verts, faces)
    nn = 2 * n - 1
    t = {k: np.zeros(nn, np.int32) for k in ("parent", "left", "right", "data")}
    t.update(lo=np.zeros((nn, 4), np.float32), hi=np.zeros((nn, 4), np.float32), area=np.zeros(nn, np.float32))
    codes = np.zeros(n, np.uint64)
    if l.oracle_atrbvh_seed(v, f, n, t["parent"], t["left"], t["right"], t["data"], t["lo"], t["hi"], t["area"],
                            codes) != 0:
        raise ValueError("oracle_atrbvh_seed failed")
    t["codes"] = codes
    return t


def soa_copy(tree):
    return {k: np.array(tree[k], copy=True) for k in SOA_FIELDS}


def atrbvh_optimize(tree, treelet_size=7, iterations=2, ci=1.2, ct=1.0):
    """The restatement's treelet optimisation of an SoA tree (a copy is
    returned) and the root SAH after each iteration."""
    l = _bind()
    t = soa_copy(tree)
    n = (len(t["parent"]) + 1) // 2
    sah = np.zeros(max(iterations, 1), np.float32)
    if l.oracle_atrbvh_optimize(n, treelet_size, iterations, ci, ct, t["parent"], t["left"], t["right"], t["data"],
                                t["lo"], t["hi"], t["area"], sah) != 0:
        raise ValueError("oracle_atrbvh_optimize failed")
    return t, sah


def atrbvh_emit(tree):
    """copyTree + refit of an SoA tree: dict of kr_bvh_node records, parents,
    counts, costs (atrbvh.cu:95-183)."""
    l = _bind()
    n = (len(tree["parent"]) + 1) // 2
    nn = 2 * n - 1
    out = {"nodes": np.zeros(nn, NODE), "parents": np.zeros(nn, np.uint32), "counts": np.zeros(nn, np.uint32),
           "costs": np.zeros(nn, np.float32)}
    t = soa_copy(tree)
    if l.oracle_atrbvh_emit(n, t["parent"], t["left"], t["right"], t["data"], t["lo"], t["hi"], t["area"],
                            out["nodes"], out["parents"], out["counts"], out["costs"]) != 0:
        raise ValueError("oracle_atrbvh_emit failed")
    return out


_ref_treelet = None


def ref_treelet_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_treelet_emu.so"))


def ref_treelet_optimize(tree, treelet_size=7, iterations=2, ci=1.2, ct=1.0):
    """The reference's own treelet kernel (AgglomerativeTreelet.cu), run as
    host code by the lockstep warp emulation in ref_treelet_emu.cpp, on a copy
    of an SoA tree; returns the optimised copy."""
    global _ref_treelet
    if _ref_treelet is None:
        r = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_treelet_emu.so"))
        r.ref_treelet_optimize.restype = ctypes.c_int
        r.ref_treelet_optimize.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_float, _i32, _i32, _i32, _i32, _f32, _f32, _f32,
                                           ctypes.POINTER(ctypes.c_char_p)]
        _ref_treelet = r
    t = soa_copy(tree)
    n = (len(t["parent"]) + 1) // 2
    err = ctypes.c_char_p()
    rc = _ref_treelet.ref_treelet_optimize(n, treelet_size, iterations, ci, ct, t["parent"], t["left"], t["right"],
                                           t["data"], t["lo"], t["hi"], t["area"], ctypes.byref(err))
    if rc != 0:
        raise ValueError((err.value or b"ref_treelet_optimize failed").decode())
    return t


def ref_atrbvh():
    """The reference's host-callable ATRBVH helpers (oracle/_ref/libref_atrbvh.so), or None."""
    path = os.path.join(HERE, "_ref", "libref_atrbvh.so")
    if not os.path.exists(path):
        return None
    r = ctypes.CDLL(path)
    c = ctypes
    for name, (res, args) in {
        "ref_morton63": (c.c_uint64, [c.c_float, c.c_float, c.c_float]),
        "ref_expand_bits64": (c.c_uint64, [c.c_uint64]),
        "ref_box_area": (c.c_float, [_f32, _f32]),
        "ref_union_area": (c.c_float, [_f32, _f32, _f32, _f32]),
        "ref_trm_index": (c.c_int, [c.c_int, c.c_int]),
        "ref_trm_row": (c.c_int, [c.c_int]),
        "ref_trm_col": (c.c_int, [c.c_int]),
    }.items():
        f = getattr(r, name)
        f.restype = res
        f.argtypes = args
    return r


# ---- the reference's own GPU tree kernels (oracle/_ref/libref_tree_gpu*.so) --
# Built for sm_100a from lbvh.cu / transforms.cu by oracle/Makefile; the calls
# below need a GPU.  variant "nofma": compiled with --fmad=false, the
# arithmetic of the restatement; "fmad": nvcc's default contraction, the
# reference as its own build compiles it.
_REF_GPU = {"nofma": "libref_tree_gpu.so", "fmad": "libref_tree_gpu_fmad.so"}
_ref_gpu = {}


def ref_gpu_available(variant: str = "nofma") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", _REF_GPU[variant]))


def ref_gpu(variant: str = "nofma"):
    if variant not in _ref_gpu:
        p = os.path.join(HERE, "_ref", _REF_GPU[variant])
        if not os.path.exists(p):
            raise FileNotFoundError(p)
        l = ctypes.CDLL(p)
        c = ctypes
        l.refgpu_lbvh.restype = c.c_int
        l.refgpu_lbvh.argtypes = [_f32, c.c_uint32, _u32, c.c_uint32, _f32, _node, _u32, _u32, _u32, _f32]
        l.refgpu_obb_from_summaries.restype = c.c_int
        l.refgpu_obb_from_summaries.argtypes = [_node, _u32, _u32, _f32, c.c_uint32, _u32, c.c_uint32, _f32, _f32,
                                                _f32, _f32, _f32]
        l.refgpu_pack.restype = c.c_int
        l.refgpu_pack.argtypes = [_node, c.c_void_p, c.c_uint32, c.c_void_p, c.c_void_p, _f32, _f32, _i32]
        l.refgpu_collapse.restype = c.c_int
        l.refgpu_collapse.argtypes = [_node, _u32, _u32, _f32, c.c_float, c.c_float, c.c_uint32, _node, _u32]
        l.refgpu_lbvh_ms.restype = c.c_int
        l.refgpu_lbvh_ms.argtypes = [_f32, c.c_uint32, _u32, c.c_uint32, _f32, c.c_int, _f32]
        l.refgpu_transform_ms.restype = c.c_int
        l.refgpu_transform_ms.argtypes = [_node, _u32, _u32, _f32, _f32, c.c_uint32, _u32, c.c_uint32, _f32, _f32,
                                          _f32, c.c_float, c.c_float, c.c_int, _f32]
        _ref_gpu[variant] = l
    return _ref_gpu[variant]


def refgpu_lbvh(verts, faces, variant: str = "nofma"):
    """The reference's LBVH kernels (codes, stable sort, Karras tree, bottom-up
    boxes, counts, costs) on the oracle's centroid box: dict as lbvh_build."""
    l = ref_gpu(variant)
    v, f, n = _mesh(verts, faces)
    _, centroid = scene_bounds(verts, faces)
    nn = 2 * n - 1
    out = {"nodes": np.zeros(nn, NODE), "parents": np.zeros(nn, np.uint32), "codes": np.zeros(n, np.uint32),
           "counts": np.zeros(nn, np.uint32), "costs": np.zeros(nn, np.float32)}
    rc = l.refgpu_lbvh(v, v.shape[0] // 3, f, n, centroid, out["nodes"], out["parents"], out["codes"], out["counts"],
                       out["costs"])
    if rc != 0:
        raise RuntimeError(f"refgpu_lbvh: CUDA error {rc}")
    return out


def refgpu_obb_tree(nodes, parents, counts, verts, faces, variant: str = "nofma"):
    """The reference's candidate, refit and finalize kernels on the oracle's
    subtree summaries: (obbs [nodes x 15], transforms [nodes x 16])."""
    l = ref_gpu(variant)
    v, f, n = _mesh(verts, faces)
    mn, mx, pairs = obb_summaries(nodes, verts, faces)
    nn = 2 * n - 1
    obbs = np.zeros((nn, 15), np.float32)
    xfs = np.zeros((nn, 16), np.float32)
    rc = l.refgpu_obb_from_summaries(np.ascontiguousarray(nodes), np.ascontiguousarray(parents, np.uint32),
                                     np.ascontiguousarray(counts, np.uint32), v, v.shape[0] // 3, f, n,
                                     mn.reshape(-1), mx.reshape(-1), pairs.reshape(-1), obbs.reshape(-1),
                                     xfs.reshape(-1))
    if rc != 0:
        raise RuntimeError(f"refgpu_obb_from_summaries: CUDA error {rc}")
    return obbs, xfs


def refgpu_collapse(nodes, parents, counts, costs, ci=1.2, ct=1.0, variant: str = "nofma"):
    """kr_cuda_bvh_collapse: (collapsed nodes, counts, primitives, costs)."""
    l = ref_gpu(variant)
    nn = nodes.shape[0]
    n = (nn + 1) // 2
    out = np.zeros(nn, NODE)
    cnt = np.ascontiguousarray(counts, np.uint32).copy()
    cst = np.ascontiguousarray(costs, np.float32).copy()
    prims = np.zeros(n, np.uint32)
    rc = l.refgpu_collapse(np.ascontiguousarray(nodes), np.ascontiguousarray(parents, np.uint32), cnt, cst, ci, ct, n,
                           out, prims)
    if rc != 0:
        raise RuntimeError(f"refgpu_collapse: CUDA error {rc}")
    return out, cnt, prims, cst


def refgpu_tree_ms(verts, faces, reps=5, variant: str = "fmad", ci=1.2, ct=1.0):
    """Mean device time (ms) of each of the reference's tree kernels on
    device-resident data: dict of morton, sort, tree, aabb (lbvh.cu's commit
    steps), candidate, refit, finalize (kr_cuda_bvh_obb_tree's stages) and
    collapse (kr_cuda_bvh_collapse's mark and gather kernels).  The subtree
    summaries and the centroid box the reference's skipped kernels would
    make come from the oracle and are not timed."""
    l = ref_gpu(variant)
    v, f, n = _mesh(verts, faces)
    _, centroid = scene_bounds(verts, faces)
    a = np.zeros(4, np.float32)
    rc = l.refgpu_lbvh_ms(v, v.shape[0] // 3, f, n, centroid, reps, a)
    if rc != 0:
        raise RuntimeError(f"refgpu_lbvh_ms: CUDA error {rc}")
    t = refgpu_lbvh(verts, faces, variant)
    mn, mx, pairs = obb_summaries(t["nodes"], verts, faces)
    b = np.zeros(4, np.float32)
    rc = l.refgpu_transform_ms(t["nodes"], t["parents"], t["counts"], t["costs"], v, v.shape[0] // 3, f, n,
                               mn.reshape(-1), mx.reshape(-1), pairs.reshape(-1), ci, ct, reps, b)
    if rc != 0:
        raise RuntimeError(f"refgpu_transform_ms: CUDA error {rc}")
    keys = ("morton", "sort", "tree", "aabb", "candidate", "refit", "finalize", "collapse")
    return dict(zip(keys, [float(x) for x in np.concatenate([a, b])]))


def refgpu_lbvh63_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_lbvh63_gpu.so"))


_ref63 = None


def refgpu_lbvh63(verts, faces):
    """The reference's ATRBVH seed build on the GPU (LBVH.cu / CubWrapper.cu):
    (sorted 63-bit codes, their triangle order, (left, right, parent, data))."""
    global _ref63
    if _ref63 is None:
        l = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_lbvh63_gpu.so"))
        l.refgpu_lbvh63.restype = ctypes.c_int
        l.refgpu_lbvh63.argtypes = [_f32, ctypes.c_uint32, _f32, _u64, _u32, _i32, _i32, _i32, _i32]
        _ref63 = l
    tri = triangles9(verts, faces)
    n = tri.shape[0]
    codes = np.zeros(n, np.uint64)
    order = np.zeros(n, np.uint32)
    arrs = [np.zeros(2 * n - 1, np.int32) for _ in range(4)]
    rc = _ref63.refgpu_lbvh63(tri.reshape(-1), n, scene_box9(tri), codes, order, *arrs)
    if rc != 0:
        raise RuntimeError(f"refgpu_lbvh63: CUDA error {rc}")
    return codes, order, tuple(arrs)


def triangles9(verts, faces):
    """The triangles as an n x 9 float32 soup."""
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    f = np.asarray(faces, np.uint32).reshape(-1, np.asarray(faces).shape[-1])[:, :3]
    return np.ascontiguousarray(v[f].reshape(-1, 9))


def scene_box9(tri9):
    """Union of the triangle boxes (min xyz, max xyz), atrbvh.cu:282-298."""
    p = tri9.reshape(-1, 3)
    return np.ascontiguousarray(np.concatenate([p.min(axis=0), p.max(axis=0)]), np.float32)


def lbvh63_seed(verts, faces):
    """The oracle's seed build: (sorted codes, order, (left, right, parent, data))."""
    tri = triangles9(verts, faces)
    box = scene_box9(tri)
    keys = np.array([morton63(t, box) for t in tri], np.uint64)
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    sorted_keys = keys[order]
    return sorted_keys, order, karras63(sorted_keys, order)


# ---- traversal packing (pack_oracle.c) ---------------------------------------
PACKED = np.dtype([("lb", "<f4", (6,)), ("rb", "<f4", (6,)), ("meta", "<i4", (4,))])
assert PACKED.itemsize == 64


def pack(nodes, transforms=None, packed=None, pairs=None):
    """bvh_persistent_prepare (transforms None) or obvh_persistent_prepare over
    every node, updating copies of packed [nodes] (PACKED) and pairs
    [internal x 32] (zeros when not given): (packed, pairs)."""
    l = _bind()
    nodes = np.ascontiguousarray(nodes)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    pk = np.zeros(nn, PACKED) if packed is None else np.array(packed, PACKED, copy=True)
    pr = np.zeros((max(ni, 1), 32), np.float32) if pairs is None else np.array(pairs, np.float32, copy=True)
    xf = None if transforms is None else np.ascontiguousarray(transforms, np.float32)
    l.oracle_pack(nodes, None if xf is None else xf.ctypes.data, nn, 0 if xf is None else 1, pk.ctypes.data,
                  pr.ctypes.data)
    return pk, pr


def soa_obvh(packed, pairs, internal_count):
    """kr_cuda_soa_obvh's arrays: (left_T [ni x 12], right_T [ni x 12], metadata [nodes x 4])."""
    l = _bind()
    pk = np.ascontiguousarray(packed, PACKED)
    pr = np.ascontiguousarray(pairs, np.float32)
    nn = pk.shape[0]
    lt = np.zeros((max(internal_count, 1), 12), np.float32)
    rt = np.zeros((max(internal_count, 1), 12), np.float32)
    meta = np.zeros((nn, 4), np.int32)
    l.oracle_soa_obvh(pk.ctypes.data, pr.ctypes.data, internal_count, nn, lt.reshape(-1), rt.reshape(-1),
                      meta.reshape(-1))
    return lt[:internal_count], rt[:internal_count], meta


def refgpu_pack(nodes, transforms=None, packed=None, pairs=None, variant: str = "nofma"):
    """The reference's kr_cuda_bvh_persistent (transforms None) or
    kr_cuda_obvh_persistent + kr_cuda_soa_obvh on the GPU, from the given
    initial buffers (zeros when not given): (packed, pairs, left_T, right_T,
    metadata); the SoA parts are None for the AABB form."""
    l = ref_gpu(variant)
    nodes = np.ascontiguousarray(nodes)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    pk = np.zeros(nn, PACKED) if packed is None else np.array(packed, PACKED, copy=True)
    pr = np.zeros((max(ni, 1), 32), np.float32) if pairs is None else np.array(pairs, np.float32, copy=True)
    lt = np.zeros((max(ni, 1), 12), np.float32)
    rt = np.zeros((max(ni, 1), 12), np.float32)
    meta = np.zeros((nn, 4), np.int32)
    xf = None if transforms is None else np.ascontiguousarray(transforms, np.float32)
    rc = l.refgpu_pack(nodes, None if xf is None else xf.ctypes.data, nn, pk.ctypes.data, pr.ctypes.data,
                       lt.reshape(-1), rt.reshape(-1), meta.reshape(-1))
    if rc != 0:
        raise RuntimeError(f"refgpu_pack: CUDA error {rc}")
    if xf is None:
        return pk, None, None, None, None
    return pk, pr, lt[:ni], rt[:ni], meta


# ---- SoA OBVH ray traversal (trace_oracle.c) ----------------------------------
ISECT = np.dtype([("normal", "<f4", (3,)), ("barys", "<f4", (2,)), ("primitive", "<u4"), ("instance", "<u4")])


def soa_obvh_intersect(left_t, right_t, metadata, verts, faces, prims, rays, threads: int = 1):
    """Closest hits of kr_ray records (8 floats each) against a SoA OBVH:
    ISECT records.  Raises if any ray meets an index outside the arrays."""
    from concurrent.futures import ThreadPoolExecutor
    l = _bind()
    lt = np.ascontiguousarray(left_t, np.float32)
    rt = np.ascontiguousarray(right_t, np.float32)
    meta = np.ascontiguousarray(metadata, np.int32).reshape(-1, 4)
    v, f, nf = _mesh(verts, faces)
    pr = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    ry = np.ascontiguousarray(rays).view(np.uint8)
    n = ry.nbytes // 32
    out = np.zeros(n, ISECT)
    ni = lt.reshape(-1, 12).shape[0]
    args = (lt.ctypes.data, rt.ctypes.data, meta.ctypes.data, ni, meta.shape[0], v.ctypes.data, f.ctypes.data, nf,
            None if pr is None else pr.ctypes.data, 0 if pr is None else pr.size, ry.ctypes.data)
    bounds = np.linspace(0, n, max(1, threads) + 1).astype(np.int64)
    with ThreadPoolExecutor(max_workers=max(1, threads)) as pool:
        bad = sum(pool.map(lambda k: l.oracle_soa_obvh_intersect(*args, int(bounds[k]), int(bounds[k + 1]),
                                                                  out.ctypes.data), range(len(bounds) - 1)))
    if bad:
        raise ValueError(f"{bad} rays met an index outside the arrays")
    return out


def refgpu_soa_obvh_intersect(left_t, right_t, metadata, verts, faces, prims, rays, variant: str = "nofma"):
    """The reference's kr_cuda_soa_obvh_intersect on the GPU: ISECT records."""
    l = ref_gpu(variant)
    c = ctypes
    f_ = l.refgpu_soa_obvh_intersect
    f_.restype = c.c_int
    f_.argtypes = [c.c_void_p] * 3 + [c.c_uint32] * 2 + [c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32,
                                                         c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32, c.c_void_p]
    lt = np.ascontiguousarray(left_t, np.float32)
    rt = np.ascontiguousarray(right_t, np.float32)
    meta = np.ascontiguousarray(metadata, np.int32).reshape(-1, 4)
    v, f, nf = _mesh(verts, faces)
    pr = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    ry = np.ascontiguousarray(rays).view(np.uint8)
    n = ry.nbytes // 32
    out = np.zeros(n, ISECT)
    rc = f_(lt.ctypes.data, rt.ctypes.data, meta.ctypes.data, lt.reshape(-1, 12).shape[0], meta.shape[0],
            v.ctypes.data, v.size // 3, f.ctypes.data, nf, None if pr is None else pr.ctypes.data,
            0 if pr is None else pr.size, ry.ctypes.data, n, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"refgpu_soa_obvh_intersect: CUDA error {rc}")
    return out


def compressed_pairs(nodes, obbs):
    """TEST INPUT: transformation pairs in the form the compressed traversal
    reads (intersectors.cu:1047-1071), one per internal node and child: column
    0 = the axis and angle / pi of the box-to-world rotation (the packer
    negates the axis, so the traversal applies world-to-box), column 1 = the
    box centre, column 2 = twice the half-extents along unit axes (their
    inverse scales the box to the unit cube).  The reference has no producer
    of this form (kr_cuda_soa_compressed_obvh has no caller); a left-handed
    frame is made right-handed by flipping its third axis, which leaves the
    symmetric box unchanged."""
    nodes = np.ascontiguousarray(nodes)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    obbs = np.asarray(obbs, np.float64).reshape(-1, 15)
    pairs = np.zeros((ni, 32), np.float32)
    for side, key in ((0, "left"), (1, "right")):
        o = obbs[nodes[key][:ni].astype(np.int64)]
        ax = o[:, 3:12].reshape(-1, 3, 3)
        ln = np.linalg.norm(ax, axis=2)
        u = ax / np.maximum(ln, 1e-300)[..., None]  # rows: unit box axes (world -> box)
        flip = np.linalg.det(u) < 0
        u[flip, 2] *= -1.0
        rt = np.transpose(u, (0, 2, 1))  # box -> world
        ang = np.arccos(np.clip((np.trace(rt, axis1=1, axis2=2) - 1.0) / 2.0, -1.0, 1.0))
        axis = np.stack([rt[:, 2, 1] - rt[:, 1, 2], rt[:, 0, 2] - rt[:, 2, 0], rt[:, 1, 0] - rt[:, 0, 1]], 1)
        norm = np.linalg.norm(axis, axis=1, keepdims=True)
        axis = np.where(norm > 1e-12, axis / np.maximum(norm, 1e-300), np.array([1.0, 0.0, 0.0]))
        m = np.zeros((ni, 16))
        m[:, 0:3] = axis
        m[:, 3] = ang / np.pi
        m[:, 4:7] = o[:, 0:3]
        m[:, 8:11] = 2.0 * o[:, 12:15] * ln
        pairs[:, 16 * side:16 * side + 16] = m
    return pairs


def refgpu_soa_compressed_obvh(packed, pairs, internal_count, node_count, variant: str = "nofma"):
    """The reference's kr_cuda_soa_compressed_obvh (a host loop between
    copies) on the GPU build: dict of lbounds, rbounds [ni, 6], metadata
    [nodes, 4]."""
    l = ref_gpu(variant)
    c = ctypes
    f_ = l.refgpu_soa_compressed_obvh
    f_.restype = c.c_int
    f_.argtypes = [c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint32, c.c_void_p, c.c_void_p, c.c_void_p]
    pk = np.ascontiguousarray(packed).view(np.uint8)
    pr = np.ascontiguousarray(pairs, np.float32)
    out = {"lbounds": np.zeros((internal_count, 6), np.float32), "rbounds": np.zeros((internal_count, 6), np.float32),
           "metadata": np.zeros((node_count, 4), np.int32)}
    rc = f_(pk.ctypes.data, pr.ctypes.data, internal_count, node_count, out["lbounds"].ctypes.data,
            out["rbounds"].ctypes.data, out["metadata"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"refgpu_soa_compressed_obvh: CUDA error {rc}")
    return out


def refgpu_compressed_intersect(lbounds, rbounds, metadata, verts, faces, prims, rays, variant: str = "nofma"):
    """The reference's kr_cuda_obvh_compressed_persistent_intersect on the
    GPU: ISECT records."""
    l = ref_gpu(variant)
    c = ctypes
    f_ = l.refgpu_compressed_intersect
    f_.restype = c.c_int
    f_.argtypes = [c.c_void_p] * 3 + [c.c_uint32] * 2 + [c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32,
                                                         c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32, c.c_void_p]
    lb = np.ascontiguousarray(lbounds, np.float32).reshape(-1, 6)
    rb = np.ascontiguousarray(rbounds, np.float32).reshape(-1, 6)
    meta = np.ascontiguousarray(metadata, np.int32).reshape(-1, 4)
    v, f, nf = _mesh(verts, faces)
    pr = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    ry = np.ascontiguousarray(rays).view(np.uint8)
    n = ry.nbytes // 32
    out = np.zeros(n, ISECT)
    rc = f_(lb.ctypes.data, rb.ctypes.data, meta.ctypes.data, lb.shape[0], meta.shape[0], v.ctypes.data, v.size // 3,
            f.ctypes.data, nf, None if pr is None else pr.ctypes.data, 0 if pr is None else pr.size, ry.ctypes.data,
            n, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"refgpu_compressed_intersect: CUDA error {rc}")
    return out


def soa_compressed_obvh(packed, pairs, internal_count, node_count):
    """The oracle's restatement of kr_cuda_soa_compressed_obvh
    (oracle_soa_compressed_obvh, pack_oracle.c): dict of lbounds, rbounds
    [ni, 6], metadata [nodes, 4]."""
    l = _bind()
    pk = np.ascontiguousarray(packed).view(np.uint8)
    pr = np.ascontiguousarray(pairs, np.float32)
    out = {"lbounds": np.zeros((internal_count, 6), np.float32), "rbounds": np.zeros((internal_count, 6), np.float32),
           "metadata": np.zeros((node_count, 4), np.int32)}
    l.oracle_soa_compressed_obvh(pk.ctypes.data, pr.ctypes.data, internal_count, node_count,
                                 out["lbounds"].ctypes.data, out["rbounds"].ctypes.data, out["metadata"].ctypes.data)
    return out


def soa_obvh_traversal_counts(left_t, right_t, metadata, verts, faces, prims, rays):
    """Per-ray means of the traversal's work on these rays: dict of internal
    nodes visited, leaves visited, triangles tested, primitive-list reads."""
    l = _bind()
    lt = np.ascontiguousarray(left_t, np.float32)
    rt = np.ascontiguousarray(right_t, np.float32)
    meta = np.ascontiguousarray(metadata, np.int32).reshape(-1, 4)
    v, f, nf = _mesh(verts, faces)
    pr = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    ry = np.ascontiguousarray(rays).view(np.uint8)
    n = ry.nbytes // 32
    out = np.zeros(n, ISECT)
    counts = np.zeros(4, np.int64)
    bad = l.oracle_soa_obvh_intersect_counts(lt.ctypes.data, rt.ctypes.data, meta.ctypes.data, lt.reshape(-1, 12).shape[0],
                                             meta.shape[0], v.ctypes.data, f.ctypes.data, nf,
                                             None if pr is None else pr.ctypes.data, 0 if pr is None else pr.size,
                                             ry.ctypes.data, 0, n, out.ctypes.data, counts.ctypes.data)
    if bad:
        raise ValueError(f"{bad} rays met an index outside the arrays")
    return {"internal_visits": counts[0] / n, "leaf_visits": counts[1] / n, "triangle_tests": counts[2] / n,
            "list_reads": counts[3] / n}


def refgpu_soa_obvh_intersect_ms(left_t, right_t, metadata, verts, faces, prims, rays, reps=5, variant="nofma"):
    """Mean device time (ms) of one launch of the reference's traversal kernel
    on device-resident data."""
    l = ref_gpu(variant)
    c = ctypes
    f_ = l.refgpu_soa_obvh_intersect_timed
    f_.restype = c.c_int
    f_.argtypes = [c.c_void_p] * 3 + [c.c_uint32] * 2 + [c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32,
                                                         c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint32, c.c_uint32,
                                                         c.POINTER(c.c_float)]
    lt = np.ascontiguousarray(left_t, np.float32)
    rt = np.ascontiguousarray(right_t, np.float32)
    meta = np.ascontiguousarray(metadata, np.int32).reshape(-1, 4)
    v, f, nf = _mesh(verts, faces)
    pr = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    ry = np.ascontiguousarray(rays).view(np.uint8)
    ms = c.c_float(0.0)
    rc = f_(lt.ctypes.data, rt.ctypes.data, meta.ctypes.data, lt.reshape(-1, 12).shape[0], meta.shape[0],
            v.ctypes.data, v.size // 3, f.ctypes.data, nf, None if pr is None else pr.ctypes.data,
            0 if pr is None else pr.size, ry.ctypes.data, ry.nbytes // 32, reps, c.byref(ms))
    if rc != 0:
        raise RuntimeError(f"refgpu_soa_obvh_intersect_timed: CUDA error {rc}")
    return ms.value


# ---- SAH cost ------------------------------------------------------------------
def ref_bvh_sah(nodes, ci=1.2, ct=1.0, obbs=None, root=0):
    """The reference's own kr_bvh_sah (host code in oracle/_ref/libref_tree_gpu.so)."""
    l = ref_gpu("nofma")
    f_ = l.kr_bvh_sah
    f_.restype = ctypes.c_float
    f_.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_char_p]
    n = np.ascontiguousarray(nodes)
    o = None if obbs is None else np.ascontiguousarray(obbs, np.float32)
    return float(f_(n.ctypes.data, root, ci, ct, None if o is None else o.ctypes.data, None))


def sah_terms(nodes, parents, obbs=None, ci=1.2, ct=1.0):
    """Per-node float32 terms of the SAH cost (0 for nodes a traversal cannot
    reach from root 0) and the root's area; their exact sum is the cost."""
    npr = nodes["n_prims"].astype(np.int64)
    nn = npr.shape[0]
    par = np.asarray(parents, np.int64).copy()
    par[par == 0xFFFFFFFF] = -1
    reached = np.ones(nn, bool)
    cur = par.copy()
    while (cur >= 0).any():
        live = cur >= 0
        reached[live] &= npr[cur[live]] == 0
        cur[live] = par[cur[live]]
    b = nodes["b"].astype(np.float32)
    d = (b[:, 3:] - b[:, :3]).astype(np.float32)
    aabb = np.float32(2) * (d[:, 0] * d[:, 1] + d[:, 0] * d[:, 2] + d[:, 1] * d[:, 2])
    if obbs is not None:
        e = (np.float32(2) * np.asarray(obbs, np.float32)[:, 12:15]).astype(np.float32)
        area = np.float32(2) * (e[:, 0] * e[:, 1] + e[:, 0] * e[:, 2] + e[:, 1] * e[:, 2])
    else:
        area = aabb
    ci, ct = np.float32(ci), np.float32(ct)
    npf = npr.astype(np.float32)
    term = np.where(npr == 0, ci * area, (ct * npf) * np.where(npr == 1, aabb, area)).astype(np.float32)
    if npr[0] != 0:
        term[0] = (ct * area[0]) * npf[0]
    term[npr == 0xFFFF] = 0
    term[~reached] = 0
    return term, float(area[0])
