"""The intersector plugins through the reference's own loading protocol.

``load(name)`` does what kr_ads_load does (src/common/ads.c:6-32): opens
``lib<name>.so`` (here, next to libobvh_b200.so), looks up
``korangar_ads_action`` and calls it with KR_ADS_ACTION_CREATE.  The ctypes
structures below mirror the reference's kr_scene / kr_object / kr_mesh /
kr_descriptor layouts (include/obvh_types.h) so a scene built here is the
scene a reference caller would hand to COMMIT.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native

PKG = os.path.dirname(os.path.abspath(__file__))

# kr_ads_action
ACTION = {name: i for i, name in enumerate([
    "NONE", "INTERSECTION_QUERY", "OCCLUSION_QUERY", "PREFERRED_QUERY_TYPE", "GET_BLAS", "GET_TLAS", "CREATE",
    "COMMIT", "INIT", "UPDATE", "SETTINGS_UPDATE", "DESTROY", "CSV_EXPORT", "CSV_IMPORT", "BVH_MODEL_EXPORT",
    "BINARY_EXPORT", "BINARY_IMPORT", "NAME"])}
KR_QUERY_TYPE_CUDA = 2
KR_OBJECT_MESH = 1


class Descriptor(ctypes.Structure):
    _fields_ = [("key", ctypes.c_char_p), ("value", ctypes.c_char_p)]


class DescriptorContainer(ctypes.Structure):
    _fields_ = [("descriptors", ctypes.POINTER(Descriptor)), ("descriptor_count", ctypes.c_uint64)]


class Mesh(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("normals", ctypes.c_void_p), ("uvs", ctypes.c_void_p),
                ("faces", ctypes.c_void_p), ("face_count", ctypes.c_uint64), ("attr_count", ctypes.c_uint64)]


class _ObjUnion(ctypes.Union):
    _fields_ = [("as_mesh", Mesh), ("as_sphere", ctypes.c_float * 4)]


class Object(ctypes.Structure):
    _anonymous_ = ("u",)
    _fields_ = [("aabb", ctypes.c_float * 6), ("type", ctypes.c_int32), ("u", _ObjUnion)]


class Instance(ctypes.Structure):
    _fields_ = [("model", ctypes.c_float * 32), ("object_id", ctypes.c_uint64)]


class Scene(ctypes.Structure):
    _fields_ = [("camera_opaque", ctypes.c_uint8 * 280), ("aabb", ctypes.c_float * 6),
                ("objects", ctypes.POINTER(Object)), ("object_count", ctypes.c_uint64),
                ("instances", ctypes.POINTER(Instance)), ("instance_count", ctypes.c_uint64),
                ("cameras", ctypes.c_void_p), ("camera_count", ctypes.c_uint64),
                ("materials", ctypes.c_void_p), ("material_count", ctypes.c_uint64),
                ("textures", ctypes.c_void_p), ("texture_count", ctypes.c_uint64),
                ("samplers", ctypes.c_void_p), ("sampler_count", ctypes.c_uint64),
                ("frame", ctypes.c_uint32 * 2), ("tile", ctypes.c_uint32 * 2),
                ("benchmark_file", ctypes.c_char_p)]


class Ads(ctypes.Structure):
    _fields_ = [("callback", ctypes.c_void_p), ("library", ctypes.c_void_p), ("context", ctypes.c_void_p),
                ("runtime", ctypes.c_void_p)]


class Blas(ctypes.Structure):
    """obvh_ads_blas (include/obvh_plugin.h)."""
    _fields_ = [(n, ctypes.c_void_p) for n in ("nodes", "collapsed", "parents", "primitive_counts", "costs", "obbs",
                                               "transforms", "primitives", "vertices", "faces")] + \
               [(n, ctypes.c_uint32) for n in ("node_count", "internal_count", "primitive_count", "primitive_slots")] + \
               [("aabb", ctypes.c_float * 6), ("build_ms", ctypes.c_float), ("commits", ctypes.c_uint32),
                ("ci", ctypes.c_float), ("ct", ctypes.c_float)] + \
               [(n, ctypes.c_int32) for n in ("collapse", "use_obbs", "save_construction_information",
                                              "intersect_bounds", "use_persistent_kernel", "intersect_bounds_level")] + \
               [(n, ctypes.c_void_p) for n in ("bvh_packed", "transformations", "soa_left_T", "soa_right_T",
                                               "soa_metadata")]


assert ctypes.sizeof(Scene) == 424 and Scene.objects.offset == 304 and Scene.benchmark_file.offset == 416
assert ctypes.sizeof(Object) == 80 and ctypes.sizeof(Mesh) == 48
assert ctypes.sizeof(Blas) == 200

KR_QUERY_TYPE_CUDA = 2


class IntersectionQuery(ctypes.Structure):
    """kr_intersection_query of CUDA kind (include/obvh_types.h)."""
    _fields_ = [("type", ctypes.c_int32), ("rays", ctypes.c_void_p), ("isects", ctypes.c_void_p),
                ("ray_count", ctypes.c_uint64)]


assert ctypes.sizeof(IntersectionQuery) == 32 and IntersectionQuery.rays.offset == 8

_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.POINTER(Ads), ctypes.c_void_p, ctypes.c_int)


class MeshScene:
    """A kr_scene of triangle-mesh objects whose host arrays stay alive with it."""

    def __init__(self, meshes, benchmark_file: str | None = None):
        self._keep = []
        objs = (Object * max(len(meshes), 1))()
        for i, (v, f) in enumerate(meshes):
            v = np.ascontiguousarray(v, np.float32).reshape(-1, 3)
            f = np.ascontiguousarray(f, np.uint32).reshape(-1, 4)
            self._keep += [v, f]
            objs[i].type = KR_OBJECT_MESH
            objs[i].as_mesh.vertices = v.ctypes.data
            objs[i].as_mesh.faces = f.ctypes.data
            objs[i].as_mesh.face_count = f.shape[0]
            objs[i].as_mesh.attr_count = v.shape[0]
        self.objects = objs
        self.scene = Scene()
        self.scene.objects = ctypes.cast(objs, ctypes.POINTER(Object))
        self.scene.object_count = len(meshes)
        self._bf = benchmark_file.encode() if benchmark_file else None
        self.scene.benchmark_file = self._bf


class Intersector:
    """One loaded plugin instance (kr_ads)."""

    def __init__(self, name: str):
        _native.lib()  # the core library the plugin links against
        path = os.path.join(PKG, f"lib{name}.so")
        if not os.path.exists(path):
            raise _native.ObvhError(f"plugin not built: {path}")
        self.dll = ctypes.CDLL(path)
        self.action_fn = _CALLBACK(("korangar_ads_action", self.dll))
        self.ads = Ads()
        self.ads.callback = ctypes.cast(self.action_fn, ctypes.c_void_p)
        self.ads.context = self.action_fn(None, None, ACTION["CREATE"])
        if not self.ads.context:
            raise _native.ObvhError("CREATE returned no context")

    def call(self, action: str, descriptor=None):
        return self.action_fn(ctypes.byref(self.ads), descriptor, ACTION[action])

    def check(self, action: str, descriptor=None):
        e = self.call(action, descriptor)
        if e:
            raise _native.ObvhError(ctypes.string_at(e).decode(errors="replace"))

    def init(self, **settings):
        items = [(k.encode(), str(v).encode()) for k, v in settings.items()]
        arr = (Descriptor * max(len(items), 1))(*[Descriptor(k, v) for k, v in items])
        cont = DescriptorContainer(ctypes.cast(arr, ctypes.POINTER(Descriptor)), len(items))
        self.check("INIT", ctypes.cast(ctypes.pointer(cont), ctypes.c_void_p))

    def commit(self, scene: MeshScene):
        self.check("COMMIT", ctypes.cast(ctypes.pointer(scene.scene), ctypes.c_void_p))

    def name(self) -> str:
        return ctypes.string_at(self.call("NAME")).decode()

    def preferred_query_type(self) -> int:
        return int(self.call("PREFERRED_QUERY_TYPE") or 0)

    def intersect(self, d_rays: int, d_isects: int, ray_count: int):
        """INTERSECTION_QUERY of CUDA kind over device rays and records."""
        q = IntersectionQuery()
        q.type = KR_QUERY_TYPE_CUDA
        q.rays, q.isects, q.ray_count = d_rays, d_isects, ray_count
        self.check("INTERSECTION_QUERY", ctypes.cast(ctypes.pointer(q), ctypes.c_void_p))

    def blas(self) -> Blas:
        p = self.call("GET_BLAS")
        return Blas.from_address(p)

    def destroy(self):
        if self.ads.context:
            self.check("DESTROY")
            self.ads.context = None
