"""obvh_b200 - B200-native (sm_100a) DiTO-14 OBB fits and AABB-BVH -> OBB-tree
transforms behind the Korangar C entry points (kr_cuda_points_obb,
kr_cuda_bvh_obb_tree, kr_cuda_bvh_collapse, the lbvh_gpu / atrbvh_gpu
intersector plugins).

The compute path is libobvh_b200.so (hand-written CUDA, see csrc/); this
package is a thin host-side mirror of its C ABI for Python callers.
"""
from ._native import ObvhError, lib  # noqa: F401
from .dito import DitoFitter, REFERENCE_GPU, kr_cuda_points_obb, points_obb  # noqa: F401

__all__ = ["ObvhError", "lib", "DitoFitter", "REFERENCE_GPU", "kr_cuda_points_obb", "points_obb"]
