"""Shared pytest configuration: the `gpu` marker and small helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")


def lattice_mesh(k: int = 12):
    """Two equal small triangles on every point of a k^3 lattice, as
    (vertices, faces): ties in the sort, the Karras split, the treelet leaf to
    expand and the pair to merge."""
    g = np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"), -1).reshape(-1, 3)
    c = np.repeat(g, 2, axis=0).astype(np.float32) * 0.5
    tri = np.array([[0, 0, 0], [0.2, 0, 0], [0, 0.2, 0]], np.float32)
    v = (c[:, None, :] + tri[None]).reshape(-1, 3)
    n = c.shape[0]
    f = np.zeros((n, 4), np.uint32)
    f[:, 0] = np.arange(0, 3 * n, 3)
    f[:, 1] = f[:, 0] + 1
    f[:, 2] = f[:, 0] + 2
    return v, f


def deep_or_tied_mesh(layout: str):
    """Trees far from balanced, as (vertices, faces): centroids on a geometric
    sequence along the diagonal ("geometric": a chain of key bits, so leaf
    ranges cross CTA and tile edges high up), or 37 centroids shared by 811
    triangles each ("duplicates": keys tied, split by index)."""
    rng = np.random.default_rng(7)
    if layout == "geometric":
        k = rng.integers(0, 10, size=30_000)
        c = (0.5 ** k)[:, None] * np.ones((1, 3)) * 0.999 + rng.uniform(0, 1e-4, size=(30_000, 1))
    else:
        c = np.repeat(rng.uniform(0, 1, size=(37, 3)), 811, axis=0)
    n = c.shape[0]
    tri = np.array([[0, 0, 0], [1e-3, 0, 0], [0, 1e-3, 0]], np.float64)
    v = (c[:, None, :] + tri[None]).reshape(-1, 3).astype(np.float32)
    f = np.zeros((n, 4), np.uint32)
    f[:, 0] = np.arange(0, 3 * n, 3)
    f[:, 1] = f[:, 0] + 1
    f[:, 2] = f[:, 0] + 2
    return v, f


def golden_dito():
    d = np.load(os.path.join(GOLDEN, "dito_golden.npz"))
    for i, name in enumerate(d["names"]):
        yield str(name), d["points"][d["offsets"][i]:d["offsets"][i + 1]], d["boxes"][i]


def obb_contains(points: np.ndarray, obb: np.ndarray, rel: float = 1e-5) -> int:
    """Number of points outside the box (FP64, tolerance rel * box scale)."""
    p = points.astype(np.float64)
    mid = obb[0:3].astype(np.float64)
    axes = obb[3:12].astype(np.float64).reshape(3, 3)
    ext = obb[12:15].astype(np.float64)
    local = (p - mid) @ axes.T
    scale = max(1.0, float(np.abs(p).max()) if len(p) else 1.0)
    return int(np.count_nonzero(np.abs(local) > ext + rel * scale))


def same_bits(a, b) -> bool:
    """Bitwise equality of float arrays, treating -0.0 == +0.0."""
    a = np.asarray(a, np.float32) + np.float32(0.0)
    b = np.asarray(b, np.float32) + np.float32(0.0)
    return bool(np.array_equal(a.view(np.uint32), b.view(np.uint32)))


def obb_overshoot(points: np.ndarray, obb: np.ndarray) -> np.ndarray:
    """World-space distance by which each point lies outside the box (FP64).

    The box is mid + sum_k c_k a_k with |c_k| <= ext_k; the axes a_k need not be
    unit length (the reference's leaf boxes keep an unnormalised third axis), so
    c_k = (p - mid).a_k / |a_k|^2 and the overshoot along a_k is
    (|c_k| - ext_k) |a_k|."""
    p = np.asarray(points, np.float64).reshape(-1, 3)
    mid = obb[0:3].astype(np.float64)
    axes = obb[3:12].astype(np.float64).reshape(3, 3)
    ext = obb[12:15].astype(np.float64)
    la = np.linalg.norm(axes, axis=1)
    c = (p - mid) @ axes.T / (la * la)
    over = (np.abs(c) - ext) * la
    return np.max(over, axis=1)


def contained(points, obb, rel: float = 1e-6) -> bool:
    """True if every point is inside the box up to rel * (1 + |p|) world units,
    i.e. a few float32 ulps of the coordinates."""
    p = np.asarray(points, np.float64).reshape(-1, 3)
    tol = rel * (1.0 + np.abs(p).max(axis=1))
    return bool(np.all(obb_overshoot(p, obb) <= tol))


def uncontained_leaves(v, f4, leaf_prims, parents, obbs, rel: float = 1e-6) -> int:
    """FP64 containment of every leaf's triangle in its leaf box and in every
    ancestor's box, for all leaves at once: the number of (leaf, box) pairs
    in which some vertex lies outside by more than rel * (1 + |p|).

    `leaf_prims[j]` is leaf j's triangle (node n-1+j); the walk moves all
    leaves one level up per step, so it takes depth steps of array work."""
    n = (len(parents) + 1) // 2
    tri = np.asarray(v, np.float64)[np.asarray(f4)[np.asarray(leaf_prims, np.int64), :3]]  # (n, 3, 3)
    tol = rel * (1.0 + np.abs(tri).max(axis=2))                                              # (n, 3)
    node = np.arange(n - 1, 2 * n - 1, dtype=np.int64)
    active = np.arange(n, dtype=np.int64)
    obbs = np.asarray(obbs, np.float64)
    bad = 0
    for _ in range(2 * n):
        if active.size == 0:
            break
        o = obbs[node[active]]
        mid, axes, ext = o[:, 0:3], o[:, 3:12].reshape(-1, 3, 3), o[:, 12:15]
        la = np.linalg.norm(axes, axis=2)                                  # (k, 3)
        c = np.einsum("kpj,kaj->kpa", tri[active] - mid[:, None, :], axes) / (la * la)[:, None, :]
        over = ((np.abs(c) - ext[:, None, :]) * la[:, None, :]).max(axis=2)  # (k, 3 vertices)
        bad += int(np.count_nonzero((~(over <= tol[active])).any(axis=1)))
        up = np.asarray(parents, np.uint32)[node[active]]
        keep = up != 0xFFFFFFFF
        active = active[keep]
        node[active] = up[keep].astype(np.int64)
    else:
        raise AssertionError("parent walk longer than the tree")
    return bad
