"""Regenerates tests/golden/dito_golden.npz from the reference's own CPU DiTO.

    python tests/golden/make_golden.py

Needs oracle/_ref/libref_dito.so, which oracle/Makefile compiles from the
reference tree (src/common/algorithm/dito/dito.cpp, unmodified) plus the
kr_points_obb clamp of src/common/geometry.cpp:249.  The inputs are seeded
synthetic point sets chosen to reach every branch of DiTO_14: regular OBBs,
the AABB kept by the final test, both degenerate cases, tiny sets that use
all points as the selection set, and inputs full of ties.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from obvh_b200 import workloads  # noqa: E402


def cases():
    out = []
    for seed in range(4):
        out.append((f"ellipsoid_{seed}", workloads.ellipsoid_points(1500, seed=seed)))
    rng = np.random.default_rng(100)
    for n in list(range(1, 21)) + [31, 64]:
        out.append((f"gauss_n{n}", rng.normal(size=(n, 3)).astype(np.float32) * np.float32(3.0)))
    out.append(("single_point", np.tile(np.float32([[1.5, -2.0, 0.25]]), (40, 1))))
    out.append(("two_points", np.float32([[0, 0, 0], [1e-4, 0, 0]] * 20)))
    t = rng.normal(size=(200, 1)).astype(np.float32)
    out.append(("collinear", (t * np.float32([1, 2, 3]) + np.float32([5, 5, 5])).astype(np.float32)))
    xs = np.round(rng.normal(size=(120, 1)) * 8) / 8
    out.append(("x_line", (xs * np.float32([1, 0, 0])).astype(np.float32)))
    ys = np.round(rng.normal(size=(90, 1)) * 4) / 4
    out.append(("diag_line", (ys * np.float32([1, 1, 0]) + np.float32([0, 0, 2])).astype(np.float32)))
    plane = rng.normal(size=(300, 3)).astype(np.float32)
    plane[:, 2] = 0
    out.append(("planar_z0", plane))
    out.append(("axis_box", np.float32([[x, y, z] for x in (0, 2) for y in (0, 3) for z in (0, 1)] * 4)))
    out.append(("integer_ties", np.round(rng.normal(size=(500, 3)) * 2).astype(np.float32)))
    out.append(("cube_grid", np.stack(np.meshgrid(*[np.arange(6, dtype=np.float32)] * 3), -1).reshape(-1, 3)))
    thin = rng.normal(size=(400, 3)).astype(np.float32) * np.float32([10, 0.001, 0.001])
    out.append(("needle", thin))
    out.append(("empty", np.zeros((0, 3), np.float32)))
    return out


def main():
    if not oracle.ref_available():
        oracle.build()
    names, offsets, pts, boxes = [], [0], [], []
    for name, p in cases():
        names.append(name)
        pts.append(p)
        offsets.append(offsets[-1] + len(p))
        boxes.append(oracle.ref_dito14(p) if len(p) else oracle.ref_dito14(np.zeros((0, 3), np.float32)))
    np.savez_compressed(os.path.join(HERE, "dito_golden.npz"), names=np.array(names),
                        offsets=np.array(offsets, np.int64), points=np.concatenate(pts).astype(np.float32),
                        boxes=np.stack(boxes).astype(np.float32))
    print(f"wrote {len(names)} cases, {offsets[-1]} points")


if __name__ == "__main__":
    main()
