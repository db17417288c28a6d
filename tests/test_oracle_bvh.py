"""The tree restatement: pinned where the reference has host-callable code
(Morton encoding, 4x4 inverse/product, AABB area) and checked structurally
elsewhere (the reference's tree kernels are GPU-only and untested)."""
import numpy as np
import pytest

import oracle
from conftest import contained
from oracle import bvh
from obvh_b200 import workloads


pytestmark = pytest.mark.skipif(not bvh.ref_vecmath_available(), reason="reference vecmath not built here")


def test_morton_matches_reference():
    l = bvh._bind()
    vm = bvh.ref_vecmath()
    rng = np.random.default_rng(0)
    pts = rng.uniform(-0.3, 1.3, size=(20000, 3)).astype(np.float32)
    pts[:100] = np.float32([0, 1, 1023 / 1024])  # clamp edges
    for x, y, z in pts:
        assert l.oracle_morton30(x, y, z) == vm.ref_v32morton3(x, y, z)


def test_matrix_helpers_match_reference():
    l = bvh._bind()
    vm = bvh.ref_vecmath()
    rng = np.random.default_rng(1)
    for t in range(2000):
        m = rng.normal(size=16).astype(np.float32)
        if t % 2:
            m[[3, 7, 11]] = 0
            m[15] = 1
        if t % 97 == 0:
            m[:] = 0  # singular: identity
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        l.oracle_minverse4(m, a)
        vm.ref_minverse4(m, b)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        r = rng.normal(size=16).astype(np.float32)
        l.oracle_mmul4(m, r, a)
        vm.ref_mmul4(m, r, b)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        box = np.sort(rng.normal(size=(2, 3)).astype(np.float32), axis=0).reshape(-1)
        assert np.float32(l.oracle_aabb_area(box)) == np.float32(vm.ref_aabb_area(box))


def _check_tree(nodes, parents, n):
    ni = n - 1
    seen = np.zeros(2 * n - 1, np.int32)
    for i in range(ni):
        l, r = nodes["left"][i], nodes["right"][i]
        assert parents[l] == i and parents[r] == i
        seen[l] += 1
        seen[r] += 1
    assert parents[0] == 0xFFFFFFFF
    assert np.all(seen[1:] == 1) and seen[0] == 0


@pytest.mark.parametrize("n", [2, 3, 7, 64, 1000, 20000])
def test_lbvh_oracle_structure(n):
    v, f = workloads.triangle_soup(n, seed=n)
    r = bvh.lbvh_build(v, f)
    nodes, parents = r["nodes"], r["parents"]
    _check_tree(nodes, parents, n)
    assert r["counts"][0] == n
    assert np.all(np.diff(r["codes"].astype(np.int64)) >= 0)
    # leaves carry every primitive once, sorted stably by code
    prims = nodes["left"][n - 1:]
    assert sorted(prims.tolist()) == list(range(n))
    # each internal node's box contains its children's
    for i in range(n - 1):
        for c in (nodes["left"][i], nodes["right"][i]):
            assert np.all(nodes["b"][i][:3] <= nodes["b"][c][:3]) and np.all(nodes["b"][i][3:] >= nodes["b"][c][3:])


def test_lbvh_oracle_duplicate_codes():
    """All centroids equal: codes tie everywhere, the index rule builds the tree."""
    n = 257
    v = np.tile(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), (n, 1))
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    r = bvh.lbvh_build(v, f)
    _check_tree(r["nodes"], r["parents"], n)
    assert r["counts"][0] == n


def test_obb_tree_oracle_contains_subtree_vertices():
    n = 3000
    v, f = workloads.triangle_soup(n, seed=5)
    r = bvh.lbvh_build(v, f)
    obbs, xfs, _ = bvh.obb_tree(r["nodes"], r["parents"], v, f)
    nodes, parents = r["nodes"], r["parents"]
    f4 = bvh._mesh(v, f)[1].reshape(-1, 4)
    for j in range(n):
        tri = v[f4[nodes["left"][n - 1 + j], :3]].astype(np.float64)
        node = n - 1 + j
        while node != 0xFFFFFFFF:
            assert contained(tri, obbs[node]), (j, node)
            node = parents[node]


def test_collapse_oracle_partition():
    n = 5000
    v, f = workloads.triangle_soup(n, seed=6)
    r = bvh.lbvh_build(v, f)
    col, cnt, prims, cst, used = bvh.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    assert used <= n
    # every collapsed leaf holds its subtree's primitives exactly once
    ni = n - 1
    for c in range(1, 2 * n - 1):
        np_ = col["n_prims"][c]
        if c < ni and 0 < np_ < 0xFFFF:
            got = prims[col["left"][c]:col["left"][c] + np_]
            stack, leaves = [c], []
            while stack:
                x = stack.pop()
                if x >= ni:
                    leaves.append(r["nodes"]["left"][x])
                else:
                    stack += [r["nodes"]["left"][x], r["nodes"]["right"][x]]
            assert sorted(got.tolist()) == sorted(leaves)
