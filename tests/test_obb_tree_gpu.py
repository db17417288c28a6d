"""GPU parity of the AABB-BVH -> OBB-tree transform and of the node collapse
against the oracle restatement, through the reference entry points
kr_cuda_bvh_obb_tree and kr_cuda_bvh_collapse."""
import numpy as np
import pytest

from conftest import contained, same_bits, uncontained_leaves
from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def builder():
    import torch
    assert torch.cuda.is_available()
    return bvh.LbvhBuilder()


def _lbvh(builder, v, f):
    mesh = bvh.Mesh(v, f)
    tree = builder.build(mesh)
    return mesh, tree


def _tree_numpy(tree):
    return bvh.nodes_numpy(tree["nodes"]), tree["parents"].cpu().numpy().view(np.uint32)


def _check_obbs(mesh, tree, v, f, sample_leaves=None):
    obbs, xfs = bvh.obb_tree(mesh, tree)
    nodes, parents = _tree_numpy(tree)
    want_o, want_x, _ = ref.obb_tree(nodes, parents, v, f)
    got_o, got_x = obbs.cpu().numpy(), xfs.cpu().numpy()
    assert same_bits(got_o, want_o)
    assert same_bits(got_x, want_x)
    # every vertex lies in its leaf's box and in every ancestor's box
    n = (len(parents) + 1) // 2
    f4 = bvh.as_faces4(f)
    if sample_leaves is None:
        assert uncontained_leaves(v, f4, nodes["left"][n - 1:], parents, got_o) == 0
        return got_o
    for j in np.random.default_rng(0).choice(n, sample_leaves, replace=False):
        tri = v[f4[nodes["left"][n - 1 + j], :3]]
        node = n - 1 + j
        while node != 0xFFFFFFFF:
            assert contained(tri, got_o[node]), (j, node)
            node = parents[node]
    return got_o


@pytest.mark.parametrize("n", [1, 2, 3, 9, 100, 5000, 100_003])
def test_obb_tree_soup(builder, n):
    v, f = workloads.triangle_soup(n, seed=100 + n)
    mesh, tree = _lbvh(builder, v, f)
    _check_obbs(mesh, tree, v, f)


def test_obb_tree_full_size(builder):
    """The 2M-triangle LBVH + OBB-tree workload: every vertex of every leaf
    inside its leaf's box and every ancestor's box (FP64)."""
    v, f = workloads.triangle_soup(2_000_000, seed=1)
    mesh, tree = _lbvh(builder, v, f)
    _check_obbs(mesh, tree, v, f)


def test_obb_tree_mesh(builder):
    v, f = workloads.torus_knot_mesh(segments=256, around=112)
    mesh, tree = _lbvh(builder, v, f)
    _check_obbs(mesh, tree, v, f)


def _random_tree(n, rng):
    """A binary tree whose depth-first leaf order is not the leaf index order."""
    ni = n - 1
    nodes = np.zeros(2 * n - 1, ref.NODE)
    parents = np.full(2 * n - 1, 0xFFFFFFFF, np.uint32)
    leaf_ids = list(rng.permutation(n) + ni)
    nodes["left"][ni:] = rng.permutation(n)
    nodes["n_prims"][ni:] = 1
    nxt = [1]

    def build_at(idx, items):
        if len(items) == 2:
            l, r = items
        else:
            cut = int(rng.integers(1, len(items)))
            kids = []
            for part in (items[:cut], items[cut:]):
                if len(part) == 1:
                    kids.append(part[0])
                else:
                    kids.append(nxt[0])
                    nxt[0] += 1
                    build_at(kids[-1], part)
            l, r = kids
        nodes["left"][idx], nodes["right"][idx] = l, r
        parents[l] = parents[r] = idx

    import sys
    sys.setrecursionlimit(100000)
    build_at(0, leaf_ids)
    return nodes, parents


def test_obb_tree_on_a_non_morton_tree():
    """kr_cuda_bvh_obb_tree on a tree not built by the LBVH (e.g. a restructured one)."""
    import torch
    rng = np.random.default_rng(3)
    n = 3000
    v, f = workloads.triangle_soup(n, seed=8)
    nodes, parents = _random_tree(n, rng)
    f4 = bvh.as_faces4(f)
    for j in range(n):  # leaf bounds (unused by the transform, kept valid)
        tri = v[f4[nodes["left"][n - 1 + j], :3]]
        nodes["b"][n - 1 + j] = np.concatenate([tri.min(0), tri.max(0)])
    mesh = bvh.Mesh(v, f)
    tree = {"nodes": torch.from_numpy(nodes.view(np.uint8).copy()).cuda(),
            "parents": torch.from_numpy(parents.view(np.int32).copy()).cuda()}
    obbs, xfs = bvh.obb_tree(mesh, tree)
    want_o, want_x, _ = ref.obb_tree(nodes, parents, v, f)
    assert same_bits(obbs.cpu().numpy(), want_o)
    assert same_bits(xfs.cpu().numpy(), want_x)


def test_obb_tree_rejects_a_parent_cycle():
    """A malformed tree ends with an error from the bounded walks, not a hang."""
    import torch
    from obvh_b200 import ObvhError
    n = 64
    v, f = workloads.triangle_soup(n, seed=9)
    rng = np.random.default_rng(4)
    nodes, parents = _random_tree(n, rng)
    parents[5] = 5  # internal node 5 is its own parent
    mesh = bvh.Mesh(v, f)
    tree = {"nodes": torch.from_numpy(nodes.view(np.uint8).copy()).cuda(),
            "parents": torch.from_numpy(parents.view(np.int32).copy()).cuda()}
    with pytest.raises(ObvhError, match="cycle|malformed"):
        bvh.obb_tree(mesh, tree)
    # the library stays usable afterwards
    v2, f2 = workloads.triangle_soup(100, seed=10)
    b = bvh.LbvhBuilder()
    mesh2 = bvh.Mesh(v2, f2)
    bvh.obb_tree(mesh2, b.build(mesh2))


@pytest.mark.parametrize("n", [2, 3, 50, 5000, 200_003])
def test_collapse(builder, n):
    v, f = workloads.triangle_soup(n, seed=200 + n)
    mesh, tree = _lbvh(builder, v, f)
    nodes, parents = _tree_numpy(tree)
    counts0 = tree["counts"].cpu().numpy().view(np.uint32).copy()
    costs0 = tree["costs"].cpu().numpy().copy()
    out = bvh.collapse(tree, 1.2, 1.0, metrics=True)
    col_w, cnt_w, prim_w, cost_w, used = ref.collapse(nodes, parents, counts0, costs0, 1.2, 1.0)
    col = bvh.nodes_numpy(out["collapsed"])
    assert same_bits(col["b"], col_w["b"])
    assert np.array_equal(col["left"], col_w["left"])
    assert np.array_equal(col["right"][: n - 1], col_w["right"][: n - 1])
    assert np.array_equal(col["n_prims"], col_w["n_prims"])
    assert np.array_equal(tree["counts"].cpu().numpy().view(np.uint32), cnt_w)
    assert same_bits(tree["costs"].cpu().numpy(), cost_w)
    assert np.array_equal(out["primitives"].cpu().numpy().view(np.uint32)[:used], prim_w[:used])
    assert out["metrics"][0] >= 0 and out["metrics"][1] >= 0


def test_collapse_full_size(builder):
    v, f = workloads.triangle_soup(2_000_000, seed=1)
    mesh, tree = _lbvh(builder, v, f)
    nodes, parents = _tree_numpy(tree)
    counts0 = tree["counts"].cpu().numpy().view(np.uint32).copy()
    costs0 = tree["costs"].cpu().numpy().copy()
    out = bvh.collapse(tree)
    col_w, cnt_w, prim_w, cost_w, used = ref.collapse(nodes, parents, counts0, costs0)
    col = bvh.nodes_numpy(out["collapsed"])
    assert np.array_equal(col["n_prims"], col_w["n_prims"]) and np.array_equal(col["left"], col_w["left"])
    assert np.array_equal(out["primitives"].cpu().numpy().view(np.uint32)[:used], prim_w[:used])
    assert same_bits(tree["costs"].cpu().numpy(), cost_w)
