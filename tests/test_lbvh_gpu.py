"""GPU parity of the LBVH build (Morton codes, sort order, topology, bounds,
counts, SAH costs) against the oracle restatement: all bit-exact."""
import numpy as np
import pytest

from conftest import same_bits
from oracle import bvh as obvh_oracle
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def builder():
    import torch
    assert torch.cuda.is_available()
    return bvh.LbvhBuilder()


def _build(builder, v, f):
    import torch
    mesh = bvh.Mesh(v, f)
    out = builder.build(mesh)
    torch.cuda.synchronize()
    return {
        "nodes": bvh.nodes_numpy(out["nodes"]),
        "parents": out["parents"].cpu().numpy().view(np.uint32),
        "counts": out["counts"].cpu().numpy().view(np.uint32),
        "costs": out["costs"].cpu().numpy(),
        "bounds": out["bounds"].cpu().numpy(),
    }


def _compare(got, want, n):
    nodes, ref = got["nodes"], want["nodes"]
    assert same_bits(nodes["b"], ref["b"])
    ni = n - 1
    assert np.array_equal(nodes["left"], ref["left"])           # children / primitive offsets
    assert np.array_equal(nodes["right"][:ni], ref["right"][:ni])
    assert np.array_equal(nodes["n_prims"], ref["n_prims"])
    assert np.array_equal(nodes["axis"], ref["axis"])
    assert np.array_equal(got["parents"], want["parents"])
    assert np.array_equal(got["counts"], want["counts"])
    assert same_bits(got["costs"], want["costs"])
    assert same_bits(got["bounds"][:6], want["scene"])
    assert same_bits(got["bounds"][6:], want["centroid"])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 33, 1000, 4095, 4096, 4097, 100_003])
def test_soup_sizes(builder, n):
    v, f = workloads.triangle_soup(n, seed=n)
    _compare(_build(builder, v, f), obvh_oracle.lbvh_build(v, f), n)


def test_full_size_soup(builder):
    """The 2,000,000-triangle LBVH workload."""
    n = 2_000_000
    v, f = workloads.triangle_soup(n, seed=1)
    _compare(_build(builder, v, f), obvh_oracle.lbvh_build(v, f), n)


def test_torus_knot_mesh(builder):
    v, f = workloads.torus_knot_mesh(segments=256, around=112)
    _compare(_build(builder, v, f), obvh_oracle.lbvh_build(v, f), f.shape[0])


def test_duplicate_codes(builder):
    """Every centroid identical: the index tie rule 32 + clz(i ^ j) shapes the tree."""
    n = 5000
    v = np.tile(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), (n, 1))
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    _compare(_build(builder, v, f), obvh_oracle.lbvh_build(v, f), n)


def test_clustered_codes(builder):
    """Few distinct codes with long runs of equal keys."""
    rng = np.random.default_rng(9)
    n = 30_000
    c = rng.integers(0, 4, size=(n, 1, 3)).astype(np.float32)
    v = (c + np.float32([[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0]])[None]).reshape(-1, 3).astype(np.float32)
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    _compare(_build(builder, v, f), obvh_oracle.lbvh_build(v, f), n)


def test_bbox_entry_points():
    v, f = workloads.triangle_soup(50_000, seed=4)
    mesh = bvh.Mesh(v, f)
    scene, centroid = obvh_oracle.scene_bounds(v, f)
    assert same_bits(bvh.bbox_calculate(mesh), scene)
    assert same_bits(bvh.bbox_calculate(mesh, centroid=True), centroid)
    # the pre-filled box is expanded, not replaced
    pre = np.float32([-5, 0.5, 0.5, 0.5, 0.5, 9])
    got = bvh.bbox_calculate(mesh, prefill=pre)
    want = np.concatenate([np.minimum(pre[:3], scene[:3]), np.maximum(pre[3:], scene[3:])])
    assert same_bits(got, want)
