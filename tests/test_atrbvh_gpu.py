"""GPU parity of the ATRBVH builder (include/obvh_atrbvh.h) against the oracle.

The tree (topology, leaf order, boxes), the sorted 63-bit codes, counts and
costs must be bit-identical to the restatement (zero signs aside); the full
commit (tree, OBB transform, collapse) must equal the oracle running the
three steps in turn.  Outputs are checked for the properties the method
guarantees at the torus-knot size of the benchmark.
"""
import numpy as np
import pytest

from conftest import contained, lattice_mesh, same_bits
from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def builder():
    import torch
    assert torch.cuda.is_available()
    return bvh.AtrbvhBuilder()


def _run(builder, v, f, flags=3, tau=9, iters=2, ci=1.2, ct=1.0):
    import torch
    mesh = bvh.Mesh(v, f)
    o = builder.build(mesh, flags=flags, ci=ci, ct=ct, treelet_size=tau, iterations=iters)
    torch.cuda.synchronize()
    err, slots = builder.status(mesh.n_faces)
    assert err == 0
    return o, slots


def _check_tree(o, r, n):
    nodes = bvh.nodes_numpy(o["nodes"])
    ni = n - 1
    assert np.array_equal(nodes["left"], r["nodes"]["left"])
    assert np.array_equal(nodes["right"][:ni], r["nodes"]["right"][:ni])
    assert np.array_equal(nodes["n_prims"], r["nodes"]["n_prims"])
    assert np.array_equal(o["parents"].cpu().numpy().view(np.uint32), r["parents"])
    assert same_bits(nodes["b"], r["nodes"]["b"])


@pytest.mark.parametrize("n", [2, 3, 9, 17, 1000, 40_000])
@pytest.mark.parametrize("tau", [7, 9])
def test_tree_matches_oracle(builder, n, tau):
    v, f = workloads.triangle_soup(n, seed=500 + n)
    o, _ = _run(builder, v, f, flags=0, tau=tau)
    r = ref.atrbvh_build(v, f, tau, 2)
    _check_tree(o, r, n)
    assert np.array_equal(o["counts"].cpu().numpy().view(np.uint32), r["counts"])
    assert same_bits(o["costs"].cpu().numpy(), r["costs"])


@pytest.mark.parametrize("iters,tau,ci,ct", [(0, 9, 1.2, 1.0), (1, 3, 1.2, 1.0), (3, 12, 2.0, 0.5), (2, 20, 1.2, 1.0)])
def test_tree_other_settings(builder, iters, tau, ci, ct):
    v, f = workloads.torus_knot_mesh(40, 20, seed=9)
    o, _ = _run(builder, v, f, flags=0, tau=tau, iters=iters, ci=ci, ct=ct)
    r = ref.atrbvh_build(v, f, tau, iters, ci=ci, ct=ct)
    _check_tree(o, r, f.shape[0])


def test_lattice_ties(builder):
    # many equal centroids and equal areas: ties in the sort, the Karras
    # split, the leaf to expand and the pair to merge
    v, f = lattice_mesh(12)
    o, _ = _run(builder, v, f, flags=0, tau=7)
    _check_tree(o, ref.atrbvh_build(v, f, 7, 2), f.shape[0])


def _pin_mesh(kind):
    if kind == "soup":
        return workloads.triangle_soup(20_000, seed=1500)
    if kind == "lattice":
        return lattice_mesh(12)
    return workloads.torus_knot_mesh(128, 56, seed=2)


@pytest.mark.skipif(not ref.ref_treelet_available(), reason="oracle/_ref/libref_treelet_emu.so not built")
@pytest.mark.parametrize("kind", ["soup", "lattice", "knot"])
@pytest.mark.parametrize("tau", [7, 9])
def test_tree_matches_the_reference_treelet_kernel(builder, kind, tau):
    """The GPU tree against the reference's own treelet kernel
    (AgglomerativeTreelet.cu, run as host code by oracle/ref_treelet_emu.cpp)
    applied to the seed tree, then copied and refit (atrbvh.cu:95-183)."""
    v, f = _pin_mesh(kind)
    n = f.shape[0]
    r = ref.atrbvh_emit(ref.ref_treelet_optimize(ref.atrbvh_seed(v, f), tau, 2))
    o, _ = _run(builder, v, f, flags=0, tau=tau)
    _check_tree(o, r, n)
    assert np.array_equal(o["counts"].cpu().numpy().view(np.uint32), r["counts"])
    assert same_bits(o["costs"].cpu().numpy(), r["costs"])


def test_full_commit_matches_the_three_steps(builder):
    v, f = workloads.torus_knot_mesh(96, 48, seed=3)
    n = f.shape[0]
    o, slots = _run(builder, v, f, flags=3, tau=7)
    r = ref.atrbvh_build(v, f, 7, 2)
    _check_tree(o, r, n)
    obbs, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    assert same_bits(o["obbs"].cpu().numpy(), obbs)
    assert same_bits(o["transforms"].cpu().numpy(), xfs)
    col, cnt, prims, cst, used = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"], 1.2, 1.0)
    c = bvh.nodes_numpy(o["collapsed"])
    assert np.array_equal(c["left"], col["left"])
    assert np.array_equal(c["n_prims"], col["n_prims"])
    assert same_bits(c["b"], col["b"])
    assert np.array_equal(o["counts"].cpu().numpy().view(np.uint32), cnt)
    assert same_bits(o["costs"].cpu().numpy(), cst)
    assert slots == used
    assert np.array_equal(o["primitives"].cpu().numpy().view(np.uint32)[:used], prims[:used])


@pytest.mark.parametrize("flags", [1, 2])
@pytest.mark.parametrize("n", [2, 3, 700, 30_000])
def test_commit_parts_match_the_steps(builder, flags, n):
    """The OBB transform alone (LBVH costs) and the collapse alone (its
    primitive lists gathered by walking subtrees) against the oracle's steps."""
    v, f = workloads.triangle_soup(n, seed=900 + n)
    o, slots = _run(builder, v, f, flags=flags, tau=7)
    r = ref.atrbvh_build(v, f, 7, 2)
    _check_tree(o, r, n)
    if flags == 1:
        assert np.array_equal(o["counts"].cpu().numpy().view(np.uint32), r["counts"])
        assert same_bits(o["costs"].cpu().numpy(), r["costs"])
        obbs, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
        assert same_bits(o["obbs"].cpu().numpy(), obbs)
        assert same_bits(o["transforms"].cpu().numpy(), xfs)
    else:
        col, cnt, prims, cst, used = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"], 1.2, 1.0)
        c = bvh.nodes_numpy(o["collapsed"])
        assert np.array_equal(c["left"], col["left"])
        assert np.array_equal(c["n_prims"], col["n_prims"])
        assert same_bits(c["b"], col["b"])
        assert np.array_equal(o["counts"].cpu().numpy().view(np.uint32), cnt)
        assert same_bits(o["costs"].cpu().numpy(), cst)
        assert slots == used
        assert np.array_equal(o["primitives"].cpu().numpy().view(np.uint32)[:used], prims[:used])


def test_knot_full_size_properties(builder):
    """The 917,504-triangle torus knot: a valid tree whose SAH is below the
    LBVH's, and every triangle inside its leaf box and every ancestor's."""
    v, f = workloads.torus_knot_mesh()
    n = f.shape[0]
    o, slots = _run(builder, v, f, flags=1, tau=7)
    nodes = bvh.nodes_numpy(o["nodes"])
    parents = o["parents"].cpu().numpy().view(np.uint32)
    ni = n - 1
    assert sorted(nodes["left"][ni:].tolist()) == list(range(n))
    seen = np.zeros(2 * n - 1, np.int8)
    stack = [0]
    while stack:
        x = stack.pop()
        seen[x] += 1
        if x < ni:
            stack += [int(nodes["left"][x]), int(nodes["right"][x])]
    assert (seen == 1).all() and parents[0] == 0xFFFFFFFF
    lb = ref.lbvh_build(v, f)
    assert o["costs"][0].item() < lb["costs"][0]
    obbs = o["obbs"].cpu().numpy()
    rng = np.random.default_rng(0)
    for leaf in rng.choice(np.arange(ni, 2 * n - 1), size=200, replace=False):
        tri = v[f[nodes["left"][leaf], :3]]
        x = leaf
        while x != 0xFFFFFFFF:
            assert contained(tri, obbs[x]), (leaf, x)
            x = parents[x]


def test_build_graph_equals_the_direct_build(builder):
    """obvh_build_atrbvh_graph_create: the ATRBVH commit captured once and
    replayed equals the direct commit bit for bit, also after the input
    buffers were given a new mesh."""
    import torch
    n = 100_000
    meshes = [workloads.triangle_soup(n, seed=90 + j) for j in range(2)]
    direct = []
    for v, f in meshes:
        o, _ = _run(builder, v, f)
        direct.append({k: t.clone() for k, t in o.items()})
    dev = bvh.Mesh(*meshes[0])
    out = builder.outputs(n)
    g = builder.capture(dev, out)
    for j in (0, 1):
        if j:
            v, f = meshes[1]
            dev.verts.copy_(torch.from_numpy(v).to(dev.verts.device))
            dev.faces.copy_(torch.from_numpy(bvh.as_faces4(f).view(np.int32)).to(dev.faces.device))
            out["primitives"].zero_()  # slots past the collapsed leaves' are not written
        g.launch()
        torch.cuda.synchronize()
        err, _ = builder.status(n)
        assert err == 0
        for k in direct[j]:
            assert torch.equal(direct[j][k].view(torch.uint8), out[k].view(torch.uint8)), (j, k)
