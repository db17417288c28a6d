"""GPU parity of the fused commit (obvh_build_async: LBVH + OBB tree +
collapse in one chain) against the oracle running the three steps in turn."""
import numpy as np
import pytest

from conftest import deep_or_tied_mesh, same_bits
from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def builder():
    import torch
    assert torch.cuda.is_available()
    return bvh.ObvhBuilder()


def _run(builder, v, f, flags, ci=1.2, ct=1.0):
    import torch
    mesh = bvh.Mesh(v, f)
    o = builder.build(mesh, flags=flags, ci=ci, ct=ct)
    torch.cuda.synchronize()
    err, slots = builder.status(mesh.n_faces)
    assert err == 0
    return o, slots


def _expect(v, f, ci=1.2, ct=1.0):
    r = ref.lbvh_build(v, f)
    obbs, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col, cnt, prims, cst, used = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"], ci, ct)
    return r, obbs, xfs, col, cnt, prims, cst, used


def _check(o, slots, exp, n, flags):
    r, obbs, xfs, col, cnt, prims, cst, used = exp
    nodes = bvh.nodes_numpy(o["nodes"])
    ni = n - 1
    assert same_bits(nodes["b"], r["nodes"]["b"])
    assert np.array_equal(nodes["left"], r["nodes"]["left"])
    assert np.array_equal(nodes["right"][:ni], r["nodes"]["right"][:ni])
    assert np.array_equal(nodes["n_prims"], r["nodes"]["n_prims"])
    assert np.array_equal(o["parents"].cpu().numpy().view(np.uint32), r["parents"])
    assert same_bits(o["bounds"].cpu().numpy(), np.concatenate([r["scene"], r["centroid"]]))
    if flags & bvh.BUILD_OBBS:
        assert same_bits(o["obbs"].cpu().numpy(), obbs)
        assert same_bits(o["transforms"].cpu().numpy(), xfs)
    counts = o["counts"].cpu().numpy().view(np.uint32)
    costs = o["costs"].cpu().numpy()
    if flags & bvh.BUILD_COLLAPSE:
        c = bvh.nodes_numpy(o["collapsed"])
        assert same_bits(c["b"], col["b"])
        assert np.array_equal(c["left"], col["left"])
        assert np.array_equal(c["right"][:ni], col["right"][:ni])
        assert np.array_equal(c["n_prims"], col["n_prims"])
        assert np.array_equal(counts, cnt)
        assert same_bits(costs, cst)
        assert slots == used
        assert np.array_equal(o["primitives"].cpu().numpy().view(np.uint32)[:used], prims[:used])
    else:
        assert np.array_equal(counts, r["counts"])
        assert same_bits(costs, r["costs"])


@pytest.mark.parametrize("n", [1, 2, 3, 17, 1000, 65_537])
def test_fused_build_matches_the_three_steps(builder, n):
    v, f = workloads.triangle_soup(n, seed=300 + n)
    o, slots = _run(builder, v, f, 3)
    _check(o, slots, _expect(v, f), n, 3)


def test_fused_build_full_size(builder):
    v, f = workloads.triangle_soup(2_000_000, seed=1)
    o, slots = _run(builder, v, f, 3)
    _check(o, slots, _expect(v, f), 2_000_000, 3)


def test_fused_build_mesh_and_other_sah_constants(builder):
    v, f = workloads.torus_knot_mesh(segments=256, around=112)
    n = f.shape[0]
    o, slots = _run(builder, v, f, 3, ci=0.8, ct=1.3)
    _check(o, slots, _expect(v, f, 0.8, 1.3), n, 3)


@pytest.mark.parametrize("flags", [0, 1, 2])
def test_fused_build_partial_flags(builder, flags):
    n = 20_000
    v, f = workloads.triangle_soup(n, seed=41)
    o, slots = _run(builder, v, f, flags)
    _check(o, slots, _expect(v, f), n, flags)


@pytest.mark.parametrize("layout", ["geometric", "duplicates"])
def test_fused_build_deep_and_tied_trees(builder, layout):
    """Trees far from balanced (conftest.deep_or_tied_mesh)."""
    v, f = deep_or_tied_mesh(layout)
    o, slots = _run(builder, v, f, 3)
    _check(o, slots, _expect(v, f), f.shape[0], 3)


def test_build_graph_replays_equal_the_three_steps(builder):
    """obvh_build_graph_create / _launch: the chain captured once per buffer
    set; every replay rebuilds from what the input buffers hold then."""
    import torch
    n = 65_537
    meshes = [workloads.triangle_soup(n, seed=70 + j) for j in range(3)]
    dev = [bvh.Mesh(v, f) for v, f in meshes[:2]]
    outs = [builder.outputs(n) for _ in range(2)]
    graphs = [builder.capture(m, o) for m, o in zip(dev, outs)]
    exps = [_expect(v, f) for v, f in meshes[:2]]
    for rep in range(2):
        for j in range(2):
            graphs[j].launch()
            torch.cuda.synchronize()
            err, slots = builder.status(n)
            assert err == 0
            _check(outs[j], slots, exps[j], n, 3)
    # new contents in mesh 0's buffers: the same graph builds them
    v2, f2 = meshes[2]
    dev[0].verts.copy_(torch.from_numpy(v2).to(dev[0].verts.device))
    dev[0].faces.copy_(torch.from_numpy(bvh.as_faces4(f2).view(np.int32)).to(dev[0].faces.device))
    graphs[0].launch()
    torch.cuda.synchronize()
    err, slots = builder.status(n)
    assert err == 0
    _check(outs[0], slots, _expect(v2, f2), n, 3)


def test_build_graph_equals_the_direct_build_at_full_size(builder):
    import torch
    v, f = workloads.triangle_soup(2_000_000, seed=5)
    mesh = bvh.Mesh(v, f)
    direct = builder.build(mesh)
    torch.cuda.synchronize()
    out = builder.outputs(mesh.n_faces)
    g = builder.capture(mesh, out)
    g.launch()
    torch.cuda.synchronize()
    for k in direct:
        assert torch.equal(direct[k].view(torch.uint8), out[k].view(torch.uint8)), k



def test_build_graph_keeps_its_buffers_when_the_builder_grows():
    """A graph captured on a small workspace still replays correctly after the
    builder moved to a larger one (the graph holds the buffers it baked in)."""
    import torch
    b = bvh.ObvhBuilder()
    n = 5_000
    v, f = workloads.triangle_soup(n, seed=81)
    mesh = bvh.Mesh(v, f)
    out = b.outputs(n)
    g = b.capture(mesh, out)
    b.build(bvh.Mesh(*workloads.triangle_soup(3 * n, seed=82)))  # reallocates the builder's workspace
    torch.cuda.synchronize()
    g.launch()
    torch.cuda.synchronize()
    direct = bvh.ObvhBuilder().build(mesh)
    torch.cuda.synchronize()
    for k in ("nodes", "parents", "counts", "costs", "bounds", "obbs", "transforms", "collapsed", "primitives"):
        assert torch.equal(direct[k].view(torch.uint8), out[k].view(torch.uint8)), k
