"""GPU parity of the batched mesh builds (include/obvh_build_batch.h).

Every mesh of a batch must come out exactly as obvh_build_async builds it
alone (the per-mesh results are in turn held to the oracle and to the
reference's own kernels by test_build_gpu.py and test_ref_gpu_pin.py): the
same node records, parents, counts, costs, boxes, OBBs, transforms, collapsed
nodes and primitive lists, bit for bit with zero signs aside.  Meshes of 2 to
cta_max_faces triangles go through the one-CTA-per-mesh kernel, the others
through the whole-GPU chain; both are covered, with ties (a lattice of equal
triangles) and closed meshes (a knot), and the captured graph replays to
the same results.
"""
import numpy as np
import pytest

from conftest import lattice_mesh, same_bits
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


def _meshes(sizes, seed):
    out = []
    for k, n in enumerate(sizes):
        if n == "lattice":
            out.append(lattice_mesh(8))
        elif n == "knot":
            out.append(workloads.torus_knot_mesh(64, 28, seed=seed + k))
        else:
            out.append(workloads.triangle_soup(n, seed=seed + k))
    return out


def _pack(meshes):
    vo, fo = [0], [0]
    for v, f in meshes:
        vo.append(vo[-1] + v.shape[0])
        fo.append(fo[-1] + f.shape[0])
    verts = np.concatenate([v for v, _ in meshes]).astype(np.float32)
    faces = np.concatenate([bvh.as_faces4(f) for _, f in meshes])
    return verts, faces, np.array(vo, np.uint64), np.array(fo, np.uint64)


def _alone(builder, v, f, flags, ci, ct):
    import torch
    o = builder.build(bvh.Mesh(v, f), flags=flags, ci=ci, ct=ct)
    torch.cuda.synchronize()
    err, slots = builder.status(f.shape[0])
    assert err == 0
    return o, slots


def _same_nodes(a, b):
    assert np.array_equal(a["left"], b["left"])
    assert np.array_equal(a["right"], b["right"])
    assert np.array_equal(a["n_prims"], b["n_prims"])
    assert same_bits(a["b"], b["b"])


def _check(meshes, flags=3, ci=1.2, ct=1.0, cta_max_faces=0, graph=False):
    import torch
    verts, faces, vo, fo = _pack(meshes)
    batch = bvh.BuildBatch(vo, fo, flags=flags, cta_max_faces=cta_max_faces)
    dv = torch.from_numpy(verts).cuda()
    df = torch.from_numpy(faces.view(np.int32)).cuda()
    out = batch.outputs()
    if graph:
        batch.capture(dv, df, out, ci=ci, ct=ct)
        batch.launch()
        batch.launch()
    else:
        batch.enqueue(dv, df, out, ci=ci, ct=ct)
    torch.cuda.synchronize()
    err, slots = batch.status()
    assert err == 0
    got = {k: v.cpu().numpy() for k, v in out.items()}
    nodes = got["nodes"].view(bvh.NODE)
    collapsed = got["collapsed"].view(bvh.NODE) if "collapsed" in got else None
    builder = bvh.ObvhBuilder()
    for m, (v, f) in enumerate(meshes):
        n = f.shape[0]
        lo, hi = batch.node_offset(m), batch.node_offset(m) + 2 * n - 1
        want, want_slots = _alone(builder, v, f, flags, ci, ct)
        w = {k: t.cpu().numpy() for k, t in want.items()}
        _same_nodes(nodes[lo:hi], w["nodes"].view(bvh.NODE))
        assert np.array_equal(got["parents"][lo:hi], w["parents"]), m
        assert np.array_equal(got["counts"][lo:hi], w["counts"]), m
        assert same_bits(got["costs"][lo:hi], w["costs"]), m
        assert same_bits(got["bounds"][m], w["bounds"]), m
        if flags & bvh.BUILD_OBBS:
            assert same_bits(got["obbs"][lo:hi], w["obbs"]), m
            assert same_bits(got["transforms"][lo:hi], w["transforms"]), m
        if flags & bvh.BUILD_COLLAPSE:
            assert slots[m] == want_slots, m
            _same_nodes(collapsed[lo:hi], w["collapsed"].view(bvh.NODE))
            p0 = int(fo[m])
            assert np.array_equal(got["primitives"][p0:p0 + slots[m]], w["primitives"][:slots[m]]), m
    return batch


SIZES = [1, 2, 3, 5, 17, 31, 32, 33, 100, 511, 512, 513, 1000, 4096, 9999, 16384, 16385, 30000, "lattice", "knot"]


def test_every_mesh_equals_its_lone_build():
    batch = _check(_meshes(SIZES, seed=10))
    info = batch.info()
    assert info["cta_meshes"] == len(SIZES) - 3  # 1, 16385 and 30000 take the chain
    assert info["chain_meshes"] == 3


@pytest.mark.parametrize("flags", [0, 1, 2])
def test_partial_builds(flags):
    _check(_meshes([2, 64, 700, 5000, 20000, "knot"], seed=20), flags=flags)


def test_other_costs_and_a_small_cta_limit():
    _check(_meshes([3, 50, 99, 100, 101, 2000, "lattice"], seed=30), ci=0.8, ct=1.3, cta_max_faces=100)


def test_many_uneven_meshes_in_a_graph():
    rng = np.random.default_rng(40)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(2), np.log(16384), size=300))]
    _check(_meshes(sizes, seed=40), graph=True)


def test_chain_meshes_in_a_graph():
    """Meshes above the CTA limit go through the whole-GPU chain, which forks
    onto helper streams (the walk up the tree beside the candidate search, the
    collapse beside the extents); captured into the batch's graph, the forks
    become parallel branches and every result stays its lone build's."""
    batch = _check(_meshes([20000, 40000, 700, "knot"], seed=50), graph=True)
    assert batch.info()["chain_meshes"] >= 2
