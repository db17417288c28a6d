"""Commits through the intersector plugins on the GPU: the device-resident
result (GET_BLAS) must equal the oracle running the reference's commit chain
(LBVH or ATRBVH, OBB tree, collapse) on the same mesh."""
import ctypes

import numpy as np
import pytest

from conftest import same_bits
from oracle import bvh as ref
from obvh_b200 import bvh, plugin, workloads

pytestmark = pytest.mark.gpu


def _d2h(ptr, dtype, count):
    import torch  # noqa: F401  (loads the CUDA runtime)
    rt = ctypes.CDLL("libcudart.so.12")
    out = np.empty(count, dtype)
    assert rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(ptr), ctypes.c_size_t(out.nbytes), 2) == 0
    return out


def _expect(kind, v, f, ci, ct):
    r = ref.lbvh_build(v, f) if kind == "lbvh_gpu" else ref.atrbvh_build(v, f, 9, 2, ci=ci, ct=ct)
    obbs, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"], ci, ct)
    return r, obbs, xfs, col


@pytest.mark.parametrize("kind", ["lbvh_gpu", "atrbvh_gpu"])
@pytest.mark.parametrize("mesh", ["soup", "knot"])
def test_commit_matches_the_reference_chain(tmp_path, kind, mesh):
    import torch
    assert torch.cuda.is_available()
    v, f = workloads.triangle_soup(30_000, seed=7) if mesh == "soup" else workloads.torus_knot_mesh(128, 64, seed=5)
    n = f.shape[0]
    a = plugin.Intersector(kind)
    a.init(collapse="y", use_obbs="y", ci="1.2", ct="1.0")
    bench = tmp_path / "bench.csv"
    a.commit(plugin.MeshScene([(v, f)], benchmark_file=str(bench)))
    b = a.blas()
    assert b.commits == 1 and b.primitive_count == n and b.node_count == 2 * n - 1
    assert b.build_ms > 0 and bench.read_text().count("\n") == 1
    r, obbs, xfs, (col, cnt, prims, cst, used) = _expect(kind, v, f, 1.2, 1.0)
    nodes = _d2h(b.nodes, ref.NODE, 2 * n - 1)
    assert np.array_equal(nodes["left"], r["nodes"]["left"])
    assert same_bits(nodes["b"], r["nodes"]["b"])
    assert np.array_equal(_d2h(b.parents, np.uint32, 2 * n - 1), r["parents"])
    assert same_bits(_d2h(b.obbs, np.float32, 15 * (2 * n - 1)).reshape(-1, 15), obbs)
    assert same_bits(_d2h(b.transforms, np.float32, 16 * (2 * n - 1)).reshape(-1, 16), xfs)
    c = _d2h(b.collapsed, ref.NODE, 2 * n - 1)
    assert np.array_equal(c["left"], col["left"]) and np.array_equal(c["n_prims"], col["n_prims"])
    assert np.array_equal(_d2h(b.primitive_counts, np.uint32, 2 * n - 1), cnt)
    assert same_bits(_d2h(b.costs, np.float32, 2 * n - 1), cst)
    assert b.primitive_slots == used
    assert np.array_equal(_d2h(b.primitives, np.uint32, n)[:used], prims[:used])
    a.destroy()


def test_recommit_and_flags_off():
    v1, f1 = workloads.triangle_soup(5_000, seed=1)
    v2, f2 = workloads.triangle_soup(9_000, seed=2)
    a = plugin.Intersector("lbvh_gpu")
    a.init(collapse="n", use_obbs="n")
    a.commit(plugin.MeshScene([(v1, f1), (v2, f2)]))  # the last object's tree stays, as in the reference
    b = a.blas()
    assert b.commits == 2 and b.primitive_count == 9_000 and not b.obbs and not b.collapsed
    r = ref.lbvh_build(v2, f2)
    assert np.array_equal(_d2h(b.nodes, ref.NODE, 2 * 9_000 - 1)["left"], r["nodes"]["left"])
    assert same_bits(_d2h(b.costs, np.float32, 2 * 9_000 - 1), r["costs"])
    a.destroy()


@pytest.mark.parametrize("kind", ["lbvh_gpu", "atrbvh_gpu"])
def test_intersection_query_matches_the_oracle(kind):
    """COMMIT with use_obbs, collapse and use_persistent_kernel packs the tree;
    INTERSECTION_QUERY then gives the oracle's closest hits (the reference's
    traversal restated) through the oracle's own build, pack and SoA OBVH."""
    import torch
    v, f = workloads.triangle_soup(20_000, seed=31)
    n = f.shape[0]
    a = plugin.Intersector(kind)
    a.init(collapse="y", use_obbs="y", use_persistent_kernel="y", ci="1.2", ct="1.0")
    a.commit(plugin.MeshScene([(v, f)]))
    b = a.blas()
    assert b.bvh_packed and b.soa_left_T and b.soa_metadata
    rays = workloads.probe_rays(30_000, [0, 0, 0], [1, 1, 1], seed=4)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    d_isects = torch.zeros(28 * len(rays), dtype=torch.uint8, device="cuda")
    a.intersect(d_rays.data_ptr(), d_isects.data_ptr(), len(rays))
    got = d_isects.cpu().numpy().view(ref.ISECT)
    r = ref.lbvh_build(v, f) if kind == "lbvh_gpu" else ref.atrbvh_build(v, f, 9, 2)
    _, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col, _, prims, _, _ = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    pk, pr = ref.pack(col, xfs)
    lt, rt, meta = ref.soa_obvh(pk, pr, n - 1)
    want = ref.soa_obvh_intersect(lt, rt, meta, v, f, prims, rays, threads=8)
    assert got.tobytes() == want.tobytes()
    assert (got["primitive"] != 0xFFFFFFFF).sum() > 0
    a.destroy()


def test_query_forms_not_built_are_errors():
    """The traversal forms the reference has but this library does not build
    answer with an error; with neither use_obbs nor use_persistent_kernel the
    query does nothing, as the reference's does."""
    import torch
    v, f = workloads.triangle_soup(1000, seed=2)
    rays = workloads.probe_rays(100, [0, 0, 0], [1, 1, 1], seed=1)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    d_isects = torch.zeros(28 * len(rays), dtype=torch.uint8, device="cuda")
    for settings, ok in (({"use_obbs": "y"}, False), ({"use_persistent_kernel": "y"}, False),
                         ({"use_obbs": "y", "use_persistent_kernel": "y", "intersect_bounds": "y"}, False), ({}, True)):
        a = plugin.Intersector("lbvh_gpu")
        a.init(**settings)
        a.commit(plugin.MeshScene([(v, f)]))
        if ok:
            a.intersect(d_rays.data_ptr(), d_isects.data_ptr(), len(rays))
            assert int(d_isects.sum().item()) == 0
        else:
            with pytest.raises(plugin._native.ObvhError, match="not built"):
                a.intersect(d_rays.data_ptr(), d_isects.data_ptr(), len(rays))
        a.destroy()
