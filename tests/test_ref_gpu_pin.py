"""The tree path pinned to the reference's own GPU kernels.

oracle/_ref/libref_tree_gpu*.so hold the reference's lbvh.cu and transforms.cu
compiled for sm_100a by oracle/Makefile (where the reference tree is present;
the built files travel with the repository).  The calls run, with the
reference's launch shapes, its Morton, sort, Karras and bottom-up box kernels,
its OBB candidate, refit and finalize kernels, and kr_cuda_bvh_collapse.  Two
of its kernels are not run, because their __syncthreads() calls follow threads
that have returned or left a loop: the subtree-summary pass and the scene-box
reductions.  The oracle supplies their outputs (summaries; the centroid box)
in the reference's own arrays.

* "nofma" is the reference built with --fmad=false, the arithmetic the
  restatement and the CUDA path use.  Every output must equal the oracle's bit
  for bit (zero signs aside), and the CUDA path's, checked directly here.
* The ATRBVH seed build (oracle/_ref/libref_lbvh63_gpu.so: LBVH.cu and
  CubWrapper.cu through their own host wrappers) must equal the oracle's
  63-bit codes, order and Karras tree exactly.  Its node boxes and the treelet
  optimiser are not run (barriers in divergent loops).
* "fmad" is the reference as its own build compiles it: nvcc's default
  contraction of multiplies and adds.  Codes, order, topology, counts, boxes
  and collapse decisions must still be identical and costs within 1e-6
  relative.  OBBs: contraction moves near-ties in the candidate score, so a
  small share of internal nodes picks another frame; the rest agree in their
  axes to about 1e-6.
"""
import numpy as np
import pytest

from conftest import deep_or_tied_mesh, same_bits
from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ref.ref_gpu_available("nofma") and ref.ref_gpu_available("fmad")),
                                 reason="oracle/_ref reference GPU libraries not built")]


def _mesh(case):
    kind, n = case
    if kind == "soup":
        return workloads.triangle_soup(n, seed=300 + n)
    if kind == "knot":
        return workloads.torus_knot_mesh(segments=256, around=112)
    return deep_or_tied_mesh(kind)


CASES = [("soup", 2), ("soup", 3), ("soup", 17), ("soup", 1000), ("soup", 65_537), ("soup", 300_000),
         ("knot", 0), ("geometric", 0), ("duplicates", 0)]


def _same_tree(a, b, n):
    ni = n - 1
    assert np.array_equal(a["nodes"]["left"], b["nodes"]["left"])
    assert np.array_equal(a["nodes"]["right"][:ni], b["nodes"]["right"][:ni])
    assert np.array_equal(a["nodes"]["n_prims"], b["nodes"]["n_prims"])
    assert np.array_equal(a["parents"], b["parents"])
    if "codes" in a and "codes" in b:
        assert np.array_equal(a["codes"], b["codes"])
    assert np.array_equal(a["counts"], b["counts"])
    assert same_bits(a["nodes"]["b"], b["nodes"]["b"])


def _root_lists(col, prims):
    """Each collapse root's primitive list (its run at its own offset)."""
    roots = np.nonzero((col["n_prims"] > 1) & (col["n_prims"] != 0xFFFF))[0]
    return {int(x): prims[col["left"][x]:col["left"][x] + col["n_prims"][x]].tolist() for x in roots}


def _same_collapse(a, pa, b, pb):
    """Collapsed trees equal but for the offsets of the collapse roots' runs,
    which the reference takes from an atomic counter."""
    la, lb = _root_lists(a, pa), _root_lists(b, pb)
    assert la == lb
    other = np.ones(a.shape[0], bool)
    other[list(la)] = False
    assert np.array_equal(a["left"][other], b["left"][other])
    assert np.array_equal(a["n_prims"], b["n_prims"])
    assert same_bits(a["b"], b["b"])


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1] or ''}")
def test_lbvh_kernels_equal_the_oracle(case):
    v, f = _mesh(case)
    o = ref.lbvh_build(v, f)
    g = ref.refgpu_lbvh(v, f, "nofma")
    _same_tree(g, o, f.shape[0])
    assert same_bits(g["costs"], o["costs"])


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1] or ''}")
def test_transform_and_collapse_kernels_equal_the_oracle(case):
    v, f = _mesh(case)
    o = ref.lbvh_build(v, f)
    obbs, xfs, _ = ref.obb_tree(o["nodes"], o["parents"], v, f)
    gb, gx = ref.refgpu_obb_tree(o["nodes"], o["parents"], o["counts"], v, f, "nofma")
    assert same_bits(gb, obbs)
    assert same_bits(gx, xfs)
    col, cnt, prims, cst, used = ref.collapse(o["nodes"], o["parents"], o["counts"], o["costs"], 1.2, 1.0)
    gc, gcnt, gprims, gcst = ref.refgpu_collapse(o["nodes"], o["parents"], o["counts"], o["costs"], 1.2, 1.0, "nofma")
    _same_collapse(gc, gprims, col, prims)
    assert np.array_equal(gcnt, cnt)
    assert same_bits(gcst, cst)


@pytest.mark.parametrize("case", [("soup", 300_000), ("knot", 0), ("duplicates", 0)],
                         ids=lambda c: f"{c[0]}{c[1] or ''}")
@pytest.mark.parametrize("ci,ct", [(1.2, 1.0), (0.8, 1.3)])
def test_cuda_path_equals_the_reference_kernels(case, ci, ct):
    """The fused build (obvh_build_async) against the reference's kernels run
    in the reference's order on the reference's own tree."""
    import torch
    v, f = _mesh(case)
    n = f.shape[0]
    builder = bvh.ObvhBuilder()
    mesh = bvh.Mesh(v, f)
    o = builder.build(mesh, flags=3, ci=ci, ct=ct)
    torch.cuda.synchronize()
    err, slots = builder.status(n)
    assert err == 0
    g = ref.refgpu_lbvh(v, f, "nofma")
    gb, gx = ref.refgpu_obb_tree(g["nodes"], g["parents"], g["counts"], v, f, "nofma")
    gc, gcnt, gprims, gcst = ref.refgpu_collapse(g["nodes"], g["parents"], g["counts"], g["costs"], ci, ct, "nofma")
    mine = {"nodes": bvh.nodes_numpy(o["nodes"]), "parents": o["parents"].cpu().numpy().view(np.uint32),
            "counts": o["counts"].cpu().numpy().view(np.uint32)}
    _same_tree(mine, {**g, "counts": gcnt}, n)
    assert same_bits(o["obbs"].cpu().numpy(), gb)
    assert same_bits(o["transforms"].cpu().numpy(), gx)
    assert same_bits(o["costs"].cpu().numpy(), gcst)
    prims = o["primitives"].cpu().numpy().view(np.uint32)
    _same_collapse(bvh.nodes_numpy(o["collapsed"]), prims, gc, gprims)
    assert slots == sum(len(x) for x in _root_lists(gc, gprims).values())


def _frame_agreement(mine, theirs, ni):
    """Share of internal nodes whose axes agree to 1e-3 (the same candidate
    frame), and the 99.9th percentile of the axis difference among them."""
    a = mine[:ni, 3:12].astype(np.float64).reshape(-1, 3, 3)
    b = theirs[:ni, 3:12].astype(np.float64).reshape(-1, 3, 3)
    d = (np.linalg.norm(a - b, axis=2) / np.maximum(np.linalg.norm(b, axis=2), 1e-30)).max(axis=1)
    same = d <= 1e-3
    return same.mean(), float(np.quantile(d[same], 0.999))


@pytest.mark.parametrize("case", [("soup", 300_000), ("knot", 0)], ids=lambda c: f"{c[0]}{c[1] or ''}")
def test_reference_as_shipped(case):
    """The reference compiled with contraction: identical codes, topology,
    boxes, counts and collapse; costs to 1e-6; OBB frames mostly the same."""
    v, f = _mesh(case)
    n = f.shape[0]
    o = ref.lbvh_build(v, f)
    g = ref.refgpu_lbvh(v, f, "fmad")
    _same_tree(g, o, n)
    np.testing.assert_allclose(g["costs"], o["costs"], rtol=1e-6, atol=0)
    col, cnt, prims, cst, used = ref.collapse(o["nodes"], o["parents"], o["counts"], o["costs"], 1.2, 1.0)
    gc, gcnt, gprims, gcst = ref.refgpu_collapse(o["nodes"], o["parents"], o["counts"], o["costs"], 1.2, 1.0, "fmad")
    _same_collapse(gc, gprims, col, prims)
    assert np.array_equal(gcnt, cnt)
    obbs, _, _ = ref.obb_tree(o["nodes"], o["parents"], v, f)
    gb, _ = ref.refgpu_obb_tree(o["nodes"], o["parents"], o["counts"], v, f, "fmad")
    share, p999 = _frame_agreement(obbs, gb, n - 1)
    assert share >= 0.98, share
    assert p999 <= 1e-5, p999


def _lattice():
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij"), -1).reshape(-1, 3)
    c = np.repeat(g, 2, axis=0).astype(np.float32) * 0.5
    tri = np.array([[0, 0, 0], [0.2, 0, 0], [0, 0.2, 0]], np.float32)
    v = (c[:, None, :] + tri[None]).reshape(-1, 3)
    n = c.shape[0]
    f = np.zeros((n, 4), np.uint32)
    f[:, 0] = np.arange(0, 3 * n, 3)
    f[:, 1] = f[:, 0] + 1
    f[:, 2] = f[:, 0] + 2
    return v, f


@pytest.mark.skipif(not ref.refgpu_lbvh63_available(), reason="oracle/_ref ATRBVH seed library not built")
@pytest.mark.parametrize("case", [("soup", 2), ("soup", 3), ("soup", 1000), ("soup", 65_537), ("knot917k", 0),
                                  ("lattice", 0), ("duplicates", 0)], ids=lambda c: f"{c[0]}{c[1] or ''}")
def test_atrbvh_seed_kernels_equal_the_oracle(case):
    if case[0] == "knot917k":
        v, f = workloads.torus_knot_mesh()
    elif case[0] == "lattice":
        v, f = _lattice()
    else:
        v, f = _mesh(case)
    codes, order, tree = ref.refgpu_lbvh63(v, f)
    ocodes, oorder, otree = ref.lbvh63_seed(v, f)
    assert np.array_equal(codes, ocodes)
    assert np.array_equal(order, oorder)
    for mine, theirs in zip(otree, tree):
        assert np.array_equal(mine, theirs)
