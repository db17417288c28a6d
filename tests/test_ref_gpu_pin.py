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
  63-bit codes, order and Karras tree exactly.  Its node-box kernel and the
  treelet kernel are not run on the GPU (barriers in divergent loops); the
  treelet kernel runs as host code instead (tests/test_ref_treelet_pin.py,
  tests/test_atrbvh_gpu.py).
* "fmad" is the reference as its own build compiles it: nvcc's default
  contraction of multiplies and adds.  Codes, order, topology, counts, boxes
  and collapse decisions must still be identical and costs within 1e-6
  relative.  OBBs: contraction moves near-ties in the candidate score, so a
  small share of internal nodes picks another frame; the rest agree in their
  axes to about 1e-6 and in surface area to rounding (a few 1e-5).
* Speed: each phase of the reference's kernels, timed on the device against
  the fused chain here on the same 2M-triangle soup.
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


def _obb_surface_area(obbs):
    """FP64 surface area of each box: half-extents times the axis lengths
    (a leaf's third axis is the unnormalised normal)."""
    o = np.asarray(obbs, np.float64)
    e = o[:, 12:15] * np.linalg.norm(o[:, 3:12].reshape(-1, 3, 3), axis=2)
    return 8.0 * (e[:, 0] * e[:, 1] + e[:, 0] * e[:, 2] + e[:, 1] * e[:, 2])


def _ms(fn, reps=5):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_tree_speed_against_the_reference_kernels(capsys):
    """Device time of each phase on the 2M-triangle soup, device-resident
    inputs: the reference's kernels (built as shipped and uncontracted) against
    the fused chain here, timed through its flags (LBVH only; + OBB tree;
    + collapse).  The reference's summary and scene-box kernels are not run,
    so its totals leave them out; the chain here includes its equivalents."""
    import torch
    v, f = workloads.triangle_soup(2_000_000, seed=1)
    theirs = {var: ref.refgpu_tree_ms(v, f, 5, var) for var in ("fmad", "nofma")}
    builder = bvh.ObvhBuilder()
    mesh = bvh.Mesh(v, f)
    out = builder.outputs(f.shape[0])
    t = {flags: _ms(lambda: builder.build(mesh, flags=flags, out=out)) for flags in (0, 1, 3)}
    assert builder.status(f.shape[0])[0] == 0
    ours = {"lbvh": t[0], "obb tree": t[1] - t[0], "collapse": t[3] - t[1], "total": t[3]}
    groups = {"lbvh": ("morton", "sort", "tree", "aabb"), "obb tree": ("candidate", "refit", "finalize"),
              "collapse": ("collapse",)}
    with capsys.disabled():
        print("\nphase      reference as shipped (uncontracted)   this build    [2M-triangle soup, ms]")
        for k, v_ in theirs["fmad"].items():
            print(f"  {k:10s} {v_:9.3f} ({theirs['nofma'][k]:7.3f})")
        for g, keys in groups.items():
            r = sum(theirs["fmad"][k] for k in keys)
            print(f"{g:10s}   {r:9.3f} ({sum(theirs['nofma'][k] for k in keys):7.3f})              {ours[g]:8.3f}")
        total = sum(theirs["fmad"].values())
        print(f"{'total':10s}   {total:9.3f} ({sum(theirs['nofma'].values()):7.3f})              {ours['total']:8.3f}")
    assert ours["total"] < total


@pytest.mark.parametrize("case", [("soup", 300_000), ("knot", 0)], ids=lambda c: f"{c[0]}{c[1] or ''}")
def test_surface_area_against_the_reference_as_shipped(case, capsys):
    """OBB surface areas (FP64, extents times axis lengths) of the CUDA path
    against the reference built as it ships (with contraction), node by node,
    split into the nodes whose candidate frame agrees and those where
    contraction moved a near-tie to another frame.  The CUDA path equals the
    reference built without contraction bit for bit (the tests above), so
    these figures are the reference's own spread between its two builds:
    rounding of fused multiply-adds, largest at leaves, whose third axis is
    the unnormalised normal.  Prints the counts outside 1e-5 relative."""
    import torch
    v, f = _mesh(case)
    n = f.shape[0]
    builder = bvh.ObvhBuilder()
    o = builder.build(bvh.Mesh(v, f), flags=1)
    torch.cuda.synchronize()
    assert builder.status(n)[0] == 0
    mine = o["obbs"].cpu().numpy()
    g = ref.refgpu_lbvh(v, f, "fmad")
    theirs, _ = ref.refgpu_obb_tree(g["nodes"], g["parents"], g["counts"], v, f, "fmad")
    sa_m, sa_t = _obb_surface_area(mine), _obb_surface_area(theirs)
    rel = np.abs(sa_m - sa_t) / np.maximum(sa_t, 1e-300)
    a = mine[:, 3:12].astype(np.float64).reshape(-1, 3, 3)
    b = theirs[:, 3:12].astype(np.float64).reshape(-1, 3, 3)
    d = (np.linalg.norm(a - b, axis=2) / np.maximum(np.linalg.norm(b, axis=2), 1e-30)).max(axis=1)
    same = d <= 1e-3
    internal = np.arange(2 * n - 1) < n - 1
    rows = {}
    for name, m in (("internal, same frame", internal & same), ("internal, other frame", internal & ~same),
                    ("leaves, same frame", ~internal & same), ("leaves, other frame", ~internal & ~same)):
        k = int(m.sum())
        rows[name] = (k, int((rel[m] > 1e-5).sum()), float(np.quantile(rel[m], 0.999)) if k else 0.0,
                      float(rel[m].max()) if k else 0.0)
    with capsys.disabled():
        print(f"\nOBB surface area vs the reference as shipped, {case[0]} {n} triangles "
              "(nodes, > 1e-5 rel, p99.9 rel, max rel):")
        for name, r in rows.items():
            print(f"  {name:22s} {r[0]:8d} {r[1]:8d} {r[2]:.2e} {r[3]:.2e}")
    # same frame: rounding-level differences only; another frame: a small share
    assert rows["internal, same frame"][3] <= 2e-4
    assert rows["leaves, same frame"][3] <= 2e-3
    assert rows["internal, other frame"][0] <= 0.02 * (n - 1)
    assert rows["leaves, other frame"][0] <= 1e-3 * n
