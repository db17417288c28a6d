"""GPU parity of the SoA OBVH traversal (include/obvh_transforms.h:
kr_cuda_soa_obvh_intersect, obvh_soa_obvh_intersect_async) against the oracle
(oracle/trace_oracle.c) and the reference's own traversal kernel (oracle/_ref,
built for sm_100a).

Each ray follows the reference's sequence of node and triangle tests, so
the intersection records (normal, barycentrics, primitive) must be
bit-identical to the oracle's and to the --fmad=false reference build's.
"""
import numpy as np
import pytest

from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


def _scene(kind, n, collapse, seed=1):
    """Mesh, fused build and SoA OBVH on the device."""
    import torch
    if kind == "soup":
        v, f = workloads.triangle_soup(n, seed=seed)
    else:
        v, f = workloads.torus_knot_mesh(segments=256, around=112)
    mesh = bvh.Mesh(v, f)
    nf = mesh.n_faces
    b = bvh.ObvhBuilder()
    o = b.build(mesh, flags=3 if collapse else 1)
    torch.cuda.synchronize()
    assert b.status(nf)[0] == 0
    nodes = o["collapsed"] if collapse else o["nodes"]
    nn, ni = 2 * nf - 1, nf - 1
    s = bvh.obvh_pack(nodes, nn, ni, o["transforms"])
    torch.cuda.synchronize()
    assert int(s["error"].item()) == 0
    prims = o["primitives"] if collapse else None
    return v, f, mesh, s, prims, nn, ni


def _soa_numpy(s, ni):
    return (s["left_T"].cpu().numpy().reshape(-1, 12)[:ni], s["right_T"].cpu().numpy().reshape(-1, 12)[:ni],
            s["metadata"].cpu().numpy().reshape(-1, 4))


def _rays(n, seed):
    return workloads.probe_rays(n, [0, 0, 0], [1, 1, 1], seed=seed)


def _dev_rays(rays):
    import torch
    return torch.from_numpy(rays.view(np.uint8).copy()).cuda()


def _isects(t, n):
    return t.cpu().numpy()[:28 * n].view(ref.ISECT)


@pytest.mark.parametrize("kind,n,collapse", [("soup", 1000, True), ("soup", 65_537, True), ("soup", 300_000, True),
                                             ("soup", 300_000, False), ("knot", 0, True)])
def test_traversal_matches_the_oracle(kind, n, collapse):
    import torch
    v, f, mesh, s, prims, nn, ni = _scene(kind, n, collapse)
    rays = _rays(40_000, seed=n + 3)
    got, err = bvh.soa_obvh_intersect(s, mesh, prims, _dev_rays(rays), nn, ni)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    lt, rt, meta = _soa_numpy(s, ni)
    want = ref.soa_obvh_intersect(lt, rt, meta, v, f, None if prims is None else prims.cpu().numpy().view(np.uint32),
                                  rays, threads=8)
    g = _isects(got, len(rays))
    assert np.array_equal(g["primitive"], want["primitive"])
    assert g.tobytes() == want.tobytes()
    assert (g["primitive"] != 0xFFFFFFFF).sum() > 0


def test_reference_entry_point_through_the_device_struct():
    """kr_cuda_obvh_persistent -> kr_cuda_soa_obvh -> kr_cuda_soa_obvh_intersect,
    the reference's own call sequence, against the stream form."""
    import ctypes
    import torch
    from obvh_b200 import _native
    v, f, mesh, s, prims, nn, ni = _scene("soup", 200_000, True, seed=8)
    lib = _native.lib()
    d_soa = ctypes.c_void_p(0)
    _native.check(lib.kr_cuda_soa_obvh(ctypes.c_void_p(s["packed"].data_ptr()), ctypes.c_void_p(s["pairs"].data_ptr()),
                                       ctypes.byref(d_soa), ni, nn))
    try:
        rays = _rays(20_000, seed=5)
        d_rays = _dev_rays(rays)
        out = torch.zeros(28 * len(rays), dtype=torch.uint8, device="cuda")
        counter = torch.zeros(1, dtype=torch.int32, device="cuda")
        _native.check(lib.kr_cuda_soa_obvh_intersect(d_soa, ctypes.c_void_p(mesh.verts.data_ptr()),
                                                     ctypes.c_void_p(mesh.faces.data_ptr()),
                                                     ctypes.c_void_p(prims.data_ptr()),
                                                     ctypes.c_void_p(d_rays.data_ptr()),
                                                     ctypes.c_void_p(out.data_ptr()), len(rays), 128, 0,
                                                     ctypes.c_void_p(counter.data_ptr())))
        want, err = bvh.soa_obvh_intersect(s, mesh, prims, d_rays, nn, ni)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert out.cpu().numpy().tobytes() == want.cpu().numpy()[:28 * len(rays)].tobytes()
    finally:
        _native.check(lib.obvh_soa_obvh_free(d_soa))


@pytest.mark.skipif(not (ref.ref_gpu_available("nofma") and ref.ref_gpu_available("fmad")),
                    reason="oracle/_ref reference GPU libraries not built")
@pytest.mark.parametrize("kind,n,collapse", [("soup", 300_000, True), ("soup", 300_000, False), ("knot", 0, True)])
def test_traversal_equals_the_reference_kernel(kind, n, collapse):
    """The reference's soa_obvh_persistent_intersect on the same SoA OBVH and
    rays: identical records from its --fmad=false build; from its contracted
    build, the same primitive for all but a few rays."""
    import torch
    v, f, mesh, s, prims, nn, ni = _scene(kind, n, collapse, seed=4)
    rays = _rays(40_000, seed=11)
    got, err = bvh.soa_obvh_intersect(s, mesh, prims, _dev_rays(rays), nn, ni)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    g = _isects(got, len(rays))
    lt, rt, meta = _soa_numpy(s, ni)
    p = None if prims is None else prims.cpu().numpy().view(np.uint32)
    r = ref.refgpu_soa_obvh_intersect(lt, rt, meta, v, f, p, rays, "nofma")
    assert g.tobytes() == r.tobytes()
    r2 = ref.refgpu_soa_obvh_intersect(lt, rt, meta, v, f, p, rays, "fmad")
    assert (r2["primitive"] == g["primitive"]).mean() >= 0.999


def test_bad_index_is_reported():
    """A child index past the tree stops the rays that meet it, with an error."""
    import torch
    v, f, mesh, s, prims, nn, ni = _scene("soup", 5000, False, seed=2)
    meta = s["metadata"].view(torch.int32).reshape(-1, 4)
    meta[0, 0] = ni + 10   # an internal index past the internal nodes
    rays = _rays(2000, seed=1)
    _, err = bvh.soa_obvh_intersect(s, mesh, prims, _dev_rays(rays), nn, ni)
    torch.cuda.synchronize()
    assert int(err.item()) & 1


@pytest.mark.skipif(not ref.ref_gpu_available("nofma"), reason="oracle/_ref reference GPU libraries not built")
def test_traversal_speed_against_the_reference_kernel(capsys):
    """Both kernels on the same device-resident SoA OBVH and 1M rays (CUDA
    events, mean of 5 launches after one warm-up): the traversal is at least
    as fast as the reference's own kernel built as it ships."""
    import torch
    v, f, mesh, s, prims, nn, ni = _scene("soup", 2_000_000, True, seed=1)
    rays = _rays(1_000_000, seed=21)
    d_rays = _dev_rays(rays)
    bvh.soa_obvh_intersect(s, mesh, prims, d_rays, nn, ni)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        out, err = bvh.soa_obvh_intersect(s, mesh, prims, d_rays, nn, ni)
    e1.record()
    torch.cuda.synchronize()
    ours = e0.elapsed_time(e1) / 5
    lt, rt, meta = _soa_numpy(s, ni)
    p = prims.cpu().numpy().view(np.uint32)
    theirs = {var: ref.refgpu_soa_obvh_intersect_ms(lt, rt, meta, v, f, p, rays, 5, var) for var in ("nofma", "fmad")}
    with capsys.disabled():
        print(f"\ntraversal of 1M rays, 2M-triangle collapsed tree: ours {ours:.3f} ms, reference kernel "
              f"{theirs['fmad']:.3f} ms as shipped, {theirs['nofma']:.3f} ms uncontracted")
    assert ours <= theirs["fmad"] * 1.05


def _compressed(s, ni, nn, pairs=None):
    """The compressed SoA OBVH of a scene's packed records and pairs (or of
    the given pairs), on the device."""
    import torch
    p = s["pairs"] if pairs is None else torch.from_numpy(np.ascontiguousarray(pairs, np.float32)).cuda()
    c = bvh.soa_compressed_obvh(s["packed"], p, ni, nn)
    torch.cuda.synchronize()
    return c


def _obb_pairs(kind, n, collapse, seed):
    """A scene with its compressed SoA OBVH built from axis-angle pairs of the
    tree's own boxes (oracle.bvh.compressed_pairs)."""
    import torch
    v, f, mesh, s, prims, nn, ni = _scene(kind, n, collapse, seed=seed)
    b = bvh.ObvhBuilder()
    o = b.build(mesh, flags=3 if collapse else 1)
    torch.cuda.synchronize()
    nodes = bvh.nodes_numpy(o["collapsed"] if collapse else o["nodes"])
    pairs = ref.compressed_pairs(nodes, o["obbs"].cpu().numpy())
    return v, f, mesh, s, prims, nn, ni, pairs


@pytest.mark.skipif(not (ref.ref_gpu_available("nofma") and ref.ref_gpu_available("fmad")),
                    reason="oracle/_ref reference GPU libraries not built")
@pytest.mark.parametrize("kind,n,collapse", [("soup", 300_000, True), ("soup", 300_000, False), ("knot", 0, True)])
def test_compressed_traversal_equals_the_reference_kernel(kind, n, collapse, capsys):
    """The reference's soa_obvh_compressed_persistent_intersect on the same
    compressed SoA OBVH and rays: identical records from its --fmad=false
    build; from its contracted build, the same primitive for nearly all rays.
    (The quantised frames do not bound the geometry, so the hits are the
    reference's, not the exact closest hits.)"""
    import torch
    v, f, mesh, s, prims, nn, ni, pairs = _obb_pairs(kind, n, collapse, seed=4)
    c = _compressed(s, ni, nn, pairs)
    rays = _rays(40_000, seed=13)
    got, err = bvh.soa_compressed_obvh_intersect(c, mesh, prims, _dev_rays(rays), nn, ni)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    g = _isects(got, len(rays))
    lb, rb = c["lbounds"].cpu().numpy()[:ni], c["rbounds"].cpu().numpy()[:ni]
    meta = c["metadata"].cpu().numpy()[:nn]
    p = None if prims is None else prims.cpu().numpy().view(np.uint32)
    r = ref.refgpu_compressed_intersect(lb, rb, meta, v, f, p, rays, "nofma")
    assert g.tobytes() == r.tobytes()
    r2 = ref.refgpu_compressed_intersect(lb, rb, meta, v, f, p, rays, "fmad")
    assert (r2["primitive"] == g["primitive"]).mean() >= 0.99
    hit = (g["primitive"] != 0xFFFFFFFF).mean()
    exact, err = bvh.soa_obvh_intersect(s, mesh, prims, _dev_rays(rays), nn, ni)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    e = _isects(exact, len(rays))
    exact_hit = (e["primitive"] != 0xFFFFFFFF).mean()
    with capsys.disabled():
        print(f"\ncompressed traversal, {kind} {n or ''}: {hit:.3f} of rays hit ({exact_hit:.3f} through the OBVH)")
    # the quantised boxes approximate the tree's boxes: most rays that hit
    # through the exact OBVH still find a triangle, and a hit is a real one
    assert hit >= 0.5 * exact_hit
    both = (g["primitive"] != 0xFFFFFFFF) & (e["primitive"] != 0xFFFFFFFF)
    assert (g["primitive"][both] == e["primitive"][both]).mean() >= 0.5


def test_compressed_reference_entry_points_through_the_device_struct():
    """kr_cuda_soa_compressed_obvh -> kr_cuda_obvh_compressed_persistent_intersect,
    the reference's call sequence for the compressed form, against the
    stream forms."""
    import ctypes
    import torch
    from obvh_b200 import _native
    v, f, mesh, s, prims, nn, ni, pairs = _obb_pairs("soup", 200_000, True, seed=8)
    d_pairs = torch.from_numpy(pairs).cuda()
    lib = _native.lib()
    d_soa = ctypes.c_void_p(0)
    _native.check(lib.kr_cuda_soa_compressed_obvh(ctypes.c_void_p(s["packed"].data_ptr()),
                                                  ctypes.c_void_p(d_pairs.data_ptr()), ctypes.byref(d_soa), ni,
                                                  nn))
    try:
        rays = _rays(20_000, seed=5)
        d_rays = _dev_rays(rays)
        out = torch.zeros(28 * len(rays), dtype=torch.uint8, device="cuda")
        counter = torch.zeros(1, dtype=torch.int32, device="cuda")
        _native.check(lib.kr_cuda_obvh_compressed_persistent_intersect(
            d_soa, ctypes.c_void_p(mesh.verts.data_ptr()), ctypes.c_void_p(mesh.faces.data_ptr()),
            ctypes.c_void_p(prims.data_ptr()), ctypes.c_void_p(d_rays.data_ptr()), ctypes.c_void_p(out.data_ptr()),
            len(rays), 128, 0, ctypes.c_void_p(counter.data_ptr())))
        want, err = bvh.soa_compressed_obvh_intersect(_compressed(s, ni, nn, pairs), mesh, prims, d_rays, nn, ni)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert out.cpu().numpy().tobytes() == want.cpu().numpy()[:28 * len(rays)].tobytes()
    finally:
        _native.check(lib.obvh_soa_obvh_compressed_free(d_soa))
