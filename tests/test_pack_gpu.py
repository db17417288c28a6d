"""GPU parity of the traversal packing (include/obvh_transforms.h:
kr_cuda_bvh_persistent, kr_cuda_obvh_persistent, kr_cuda_soa_obvh and the
fused obvh_obvh_pack_async) against the oracle and against the reference's
own packing functions (oracle/_ref, built for sm_100a).

Packing moves bytes, so every output must be identical, including the fields
the reference leaves alone: the buffers are also prefilled with random bytes,
which must survive exactly where the reference does not write.
"""
import numpy as np
import pytest

from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


def _tree(n, seed, collapse=True):
    """A fused build's plain or collapsed tree with its OBB transforms, as numpy."""
    import torch
    v, f = workloads.triangle_soup(n, seed=seed)
    b = bvh.ObvhBuilder()
    o = b.build(bvh.Mesh(v, f), flags=3 if collapse else 1)
    torch.cuda.synchronize()
    assert b.status(n)[0] == 0
    nodes = bvh.nodes_numpy(o["collapsed"] if collapse else o["nodes"])
    return nodes, o["transforms"].cpu().numpy().reshape(-1, 16)


def _garbage(shape_bytes, seed):
    return np.random.default_rng(seed).integers(0, 256, size=shape_bytes, dtype=np.uint8)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()


def _host(t, dtype, shape):
    return t.cpu().numpy().view(np.uint8).view(dtype).reshape(shape)


@pytest.mark.parametrize("n,collapse", [(1, False), (2, True), (3, False), (1000, True), (65_537, True),
                                        (300_000, True), (300_000, False)])
@pytest.mark.parametrize("prefill", [False, True])
def test_obvh_persistent_and_soa_match_the_oracle(n, collapse, prefill):
    import torch
    nodes, xfs = _tree(n, 700 + n, collapse)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    pk0 = _garbage(nn * 64, 1).view(ref.PACKED) if prefill else np.zeros(nn, ref.PACKED)
    pr0 = _garbage(max(ni, 1) * 128, 2).view(np.float32).reshape(-1, 32) if prefill else \
        np.zeros((max(ni, 1), 32), np.float32)
    want_pk, want_pr = ref.pack(nodes, xfs, pk0, pr0)
    want_lt, want_rt, want_meta = ref.soa_obvh(want_pk, want_pr, ni)

    # the two synchronous entry points, in the reference's order
    o = bvh.persistent(_dev(nodes), nn, _dev(xfs), _dev(pk0), _dev(pr0).view(torch.float32))
    got_pk = _host(o["packed"], ref.PACKED, (nn,))
    got_pr = _host(o["pairs"], np.float32, (-1, 32))
    assert got_pk.tobytes() == want_pk.tobytes()
    assert got_pr.tobytes() == want_pr.tobytes()
    s = bvh.soa_obvh(o["packed"], o["pairs"], ni, nn)
    assert s["left_T"].tobytes() == want_lt.tobytes()
    assert s["right_T"].tobytes() == want_rt.tobytes()
    assert s["metadata"].tobytes() == want_meta.tobytes()

    # the fused pass
    f = bvh.obvh_pack(_dev(nodes), nn, ni, _dev(xfs), _dev(pk0), _dev(pr0).view(torch.float32))
    torch.cuda.synchronize()
    assert int(f["error"].item()) == 0
    assert _host(f["packed"], ref.PACKED, (nn,)).tobytes() == want_pk.tobytes()
    assert _host(f["pairs"], np.float32, (-1, 32)).tobytes() == want_pr.tobytes()
    assert _host(f["left_T"], np.float32, (-1, 12))[:ni].tobytes() == want_lt.tobytes()
    assert _host(f["right_T"], np.float32, (-1, 12))[:ni].tobytes() == want_rt.tobytes()
    assert _host(f["metadata"], np.int32, (-1, 4))[:nn].tobytes() == want_meta.tobytes()


@pytest.mark.parametrize("prefill", [False, True])
def test_bvh_persistent_matches_the_oracle(prefill):
    nodes, _ = _tree(100_000, 5, collapse=True)
    nn = nodes.shape[0]
    pk0 = _garbage(nn * 64, 3).view(ref.PACKED) if prefill else np.zeros(nn, ref.PACKED)
    want, _ = ref.pack(nodes, None, pk0)
    o = bvh.persistent(_dev(nodes), nn, None, _dev(pk0))
    assert _host(o["packed"], ref.PACKED, (nn,)).tobytes() == want.tobytes()
    import torch
    f = bvh.obvh_pack(_dev(nodes), nn, (nn - 1) // 2, None, _dev(pk0))
    torch.cuda.synchronize()
    assert _host(f["packed"], ref.PACKED, (nn,)).tobytes() == want.tobytes()


@pytest.mark.skipif(not ref.ref_gpu_available("nofma"), reason="oracle/_ref reference GPU libraries not built")
@pytest.mark.parametrize("n,collapse,obbs", [(2, True, True), (1000, True, True), (300_000, True, True),
                                             (300_000, False, True), (300_000, True, False)])
def test_packing_equals_the_reference_functions(n, collapse, obbs):
    """The reference's kr_cuda_(o)bvh_persistent and kr_cuda_soa_obvh on the
    same tree and the same prefilled buffers."""
    import torch
    nodes, xfs = _tree(n, 900 + n, collapse)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    pk0 = _garbage(nn * 64, 4).view(ref.PACKED)
    pr0 = _garbage(max(ni, 1) * 128, 5).view(np.float32).reshape(-1, 32)
    rpk, rpr, rlt, rrt, rmeta = ref.refgpu_pack(nodes, xfs if obbs else None, pk0, pr0)
    f = bvh.obvh_pack(_dev(nodes), nn, ni, _dev(xfs) if obbs else None, _dev(pk0), _dev(pr0).view(torch.float32))
    torch.cuda.synchronize()
    assert _host(f["packed"], ref.PACKED, (nn,)).tobytes() == rpk.tobytes()
    if obbs:
        assert _host(f["pairs"], np.float32, (-1, 32))[:ni].tobytes() == rpr[:ni].tobytes()
        assert _host(f["left_T"], np.float32, (-1, 12))[:ni].tobytes() == rlt.tobytes()
        assert _host(f["right_T"], np.float32, (-1, 12))[:ni].tobytes() == rrt.tobytes()
        assert _host(f["metadata"], np.int32, (-1, 4))[:nn].tobytes() == rmeta.tobytes()


def test_malformed_tree_is_reported():
    """A child index past the end is skipped and reported, not followed."""
    import torch
    nodes, xfs = _tree(1000, 11, collapse=False)
    bad = nodes.copy()
    bad["right"][5] = 10 ** 7
    nn = nodes.shape[0]
    with pytest.raises(bvh._native.ObvhError, match="outside the tree"):
        bvh.persistent(_dev(bad), nn, _dev(xfs))
    f = bvh.obvh_pack(_dev(bad), nn, (nn - 1) // 2, _dev(xfs))
    torch.cuda.synchronize()
    assert int(f["error"].item()) == 1


@pytest.mark.parametrize("n,collapse", [(2, True), (3, False), (1000, True), (65_537, True), (300_000, True)])
@pytest.mark.parametrize("prefill", [False, True])
def test_compressed_soa_matches_the_oracle_and_the_reference(n, collapse, prefill):
    """kr_cuda_soa_compressed_obvh on the persistent packing's records and
    pairs (prefilled records carry random metadata words, which the
    compression shifts through): byte-identical to the oracle's restatement
    and to the reference's own host loop; the stream form equals both."""
    import torch
    nodes, xfs = _tree(n, 900 + n, collapse)
    nn = nodes.shape[0]
    ni = (nn - 1) // 2
    pk0 = _garbage(nn * 64, 3).view(ref.PACKED) if prefill else np.zeros(nn, ref.PACKED)
    pr0 = np.zeros((max(ni, 1), 32), np.float32)
    pk, pr = ref.pack(nodes, xfs, pk0, pr0)
    want = ref.soa_compressed_obvh(pk, pr, ni, nn)
    got = bvh.soa_compressed_obvh_sync(_dev(pk), _dev(pr), ni, nn)
    for k in ("lbounds", "rbounds", "metadata"):
        assert got[k].tobytes() == want[k].tobytes(), k
    if ref.ref_gpu_available("nofma"):
        theirs = ref.refgpu_soa_compressed_obvh(pk, pr, ni, nn)
        for k in ("lbounds", "rbounds", "metadata"):
            assert theirs[k].tobytes() == want[k].tobytes(), k
    s = bvh.soa_compressed_obvh(_dev(pk), _dev(pr).view(torch.float32), ni, nn)
    torch.cuda.synchronize()
    assert s["lbounds"].cpu().numpy()[:ni].tobytes() == want["lbounds"].tobytes()
    assert s["rbounds"].cpu().numpy()[:ni].tobytes() == want["rbounds"].tobytes()
    assert s["metadata"].cpu().numpy()[:nn].tobytes() == want["metadata"].tobytes()
