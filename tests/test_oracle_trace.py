"""The oracle's SoA OBVH traversal (oracle/trace_oracle.c) finds the closest
hit a brute-force test of every triangle finds, on plain and collapsed trees
(the OBB tree is conservative, so culling never loses the nearest triangle)."""
import numpy as np
import pytest

from oracle import bvh as ref
from obvh_b200 import workloads


def _brute(v, f, rays):
    """Closest hit per ray over every triangle, kr_ray_triangle_intersect's
    float32 arithmetic step by step."""
    f = np.asarray(f)[:, :3]
    p1, p2, p3 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    e1, e2 = (p2 - p1).astype(np.float32), (p3 - p1).astype(np.float32)
    prim = np.full(len(rays), 0xFFFFFFFF, np.uint32)
    for k, r in enumerate(rays):
        d = r["direction"].astype(np.float32)
        o = r["origin"].astype(np.float32)
        s1 = np.stack([d[1] * e2[:, 2] - d[2] * e2[:, 1], d[2] * e2[:, 0] - d[0] * e2[:, 2],
                       d[0] * e2[:, 1] - d[1] * e2[:, 0]], 1)
        with np.errstate(all="ignore"):
            invd = np.float32(1.0) / (s1[:, 0] * e1[:, 0] + s1[:, 1] * e1[:, 1] + s1[:, 2] * e1[:, 2])
            dd = (o - p1).astype(np.float32)
            b1 = (dd[:, 0] * s1[:, 0] + dd[:, 1] * s1[:, 1] + dd[:, 2] * s1[:, 2]) * invd
            s2 = np.stack([dd[:, 1] * e1[:, 2] - dd[:, 2] * e1[:, 1], dd[:, 2] * e1[:, 0] - dd[:, 0] * e1[:, 2],
                           dd[:, 0] * e1[:, 1] - dd[:, 1] * e1[:, 0]], 1)
            b2 = (d[0] * s2[:, 0] + d[1] * s2[:, 1] + d[2] * s2[:, 2]) * invd
            t = (e2[:, 0] * s2[:, 0] + e2[:, 1] * s2[:, 1] + e2[:, 2] * s2[:, 2]) * invd
            ok = ~((b1 < 0) | (b1 > 1) | (b2 < 0) | (b1 + b2 > 1) | (t < 0) | (t > r["tmax"]))
        if ok.any():
            prim[k] = np.argmin(np.where(ok, t, np.inf))
    return prim


@pytest.mark.parametrize("n", [2, 17, 5000])
@pytest.mark.parametrize("collapsed", [False, True])
def test_oracle_traversal_finds_the_closest_hit(n, collapsed):
    v, f = workloads.triangle_soup(n, seed=40 + n, rmin=0.02, rmax=0.2)
    r = ref.lbvh_build(v, f)
    _, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col, _, prims, _, _ = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    tree = col if collapsed else r["nodes"]
    if tree["n_prims"][0] not in (0,):
        pytest.skip("the whole tree collapsed into its root: no internal node to traverse")
    pk, pr = ref.pack(tree, xfs)
    lt, rt, meta = ref.soa_obvh(pk, pr, n - 1)
    rays = workloads.probe_rays(1500, [0, 0, 0], [1, 1, 1], seed=n)
    hits = ref.soa_obvh_intersect(lt, rt, meta, v, f, prims if collapsed else None, rays, threads=4)
    want = _brute(v, f, rays)
    assert np.array_equal(hits["primitive"], want)
    miss = want == 0xFFFFFFFF
    assert np.all(hits["barys"][miss] == 0.5)
    assert np.array_equal(hits["normal"][miss], rays["direction"][miss])


def _quant(v, negate):
    """kr_cuda_soa_compressed_obvh's byte of a float (transforms.cu:1482-1485):
    x86 truncation to int32 (0x80000000 outside the range), then the low
    8 bits, of -(v * 127) or v * 127, in float arithmetic."""
    x = np.float32(v) * np.float32(127.0)
    q = int(np.trunc(x)) & 0xFFFFFFFF if abs(float(x)) < 2.0 ** 31 else 0x80000000
    return ((-q if negate else q) & 0xFF)


def test_compressed_packing_restatement():
    """The oracle's compressed packing on hand-made records and pairs, held to
    a separate evaluation of the reference's host loop: boxes (column 1,
    1 / column 2) and metadata words shifted through the quantised bytes,
    on top of the records' own words; leaf records copied unchanged."""
    rng = np.random.default_rng(5)
    nn, ni = 7, 3
    packed = np.zeros(nn, ref.PACKED)
    packed["meta"] = rng.integers(-2 ** 31, 2 ** 31, size=(nn, 4), dtype=np.int64).astype(np.int32)
    pairs = rng.uniform(-3, 3, size=(ni, 32)).astype(np.float32)
    pairs[0, 0] = 1e12    # out of the int32 range after scaling
    pairs[1, 17] = -0.0
    pairs[2, 3] = np.nan
    got = ref.soa_compressed_obvh(packed, pairs, ni, nn)
    for i in range(nn):
        m = packed["meta"][i].astype(np.int64) & 0xFFFFFFFF
        want = [int(m[0]), int(m[1]), int(m[2]), int(m[3])]
        if i < ni:
            for side in range(2):
                c = pairs[i, 16 * side:16 * side + 16]
                w = want[2 + side]
                for k in range(3):
                    w = ((w | _quant(c[k], True)) << 8) & 0xFFFFFFFF
                w |= _quant(c[3], False)
                want[2 + side] = w
                box = got["lbounds" if side == 0 else "rbounds"][i]
                assert np.array_equal(box[:3].view(np.uint32), c[4:7].view(np.uint32))
                inv = (np.float32(1.0) / c[8:11]).astype(np.float32)
                assert np.array_equal(box[3:].view(np.uint32), inv.view(np.uint32))
        assert [int(x) & 0xFFFFFFFF for x in got["metadata"][i]] == want, i
