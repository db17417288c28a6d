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
