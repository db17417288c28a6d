"""The SAH cost (include/obvh_transforms.h: kr_bvh_sah, obvh_bvh_sah_async).

* kr_bvh_sah (host arrays, as in the reference) must return the reference's
  own kr_bvh_sah result bit for bit (oracle/_ref holds the reference's
  function, compiled from its sources).
* obvh_bvh_sah_async sums the same float terms on the device in double: it
  must equal the exact sum of the oracle's terms (oracle.bvh.sah_terms) to
  1e-12 relative, and the reference's sequential float sum to that sum's
  drift (0.23% at 2M triangles; bounded here by 0.5%).
"""
import math

import numpy as np
import pytest

from oracle import bvh as ref
from obvh_b200 import bvh, workloads

pytestmark = pytest.mark.gpu


def _tree(n, seed, collapse):
    import torch
    v, f = workloads.triangle_soup(n, seed=seed)
    b = bvh.ObvhBuilder()
    o = b.build(bvh.Mesh(v, f), flags=3 if collapse else 1)
    torch.cuda.synchronize()
    assert b.status(n)[0] == 0
    return o


@pytest.mark.parametrize("n", [3, 1000, 300_000, 2_000_000])
@pytest.mark.parametrize("collapse", [False, True])
@pytest.mark.parametrize("with_obbs", [False, True])
def test_sah_device_and_host(n, collapse, with_obbs):
    import torch
    o = _tree(n, 60 + n, collapse)
    nodes_t = o["collapsed"] if collapse else o["nodes"]
    obbs_t = o["obbs"] if with_obbs else None
    got = bvh.bvh_sah(nodes_t, o["parents"], obbs_t).cpu().numpy()
    torch.cuda.synchronize()
    nodes = bvh.nodes_numpy(nodes_t)
    parents = o["parents"].cpu().numpy().view(np.uint32)
    obbs = None if obbs_t is None else obbs_t.cpu().numpy().reshape(-1, 15)
    terms, root_area = ref.sah_terms(nodes, parents, obbs)
    exact = math.fsum(terms.astype(np.float64))
    assert got[0] == pytest.approx(exact, rel=1e-12)
    assert got[1] == pytest.approx(exact / root_area, rel=1e-12)
    host = bvh.bvh_sah_host(nodes, obbs=obbs)
    if ref.ref_gpu_available("nofma"):
        assert host == ref.ref_bvh_sah(nodes, obbs=obbs)
    assert host == pytest.approx(got[1], rel=5e-3)
