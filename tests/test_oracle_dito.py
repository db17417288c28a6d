"""The DiTO oracle restatement, pinned against the reference's own DiTO_14."""
import numpy as np
import pytest

import oracle
from conftest import golden_dito, obb_contains, same_bits
from obvh_b200 import workloads


def test_oracle_matches_golden_fixtures():
    """Bit-exact against outputs of the reference's DiTO_14 + kr_points_obb clamp."""
    for name, pts, box in golden_dito():
        out, _, _ = oracle.dito14(pts)
        assert np.array_equal(out.view(np.uint32), box.view(np.uint32)), name


def test_golden_fixtures_reach_every_path():
    kinds = {oracle.dito14(p)[2] for _, p, _ in golden_dito()}
    assert kinds == {0, 1, 2, 3, 4}


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU DiTO not built here")
@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_reference_random(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(1, 5000))
    p = rng.normal(size=(n, 3)).astype(np.float32) * rng.uniform(0.01, 20, size=3).astype(np.float32)
    if seed % 5 == 0:
        p = np.round(p)
    out, _, _ = oracle.dito14(p)
    ref = oracle.ref_dito14(p)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("seed", range(3))
def test_oracle_box_contains_points(seed):
    p = workloads.ellipsoid_points(20000, seed=seed)
    out, _, kind = oracle.dito14(p)
    assert kind in (3, 4)
    assert obb_contains(p, out) == 0
    # the reference GPU semantics give a box containing the points too
    outg, _, _ = oracle.dito14(p, oracle.DITO_GPU)
    assert obb_contains(p, outg) == 0


def test_oracle_extremal_first_index_ties():
    p = np.float32([[1, 0, 0], [0, 0, 0], [1, 0, 0], [0, 0, 0]])
    mn, mx, amn, amx = oracle.extremal7(p)
    assert amn[0] == 1 and amx[0] == 0   # first point reaching x min / x max
    assert same_bits(mn[:3], [0, 0, 0])
