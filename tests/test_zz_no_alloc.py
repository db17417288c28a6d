"""The allocation-free DiTO entry point (obvh_points_obb_noalloc).

It exists for callers that may not allocate device memory when they fit a
box: a plugin whose host application owns every byte of GPU memory, or a
service that reserves its whole budget at start-up and forbids allocations
afterwards.  Its scratch lives in static device arrays that all calls share.

Checked through the C ABI against the regular entry point (obvh_points_obb)
on two calls in a row (the second call must not see anything the first one
left in the shared arrays), and against the oracle and the golden cases,
bit for bit like every DiTO test here.  This file is collected last so that
a failure here cannot stop the other GPU tests from running.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_dito, same_bits
from obvh_b200 import REFERENCE_GPU, _native, points_obb, workloads

pytestmark = pytest.mark.gpu

MAX_POINTS = 1 << 20


def _noalloc(pts, flags=0):
    lib = _native.lib()
    p = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(15, np.float32)
    e = lib.obvh_points_obb_noalloc(p.ctypes.data if p.size else None, p.shape[0], flags, out.ctypes.data, None)
    _native.check(e)
    return out


def test_noalloc_matches_regular_entry_point_twice():
    big = workloads.ellipsoid_points(MAX_POINTS, seed=11)   # the largest allowed input
    small = workloads.ellipsoid_points(3_001, seed=12)[1:]  # smaller than the first call's input
    for pts in (big, small):
        want = points_obb(pts)
        got = _noalloc(pts)
        assert same_bits(got, want), (got, want)


def test_noalloc_matches_the_oracle_and_the_golden_cases():
    for name, pts, box in golden_dito():
        assert same_bits(_noalloc(pts), box), name
        want, _, _ = oracle.dito14(pts, oracle.DITO_GPU)
        assert same_bits(_noalloc(pts, REFERENCE_GPU), want), name
    pts = workloads.ellipsoid_points(200_000, seed=13)
    want, _, _ = oracle.dito14(pts)
    assert same_bits(_noalloc(pts), want)


def test_noalloc_empty_input():
    want, _, _ = oracle.dito14(np.zeros((0, 3), np.float32))
    assert same_bits(_noalloc(np.zeros((0, 3), np.float32)), want)


def test_noalloc_reports_bad_input_then_recovers():
    # Non-finite points leave no finite projection: the kernel records a
    # status word (it does not fault) and the call returns an error.  The
    # next call must start from a clean control block.
    bad = np.full((1000, 3), np.nan, np.float32)
    with pytest.raises(_native.ObvhError, match="invalid input"):
        _noalloc(bad)
    pts = workloads.ellipsoid_points(50_000, seed=14)
    assert same_bits(_noalloc(pts), points_obb(pts))


def test_noalloc_rejects_more_than_the_maximum():
    pts = np.zeros((MAX_POINTS + 1, 3), np.float32)
    with pytest.raises(_native.ObvhError, match="maximum"):
        _noalloc(pts)
