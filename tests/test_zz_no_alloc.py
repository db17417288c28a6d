"""The allocation-free DiTO entry point (obvh_points_obb_noalloc).

It exists for callers that may not allocate device memory when they fit a box;
its scratch lives in static device arrays shared by all calls.  Checked through
the C ABI against the regular entry point (obvh_points_obb), bit for bit as
every DiTO test here, on two calls in a row: the second call must not see
anything the first one left in the shared arrays.  This file is collected last
so that a failure here cannot stop the other GPU tests from running.
"""
import ctypes

import numpy as np
import pytest

from conftest import same_bits
from obvh_b200 import _native, points_obb, workloads

pytestmark = pytest.mark.gpu

MAX_POINTS = 1 << 20


def _noalloc(pts, flags=0):
    lib = _native.lib()
    p = np.ascontiguousarray(pts, dtype=np.float32)
    out = np.zeros(15, np.float32)
    e = lib.obvh_points_obb_noalloc(p.ctypes.data if p.size else None, p.shape[0], flags, out.ctypes.data, None)
    _native.check(e)
    return out


def test_noalloc_matches_regular_entry_point_twice():
    big = workloads.ellipsoid_points(MAX_POINTS, seed=11)        # the largest allowed input
    small = workloads.ellipsoid_points(3_001, seed=12)[1:]      # smaller, misaligned start
    for pts in (big, small):
        want = points_obb(pts)
        got = _noalloc(pts)
        assert same_bits(got, want), (got, want)


def test_noalloc_rejects_more_than_the_maximum():
    pts = np.zeros((MAX_POINTS + 1, 3), np.float32)
    with pytest.raises(_native.ObvhError, match="maximum"):
        _noalloc(pts)
