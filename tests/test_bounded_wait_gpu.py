"""The library's spins are bounded: a wait on a flag that nothing sets gives
up after its limit, reports the timeout in the device error word, and leaves
the context usable (a fit right after still matches the oracle)."""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import same_bits
from obvh_b200 import _native, dito, workloads

pytestmark = pytest.mark.gpu


def test_wait_on_an_unset_flag_times_out_and_reports_it():
    lib = _native.lib()
    err = ctypes.c_uint32(0)
    _native.check(lib.obvh_check_bounded_wait(20_000, ctypes.byref(err)))  # 20 ms
    assert err.value == 1  # kErrWaitTimeout
    pts = workloads.ellipsoid_points(10_000, seed=3)
    assert same_bits(dito.points_obb(pts), oracle.dito14(pts)[0])


def test_limit_is_capped():
    lib = _native.lib()
    err = ctypes.c_uint32(0)
    with pytest.raises(_native.ObvhError):
        _native.check(lib.obvh_check_bounded_wait(5_000_000, ctypes.byref(err)))
