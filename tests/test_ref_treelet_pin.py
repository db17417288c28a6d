"""The ATRBVH treelet restatement pinned to the reference's own kernel.

oracle/_ref/libref_treelet_emu.so runs the reference's
agglomerativeSmallTreeletKernel (AgglomerativeTreelet.cu:14-222,405-570,
Treelet.cuh:21-129) as host code, one lockstep-emulated warp at a time, under
the reference's own optimisation loop and schedule
(AgglomerativeTreeletOptimizer.cpp:73-98, AgglomerativeScheduler.cpp:43-82).
From the same seed tree it must produce the SoA tree of the restatement in
oracle/atrbvh_oracle.c bit for bit (zero signs aside): parents, children,
leaf data, boxes and areas.  The GPU path is held to the same emulated
reference in tests/test_atrbvh_gpu.py.
"""
import numpy as np
import pytest

from conftest import lattice_mesh, same_bits
from oracle import bvh as ref
from obvh_b200 import workloads

pytestmark = pytest.mark.skipif(not ref.ref_treelet_available(),
                                reason="oracle/_ref/libref_treelet_emu.so not built (no reference tree)")


def _same_tree(a, b):
    for k in ref.SOA_FIELDS:
        if a[k].dtype.kind == "f":
            assert same_bits(a[k], b[k]), k
        else:
            assert np.array_equal(a[k], b[k]), k


def _pin(v, f, tau, iters=2, ci=1.2, ct=1.0):
    seed = ref.atrbvh_seed(v, f)
    want = ref.ref_treelet_optimize(seed, tau, iters, ci, ct)
    got, _ = ref.atrbvh_optimize(seed, tau, iters, ci, ct)
    _same_tree(got, want)
    return seed, want


@pytest.mark.parametrize("n", [2, 3, 4, 9, 17, 31, 32, 33, 64, 65, 129, 1000, 5000])
@pytest.mark.parametrize("tau", [7, 9])
def test_soup(n, tau):
    v, f = workloads.triangle_soup(n, seed=1300 + n)
    seed, want = _pin(v, f, tau)
    if n >= 1000:  # the optimiser rewrites the tree: the pin is not vacuous
        assert not np.array_equal(seed["left"], want["left"])


@pytest.mark.parametrize("tau", [3, 4, 5, 6, 8, 12, 16, 20])
@pytest.mark.parametrize("iters", [1, 3])
def test_treelet_sizes_and_iterations(tau, iters):
    v, f = workloads.triangle_soup(2000, seed=77)
    _pin(v, f, tau, iters)


def test_other_costs():
    v, f = workloads.triangle_soup(3000, seed=78)
    _pin(v, f, 7, 2, ci=2.0, ct=0.5)


@pytest.mark.parametrize("tau", [7, 9])
def test_lattice_ties(tau):
    v, f = lattice_mesh(12)
    _pin(v, f, tau)


@pytest.mark.parametrize("segments,around,tau", [(64, 28, 7), (64, 28, 9), (128, 56, 7)])
def test_reduced_knot(segments, around, tau):
    v, f = workloads.torus_knot_mesh(segments, around, seed=2)
    _pin(v, f, tau)


def test_no_iterations_leaves_the_seed():
    v, f = workloads.triangle_soup(500, seed=79)
    seed = ref.atrbvh_seed(v, f)
    _same_tree(ref.ref_treelet_optimize(seed, 7, 0), {k: seed[k] for k in ref.SOA_FIELDS})
