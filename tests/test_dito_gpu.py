"""GPU parity of the DiTO-14 fit against the oracle, through the C ABI.

The fit is required to be bit-identical to the reference's CPU DiTO_14 plus
the kr_points_obb clamp (zero signs aside): both evaluate the same
uncontracted float32 operations and keep the first point on ties.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_dito, obb_contains, same_bits
from obvh_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def fitter(torch):
    from obvh_b200 import DitoFitter
    return DitoFitter()


def _device_fit(torch, fitter, pts, flags=0, pad=0):
    """Fits pts placed `pad` points into a device buffer (pad 1..3 misaligns it)."""
    buf = torch.zeros((len(pts) + pad + 1, 3), dtype=torch.float32, device="cuda")
    if len(pts):
        buf[pad:pad + len(pts)] = torch.from_numpy(pts).cuda()
    view = buf[pad:pad + len(pts)]
    out = fitter.fit(view, flags=flags)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_golden_through_reference_entry_point():
    from obvh_b200 import kr_cuda_points_obb
    for name, pts, box in golden_dito():
        out, ms = kr_cuda_points_obb(pts)
        assert same_bits(out, box), (name, out, box)
        assert ms >= 0


def test_golden_through_device_entry_point(torch, fitter):
    for name, pts, box in golden_dito():
        for pad in (0, 1, 2, 3):
            out = _device_fit(torch, fitter, pts, pad=pad)
            assert same_bits(out, box), (name, pad, out, box)


def test_reference_gpu_semantics(torch, fitter):
    from obvh_b200 import REFERENCE_GPU
    for name, pts, _ in golden_dito():
        want, _, _ = oracle.dito14(pts, oracle.DITO_GPU)
        out = _device_fit(torch, fitter, pts, flags=REFERENCE_GPU)
        assert same_bits(out, want), (name, out, want)


@pytest.mark.parametrize("n", [15, 100, 2047, 2048, 2049, 8191, 24577, 100003, 1 << 20])
def test_sizes_around_tile_boundaries(torch, fitter, n):
    rng = np.random.default_rng(n)
    pts = (rng.normal(size=(n, 3)) * rng.uniform(0.1, 10, size=3)).astype(np.float32)
    want, axes, kind = oracle.dito14(pts)
    for pad in (0, 3):
        out = _device_fit(torch, fitter, pts, pad=pad)
        assert same_bits(out, want), (n, pad)
    path, got_axes, err = fitter.report()
    assert err == 0 and path == kind
    assert obb_contains(pts, out) == 0


def test_first_index_ties_on_lattice(torch, fitter):
    """Millions of ties: the argmin/argmax must pick the first point like the CPU scan."""
    rng = np.random.default_rng(7)
    pts = rng.integers(-10, 11, size=(3_000_000, 3)).astype(np.float32)
    pts = pts @ np.float32([[0.8, 0.6, 0], [-0.6, 0.8, 0], [0, 0, 1]])
    pts = pts.astype(np.float32)
    mn, mx, amn, amx = oracle.extremal7(pts)
    want, _, _ = oracle.dito14(pts)
    out = _device_fit(torch, fitter, pts)
    assert same_bits(out, want)


def test_many_fits_reuse_workspace(torch, fitter):
    rng = np.random.default_rng(3)
    for i in range(30):
        n = int(rng.integers(0, 300000))
        pts = workloads.ellipsoid_points(n, seed=i) if n else np.zeros((0, 3), np.float32)
        want, _, _ = oracle.dito14(pts)
        out = _device_fit(torch, fitter, pts, pad=i % 4)
        assert same_bits(out, want), (i, n)


def test_ellipsoid_config_full_size(torch, fitter):
    """The plain-fit workload: 100,000 points (seeds 0..9) and the 100M roofline size."""
    from obvh_b200 import points_obb
    for seed in range(10):
        pts = workloads.ellipsoid_points(100_000, seed=seed)
        want = oracle.ref_dito14(pts) if oracle.ref_available() else oracle.dito14(pts)[0]
        assert same_bits(points_obb(pts), want)
    dev = workloads.ellipsoid_points_torch(100_000_000, seed=0)
    pts = dev.cpu().numpy()
    want, _, _ = oracle.dito14(pts)
    out = fitter.fit(dev).cpu().numpy()
    assert same_bits(out, want)
    assert obb_contains(pts[::97], out) == 0


def test_empty_and_tiny_inputs(torch, fitter):
    for n in range(0, 20):
        pts = np.arange(3 * n, dtype=np.float32).reshape(n, 3) ** 1.5
        want, _, _ = oracle.dito14(pts)
        assert same_bits(_device_fit(torch, fitter, pts), want), n
