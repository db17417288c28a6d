"""GPU parity of the batched DiTO-14 fit (include/obvh_batch.h).

Every box of a batch must be the oracle's box for that set alone, bit for bit
(zero signs aside), whichever way the planner splits the work: one warp per
set, one CTA per set, or a large set in chunks over many CTAs with a second
pass that waits for the first.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_dito, same_bits
from obvh_b200 import workloads

pytestmark = pytest.mark.gpu

# Knob settings that force each path of the planner.
TUNINGS = {
    "default": None,
    "all_warp": dict(points_per_thread=4, chunk_points=1024, warp_max_points=1 << 30, cta_max_points=1 << 30,
                     lag_tasks=0, ctas_per_sm=2),
    "all_cta": dict(points_per_thread=16, chunk_points=1024, warp_max_points=0, cta_max_points=1 << 30,
                    lag_tasks=0, ctas_per_sm=1),
    "all_chunks": dict(points_per_thread=8, chunk_points=1024, warp_max_points=0, cta_max_points=0,
                       lag_tasks=1, ctas_per_sm=2),
    "chunks_no_lag": dict(points_per_thread=4, chunk_points=1024, warp_max_points=16, cta_max_points=2048,
                          lag_tasks=1, ctas_per_sm=1),
    # pass 2 of a chunked set by the CTA that completes its pass 1
    "chunks_finisher": dict(points_per_thread=8, chunk_points=1024, warp_max_points=0, cta_max_points=0,
                            lag_tasks=0, ctas_per_sm=2),
}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _csr(sets):
    sizes = [len(s) for s in sets]
    offsets = np.zeros(len(sets) + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    pts = np.concatenate([np.asarray(s, np.float32).reshape(-1, 3) for s in sets]) if offsets[-1] else \
        np.zeros((0, 3), np.float32)
    return pts, offsets


def _run(torch, pts, offsets, tuning=None, flags=0, pad=0):
    from obvh_b200.batch import DitoBatch
    buf = torch.zeros((len(pts) + pad + 1, 3), dtype=torch.float32, device="cuda")
    if len(pts):
        buf[pad:pad + len(pts)] = torch.from_numpy(pts).cuda()
    view = buf[pad:pad + len(pts)] if len(pts) else buf[pad:pad + 1]
    sets = len(offsets) - 1
    out = torch.zeros((max(sets, 1), 15), dtype=torch.float32, device="cuda")
    b = DitoBatch(offsets, flags=flags, tuning=tuning)
    b.run(view, out)
    assert b.status() == 0
    return out[:sets].cpu().numpy(), b


def _expect(pts, offsets, mode=oracle.DITO_CPU):
    return [oracle.dito14(pts[offsets[s]:offsets[s + 1]], mode)[0] for s in range(len(offsets) - 1)]


def _mixed_sets(seed, count, lo=1, hi=60000):
    rng = np.random.default_rng(seed)
    sets = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        kind = i % 4
        if kind == 0:
            p = workloads.ellipsoid_points(n, seed=seed * 1000 + i)
        elif kind == 1:  # lattice: many ties
            p = rng.integers(-3, 4, size=(n, 3)).astype(np.float32)
        elif kind == 2:  # collinear
            t = rng.normal(size=(n, 1)).astype(np.float32)
            p = (t * np.array([[1.0, 2.0, -0.5]], np.float32) + 3.0).astype(np.float32)
        else:
            sig = np.exp(rng.uniform(np.log(0.01), np.log(5.0), size=3))
            p = (rng.normal(size=(n, 3)) * sig + rng.uniform(-100, 100, size=3)).astype(np.float32)
        sets.append(p)
    return sets


def test_golden_sets_as_one_batch(torch):
    names, sets, boxes = zip(*golden_dito())
    pts, offsets = _csr(sets)
    for tname, tuning in TUNINGS.items():
        for pad in (0, 1, 3):
            out, _ = _run(torch, pts, offsets, tuning, pad=pad)
            for i, name in enumerate(names):
                assert same_bits(out[i], boxes[i]), (tname, pad, name, out[i], boxes[i])


@pytest.mark.parametrize("tname", list(TUNINGS))
def test_mixed_sets_match_oracle(torch, tname):
    sets = _mixed_sets(7, 48)
    sets.insert(5, np.zeros((0, 3), np.float32))            # empty set
    sets.insert(9, np.ones((1, 3), np.float32))             # one point
    sets.insert(11, np.full((40, 3), 2.5, np.float32))      # all points equal
    pts, offsets = _csr(sets)
    want = _expect(pts, offsets)
    out, b = _run(torch, pts, offsets, TUNINGS[tname], pad=2)
    for s in range(len(sets)):
        assert same_bits(out[s], want[s]), (tname, s, len(sets[s]), out[s], want[s])


def test_reference_gpu_semantics(torch):
    from obvh_b200 import REFERENCE_GPU
    sets = _mixed_sets(11, 24)
    pts, offsets = _csr(sets)
    want = _expect(pts, offsets, oracle.DITO_GPU)
    for tname in ("default", "all_chunks"):
        out, _ = _run(torch, pts, offsets, TUNINGS[tname], flags=REFERENCE_GPU)
        for s in range(len(sets)):
            assert same_bits(out[s], want[s]), (tname, s, out[s], want[s])


def test_batch_equals_single_fits(torch):
    from obvh_b200 import DitoFitter
    pts, offsets = workloads.gaussian_sets(n_sets=96, seed=5, size_max=150000)
    out, _ = _run(torch, pts, offsets)
    f = DitoFitter()
    dp = torch.from_numpy(pts).cuda()
    for s in range(96):
        one = f.fit(dp[offsets[s]:offsets[s + 1]]).cpu().numpy()
        assert same_bits(out[s], one), (s, out[s], one)


def test_graph_replay_and_autotune(torch):
    from obvh_b200.batch import DitoBatch
    pts, offsets = workloads.gaussian_sets(n_sets=200, seed=6, size_max=100000)
    want = _expect(pts, offsets)
    dp = torch.from_numpy(pts).cuda()
    out = torch.zeros((200, 15), dtype=torch.float32, device="cuda")
    b = DitoBatch(offsets)
    tuning, ms = b.autotune(dp, out, repeats=2)
    assert ms > 0 and tuning["points_per_thread"] in (4, 8, 16)
    b.capture(dp, out)
    for _ in range(3):
        out.zero_()
        b.launch()
        assert b.status() == 0
        got = out.cpu().numpy()
        for s in range(200):
            assert same_bits(got[s], want[s]), (s, got[s], want[s])


def test_host_entry_point(torch):
    from obvh_b200.batch import points_obb_batch
    pts, offsets = workloads.gaussian_sets(n_sets=64, seed=8, size_max=80000)
    out, ms = points_obb_batch(pts, offsets, return_time=True)
    want = _expect(pts, offsets)
    assert ms > 0
    for s in range(64):
        assert same_bits(out[s], want[s]), (s, out[s], want[s])
    empty = points_obb_batch(np.zeros((0, 3), np.float32), np.zeros(1, np.int64))
    assert empty.shape == (0, 15)


def test_bad_arguments(torch):
    from obvh_b200 import _native
    from obvh_b200.batch import DitoBatch
    with pytest.raises(_native.ObvhError):
        DitoBatch(np.array([0, 5, 3]))        # decreasing offsets
    with pytest.raises(_native.ObvhError):
        DitoBatch(np.array([1, 5]))           # not starting at 0
    with pytest.raises(_native.ObvhError):
        DitoBatch(np.array([0, 5]), tuning=dict(points_per_thread=3, chunk_points=4096, warp_max_points=0,
                                                  cta_max_points=0, lag_tasks=0, ctas_per_sm=1))
