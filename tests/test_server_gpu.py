"""The request server (include/obvh_server.h) on the GPU.

Every result must be the one the plain path gives for the same input alone
(obvh_points_obb for a fit, obvh_build_async for a build), bit for bit,
whatever else was in flight: fits batched with others, builds overlapping on
several streams, inputs from host memory or already on the device.  Admission
must keep the arena within its budget and still complete everything.
"""
import random
import threading
import time

import numpy as np
import pytest

from conftest import same_bits
from obvh_b200 import bvh, dito, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _fit_inputs(rng, k):
    sizes = [0, 1, 2, 3, 13, 14, 15, 16, 17] + [int(np.exp(rng.uniform(np.log(20), np.log(300_000)))) for _ in range(k)]
    out = []
    for i, n in enumerate(sizes):
        sig = np.exp(rng.uniform(np.log(0.01), np.log(5.0), size=3))
        rot = workloads.random_rotation(rng)
        p = (rng.normal(size=(n, 3)) * sig) @ rot.T + rng.uniform(-100, 100, size=3)
        out.append(p.astype(np.float32))
    return out


def _build_inputs(rng, k):
    return [workloads.triangle_soup(int(np.exp(rng.uniform(np.log(1), np.log(80_000)))) + 1, seed=900 + i)
            for i in range(k)]


def _alone_build(builder, v, f, flags, ci, ct):
    import torch
    o = builder.build(bvh.Mesh(v, f), flags=flags, ci=ci, ct=ct)
    torch.cuda.synchronize()
    err, slots = builder.status(f.shape[0])
    assert err == 0
    return o, slots


def _check_build(got, alone, slots, flags):
    nodes = bvh.nodes_numpy(alone["nodes"])
    assert np.array_equal(got["nodes"].view(np.uint8), nodes.view(np.uint8))
    assert np.array_equal(got["parents"], alone["parents"].cpu().numpy().view(np.uint32))
    assert np.array_equal(got["counts"], alone["counts"].cpu().numpy().view(np.uint32))
    assert same_bits(got["costs"], alone["costs"].cpu().numpy())
    if flags & bvh.BUILD_OBBS:
        assert same_bits(got["obbs"], alone["obbs"].cpu().numpy())
        assert same_bits(got["transforms"], alone["transforms"].cpu().numpy())
    if flags & bvh.BUILD_COLLAPSE:
        assert got["slots"] == slots
        c = bvh.nodes_numpy(alone["collapsed"])
        assert np.array_equal(got["collapsed"].view(np.uint8), c.view(np.uint8))
        assert np.array_equal(got["primitives"][:slots], alone["primitives"].cpu().numpy().view(np.uint32)[:slots])


def test_results_alone_equal_results_in_the_mix(torch):
    from obvh_b200.server import Server
    rng = np.random.default_rng(11)
    fits = _fit_inputs(rng, 60)
    builds = _build_inputs(rng, 10)
    srv = Server(budget_bytes=6 << 30, build_lanes=3)
    jobs = [("fit", i) for i in range(len(fits))] + [("build", i) for i in range(len(builds))]
    random.Random(3).shuffle(jobs)
    ids = {}
    dev_fits = {i: torch.from_numpy(fits[i]).cuda() for i in range(0, len(fits), 2)}
    dev_builds = {i: (torch.from_numpy(builds[i][0]).cuda(), torch.from_numpy(bvh.as_faces4(builds[i][1]).view(np.int32)).cuda())
                  for i in range(1, len(builds), 2)}
    torch.cuda.synchronize()
    flags_of = {i: [3, 1, 2, 0][i % 4] for i in range(len(builds))}

    def producer():
        r = random.Random(5)
        for kind, i in jobs:
            if kind == "fit":
                ids[jobs.index((kind, i))] = srv.submit_fit(dev_fits.get(i, fits[i]))
            else:
                v, f = dev_builds.get(i, builds[i])
                ids[jobs.index((kind, i))] = srv.submit_build(v, f, flags=flags_of[i], ci=1.2, ct=1.0)
            time.sleep(r.uniform(0, 0.002))

    t = threading.Thread(target=producer)
    t.start()
    t.join()
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["fit_batches"] >= 1 and st["peak_bytes"] <= st["arena_bytes"]
    assert st["build_batches"] >= 1  # the builds of up to 16,384 triangles went through batch rounds
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]

    builder = bvh.ObvhBuilder()
    for k, (kind, i) in enumerate(jobs):
        rid = ids[k]
        if kind == "fit":
            alone = dito.points_obb(fits[i])
            assert same_bits(srv.fit_result(rid), alone), (i, len(fits[i]))
        else:
            v, f = builds[i]
            alone, slots = _alone_build(builder, v, f, flags_of[i], 1.2, 1.0)
            _check_build(srv.build_result(rid), alone, slots, flags_of[i])
        assert srv.latency_ms(rid) > 0
        srv.release(rid)
    assert srv.stats()["in_use_bytes"] == 0
    srv.close()


def test_budget_admission_and_oversize_requests(torch):
    from obvh_b200 import _native
    from obvh_b200.server import Server
    v, f = workloads.triangle_soup(200_000, seed=21)
    # about 1.5 builds of this size fit: they must run one after another
    srv = Server(budget_bytes=260 << 20, build_lanes=4)
    ids = [srv.submit_build(v, f, flags=3) for _ in range(4)]
    big = srv.submit_fit(np.zeros((30_000_000, 3), np.float32))  # 360 MB: more than the whole budget
    small = srv.submit_fit(workloads.ellipsoid_points(10_000, seed=2))
    # a completed build's outputs stay resident until released, and later
    # builds wait for that memory: the client consumes results in order
    outs = []
    for rid in ids:
        assert srv.wait(rid, 120_000)
        outs.append(srv.build_result(rid))
        assert srv.stats()["in_use_bytes"] > 0
        srv.release(rid)
    srv.drain()
    with pytest.raises(_native.ObvhError, match="budget"):
        srv.fit_result(big)
    assert same_bits(srv.fit_result(small), dito.points_obb(workloads.ellipsoid_points(10_000, seed=2)))
    st = srv.stats()
    assert st["completed"] == 5 and st["failed"] == 1
    assert st["peak_bytes"] <= 260 << 20
    for got in outs[1:]:
        assert np.array_equal(got["nodes"].view(np.uint8), outs[0]["nodes"].view(np.uint8))
        assert same_bits(got["obbs"], outs[0]["obbs"])
    for rid in (small, big):
        srv.release(rid)
    assert srv.stats()["in_use_bytes"] == 0
    srv.close()


def test_many_small_fits_are_batched(torch):
    from obvh_b200.server import Server
    rng = np.random.default_rng(4)
    sets = [rng.normal(size=(int(rng.integers(1, 3000)), 3)).astype(np.float32) for _ in range(2000)]
    srv = Server(budget_bytes=1 << 30)
    ids = [srv.submit_fit(s) for s in sets]
    srv.drain()
    st = srv.stats()
    assert st["completed"] == 2000 and st["fit_batches"] < 2000
    for s, rid in zip(sets[::50], ids[::50]):
        assert same_bits(srv.fit_result(rid), dito.points_obb(s))
    srv.close()


def test_small_builds_batched_in_one_round_equal_their_lone_builds(torch):
    """Builds of up to 16,384 triangles admitted together go to one launch of
    the one-CTA-per-mesh kernel, each into its own arena blocks, with its own
    flags and SAH constants; every result equals its lone obvh_build_async,
    bit for bit, and the larger builds beside them still go through lanes."""
    from obvh_b200.server import Server
    rng = np.random.default_rng(21)
    sizes = [2, 3, 64, 255, 256, 257, 1000, 5000, 16384, 16385, 40000] + \
            [int(np.exp(rng.uniform(np.log(2), np.log(16384)))) for _ in range(40)]
    meshes = [workloads.triangle_soup(n, seed=1300 + i) for i, n in enumerate(sizes)]
    flags = [[3, 1, 2, 0][i % 4] for i in range(len(meshes))]
    consts = [(1.2, 1.0) if i % 3 else (0.8, 1.3) for i in range(len(meshes))]
    srv = Server(budget_bytes=4 << 30, build_lanes=2)
    ids = [srv.submit_build(v, f, flags=flags[i], ci=consts[i][0], ct=consts[i][1]) for i, (v, f) in enumerate(meshes)]
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(meshes) and st["failed"] == 0
    assert 1 <= st["build_batches"] < len(meshes)
    builder = bvh.ObvhBuilder()
    for i, (v, f) in enumerate(meshes):
        alone, slots = _alone_build(builder, v, f, flags[i], *consts[i])
        _check_build(srv.build_result(ids[i]), alone, slots, flags[i])
        srv.release(ids[i])
    assert srv.stats()["in_use_bytes"] == 0
    srv.close()
