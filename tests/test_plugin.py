"""The intersector plugins (liblbvh_gpu.so, libatrbvh_gpu.so) through the
reference's loading protocol: dlopen, dlsym("korangar_ads_action"), CREATE,
then actions.  These checks make no CUDA call; the commits are in
test_plugin_gpu.py."""
import ctypes

import numpy as np
import pytest

from obvh_b200 import _native, plugin


@pytest.fixture(scope="module", params=["lbvh_gpu", "atrbvh_gpu"])
def ads(request):
    from obvh_b200 import build
    build.build_plugins()
    a = plugin.Intersector(request.param)
    yield request.param, a
    a.destroy()


def test_exports_only_the_action_symbol(ads):
    name, a = ads
    assert hasattr(a.dll, "korangar_ads_action")


def test_name_and_query_type(ads):
    name, a = ads
    assert a.name() == {"lbvh_gpu": "LBVH GPU", "atrbvh_gpu": "ATRBVH"}[name]
    assert a.preferred_query_type() == plugin.KR_QUERY_TYPE_CUDA


def test_init_reads_the_reference_descriptors(ads):
    _, a = ads
    a.init(collapse="y", use_obbs="y", ci="1.5", ct="0.75", intersect_bounds="n", intersect_bounds_level="3",
           use_persistent_kernel="y", save_construction_information="n", unknown_key="ignored")
    b = a.blas()
    assert (b.collapse, b.use_obbs, b.use_persistent_kernel, b.intersect_bounds) == (1, 1, 1, 0)
    assert b.intersect_bounds_level == 3
    assert np.float32(b.ci) == np.float32(1.5) and np.float32(b.ct) == np.float32(0.75)
    assert b.commits == 0 and b.nodes is None


def test_empty_scene_and_queries_are_errors(ads):
    _, a = ads
    with pytest.raises(_native.ObvhError, match="no intersectable primitives"):
        a.commit(plugin.MeshScene([(np.zeros((0, 3), np.float32), np.zeros((0, 4), np.uint32))]))
    assert a.call("INTERSECTION_QUERY")  # a null query: an error string, never a silent success
    assert a.call("OCCLUSION_QUERY")  # not built: an error string
    assert a.call("SETTINGS_UPDATE") is None and a.call("CSV_EXPORT") is None


def test_layouts_match_the_reference_headers():
    assert ctypes.sizeof(plugin.Scene) == 424
    assert plugin.Scene.objects.offset == 304 and plugin.Scene.benchmark_file.offset == 416
    assert ctypes.sizeof(plugin.Object) == 80
