"""The C ABI: the library loads and exports every symbol include/*.h declares,
and the shared structs keep the reference's byte layout."""
import ctypes
import os
import subprocess

import pytest

from obvh_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _native.lib()
    names = _native.declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in _native.lib().obvh_version()


def test_struct_layouts_compile_against_headers(tmp_path):
    """The static asserts in obvh_types.h encode the reference's sizes/offsets."""
    src = tmp_path / "t.c"
    src.write_text('#include "obvh_types.h"\n#include "obvh_dito.h"\n#include "obvh_api.h"\nint main(void){return 0;}\n')
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "t")],
                   check=True)
    src2 = tmp_path / "t.cpp"
    src2.write_text('#include "obvh_types.h"\n#include "obvh_dito.h"\nint main(){return 0;}\n')
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src2), "-o", str(tmp_path / "t2")],
                   check=True)


def test_workspace_size_is_reported():
    assert _native.lib().obvh_dito_workspace_bytes() > 256


def test_build_graph_entry_points_check_their_handles():
    """No CUDA call is made for a null handle: launch names the error,
    destroy is a no-op, create wants somewhere to write the handle."""
    lib = _native.lib()
    assert b"null graph" in ctypes.string_at(lib.obvh_build_graph_launch(None, None))
    assert lib.obvh_build_graph_destroy(None) is None
    args = [None, None, 0, 0, 1.2, 1.0] + [None] * 10 + [None]
    assert b"null output" in ctypes.string_at(lib.obvh_build_graph_create(*args))


def test_build_headers_compile_as_c(tmp_path):
    src = tmp_path / "b.c"
    src.write_text('#include "obvh_build.h"\n#include "obvh_atrbvh.h"\nint main(void){obvh_build_graph g = 0;'
                   'return g != 0;}\n')
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(tmp_path / "b")], check=True)
