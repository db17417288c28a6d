"""Build recipe for the native libraries (sm_100a only).

    python -m obvh_b200.build            # build what is out of date
    python -m obvh_b200.build --force    # rebuild everything

Produces, in-tree next to this file:

* ``libobvh_b200.so``  - every kernel and the C ABI declared in include/*.h
* ``liblbvh_gpu.so``   - the ``lbvh_gpu`` intersector plugin (``korangar_ads_action``)
* ``libatrbvh_gpu.so`` - the ``atrbvh_gpu`` intersector plugin

All CUDA is compiled for ``compute_100a``/``sm_100a`` with ``--fmad=false``
(uncontracted float arithmetic, matching the reference's CPU evaluation order)
and IEEE division/square root.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
    "-I", INCLUDE, "-I", CSRC,
]

LIB_CORE = os.path.join(PKG, "libobvh_b200.so")
PLUGINS = {
    "lbvh_gpu": os.path.join(PKG, "liblbvh_gpu.so"),
    "atrbvh_gpu": os.path.join(PKG, "libatrbvh_gpu.so"),
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build obvh_b200")
    return exe


def _core_sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return (_core_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(INCLUDE, "*.h")) + [os.path.abspath(__file__)])


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_core(force: bool = False, verbose: bool = False, jobs: int = 0) -> str:
    """Compiles every csrc/*.cu into libobvh_b200.so (objects under _build/)."""
    deps = _deps()
    if not force and not _stale(LIB_CORE, deps):
        return LIB_CORE
    objdir = os.path.join(ROOT, "_build", "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [d for d in deps if d.endswith((".h", ".cuh", ".py"))]
    newest_header = max(os.path.getmtime(h) for h in headers)
    procs, objs = [], []
    for src in _core_sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((subprocess.Popen(cmd), src))
    failed = [src for p, src in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on: " + ", ".join(failed))
    tmp = LIB_CORE + ".tmp"
    _run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"], verbose)
    os.replace(tmp, LIB_CORE)
    return LIB_CORE


def build_plugins(force: bool = False, verbose: bool = False):
    """The two intersector plugins; each links against libobvh_b200.so."""
    out = []
    for name, target in PLUGINS.items():
        src = os.path.join(PKG, "plugins", name + ".cpp")
        if not os.path.exists(src):
            continue
        deps = [src, LIB_CORE] + glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(PKG, "plugins", "*.h"))
        if force or _stale(target, deps):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", INCLUDE, "-I", os.path.join(PKG, "plugins"),
                   "-I", "/usr/local/cuda/include", "-o", target, src,
                   "-L", PKG, "-lobvh_b200", "-Wl,-rpath,$ORIGIN"]
            _run(cmd, verbose)
        out.append(target)
    return out


def build(force: bool = False, verbose: bool = False) -> None:
    build_core(force, verbose)
    build_plugins(force, verbose)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    build(a.force, a.verbose)
    print("built:", LIB_CORE, file=sys.stderr)
