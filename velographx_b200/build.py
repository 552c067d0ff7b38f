"""Build recipe of the B200 library and its Python module (in-tree).

* ``libvx_b200.so``   -- every ``csrc/*.cu`` compiled by nvcc for sm_100a
                         (``-gencode arch=compute_100a,code=sm_100a -lineinfo``)
                         and linked as one shared library (static cudart).
* ``_velographx*.so`` -- ``python/bindings.cpp`` (pybind11) linked against it
                         with an ``$ORIGIN`` rpath.

Objects go to ``velographx_b200/_build`` (git-ignored).  Rebuilds only what
changed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvx_b200.so")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INCLUDE, "vx_b200.h")]
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        if _newer(obj, [src] + headers):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj])
        objs.append(obj)
    # relink when an object changed or the set of sources did
    manifest = os.path.join(BUILD, "objects.txt")
    listing = "\n".join(objs)
    old = open(manifest).read() if os.path.exists(manifest) else None
    if _newer(LIB, objs) or old != listing:
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
        with open(manifest, "w") as f:
            f.write(listing)
    return LIB


def build_module() -> str:
    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(HERE, "_velographx" + suffix)
    src = os.path.join(HERE, "python", "bindings.cpp")
    deps = [src, LIB] + glob.glob(os.path.join(INCLUDE, "**", "*.h*"), recursive=True)
    if _newer(out, deps):
        py_inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-std=c++20", "-shared", "-fPIC", "-fvisibility=hidden", src, "-o", out,
              "-I" + INCLUDE, "-I" + pybind11.get_include(), "-I" + py_inc, "-L" + HERE, "-l:libvx_b200.so",
              "-Wl,-rpath,$ORIGIN"])
    return out


def build(verbose_ptxas: bool = False) -> None:
    build_library(verbose_ptxas)
    build_module()


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
