"""Build recipe of the product library ``fastlbp_b200/libfastlbp_b200.so``.

nvcc compiles the CUDA engine for sm_100a (``-gencode arch=compute_100a,code=sm_100a``)
and the host C++ API; everything links into one shared library that the
Python layer loads with ctypes and C++ callers link with ``-lfastlbp_b200``.
The library is built in-tree so it travels with the repository.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfastlbp_b200.so")

SOURCES = ["engine.cu", "direct.cu", "dlayout.cu", "layout.cpp", "model.cpp", "causal_bp.cpp", "fg_capi.cpp", "noalloc.cu", "schedule.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
# -ftz=true: FP32 device arithmetic flushes subnormal results to zero (fewer instructions around the
# approximate transcendentals). The message formulas take any product that falls below the smallest
# normal in log space, so no FP32 message depends on a subnormal value.
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-ccbin", "g++", "-Xcompiler", "-fPIC", "-ftz=true", "-I" + INCLUDE]
OPENMP = ["-Xcompiler", "-fopenmp"]  # the host layout build runs on all host threads


def _obj(src: str) -> str:
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _needs(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    for d, _, fs in os.walk(INCLUDE):
        hs += [os.path.join(d, f) for f in fs if f.endswith(".h")]
    return hs


def _compile(src: str, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    cmd = [NVCC] + COMMON + OPENMP + ARCH + ["-c", path, "-o", _obj(src)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return _obj(src)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile changed sources and relink; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    todo = [s for s in SOURCES if force or _needs(_obj(s), [os.path.join(CSRC, s)] + hdrs)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [_obj(s) for s in SOURCES]
    if force or todo or _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", "g++", "-o", LIB] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
