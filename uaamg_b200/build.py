"""Builds the in-tree CUDA library ``uaamg_b200/libuaamg_b200.so`` for sm_100a.

nvcc compiles the two engine translation units (the FP64 one with -fmad=false
so its per-cell arithmetic rounds exactly like the reference's x86-64 build) and
the C-ABI layer, then links them with the static CUDA runtime.  The library is
rebuilt only when a source is newer than it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libuaamg_b200.so")
WL_LIB = os.path.join(HERE, "libuaamg_workloads.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", f"-I{INCLUDE}"] + ARCH

# (source, extra nvcc flags)
UNITS = [
    ("kernels_f64.cu", ["-fmad=false"]),
    ("kernels_f32.cu", []),
    ("api.cpp", ["-x", "cu"]),
    ("runtime.cpp", ["-x", "cu"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("tunecache.cpp", ["-x", "cu"]),
    ("project.cu", ["-fmad=false"]),
]
HEADERS = ["common.cuh", "kernels.cuh", "march.cuh", "fused.cuh", "tail.cuh", "vec.cuh", "tma.cuh",
           "engine.cuh", "engine.h", "handle.h"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _newest_input() -> float:
    files = [os.path.join(CSRC, u[0]) for u in UNITS] + [os.path.join(CSRC, h) for h in HEADERS]
    files += [os.path.join(INCLUDE, "uaamg.h"), os.path.abspath(__file__)]
    return max(os.path.getmtime(f) for f in files)


def build_workloads(force: bool = False, verbose: bool = False) -> str:
    """Host-only workload generators (g++), libuaamg_workloads.so."""
    src = os.path.join(CSRC, "workloads.cpp")
    if not force and os.path.exists(WL_LIB) and os.path.getmtime(WL_LIB) >= os.path.getmtime(src):
        return WL_LIB
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    tmp = WL_LIB + ".tmp"
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
           "-Wl,--exclude-libs,ALL", src, "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, WL_LIB)
    return WL_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_workloads(force, verbose)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src, extra in UNITS:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc] + NVCC_COMMON + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
