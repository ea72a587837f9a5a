"""Builds oracle/_ref/integration_drive (test infrastructure): the reference-side
code of INTEGRATION.md section 2 -- the GpuUAAMGPCG[3D] subclass, the Factory and
Factory3D lines and the SolverKind mirror, extracted verbatim from that section --
compiled with oracle/integration_drive.cpp, the reference's own pressure, PCG,
UAAMG and grid sources (read in place from the reference tree) and linked
against this repository's uaamg_b200/libuaamg_b200.so.

    python oracle/build_integration.py [REFERENCE_TREE]

The program is run by tests/test_gpu_integration.py on a GPU; outputs go to
oracle/_ref/ only.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "integration_gen")
EXE = os.path.join(OUT, "integration_drive")
REF_SRCS = ["src/core/grid.cpp", "src/core/grid_3d.cpp", "src/solver/pcg.cpp",
            "src/solver/pcg_3d.cpp", "src/solver/preconditioner/uaamg_preconditioner.cpp",
            "src/solver/preconditioner/uaamg_preconditioner_3d.cpp",
            "src/pressure/pressure.cpp", "src/pressure/pressure_3d.cpp"]


def extract() -> dict:
    """The four C++ blocks of INTEGRATION.md section 2, in order: the subclass header,
    the Factory lines, the Factory3D lines, the SolverKind mirror."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## 2. The Solver subclass"):text.index("## 3.")]
    blocks = re.findall(r"```cpp\n(.*?)```", sec, re.S)
    if len(blocks) < 4:
        raise RuntimeError("INTEGRATION.md section 2: expected 4 C++ blocks")
    return {"gpu_uaamg_pcg.h": blocks[0], "factory2d_lines.inc": blocks[1],
            "factory3d_lines.inc": blocks[2], "solver_kind.h": "#pragma once\n" + blocks[3]}


def build(ref: str, verbose: bool = False) -> str:
    lib = os.path.join(ROOT, "uaamg_b200", "libuaamg_b200.so")
    if not os.path.exists(lib):
        raise FileNotFoundError(lib)
    os.makedirs(GEN, exist_ok=True)
    for name, body in extract().items():
        with open(os.path.join(GEN, name), "w") as f:
            f.write(body)
    srcs = [os.path.join(HERE, "integration_drive.cpp")] + [os.path.join(ref, s) for s in REF_SRCS]
    # the reference's release flags (CMakeLists.txt:13) without FMA contraction, as
    # oracle/Makefile builds it
    cmd = ["g++", "-std=c++17", "-O2", "-DNDEBUG", "-ffp-contract=off", "-include", "array",
           "-I", os.path.join(ref, "include"), "-I", GEN, "-I", os.path.join(ROOT, "include"),
           *srcs, lib, "-Wl,-rpath,$ORIGIN/../../uaamg_b200", "-o", EXE + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(EXE + ".tmp", EXE)
    return EXE


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UAAMG_REFERENCE_TREE",
                                                                 "/root/reference")
    print(build(tree, verbose=True))
