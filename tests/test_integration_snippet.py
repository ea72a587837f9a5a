"""The reference-side binding shown in INTEGRATION.md (the Solver / Solver3D subclass
and its factory lines) compiles against the reference's own headers and links
against the built library.  Needs the reference tree (for its headers and
src/core/grid.cpp) and g++; skipped where either is absent.  No GPU: the program is
built, not run."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

REF_TREE = None
try:
    import __graft_entry__ as _ge
    REF_TREE = _ge.REF_TREE
except Exception:  # pragma: no cover - the entry module always imports here
    pass

LIB = os.path.join(ROOT, "uaamg_b200", "libuaamg_b200.so")


def _snippet():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## 2. The Solver subclass"):text.index("## 3.")]
    header, factory, factory3d, kind = re.findall(r"```cpp\n(.*?)```", sec, re.S)[:4]
    header = header.replace("#pragma once\n", "")
    return header + kind + """
#include <memory>
#include <string>
#include "core/grid.h"
#include "core/grid_3d.h"
#include "solver/pcg_3d.h"
#include "solver/preconditioner/uaamg_preconditioner_3d.h"

std::unique_ptr<Solver> make_solver(const std::string& name) {
""" + factory + """
    return nullptr;
}

std::unique_ptr<Solver3D> make_solver_3d(const std::string& name) {
""" + factory3d + """
    return nullptr;
}

int main(int argc, char**) {
    if (argc > 1) {  // never taken in this test (tests/test_gpu_integration.py runs it)
        auto s = make_solver(solver_key(solver_kind("pcg_uaamg_gpu")));
        auto s3d = make_solver_3d("pcg_uaamg_gpu");
        Grid g(8, 4, 1.0, 0.5);
        g.init_variable_lap();
        s->solve(g, g.p, 10, 1e-6);
        GpuUAAMGPCG3D s3(UAAMG_MIXED);
    }
    return 0;
}
"""


@pytest.mark.skipif(not (REF_TREE and os.path.isdir(os.path.join(REF_TREE, "include"))),
                    reason="reference tree not present")
@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not present")
def test_integration_binding_compiles_and_links(tmp_path):
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    src = tmp_path / "binding.cpp"
    src.write_text(_snippet())
    exe = tmp_path / "binding"
    cmd = ["g++", "-std=c++17", "-include", "array",
           "-I", os.path.join(REF_TREE, "include"), "-I", os.path.join(ROOT, "include"),
           str(src), os.path.join(REF_TREE, "src", "core", "grid.cpp"),
           os.path.join(REF_TREE, "src", "core", "grid_3d.cpp"),
           os.path.join(REF_TREE, "src", "solver", "pcg_3d.cpp"),
           os.path.join(REF_TREE, "src", "solver", "preconditioner", "uaamg_preconditioner_3d.cpp"),
           LIB, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert exe.exists()
