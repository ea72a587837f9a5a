"""The drop-in as a reference maintainer uses it: oracle/_ref/integration_drive runs
the reference's own PressureProjection::project and PressureProjection3D::project
(src/pressure/pressure.cpp:5-33, pressure_3d.cpp:5-40) with the GpuUAAMGPCG[3D]
subclass, factory lines and SolverKind mirror of INTEGRATION.md section 2, against
the same projections with the reference's PCG(UAAMGPreconditioner) and
PCG3D(UAAMGPreconditioner3D) (the latter through the Factory3D line that replaces the
Jacobi3D fallback), two steps each with a moving obstacle.  Pressure and projected
face velocities must agree to 1e-10 (the reference's own GPU-vs-CPU PCG bar).

The program is compiled where the reference tree is present (build(), via
oracle/build_integration.py); this test runs the prebuilt binary."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "integration_drive")


@pytest.mark.skipif(not os.path.exists(EXE),
                    reason="oracle/_ref/integration_drive not built (needs the reference tree)")
def test_reference_projection_with_gpu_solver():
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    out = r.stdout
    assert r.returncode == 0, out + r.stderr
    assert "integration ok" in out
    lines = [l for l in out.splitlines() if l.startswith(("2d step", "3d step"))]
    assert len(lines) == 4, out
    for l in lines:
        diffs = [float(v) for v in re.findall(r"d[puvw] ([0-9.e+-]+)", l)]
        assert diffs and max(diffs) <= 1e-10, l
    assert "PCG(B200-UAAMG)" in out
