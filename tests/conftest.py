"""Shared pytest set-up.

* ``gpu`` marker: tests that need a CUDA device (the parity tests proper, which
  call the CUDA library through its C-ABI).
* The oracle (test infrastructure, ``oracle/``) is built on demand with make.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def golden_names(prefix=""):
    """Golden cases (one solve or V-cycle each); the 256^3 reference pressure samples
    (spheres_256_reference_p.npz) are read by their own tests."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and f.startswith(prefix) and not f.startswith("spheres_256_"))


def load_golden(name):
    import numpy as np
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    for k in ("dx", "dy", "dz", "dt", "tol"):
        if k in d:
            d[k] = float(d[k])
    for k in ("max_iter", "applies"):
        if k in d:
            d[k] = int(d[k])
    d["kind"] = str(d["kind"])
    return d


@pytest.fixture(scope="session")
def handle():
    """One solver handle on cuda:0 for the GPU tests."""
    from uaamg_b200.solver import Handle
    h = Handle(0)
    yield h
    h.close()
