"""The flat 2D finest-level V-cycle steps (uaamg_b200/csrc/flat2d.cuh) built for the
host and checked against the oracle's V-cycle stage by stage, on the CPU:

  forward sweep from x = 0         == the oracle's level-0 x after smooth(forward)
  residual + restriction           == its level-1 b after restrict_residual
  prolongation + reverse sweep     == its final z, given its level-1 solution

bit for bit in FP64 (the GPU instantiation is compiled with -fmad=false and uses the
same functions); FP32 within 1e-5 relative of the FP64 stages.  The CG's z sums of the
odd-colour step are checked against numpy.  Needs nvcc (the header is CUDA source).
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

KACTIVE, KODD = 64, 128
NVCC = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def f2h(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not present")
    out = str(tmp_path_factory.mktemp("f2h") / "libf2h.so")
    cmd = [NVCC, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           "-I", os.path.join(ROOT, "uaamg_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "flat2d_host.cu"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    lib = C.CDLL(out)
    p, i, d = C.c_void_p, C.c_int, C.c_double
    for t in ("f64", "f32"):
        getattr(lib, f"f2h_fwd_{t}").argtypes = [i, i, d, d, i, p, p, p]
        getattr(lib, f"f2h_res_{t}").argtypes = [i, i, i, i, d, d, i, p, p, p, p, p]
        getattr(lib, f"f2h_up_{t}").argtypes = [i, i, i, i, d, d, i, p, p, p, p, p]
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def codes(solid, fine=True):
    """Cell codes as the engine builds them (k_codes): bit 6 interior fluid, bit 7
    colour (i + j) & 1, and on the finest level bits 0-3 'the +x, -x, +y, -y
    neighbour is interior fluid'."""
    ny, nx = solid.shape[0] - 2, solid.shape[1] - 2
    c = np.zeros(solid.shape, np.uint8)
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            v = KODD if (i + j) & 1 else 0
            if not solid[j, i]:
                v |= KACTIVE
                if fine:
                    if i < nx and not solid[j, i + 1]:
                        v |= 1
                    if i > 1 and not solid[j, i - 1]:
                        v |= 2
                    if j < ny and not solid[j + 1, i]:
                        v |= 4
                    if j > 1 and not solid[j - 1, i]:
                        v |= 8
            c[j, i] = v
    return c


def case(seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(4, 40)), int(rng.integers(4, 40))
    frac = [0.0, 0.1, 0.3][seed % 3]
    solid = (rng.random((ny + 2, nx + 2)) < frac).astype(np.uint8)
    solid[[0, -1], :] = 0
    solid[:, [0, -1]] = 0
    r = np.zeros(solid.shape)
    r[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    dx, dy = float(rng.uniform(0.01, 1.0)), float(rng.uniform(0.01, 1.0))
    return solid, r, dx, dy, seed % 4 == 3


@pytest.mark.parametrize("seed", range(12))
def test_flat2d_steps_equal_oracle_stages(f2h, seed):
    solid, r, dx, dy, dirichlet = case(seed)
    ny, nx = solid.shape[0] - 2, solid.shape[1] - 2
    H = O.Hierarchy(solid, dx, dy, 1.0, dirichlet=dirichlet)
    if H.nlevels < 2:
        pytest.skip("a single level: no finest-level marches")
    x_fwd, b1, x1, z = H.vcycle_stages(r)
    cny, cnx = b1.shape[0] - 2, b1.shape[1] - 2
    c0 = codes(solid)
    c1 = codes(H.level_solid(1), fine=False)
    dr = int(dirichlet)
    inner = (slice(1, -1), slice(1, -1))

    # FP64: bit for bit
    x = np.zeros_like(r)
    f2h.f2h_fwd_f64(nx, ny, dx, dy, dr, _p(c0), _p(r), _p(x))
    assert np.array_equal(x[inner], x_fwd[inner])
    cb = np.zeros_like(b1)
    f2h.f2h_res_f64(nx, ny, cnx, cny, dx, dy, dr, _p(c0), _p(r), _p(x_fwd), _p(c1), _p(cb))
    assert np.array_equal(cb[inner], b1[inner])
    xu = np.zeros_like(r)
    sums = np.zeros(3)
    f2h.f2h_up_f64(nx, ny, cnx, cny, dx, dy, dr, _p(c0), _p(r), _p(x1), _p(xu), _p(sums))
    assert np.array_equal(xu[inner], z[inner])
    fl = np.zeros(solid.shape, bool)
    fl[inner] = solid[inner] == 0
    want = np.array([z[fl].sum(), (r[fl] * z[fl]).sum(), r[fl].sum()])
    np.testing.assert_allclose(sums, want, rtol=1e-10, atol=1e-10 * np.abs(z[fl]).sum())

    # FP32: the same steps from the FP64 stages' inputs, within FP32 rounding
    def rel(a, b):
        return np.linalg.norm(a[inner] - b[inner]) / max(np.linalg.norm(b[inner]), 1e-300)

    r32 = r.astype(np.float32)
    x32 = np.zeros_like(r32)
    f2h.f2h_fwd_f32(nx, ny, dx, dy, dr, _p(c0), _p(r32), _p(x32))
    assert rel(x32.astype(np.float64), x_fwd) <= 1e-5
    cb32 = np.zeros(b1.shape, np.float32)
    xf32 = x_fwd.astype(np.float32)
    f2h.f2h_res_f32(nx, ny, cnx, cny, dx, dy, dr, _p(c0), _p(r32), _p(xf32), _p(c1), _p(cb32))
    assert rel(cb32.astype(np.float64), b1) <= 1e-4
    xu32 = np.zeros_like(r32)
    x132 = x1.astype(np.float32)
    f2h.f2h_up_f32(nx, ny, cnx, cny, dx, dy, dr, _p(c0), _p(r32), _p(x132), _p(xu32), _p(sums))
    assert rel(xu32.astype(np.float64), z) <= 1e-5
