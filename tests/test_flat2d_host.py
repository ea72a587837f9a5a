"""The flat 2D V-cycle steps (uaamg_b200/csrc/flat2d.cuh) built for the host and
checked against the oracle's V-cycle stage by stage, on the CPU, on every level that
runs as marches (the finest, with couplings from the cell codes, and the coarse ones,
with their stored Galerkin couplings and diagonal):

  forward sweep from x = 0         == the oracle's x after smooth(forward)
  residual + restriction           == the next level's b after restrict_residual
  prolongation + reverse sweep     == the level's x on exit, given the next level's x

bit for bit in FP64 (the GPU instantiation is compiled with -fmad=false and uses the
same functions); FP32 within 1e-5 relative of the FP64 stages.  The CG's z sums of the
finest level's odd-colour step are checked against numpy.  Needs nvcc (the header is
CUDA source).
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
        getattr(lib, f"f2h_step_{t}").argtypes = [i, i, i, i, i, i, d, d, i, p, p, p, p, p, p, p,
                                                  p, p, p]
    lib.f2h_step_mixed.argtypes = [i, i, i, i, i, d, d, p, p, p, p, p, p, p, p, p, p]
    return lib


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


def run(f2h, t, step, lvl, b, x=None, ccode=None, cb=None, xc=None):
    """One flat step on level `lvl` (a dict of the level's data) in type t."""
    dt = np.float64 if t == "f64" else np.float32
    cast = (lambda a: None if a is None else np.ascontiguousarray(a, dtype=dt))
    dg, cx, cy = (cast(a) for a in lvl["op"])
    b = cast(b)
    x = cast(x) if x is not None else np.zeros(b.shape, dt)
    cb = cast(cb) if cb is not None else None
    xc = cast(xc)
    sums = np.zeros(3)
    getattr(f2h, f"f2h_step_{t}")(step, int(lvl["fine"]), lvl["nx"], lvl["ny"], lvl["cnx"],
                                  lvl["cny"], lvl["dx"], lvl["dy"], lvl["dir"], _p(dg), _p(cx),
                                  _p(cy), _p(lvl["code"]), _p(b), _p(x), _p(ccode), _p(cb),
                                  _p(xc), _p(sums))
    return x, cb, sums


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


@pytest.mark.parametrize("seed", range(12))
def test_flat2d_steps_equal_oracle_stages(f2h, seed):
    """Every level that runs as marches: the finest (couplings from the codes, the
    CG's z sums) and the coarse ones (stored Galerkin couplings and diagonal)."""
    solid, r, dx, dy, dirichlet = case(seed)
    H = O.Hierarchy(solid, dx, dy, 1.0, dirichlet=dirichlet)
    if H.nlevels < 2:
        pytest.skip("a single level: no marches")
    inner = (slice(1, -1), slice(1, -1))
    for l in range(H.nlevels - 1):
        b_l, x_fwd, b1, x1, x_out = H.vcycle_stages(r, l)
        nx, ny, _ = H.dims(l)
        cnx, cny, _ = H.dims(l + 1)
        sl = H.level_solid(l)
        cx, cy, _, dg = H.level_coeffs(l)
        lvl = dict(fine=l == 0, nx=nx, ny=ny, cnx=cnx, cny=cny, dx=dx, dy=dy,
                   dir=int(dirichlet and l == 0), code=codes(sl, fine=l == 0),
                   op=(dg, cx, cy) if l > 0 else (None, None, None))
        c1 = codes(H.level_solid(l + 1), fine=False)

        # FP64: bit for bit
        x, _, _ = run(f2h, "f64", 0, lvl, b_l)
        assert np.array_equal(x[inner], x_fwd[inner]), f"level {l}: forward sweep"
        _, cb, _ = run(f2h, "f64", 1, lvl, b_l, x=x_fwd, ccode=c1, cb=np.zeros_like(b1))
        assert np.array_equal(cb[inner], b1[inner]), f"level {l}: restriction"
        xu, _, sums = run(f2h, "f64", 2, lvl, b_l, xc=x1)
        assert np.array_equal(xu[inner], x_out[inner]), f"level {l}: prolongation + reverse sweep"
        if l == 0:
            fl = np.zeros(solid.shape, bool)
            fl[inner] = solid[inner] == 0
            z = x_out
            want = np.array([z[fl].sum(), (r[fl] * z[fl]).sum(), r[fl].sum()])
            np.testing.assert_allclose(sums, want, rtol=1e-10, atol=1e-10 * np.abs(z[fl]).sum())

        # FP32: the same steps from the FP64 stages' inputs, within FP32 rounding
        def rel(a, b):
            return np.linalg.norm(a[inner] - b[inner]) / max(np.linalg.norm(b[inner]), 1e-300)

        x, _, _ = run(f2h, "f32", 0, lvl, b_l)
        assert rel(x.astype(np.float64), x_fwd) <= 1e-5
        _, cb, _ = run(f2h, "f32", 1, lvl, b_l, x=x_fwd, ccode=c1, cb=np.zeros_like(b1))
        assert rel(cb.astype(np.float64), b1) <= 1e-4
        xu, _, _ = run(f2h, "f32", 2, lvl, b_l, xc=x1)
        assert rel(xu.astype(np.float64), x_out) <= 1e-5


@pytest.mark.parametrize("seed", range(6))
def test_flat2d_coarse_fp16_couplings(f2h, seed):
    """The mixed form's coarse levels: couplings stored as FP16 face counts (exact up
    to 2048 faces) and decoded as count * (finest 1/h^2), FP32 values; within FP32
    rounding of the oracle's FP64 stages (the host divides exactly where the GPU uses
    the fast reciprocal)."""
    solid, r, dx, dy, _ = case(seed)
    H = O.Hierarchy(solid, dx, dy, 1.0)
    if H.nlevels < 3:
        pytest.skip("no coarse march level")
    csx, csy = 1.0 / (dx * dx), 1.0 / (dy * dy)
    inner = (slice(1, -1), slice(1, -1))
    for l in range(1, H.nlevels - 1):
        b_l, x_fwd, b1, x1, x_out = H.vcycle_stages(r, l)
        nx, ny, _ = H.dims(l)
        cnx, cny, _ = H.dims(l + 1)
        cx, cy, _, dg = H.level_coeffs(l)
        counts_x, counts_y = np.rint(cx / csx), np.rint(cy / csy)
        assert np.array_equal(counts_x * csx, cx) or np.allclose(counts_x * csx, cx, rtol=1e-15)
        hcx = counts_x.astype(np.float16).view(np.uint16).copy()
        hcy = counts_y.astype(np.float16).view(np.uint16).copy()
        code = codes(H.level_solid(l), fine=False)
        c1 = codes(H.level_solid(l + 1), fine=False)
        f32 = (lambda a: np.ascontiguousarray(a, dtype=np.float32))
        dg32, b32 = f32(dg), f32(b_l)

        def step(k, x=None, cb=None, xc=None):
            x = f32(x) if x is not None else np.zeros(b32.shape, np.float32)
            sums = np.zeros(3)
            f2h.f2h_step_mixed(k, nx, ny, cnx, cny, csx, csy, _p(dg32), _p(hcx), _p(hcy), _p(code),
                               _p(b32), _p(x), _p(c1), _p(cb), _p(f32(xc) if xc is not None else None),
                               _p(sums))
            return x, cb

        def rel(a, b):
            return np.linalg.norm(a[inner] - b[inner]) / max(np.linalg.norm(b[inner]), 1e-300)

        x, _ = step(0)
        assert rel(x.astype(np.float64), x_fwd) <= 1e-5, f"level {l}: forward sweep"
        cb = np.zeros(b1.shape, np.float32)
        step(1, x=x_fwd, cb=cb)
        assert rel(cb.astype(np.float64), b1) <= 1e-4, f"level {l}: restriction"
        xu, _ = step(2, xc=x1)
        assert rel(xu.astype(np.float64), x_out) <= 1e-5, f"level {l}: reverse sweep"
