"""The oracle (plain-C restatement) pinned against the reference: the golden
fixtures generated from the reference's own code, the compiled reference itself
where available, and the reference's own known-answer test."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden_names, load_golden


@pytest.mark.parametrize("name", golden_names())
def test_restatement_matches_golden_bit_exact(name):
    g = load_golden(name)
    if g["kind"] == "vcycle":
        z = O.Hierarchy(g["solid"], g["dx"], g["dy"], g["dz"]).vcycle(g["r"])
        inner = z.copy()
        assert np.array_equal(inner, g["z"]), f"max diff {np.abs(inner - g['z']).max()}"
    elif g["kind"] == "pcg":
        p, n, _ = O.pcg(g["solid"], g["r"], g["dx"], g["dy"], g["dz"], g["max_iter"], g["tol"],
                        tol_mode=0)
        assert np.array_equal(p, g["p"]), f"max diff {np.abs(p - g['p']).max()}"
    elif g["kind"] == "pcg_var":
        lap = (g["lap_diag"], g["lap_off_x"], g["lap_off_y"])
        p, n, _ = O.pcg_var(g["solid"], lap, g["r"], g["dx"], g["dy"], g["max_iter"], g["tol"],
                            tol_mode=0)
        assert np.array_equal(p, g["p"]), f"max diff {np.abs(p - g['p']).max()}"
    else:
        w = g["w"] if g["w"].size else None
        rhs = O.divergence_rhs(g["solid"], g["u"], g["v"], w, g["dx"], g["dy"], g["dz"], g["dt"])
        p, n, _ = O.pcg(g["solid"], rhs, g["dx"], g["dy"], g["dz"], g["max_iter"], g["tol"],
                        tol_mode=0)
        assert np.array_equal(p, g["p"])
        u, v, w2 = O.correct_velocity(g["solid"], p, g["dt"], g["u"], g["v"], w, g["dx"], g["dy"],
                                      g["dz"])
        assert np.array_equal(u, g["u_out"]) and np.array_equal(v, g["v_out"])
        if w is not None:
            assert np.array_equal(w2, g["w_out"])


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(6))
def test_restatement_matches_compiled_reference_random(seed):
    rng = np.random.default_rng(100 + seed)
    dim = 2 + seed % 2
    shape = tuple(int(x) + 2 for x in rng.integers(2, 21, size=dim))
    frac = [0.0, 0.1, 0.3, 0.55][seed % 4]
    solid = (rng.random(shape) < frac).astype(np.uint8)
    r = rng.standard_normal(shape)
    sp = rng.uniform(0.05, 2.0, size=3)
    z_ref = O.ref_vcycle(solid, r, *sp)
    z = O.Hierarchy(solid, *sp).vcycle(r)
    assert np.array_equal(z, z_ref)
    p_ref, _ = O.ref_pcg(solid, r, *sp, max_iter=20, tol=1e-10)
    p, _, _ = O.pcg(solid, r, *sp, max_iter=20, tol=1e-10, tol_mode=0)
    assert np.array_equal(p, p_ref)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "test_amgpcg")),
                    reason="compiled reference test not present")
def test_reference_known_answer_amgpcg_passes():
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "test_amgpcg")],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout
    assert "Failed: 0" in out.stdout


def _dirichlet_problem(n):
    h = 1.0 / n
    x = (np.arange(n + 2) - 0.5) * h
    X, Y = np.meshgrid(x, x, indexing="xy")  # [j, i]
    exact = np.sin(np.pi * X) * np.sin(np.pi * Y)
    f = 2 * np.pi ** 2 * exact
    rhs = np.zeros((n + 2, n + 2))
    rhs[1:-1, 1:-1] = -f[1:-1, 1:-1]       # lap(p) = rhs  <=>  -lap(p) = f
    return h, rhs, exact


def test_dirichlet_64_analytic_error():
    """The CPU-runnable plain method: 64x64 cells on [0,1]^2, h = 1/64, Dirichlet
    p = 0 walls, f = 2 pi^2 sin sin, one V-cycle per iteration, rel. residual
    1e-10; the error against sin(pi x) sin(pi y) is second order in h."""
    n = 64
    h, rhs, exact = _dirichlet_problem(n)
    solid = np.zeros((n + 2, n + 2), np.uint8)
    p, it, st = O.pcg(solid, rhs, h, h, max_iter=100, tol=1e-10, tol_mode=1, dirichlet=True)
    assert st == 0 and it <= 30
    err = np.abs(p - exact)[1:-1, 1:-1].max()
    assert err < 1e-3                         # O(h^2): pi^2 h^2 / 8 ~ 3e-4
    hier = O.Hierarchy(solid, h, h, dirichlet=True)
    assert hier.nlevels == 5 and hier.dims(4)[:2] == (4, 4)
    # halving h divides the error by ~4
    h2, rhs2, exact2 = _dirichlet_problem(32)
    p2, _, _ = O.pcg(np.zeros((34, 34), np.uint8), rhs2, h2, h2, max_iter=100, tol=1e-10,
                     tol_mode=1, dirichlet=True)
    err2 = np.abs(p2 - exact2)[1:-1, 1:-1].max()
    assert 3.0 < err2 / err < 5.0


def test_oracle_relative_mode_reaches_tolerance():
    rng = np.random.default_rng(7)
    shape = (14, 18, 22)
    solid = np.zeros(shape, np.uint8)
    solid[1:-1, 1:-1, 1:-1] = rng.random((12, 16, 20)) < 0.1
    rhs = rng.standard_normal(shape)
    p, it, st = O.pcg(solid, rhs, 0.1, 0.1, 0.1, max_iter=200, tol=1e-8, tol_mode=1)
    res, bn = O.true_residual(solid, rhs, p, 0.1, 0.1, 0.1)
    assert st == 0 and res / bn < 2e-8
    # warm start from the answer converges at once
    p2, it2, st2 = O.pcg(solid, rhs, 0.1, 0.1, 0.1, max_iter=200, tol=1e-6, tol_mode=1, x0=p,
                         warm=True)
    assert it2 <= 1


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(4))
def test_static_pressure_rhs_matches_compiled_reference(seed):
    """recoverStaticPressure's right-hand side (pressure.cpp:35-66): the restatement
    equals what the reference's own function hands its solver, bit for bit, with
    solids touching walls and each other (the clamped and dropped stencil branches)."""
    rng = np.random.default_rng(seed)
    nx, ny = [(17, 11), (32, 24), (9, 40), (64, 48)][seed]
    dx, dy = rng.uniform(0.01, 1.0, size=2)
    solid = (rng.random((ny + 2, nx + 2)) < [0.0, 0.1, 0.3, 0.05][seed]).astype(np.uint8)
    u = rng.standard_normal((ny + 2, nx + 1))
    v = rng.standard_normal((ny + 1, nx + 2))
    assert np.array_equal(O.static_rhs(solid, u, v, dx, dy), O.ref_static_rhs(solid, u, v, dx, dy))


class _OracleSolver:
    """A Solver-interface stand-in whose solve is the oracle's PCG (the reference's
    PCG::solve with its absolute stop), for checking the Python host projection."""

    def solve(self, g, rhs, max_iter, tol):
        p, _, _ = O.pcg(g.solid, rhs, g.dx, g.dy, g.dz, max_iter=max_iter, tol=tol, tol_mode=0)
        g.p[...] += p


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(3))
def test_host_projection_mirror_matches_compiled_reference(seed):
    """PressureProjection.project's host path (numpy divergence and face correction
    around any Solver) against the reference's own PressureProjection::project: the
    same pressure and corrected velocities, bit for bit."""
    from uaamg_b200.solver import Grid, PressureProjection
    rng = np.random.default_rng(300 + seed)
    nx, ny = [(20, 14), (31, 9), (16, 26)][seed]
    dx, dy = rng.uniform(0.05, 1.0, size=2)
    solid = (rng.random((ny + 2, nx + 2)) < 0.1).astype(np.uint8)
    u = rng.standard_normal((ny + 2, nx + 1))
    v = rng.standard_normal((ny + 1, nx + 2))
    dt = 0.01
    ur, vr, _, pr, _ = O.ref_project(solid, u, v, None, dx, dy, 1.0, dt, 40, 1e-9)
    g = Grid(nx, ny, nx * dx, ny * dy)
    g.dx, g.dy = dx, dy
    g.solid[...] = solid
    g.u[...], g.v[...] = u, v
    PressureProjection.project(g, dt, _OracleSolver(), 40, 1e-9)
    assert np.array_equal(g.p, pr)
    assert np.array_equal(g.u, ur) and np.array_equal(g.v, vr)


# --- variable-coefficient Laplacian (Grid::lap_*, pcg.cpp:35-46) -------------


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("case", [(40, 32, 0.5, 0.5, 0.35, 0.0), (57, 31, 0.3, 0.6, 0.2, 0.05),
                                  (16, 16, 0.5, 0.5, 0.6, 0.0)])
def test_smooth_cylinder_restatement_matches_compiled_reference(case):
    nx, ny, cx, cy, r, tw = case
    dx, dy = 1.0 / nx, 1.0 / ny
    rng = np.random.default_rng(nx)
    solid = np.zeros((ny + 2, nx + 2), np.uint8)
    solid[1:-1, 1:-1] = rng.random((ny, nx)) < 0.05
    s1, l1 = O.smooth_cylinder(solid, dx, dy, cx, cy, r, tw)
    s2, l2 = O.ref_smooth_cylinder(solid, dx, dy, cx, cy, r, tw)
    assert np.array_equal(s1, s2)
    for a, b in zip(l1, l2):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("seed", range(4))
def test_variable_pcg_restatement_matches_compiled_reference(seed):
    """Restated PCG with lap_* against PCG::solve on a grid with init_variable_lap:
    the reference's own SmoothCylinder coefficients (fixed iterations: that operator
    is non-symmetric) and random layered media (to convergence), bit for bit."""
    from uaamg_b200 import workloads as W
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(20, 70)), int(rng.integers(20, 70))
    dx, dy = 1.0 / nx, float(rng.uniform(0.5, 2.0)) / ny
    solid = np.zeros((ny + 2, nx + 2), np.uint8)
    if seed % 2:
        solid, lap = O.ref_smooth_cylinder(solid, dx, dy, 0.5, 0.5 * ny * dy, 0.4)
        max_iter, tol = 15, 0.0
    else:
        solid[1:-1, 1:-1] = rng.random((ny, nx)) < 0.03
        lap = W.layered_lap_2d(solid, dx, dy, float(rng.uniform(0.1, 0.8)))
        max_iter, tol = 300, 1e-9
    rhs = np.where(solid == 0, rng.standard_normal(solid.shape), 0.0)
    rhs[[0, -1], :] = 0.0
    rhs[:, [0, -1]] = 0.0
    p, n, _ = O.pcg_var(solid, lap, rhs, dx, dy, max_iter, tol, tol_mode=0)
    pr, nr = O.ref_pcg_var(solid, lap, rhs, dx, dy, max_iter, tol)
    assert np.array_equal(p, pr), f"max diff {np.abs(p - pr).max()}"
    assert nr in (n, n + 1)


def test_layered_coefficients_generator():
    """The bench's layered-medium generator equals the fixture script's formula and
    gives a symmetric operator with zero row sums (so a zero-mean RHS is solvable)."""
    import importlib.util
    from uaamg_b200 import workloads as W
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    nx, ny, dx, dy = 45, 29, 1e-3, 1.5e-3
    rng = np.random.default_rng(3)
    solid = np.zeros((ny + 2, nx + 2), np.uint8)
    solid[1:-1, 1:-1] = rng.random((ny, nx)) < 0.1
    lap = W.layered_lap_2d(solid, dx, dy, 0.5)
    for a, b in zip(lap, mg.layered_lap(solid, dx, dy, 0.5)):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=0)
    x = rng.standard_normal(solid.shape)
    y = rng.standard_normal(solid.shape)
    fl = (solid == 0)
    fl[[0, -1], :] = False
    fl[:, [0, -1]] = False
    x, y = np.where(fl, x, 0.0), np.where(fl, y, 0.0)
    ax, ay = O.matvec_var(solid, lap, x), O.matvec_var(solid, lap, y)
    assert abs(np.sum(y * ax) - np.sum(x * ay)) <= 1e-12 * np.sum(np.abs(y * ax))
    one = np.where(fl, 1.0, 0.0)
    assert np.abs(O.matvec_var(solid, lap, one)).max() <= 1e-9 * np.abs(lap[0][fl]).max()


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference CUDA solver (oracle/_ref) not built")
def test_reference_gpu_library_loads_and_exports():
    """The reference's own CUDA 3D solver, compiled for sm_100a behind ref_gpu_shim.cu,
    loads without a GPU and exports its entry point (it runs only under
    bench.py --impl reference --reference-gpu)."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libuaamg_ref_gpu.so"))
    assert hasattr(lib, "ref_gpu_pcg3d")


@pytest.mark.skipif(not O.have_ref(), reason="compiled reference (oracle/_ref) not present")
def test_restatement_matches_compiled_reference_property():
    """Property check over many small grids (2 to 13 cells an axis, so odd sizes,
    single-cell coarse levels and all-solid rows occur): the restated V-cycle and a
    fixed number of PCG iterations equal the compiled reference bit for bit, with
    and without variable coefficients in 2D."""
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    @settings(max_examples=120, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.too_slow])
    @given(dim=st.sampled_from([2, 3]), dims=st.lists(st.integers(2, 13), min_size=3, max_size=3),
           frac=st.sampled_from([0.0, 0.1, 0.3, 0.6]), seed=st.integers(0, 2**31 - 1),
           var=st.booleans())
    def check(dim, dims, frac, seed, var):
        rng = np.random.default_rng(seed)
        shape = tuple(d + 2 for d in dims[:dim])[::-1]
        solid = (rng.random(shape) < frac).astype(np.uint8)
        r = rng.standard_normal(shape)
        sp = rng.uniform(0.05, 2.0, size=3)
        z = O.Hierarchy(solid, *sp).vcycle(r)
        assert np.array_equal(z, O.ref_vcycle(solid, r, *sp))
        if dim == 2 and var:
            lap = tuple(rng.uniform(-2.0, 4.0, size=shape) for _ in range(3))
            p, _, _ = O.pcg_var(solid, lap, r, sp[0], sp[1], 8, 0.0, tol_mode=0)
            p_ref, _ = O.ref_pcg_var(solid, lap, r, sp[0], sp[1], 8, 0.0)
        else:
            p, _, _ = O.pcg(solid, r, *sp, max_iter=8, tol=0.0, tol_mode=0)
            p_ref, _ = O.ref_pcg(solid, r, *sp, max_iter=8, tol=0.0)
        assert np.array_equal(p, p_ref, equal_nan=True)

    check()
