"""The variable-coefficient Laplacian of PCG::solve (Grid::lap_diag / lap_off_x /
lap_off_y, src/solver/pcg.cpp:35-46; include/core/grid.h:23-31) on the GPU, through
the C-ABI (uaamg_set_variable_laplacian): against the reference's own outputs (the
varlap_* golden fixtures) and the oracle.

Tolerances, as for the uniform operator:
  FP64          |p - p_ref| <= 1e-10 * max(1, |p_ref|)
  mixed         FP64 true residual <= 1e-6 and relative L2 <= 1e-5 of the
                fluid-mean-removed pressure against the FP64 solution
  plain FP32    relative L2 <= 1e-2 (its solution is stored in FP32)
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden_names, load_golden
from uaamg_b200 import _capi
from uaamg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def fluid_interior(solid):
    m = np.zeros(solid.shape, bool)
    m[1:-1, 1:-1] = solid[1:-1, 1:-1] == 0
    return m


def meanfree(p, solid):
    m = fluid_interior(solid)
    out = np.zeros_like(p)
    out[m] = p[m] - p[m].mean()
    return out


def rel_l2_meanfree(a, b, solid):
    x, y = meanfree(a, solid), meanfree(b, solid)
    return np.linalg.norm(x - y) / np.linalg.norm(y)


def lap_of(g):
    return g["lap_diag"], g["lap_off_x"], g["lap_off_y"]


@pytest.fixture(params=["fused", "sweeps", "fused_all", "march", "march_all"])
def vkernels(request, handle):
    handle.set_vcycle_kernels({"fused": 0, "sweeps": 1, "fused_all": 2, "march": 3,
                               "march_all": 4}[request.param])
    yield request.param
    handle.set_vcycle_kernels(0)


def layered_case(seed, nx=160, ny=96, amp=0.5):
    """A 2D layered-medium problem with random solid boxes and a smoothed RHS."""
    solid, rhs = W.boxes(2, nx, ny, 0, 0.1, seed=seed)
    from scipy import ndimage
    fl = fluid_interior(solid)
    lab, n = ndimage.label(fl)
    if n > 1:  # one connected fluid region: the constant is the only null vector
        sizes = ndimage.sum(fl, lab, index=np.arange(1, n + 1))
        keep = 1 + int(np.argmax(sizes))
        solid = np.where(fl & (lab != keep), 1, solid).astype(np.uint8)
        rhs = np.where(solid == 0, rhs, 0.0)
    dx, dy = 1e-3, 1.5e-3
    return solid, rhs, dx, dy, W.layered_lap_2d(solid, dx, dy, amp)


@pytest.mark.parametrize("name", golden_names("varlap_"))
def test_varlap_fp64_vs_reference(handle, vkernels, name):
    g = load_golden(name)
    handle.set_problem(g["solid"], g["dx"], g["dy"])
    handle.set_variable_laplacian(*lap_of(g))
    p = np.zeros_like(g["r"])
    st = handle.solve(g["r"], p, handle.options("fp64", g["tol"], g["max_iter"], "abs"))
    ref = g["p"]
    d = meanfree(p, g["solid"]) - meanfree(ref, g["solid"])
    assert np.abs(d).max() <= 1e-10 * max(1.0, np.abs(ref).max())
    assert abs((st.iterations + 1) - g["applies"]) <= 1 or st.iterations == g["max_iter"]


@pytest.mark.parametrize("seed", range(4))
def test_varlap_fp64_vs_oracle(handle, seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(40, 200)), int(rng.integers(40, 200))
    solid, rhs, dx, dy, lap = layered_case(seed, nx, ny, float(rng.uniform(0.1, 0.8)))
    handle.set_problem(solid, dx, dy)
    handle.set_variable_laplacian(*lap)
    p = np.zeros_like(rhs)
    handle.solve(rhs, p, handle.options("fp64", 1e-11, 600, "rel"))
    po, _, _ = O.pcg_var(solid, lap, rhs, dx, dy, max_iter=600, tol=1e-11, tol_mode=1)
    assert rel_l2_meanfree(p, po, solid) <= 1e-8
    # the exit diagnostics use the same operator
    res, bn = O.true_residual_var(solid, lap, rhs, p)
    assert res / bn <= 1e-10


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
@pytest.mark.parametrize("seed", range(3))
def test_varlap_reduced_precision_vs_fp64(handle, prec, seed):
    solid, rhs, dx, dy, lap = layered_case(seed + 7)
    handle.set_problem(solid, dx, dy)
    handle.set_variable_laplacian(*lap)
    p64 = np.zeros_like(rhs)
    handle.solve(rhs, p64, handle.options("fp64", 1e-12, 400, "rel"), strict=True)
    p = np.zeros_like(rhs)
    st = handle.solve(rhs, p, handle.options(prec, 1e-6, 400, "rel"))
    res, bn = O.true_residual_var(solid, lap, rhs, p)
    if prec == "mixed":
        assert st.status == 0 and res / bn <= 1e-6
        assert abs(st.rel_residual - res / bn) <= 1e-3 * res / bn
        assert rel_l2_meanfree(p, p64, solid) <= 1e-5
    else:
        assert rel_l2_meanfree(p, p64, solid) <= 1e-2


def test_varlap_warm_start(handle):
    solid, rhs, dx, dy, lap = layered_case(3)
    handle.set_problem(solid, dx, dy)
    handle.set_variable_laplacian(*lap)
    p = np.zeros_like(rhs)
    cold = handle.solve(rhs, p, handle.options("mixed", 1e-6, 400, "rel"), strict=True)
    rhs2 = rhs * (1.0 + 1e-3 * np.cos(np.arange(rhs.size).reshape(rhs.shape)))
    warm = handle.solve(rhs2, p, handle.options("mixed", 1e-6, 400, "rel", warm_start=True),
                        strict=True)
    res, bn = O.true_residual_var(solid, lap, rhs2, p)
    assert res / bn <= 1e-6
    assert warm.iterations < cold.iterations


def test_varlap_set_clear_and_new_problem(handle):
    solid, rhs, dx, dy, lap = layered_case(5, 96, 64)
    opts = handle.options("fp64", 1e-10, 300, "rel")
    handle.set_problem(solid, dx, dy)
    pu = np.zeros_like(rhs)
    handle.solve(rhs, pu, opts)
    # the uniform operator written as coefficients gives the uniform solution
    fl = fluid_interior(solid)
    ix, iy = 1.0 / dx**2, 1.0 / dy**2
    uni = (np.where(fl, 2 * ix + 2 * iy, 0.0), np.where(fl, -ix, 0.0), np.where(fl, -iy, 0.0))
    handle.set_variable_laplacian(*uni)
    pv = np.zeros_like(rhs)
    handle.solve(rhs, pv, opts)
    assert rel_l2_meanfree(pv, pu, solid) <= 1e-9
    handle.set_variable_laplacian(*lap)
    pl = np.zeros_like(rhs)
    handle.solve(rhs, pl, opts)
    assert rel_l2_meanfree(pl, pu, solid) > 1e-3
    # cleared: back to the uniform operator, bit for bit
    handle.set_variable_laplacian()
    p2 = np.zeros_like(rhs)
    handle.solve(rhs, p2, opts)
    assert np.array_equal(p2, pu)
    # a new problem starts with the uniform operator
    handle.set_variable_laplacian(*lap)
    handle.set_problem(solid, dx, dy)
    p3 = np.zeros_like(rhs)
    handle.solve(rhs, p3, opts)
    assert np.array_equal(p3, pu)


def test_varlap_rejects_3d_and_partial_arrays(handle):
    solid3 = np.zeros((10, 10, 10), np.uint8)
    handle.set_problem(solid3, 0.1, 0.1, 0.1)
    z3 = np.zeros((10, 10, 10))
    with pytest.raises(_capi.UaamgError):
        handle.set_variable_laplacian(z3, z3, z3)
    solid2 = np.zeros((10, 12), np.uint8)
    handle.set_problem(solid2, 0.1, 0.1)
    z = np.zeros((10, 12))
    with pytest.raises(_capi.UaamgError):
        handle.set_variable_laplacian(z, None, z)


def test_varlap_solver_surface_and_projection():
    """Grid.init_variable_lap + GpuUAAMGPCG (the Solver drop-in) against the
    reference's output, and the device projection with that operator."""
    from uaamg_b200 import GpuUAAMGPCG, Grid, PressureProjection
    gd = load_golden("varlap_2d_layered")
    s = gd["solid"]
    ny, nx = s.shape[0] - 2, s.shape[1] - 2
    g = Grid(nx, ny, nx * gd["dx"], ny * gd["dy"])
    g.dx, g.dy = gd["dx"], gd["dy"]
    g.solid[:] = s
    g.init_variable_lap()
    g.lap_diag[:], g.lap_off_x[:], g.lap_off_y[:] = lap_of(gd)
    solver = GpuUAAMGPCG("fp64", "abs")
    solver.solve(g, gd["r"], gd["max_iter"], gd["tol"])
    d = meanfree(g.p, s) - meanfree(gd["p"], s)
    assert np.abs(d).max() <= 1e-10 * max(1.0, np.abs(gd["p"]).max())

    # projection: the device path (divergence, solve, correction) and the host
    # mirror agree, and the pressure is the variable-operator solution
    rng = np.random.default_rng(0)
    u0 = 1.0 + 0.1 * rng.standard_normal(g.u.shape)
    v0 = 0.1 * rng.standard_normal(g.v.shape)
    dt = 1e-3
    solver = GpuUAAMGPCG("fp64", "rel")
    g.u[:], g.v[:], g.p[:] = u0, v0, 0.0
    PressureProjection.project(g, dt, solver, 400, 1e-10, on_device=True)
    pd, ud, vd = g.p.copy(), g.u.copy(), g.v.copy()
    g.u[:], g.v[:], g.p[:] = u0, v0, 0.0
    PressureProjection.project(g, dt, solver, 400, 1e-10, on_device=False)
    scale = max(1.0, np.abs(g.p).max())
    assert np.abs(pd - g.p).max() <= 1e-10 * scale
    assert np.abs(ud - g.u).max() <= 1e-10 * max(1.0, np.abs(g.u).max())
    assert np.abs(vd - g.v).max() <= 1e-10 * max(1.0, np.abs(g.v).max())
    rhs = O.divergence_rhs(s, u0, v0, None, g.dx, g.dy, 1.0, dt)
    po, _, _ = O.pcg_var(s, lap_of(gd), rhs, g.dx, g.dy, 400, 1e-10, tol_mode=1)
    assert rel_l2_meanfree(pd, po, s) <= 1e-8


def test_varlap_new_contents_reach_every_precision(handle):
    """Re-sending different coefficients (same device buffers) is seen by the FP32
    forms too, whose converted copies are refreshed."""
    solid, rhs, dx, dy, lap_a = layered_case(11, 128, 80, 0.3)
    lap_b = W.layered_lap_2d(solid, dx, dy, 0.7)
    handle.set_problem(solid, dx, dy)
    for lap in (lap_a, lap_b, lap_a):
        handle.set_variable_laplacian(*lap)
        for prec in ("mixed", "fp32"):
            p = np.zeros_like(rhs)
            st = handle.solve(rhs, p, handle.options(prec, 1e-6, 400, "rel"))
            res, bn = O.true_residual_var(solid, lap, rhs, p)
            if prec == "mixed":
                assert st.status == 0 and res / bn <= 1e-6
            else:
                assert res / bn <= 1e-3
