"""Host-side logic without a GPU: the Python mirror of the reference surface
(grids, factory keys, pressure-projection pieces) against the oracle, and the
seeded workload generators."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_names, load_golden
from uaamg_b200 import Factory, Grid, Grid3D, PressureProjection, SolverKind, workloads


def test_grid_layouts_match_reference_sizes():
    g = Grid(8, 4, 2.0, 1.0)
    assert g.u.size == 9 * 6 and g.v.size == 10 * 5 and g.p.size == 10 * 6
    assert g.dx == 0.25 and g.dy == 0.25 and g.ip(3, 2) == 3 + 2 * 10
    g3 = Grid3D(4, 3, 2, 1.0, 1.0, 1.0)
    assert g3.u.size == 5 * 5 * 4 and g3.w.size == 6 * 5 * 3 and g3.p.size == 6 * 5 * 4
    assert g3.ip(1, 2, 1) == 1 + 2 * 6 + 1 * 6 * 5


@pytest.mark.parametrize("name", golden_names("project_"))
def test_projection_pieces_bit_exact_against_reference(name):
    gd = load_golden(name)
    s = gd["solid"]
    if s.ndim == 2:
        g = Grid(s.shape[1] - 2, s.shape[0] - 2, 1.0, 1.0)
    else:
        g = Grid3D(s.shape[2] - 2, s.shape[1] - 2, s.shape[0] - 2, 1.0, 1.0, 1.0)
        g.w = gd["w"].copy()
    g.dx, g.dy, g.dz = gd["dx"], gd["dy"], gd["dz"]
    g.solid[...] = s
    g.u, g.v = gd["u"].copy(), gd["v"].copy()
    rhs = PressureProjection.rhs(g, gd["dt"])
    w = gd["w"] if gd["w"].size else None
    rhs_o = O.divergence_rhs(s, gd["u"], gd["v"], w, gd["dx"], gd["dy"], gd["dz"], gd["dt"])
    assert np.array_equal(rhs, rhs_o)
    g.p = gd["p"].copy()
    PressureProjection.correct(g, gd["dt"])
    assert np.array_equal(g.u, gd["u_out"]) and np.array_equal(g.v, gd["v_out"])
    if w is not None:
        assert np.array_equal(g.w, gd["w_out"])


def test_factory_keys():
    assert {k.value for k in SolverKind} == {"cg_gpu", "pcg_uaamg_gpu", "pcg_uaamg_gpu_fp32",
                                            "pcg_uaamg_gpu_mixed"}
    with pytest.raises(ValueError):
        Factory.create("jacobi")


def test_workloads_are_deterministic_and_shaped():
    s1, r1 = workloads.spheres_3d(40, 36, 32, nspheres=4, rmin=3, rmax=6, seed=5)
    s2, r2 = workloads.spheres_3d(40, 36, 32, nspheres=4, rmin=3, rmax=6, seed=5)
    assert np.array_equal(s1, s2) and np.array_equal(r1, r2)
    assert s1.shape == (34, 38, 42) and 0 < s1.sum() < 40 * 36 * 32
    fluid = (s1 == 0)
    fluid[0, :, :] = fluid[-1, :, :] = fluid[:, 0, :] = fluid[:, -1, :] = False
    fluid[:, :, 0] = fluid[:, :, -1] = False
    assert abs(r1[fluid].mean()) < 1e-14 and np.all(r1[s1 == 1] == 0)
    s, u, v, rhs = workloads.obstacle_flow_2d(64, 32, 1e-3, 1.5e-3, 1e-3)
    assert u.shape == (34, 65) and v.shape == (33, 66)
    rhs_o = O.divergence_rhs(s, u, v, None, 1e-3, 1.5e-3, 1.0, 1e-3)
    assert np.array_equal(rhs, rhs_o)
    sb, rb = workloads.boxes(2, 128, 64, 0, 0.15, seed=11)
    frac = sb[1:-1, 1:-1].mean()
    assert 0.15 <= frac < 0.5


def test_variable_lap_mirror_and_solver_sync(monkeypatch):
    """Grid.init_variable_lap mirrors Grid::init_variable_lap (grid.cpp:12-17), and
    GpuUAAMGPCG sends the grid's lap_* arrays on every call (PCG::solve reads them
    each time), clears them once they are gone and re-sends after a new mask."""
    import uaamg_b200.solver as S

    g = Grid(6, 4, 1.0, 1.0)
    assert not g.has_variable_lap()
    g.init_variable_lap()
    assert g.has_variable_lap() and g.lap_diag.shape == g.p.shape
    assert not g.lap_diag.any() and not g.lap_off_x.any() and not g.lap_off_y.any()

    calls = []

    class FakeHandle:
        options = staticmethod(S.Handle.options)

        def __init__(self, device=0):
            pass

        def set_problem(self, solid, dx, dy, dz=1.0):
            calls.append("problem")

        def set_variable_laplacian(self, *arrs):
            calls.append("lap" if arrs else "clear")

        def solve(self, rhs, p, opts, strict=False):
            calls.append("solve")
            return None

    monkeypatch.setattr(S, "Handle", FakeHandle)
    solver = S.GpuUAAMGPCG("fp64")
    rhs = np.zeros(g.p.shape)
    solver.solve(g, rhs, 10, 1e-6)
    solver.solve(g, rhs, 10, 1e-6)
    assert calls == ["problem", "lap", "solve", "lap", "solve"]
    calls.clear()
    g.lap_diag = g.lap_off_x = g.lap_off_y = np.zeros(0)
    solver.solve(g, rhs, 10, 1e-6)
    solver.solve(g, rhs, 10, 1e-6)
    assert calls == ["clear", "solve", "solve"]
    calls.clear()
    g.init_variable_lap()
    g.solid[2, 3] = 1
    solver.solve(g, rhs, 10, 1e-6)
    assert calls == ["problem", "lap", "solve"]
