"""Device-side pressure projection (uaamg_project / uaamg_project_device) against the
reference's host steps on identical inputs: the oracle's divergence (pressure.cpp:10-14,
fvc::divergence) fed to the same GPU solve, and the oracle's face correction
(pressure.cpp:21-32, pressure_3d.cpp:21-39) of that pressure.  The device divergence
and correction are the reference's FP64 expressions, so pressure and velocities must
match bit for bit."""
import numpy as np
import pytest

from uaamg_b200 import workloads
from uaamg_b200.solver import Grid, Grid3D, Handle, Factory, PressureProjection

import oracle as O

pytestmark = pytest.mark.gpu


def _case(dim, seed):
    if dim == 2:
        nx, ny = 192, 128
        dx, dy, dz = 1e-3, 1.5e-3, 1.0
        s, u, v, _ = workloads.obstacle_flow_2d(nx, ny, dx, dy, 1e-3, 8, seed)
        return s, u, v, None, dx, dy, dz
    n = 40
    h = 1.0 / n
    s, u, v, w, _ = workloads.obstacle_flow_3d(n, n, n, h, h, h, 1e-3, 4, seed)
    return s, u, v, w, h, h, h


def _host_steps(hd, s, u, v, w, dx, dy, dz, dt, opts):
    rhs = O.divergence_rhs(s, u, v, w, dx, dy, dz, dt)
    p = np.zeros_like(rhs)
    hd.solve(rhs, p, opts)
    uo, vo, wo = O.correct_velocity(s, p, dt, u, v, w, dx, dy, dz)
    return p, uo, vo, wo


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("dim", [2, 3])
def test_project_matches_host_divergence_solve_and_correction(dim, prec):
    s, u, v, w, dx, dy, dz = _case(dim, 31 + dim)
    dt = 1e-3
    hd = Handle(0)
    hd.set_problem(s, dx, dy, dz)
    opts = hd.options(prec, 1e-8 if prec == "fp64" else 1e-6, 500, "rel")
    p_ref, u_ref, v_ref, w_ref = _host_steps(hd, s, u, v, w, dx, dy, dz, dt, opts)
    ug, vg = u.copy(), v.copy()
    wg = w.copy() if w is not None else None
    p = np.full(s.shape, 7.0)  # overwritten: the projection starts from p = 0
    st = hd.project(ug, vg, wg, p, dt, opts)
    assert st.status == 0
    assert np.array_equal(p, p_ref)
    assert np.array_equal(ug, u_ref) and np.array_equal(vg, v_ref)
    if dim == 3:
        assert np.array_equal(wg, w_ref)
    # the corrected field's divergence is the constant that Neumann walls cannot
    # remove (the net flux through the domain walls), up to the solve tolerance
    fl = np.zeros(s.shape, bool)
    fl[(slice(1, -1),) * s.ndim] = True
    fl &= s == 0
    div = O.divergence_rhs(s, ug, vg, wg, dx, dy, dz, dt)[fl]
    div0 = O.divergence_rhs(s, u, v, w, dx, dy, dz, dt)[fl]
    assert np.linalg.norm(div - div.mean()) <= 1e-4 * np.linalg.norm(div0 - div0.mean())
    hd.close()


def test_project_device_equals_host_array_call():
    torch = pytest.importorskip("torch")
    s, u, v, w, dx, dy, dz = _case(3, 7)
    dt = 1e-3
    hd = Handle(0)
    hd.set_problem(s, dx, dy, dz)
    opts = hd.options("mixed", 1e-6, 500, "rel")
    uh, vh, wh, ph = u.copy(), v.copy(), w.copy(), np.zeros(s.shape)
    hd.project(uh, vh, wh, ph, dt, opts)
    du, dv, dw = (torch.from_numpy(a.copy()).cuda() for a in (u, v, w))
    dp = torch.zeros(s.shape, dtype=torch.float64, device="cuda")
    hd.project_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr(), dp.data_ptr(), dt, opts)
    torch.cuda.synchronize()
    assert np.array_equal(dp.cpu().numpy(), ph)
    assert np.array_equal(du.cpu().numpy(), uh) and np.array_equal(dv.cpu().numpy(), vh)
    assert np.array_equal(dw.cpu().numpy(), wh)
    hd.close()


def test_pressure_projection_uses_the_device_path():
    """PressureProjection.project with a GPU solver runs divergence, solve and
    correction on the device; the host steps give the same fields."""
    s, u, v, _, dx, dy, _ = _case(2, 11)
    ny, nx = s.shape[0] - 2, s.shape[1] - 2
    dt = 1e-3
    results = []
    for on_device in (True, False):
        g = Grid(nx, ny, nx * dx, ny * dy)
        g.solid[...] = s
        g.u[...] = u
        g.v[...] = v
        solver = Factory.create("pcg_uaamg_gpu")
        PressureProjection.project(g, dt, solver, 500, 1e-10, on_device=on_device)
        results.append((g.p.copy(), g.u.copy(), g.v.copy()))
    (p1, u1, v1), (p2, u2, v2) = results
    assert np.array_equal(p1, p2) and np.array_equal(u1, u2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_static_pressure_matches_reference_rhs_and_solve(prec):
    """recoverStaticPressure (pressure.cpp:35-66): the device right-hand side is the
    reference's, so the pressure equals the same solve of the oracle's RHS bit for bit;
    the host- and device-array forms agree; 3D is rejected as in the reference."""
    torch = pytest.importorskip("torch")
    s, u, v, _, dx, dy, dz = _case(2, 23)
    hd = Handle(0)
    hd.set_problem(s, dx, dy, dz)
    opts = hd.options(prec, 1e-8 if prec == "fp64" else 1e-6, 500, "rel")
    rhs = O.static_rhs(s, u, v, dx, dy)
    p_ref = np.zeros_like(rhs)
    hd.solve(rhs, p_ref, opts)
    p = np.full(s.shape, 3.0)  # overwritten: the recovery starts from p = 0
    st = hd.static_pressure(u.copy(), v.copy(), p, opts)
    assert st.status == 0 and np.array_equal(p, p_ref)
    du, dv = torch.from_numpy(u.copy()).cuda(), torch.from_numpy(v.copy()).cuda()
    dp = torch.zeros(s.shape, dtype=torch.float64, device="cuda")
    hd.static_pressure_device(du.data_ptr(), dv.data_ptr(), dp.data_ptr(), opts)
    torch.cuda.synchronize()
    assert np.array_equal(dp.cpu().numpy(), p_ref)
    hd.close()
    s3, u3, v3, w3, h3, _, _ = _case(3, 5)
    hd3 = Handle(0)
    hd3.set_problem(s3, h3, h3, h3)
    with pytest.raises(Exception):
        hd3.static_pressure_device(1, 1, 1, hd3.options("fp64"))
    hd3.close()
