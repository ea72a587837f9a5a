"""Generates the golden fixtures in this folder from the REFERENCE ITSELF.

Each fixture is the output of the reference's own CPU code (PCG / PCG3D with
UAAMGPreconditioner[3D], PressureProjection::project), compiled unchanged from
the reference tree by ``oracle/Makefile`` into ``oracle/_ref/libuaamg_ref.so``,
on small deterministic inputs.  The case shapes mirror the reference's own GPU
parity tests:

  vcycle_2d_uniform   src/solver/cuda/test_cuda_uaamg.cu:19-60   (32x16, r = 1)
  pcg_2d_gauss        src/solver/cuda/test_cuda_uaamg.cu:63-130  (32x16, 50 it, tol 1e-10)
  vcycle_2d_cylinder  src/solver/cuda/test_cuda_uaamg.cu:134-185 (64x16, Lx = 4, R = 0.1)
  vcycle_3d_uniform   src/solver/cuda/test_cuda_uaamg_3d.cu:15-58 (16x8x4)
  pcg_3d_gauss        src/solver/cuda/test_cuda_uaamg_3d.cu:60-96 (30 it, tol 1e-10)
plus random-solid / odd-size / anisotropic cases and a 2D and 3D projection, and the
variable-coefficient branch of PCG::solve (pcg.cpp:35-46, Grid::init_variable_lap):

  varlap_2d_smooth_cylinder  the coefficients of the reference's own
                             SmoothCylinder::applyToLaplacian (cylinder_model.cpp:50-71)
  varlap_2d_layered          a layered medium (layered_lap below)

Run from the repository root after ``make -C oracle ref``:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def _interior(shape):
    m = np.zeros(shape, bool)
    if len(shape) == 2:
        m[1:-1, 1:-1] = True
    else:
        m[1:-1, 1:-1, 1:-1] = True
    return m


def _gauss(shape, c=0.01):
    """exp(-c*|x - centre|^2) in cell-index units on the interior (the
    reference tests' RHS), 0 on ghosts."""
    if len(shape) == 2:
        ny, nx = shape[0] - 2, shape[1] - 2
        j, i = np.meshgrid(np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
        d2 = (i - nx / 2.0) ** 2 + (j - ny / 2.0) ** 2
    else:
        nz, ny, nx = (s - 2 for s in shape)
        k, j, i = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2),
                              indexing="ij")
        d2 = (i - nx / 2.0) ** 2 + (j - ny / 2.0) ** 2 + (k - nz / 2.0) ** 2
    return np.where(_interior(shape), np.exp(-c * d2), 0.0)


def _cylinder(nx, ny, dx, dy, cx, cy, R):
    s = np.zeros((ny + 2, nx + 2), np.uint8)
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            x, y = (i - 0.5) * dx, (j - 0.5) * dy
            if np.sqrt((x - cx) ** 2 + (y - cy) ** 2) < R:
                s[j, i] = 1
    return s


def _random_solid(shape, frac, rng):
    s = (rng.random(shape) < frac).astype(np.uint8)
    s[~_interior(shape)] = 0
    return s


def layered_lap(solid, dx, dy, amp):
    """lap_diag / lap_off_x / lap_off_y of a layered medium: x conductivity
    1 + amp sin(2 pi (j - 1/2) / ny) by row, y conductivity 1 + amp cos(2 pi (i - 1/2) / nx)
    by column (a symmetric operator with zero row sums); solid cells d = 1e15."""
    ny, nx = solid.shape[0] - 2, solid.shape[1] - 2
    j, i = np.meshgrid(np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
    kx = 1.0 + amp * np.sin(2.0 * np.pi * (j - 0.5) / ny)
    ky = 1.0 + amp * np.cos(2.0 * np.pi * (i - 0.5) / nx)
    fl = _interior(solid.shape) & (solid == 0)
    ix, iy = 1.0 / (dx * dx), 1.0 / (dy * dy)
    ox = np.where(fl, -kx * ix, 0.0)
    oy = np.where(fl, -ky * iy, 0.0)
    d = np.where(fl, 2.0 * kx * ix + 2.0 * ky * iy, 0.0)
    d[_interior(solid.shape) & (solid != 0)] = 1e15
    return d, ox, oy


def cases():
    rng = np.random.default_rng(20260101)
    out = []
    # --- mirrors of the reference's GPU parity tests -------------------------
    sh = (16 + 2, 32 + 2)
    out.append(dict(name="vcycle_2d_uniform", kind="vcycle", solid=np.zeros(sh, np.uint8),
                    r=np.where(_interior(sh), 1.0, 0.0), dx=1 / 32, dy=1 / 16, dz=1.0))
    out.append(dict(name="pcg_2d_gauss", kind="pcg", solid=np.zeros(sh, np.uint8),
                    r=_gauss(sh), dx=1 / 32, dy=1 / 16, dz=1.0, max_iter=50, tol=1e-10))
    s = _cylinder(64, 16, 4.0 / 64, 1.0 / 16, 1.0, 0.5, 0.1)
    out.append(dict(name="vcycle_2d_cylinder", kind="vcycle", solid=s,
                    r=np.where(_interior(s.shape) & (s == 0), 1.0, 0.0), dx=4.0 / 64,
                    dy=1.0 / 16, dz=1.0))
    sh3 = (4 + 2, 8 + 2, 16 + 2)
    out.append(dict(name="vcycle_3d_uniform", kind="vcycle", solid=np.zeros(sh3, np.uint8),
                    r=np.where(_interior(sh3), 1.0, 0.0), dx=1 / 16, dy=1 / 8, dz=1 / 4))
    out.append(dict(name="pcg_3d_gauss", kind="pcg", solid=np.zeros(sh3, np.uint8),
                    r=_gauss(sh3), dx=1.0 / 16, dy=1.0 / 8, dz=1.0 / 4, max_iter=30, tol=1e-10))
    # --- random solids, odd and anisotropic shapes ---------------------------
    for name, shape, sp, frac, kind in [
        ("vcycle_2d_odd_rand", (37 + 2, 53 + 2), (1e-3, 1.5e-3, 1.0), 0.15, "vcycle"),
        ("pcg_2d_odd_rand", (37 + 2, 53 + 2), (1e-3, 1.5e-3, 1.0), 0.15, "pcg"),
        ("vcycle_3d_odd_rand", (11 + 2, 19 + 2, 23 + 2), (0.5, 0.25, 0.125), 0.2, "vcycle"),
        ("pcg_3d_odd_rand", (11 + 2, 19 + 2, 23 + 2), (0.5, 0.25, 0.125), 0.2, "pcg"),
        ("pcg_3d_dense_solid", (12 + 2, 12 + 2, 12 + 2), (1 / 12, 1 / 12, 1 / 12), 0.45, "pcg"),
        ("vcycle_3d_tiny", (3 + 2, 3 + 2, 3 + 2), (1.0, 1.0, 1.0), 0.0, "vcycle"),
        ("pcg_2d_tiny", (2 + 2, 2 + 2), (1.0, 1.0, 1.0), 0.0, "pcg"),
    ]:
        s = _random_solid(shape, frac, rng)
        r = np.where(_interior(shape), rng.standard_normal(shape), 0.0)
        c = dict(name=name, kind=kind, solid=s, r=r, dx=sp[0], dy=sp[1], dz=sp[2])
        if kind == "pcg":
            # A random mask leaves isolated fluid pockets, so a random RHS has no
            # solution; rhs = -A x_true is always compatible (lap(p) = rhs).  The
            # solution is still defined only up to a constant per pocket, so these
            # cases compare a fixed number of iterations (tol = 0), as the
            # reference's own GPU tests do (test_cuda_uaamg_3d.cu:68-94).  On such
            # masks the reference's own result moves by ~1e-7 after 25 iterations
            # when its RHS is perturbed by 1e-15, so 10 iterations are compared,
            # where it is stable to ~1e-11.
            x_true = np.where(_interior(shape) & (s == 0), rng.standard_normal(shape), 0.0)
            c["r"] = -O.matvec(s, x_true, sp[0], sp[1], sp[2])
            c.update(max_iter=10, tol=0.0)
        out.append(c)
    # --- pressure projection --------------------------------------------------
    nx, ny, dx, dy, dt = 48, 24, 1.0 / 48, 0.5 / 24, 1e-2
    s = _cylinder(nx, ny, dx, dy, 0.25, 0.25, 0.06)
    u = 1.0 + 0.1 * rng.standard_normal((ny + 2, nx + 1))
    v = 0.1 * rng.standard_normal((ny + 1, nx + 2))
    out.append(dict(name="project_2d", kind="project", solid=s, u=u, v=v, w=None, dx=dx, dy=dy,
                    dz=1.0, dt=dt, max_iter=200, tol=1e-5))
    nx, ny, nz, h = 12, 10, 8, 0.1
    s = _random_solid((nz + 2, ny + 2, nx + 2), 0.1, rng)
    u = 1.0 + 0.1 * rng.standard_normal((nz + 2, ny + 2, nx + 1))
    v = 0.1 * rng.standard_normal((nz + 2, ny + 1, nx + 2))
    w = 0.1 * rng.standard_normal((nz + 1, ny + 2, nx + 2))
    out.append(dict(name="project_3d", kind="project", solid=s, u=u, v=v, w=w, dx=h, dy=h, dz=h,
                    dt=dt, max_iter=200, tol=1e-5))
    # --- variable-coefficient Laplacian (2D) ---------------------------------
    # The reference's SmoothCylinder takes the solid fraction as 1 OUTSIDE the disk
    # (cylinder_model.cpp:45-48), so the fluid is the disk itself, and its per-cell
    # off-diagonals make the operator non-symmetric: CG on it stalls, so a fixed
    # number of iterations is compared (tol = 0).
    nx, ny, dx, dy = 40, 32, 1.0 / 40, 1.0 / 32
    s, (d, ox, oy) = O.ref_smooth_cylinder(np.zeros((ny + 2, nx + 2), np.uint8), dx, dy,
                                           0.5, 0.5, 0.35)
    r = np.where(_interior(s.shape) & (s == 0), rng.standard_normal(s.shape), 0.0)
    out.append(dict(name="varlap_2d_smooth_cylinder", kind="pcg_var", solid=s, r=r, lap_diag=d,
                    lap_off_x=ox, lap_off_y=oy, dx=dx, dy=dy, dz=1.0, max_iter=12, tol=0.0))
    nx, ny, dx, dy = 53, 37, 1e-3, 1.5e-3
    s = _cylinder(nx, ny, dx, dy, 0.25 * nx * dx, 0.5 * ny * dy, 0.1 * ny * dy)
    d, ox, oy = layered_lap(s, dx, dy, 0.5)
    r = np.where(_interior(s.shape) & (s == 0), _gauss(s.shape), 0.0)
    out.append(dict(name="varlap_2d_layered", kind="pcg_var", solid=s, r=r, lap_diag=d,
                    lap_off_x=ox, lap_off_y=oy, dx=dx, dy=dy, dz=1.0, max_iter=200, tol=1e-9))
    return out


def main():
    for c in cases():
        name = c.pop("name")
        if c["kind"] == "vcycle":
            c["z"] = O.ref_vcycle(c["solid"], c["r"], c["dx"], c["dy"], c["dz"])
        elif c["kind"] == "pcg_var":
            lap = (c["lap_diag"], c["lap_off_x"], c["lap_off_y"])
            p, n = O.ref_pcg_var(c["solid"], lap, c["r"], c["dx"], c["dy"], c["max_iter"],
                                 c["tol"])
            c["p"] = p
            c["applies"] = n
        elif c["kind"] == "pcg":
            p, n = O.ref_pcg(c["solid"], c["r"], c["dx"], c["dy"], c["dz"], c["max_iter"], c["tol"])
            c["p"] = p
            c["applies"] = n
        else:
            u, v, w, p, n = O.ref_project(c["solid"], c["u"], c["v"], c["w"], c["dx"], c["dy"],
                                          c["dz"], c["dt"], c["max_iter"], c["tol"])
            c.update(u_out=u, v_out=v, p=p, applies=n)
            if w is not None:
                c["w_out"] = w
        arrays = {k: (np.asarray(v) if v is not None else np.zeros(0)) for k, v in c.items()}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, {k: getattr(v, "shape", v) for k, v in arrays.items()})


if __name__ == "__main__":
    main()
