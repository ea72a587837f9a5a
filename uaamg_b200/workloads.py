"""Seeded synthetic workloads (ctypes over libuaamg_workloads.so, host code).

Every generator returns padded numpy arrays in the reference's memory order
(C-order shape (nz+2, ny+2, nx+2) / (ny+2, nx+2)).  The named workloads:

* ``spheres_256``: 256^3, h = 1/256, 32 solid spheres with radius U[8, 24] cells,
  RHS = N(0,1) noise blurred with a sigma = 4 cell Gaussian (+-16 taps), zero at
  solids, zero fluid mean; seed 20260303.
* ``obstacle_2d``: 2048 x 1024, dx = 1e-3, dy = 1.5e-3, disk of radius 0.05*Ly at
  (0.25 Lx, 0.5 Ly); u = 1 + Fourier modes |k| <= 16 with N(0,1)/|k|^2
  amplitudes, v = modes; RHS = div(u)/dt, dt = 1e-3; seed 20260202.
* ``layered_2d``: the obstacle_2d grid, mask and RHS, solved with the 2D
  variable-coefficient operator (lap_diag / lap_off_x / lap_off_y) of a layered
  medium: x conductivity 1 + 0.5 sin(2 pi y / Ly), y conductivity 1 + 0.5 cos(2 pi x / Lx).
* ``batch96``: 64 2D problems with nx, ny uniform on {64, 128, ..., 1024} and 32 3D
  problems with nx, ny, nz uniform on {32, 48, 64, 96, 128}; h = 1/max(dims);
  random solid boxes up to a coverage U[0, 0.2]; smoothed-noise RHS; seed 20260404.
* ``serve10k``: 500 simulation ids x 20 steps; 70 % 2D n x n with
  n = clip(round(exp(N(ln 384, 0.5))), 64, 2048), 30 % 3D n^3 with
  n = clip(round(exp(N(ln 96, 0.4))), 32, 256); obstacle disk / sphere; RHS of step
  t = rhs0 + (t/20) rhs1 (wl_serve_fields); seed 20260505.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "libuaamg_workloads.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            from . import build as _b
            _b.build_workloads()
        L = C.CDLL(_LIB)
        p, i, d, u64 = C.c_void_p, C.c_int, C.c_double, C.c_uint64
        L.wl_spheres_3d.argtypes = [i, i, i, i, d, d, u64, d, i, p, p]
        L.wl_spheres_3d.restype = C.c_long
        L.wl_boxes.argtypes = [i, i, i, i, d, u64, d, i, p, p]
        L.wl_boxes.restype = C.c_long
        L.wl_obstacle_flow_2d.argtypes = [i, i, d, d, d, i, u64, d, p, p, p, p]
        L.wl_obstacle_flow_2d.restype = C.c_long
        L.wl_obstacle_flow_3d.argtypes = [i, i, i, d, d, d, d, i, u64, d, p, p, p, p, p]
        L.wl_obstacle_flow_3d.restype = C.c_long
        L.wl_layered_lap_2d.argtypes = [i, i, d, d, d, p, p, p, p]
        L.wl_layered_lap_2d.restype = C.c_long
        L.wl_serve_fields.argtypes = [i, i, i, u64, p, p, p]
        L.wl_serve_fields.restype = C.c_long
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def spheres_3d(nx, ny, nz, nspheres=32, rmin=8.0, rmax=24.0, seed=20260303, sigma=4.0,
               trunc=16):
    solid = np.zeros((nz + 2, ny + 2, nx + 2), np.uint8)
    rhs = np.zeros((nz + 2, ny + 2, nx + 2))
    _load().wl_spheres_3d(nx, ny, nz, nspheres, rmin, rmax, seed, sigma, trunc, _p(solid), _p(rhs))
    return solid, rhs


def boxes(dim, nx, ny, nz, coverage, seed, sigma=4.0, trunc=16):
    shape = (nz + 2, ny + 2, nx + 2) if dim == 3 else (ny + 2, nx + 2)
    solid = np.zeros(shape, np.uint8)
    rhs = np.zeros(shape)
    _load().wl_boxes(dim, nx, ny, nz if dim == 3 else 0, coverage, seed, sigma, trunc, _p(solid),
                     _p(rhs))
    return solid, rhs


def obstacle_flow_2d(nx, ny, dx, dy, dt=1e-3, kmax=16, seed=20260202, t=0.0):
    solid = np.zeros((ny + 2, nx + 2), np.uint8)
    u = np.zeros((ny + 2, nx + 1))
    v = np.zeros((ny + 1, nx + 2))
    rhs = np.zeros((ny + 2, nx + 2))
    _load().wl_obstacle_flow_2d(nx, ny, dx, dy, dt, kmax, seed, t, _p(solid), _p(u), _p(v), _p(rhs))
    return solid, u, v, rhs


def obstacle_flow_3d(nx, ny, nz, dx, dy, dz, dt=1e-3, kmax=8, seed=20260505, t=0.0):
    solid = np.zeros((nz + 2, ny + 2, nx + 2), np.uint8)
    u = np.zeros((nz + 2, ny + 2, nx + 1))
    v = np.zeros((nz + 2, ny + 1, nx + 2))
    w = np.zeros((nz + 1, ny + 2, nx + 2))
    rhs = np.zeros((nz + 2, ny + 2, nx + 2))
    _load().wl_obstacle_flow_3d(nx, ny, nz, dx, dy, dz, dt, kmax, seed, t, _p(solid), _p(u),
                                _p(v), _p(w), _p(rhs))
    return solid, u, v, w, rhs


def layered_lap_2d(solid, dx, dy, amp=0.5):
    """(lap_diag, lap_off_x, lap_off_y) of a layered medium on a padded 2D mask,
    see wl_layered_lap_2d: symmetric, zero row sums, conductivities in [1-amp, 1+amp]."""
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    ny, nx = (s - 2 for s in solid.shape)
    lap = tuple(np.zeros(solid.shape) for _ in range(3))
    _load().wl_layered_lap_2d(nx, ny, dx, dy, amp, _p(solid), *(_p(a) for a in lap))
    return lap


def spheres_256():
    """The 256^3 mixed-precision workload: (solid, rhs, h)."""
    s, r = spheres_3d(256, 256, 256)
    return s, r, 1.0 / 256


def obstacle_2d():
    """The 2048 x 1024 projection workload: (solid, u, v, rhs, dx, dy, dt)."""
    dx, dy, dt = 1.0e-3, 1.5e-3, 1.0e-3
    s, u, v, r = obstacle_flow_2d(2048, 1024, dx, dy, dt)
    return s, u, v, r, dx, dy, dt


def layered_2d(amp=0.5):
    """The obstacle_2d grid, mask and RHS with the variable-coefficient Laplacian of
    a layered medium (layered_lap_2d, conductivities in [0.5, 1.5]):
    (solid, rhs, dx, dy, (lap_diag, lap_off_x, lap_off_y))."""
    s, _, _, r, dx, dy, _ = obstacle_2d()
    return s, r, dx, dy, layered_lap_2d(s, dx, dy, amp)


def serve_fields(dim, n, seed, kmax=None):
    """One serving simulation id: (solid, rhs0, rhs1), see wl_serve_fields."""
    kmax = kmax if kmax is not None else (4 if dim == 2 else 2)
    shape = (n + 2, n + 2, n + 2) if dim == 3 else (n + 2, n + 2)
    solid = np.zeros(shape, np.uint8)
    r0 = np.zeros(shape)
    r1 = np.zeros(shape)
    _load().wl_serve_fields(dim, n, kmax, seed, _p(solid), _p(r0), _p(r1))
    return solid, r0, r1


def batch96(seed=20260404):
    """The 96 uneven batch problems: list of (solid, rhs, dx, dy, dz)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    sizes2 = list(range(64, 1025, 64))
    sizes3 = [32, 48, 64, 96, 128]
    for q in range(96):
        if q < 64:
            nx, ny, nz, dim = int(rng.choice(sizes2)), int(rng.choice(sizes2)), 0, 2
        else:
            dim = 3
            nx, ny, nz = (int(rng.choice(sizes3)) for _ in range(3))
        cov = float(rng.uniform(0.0, 0.2))
        s, r = boxes(dim, nx, ny, nz, cov, seed + 1 + q)
        h = 1.0 / max(nx, ny, nz)
        out.append((s, r, h, h, h if dim == 3 else 1.0))
    return out


def serve_plan(n_ids=500, steps=20, seed=20260505):
    """The serving mix: list of (sim_id, dim, n, field_seed) for every id."""
    rng = np.random.Generator(np.random.MT19937(seed))
    plan = []
    for sid in range(n_ids):
        if rng.uniform() < 0.7:
            dim, n = 2, int(np.clip(round(float(np.exp(rng.normal(np.log(384), 0.5)))), 64, 2048))
        else:
            dim, n = 3, int(np.clip(round(float(np.exp(rng.normal(np.log(96), 0.4)))), 32, 256))
        plan.append((sid, dim, n, seed * 1000 + sid))
    return plan
