"""Test infrastructure only: ctypes bindings for the oracle.

Two libraries, both built by ``oracle/Makefile``:

* ``liboracle.so`` -- the plain-C restatement (``uaamg_oracle.c``) of the
  reference's CPU UAAMG-PCG (``src/solver/pcg_3d.cpp``, ``pcg.cpp``,
  ``src/solver/preconditioner/uaamg_preconditioner{,_3d}.cpp``);
* ``_ref/libuaamg_ref.so`` -- the reference's OWN CPU source files compiled
  unchanged, behind ``ref_shim.cpp``.  Present only where the reference tree was
  available at build time (it then travels with the repository snapshot).
* ``_ref/libuaamg_ref_gpu.so`` -- the reference's OWN CUDA 3D solver (CudaPCG3D)
  compiled unchanged for sm_100a, behind ``ref_gpu_shim.cu`` (same conditions).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  Arrays are numpy, padded and column-major with i fastest, stored
here as C-order arrays of shape (nz+2, ny+2, nx+2) (3D) or (ny+2, nx+2) (2D),
which is the same memory order.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libuaamg_ref.so")
_REF_GPU = os.path.join(HERE, "_ref", "libuaamg_ref_gpu.so")

_d = C.c_double
_i = C.c_int
_p = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _load(path):
    lib = C.CDLL(path)
    return lib


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise FileNotFoundError(f"{_LIB} missing: run `make -C oracle`")
        _lib = _load(_LIB)
        L = _lib
        L.oh_create.restype = _p
        L.oh_create.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _i]
        L.oh_destroy.argtypes = [_p]
        L.oh_nlevels.argtypes = [_p]
        L.oh_nlevels.restype = _i
        L.oh_level_dims.argtypes = [_p, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]
        L.oh_level_solid.argtypes = [_p, _i, _p]
        L.oh_level_coeffs.argtypes = [_p, _i, _p, _p, _p, _p]
        L.oh_vcycle.argtypes = [_p, _p, _p]
        L.oracle_pcg.restype = _i
        L.oracle_pcg.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _p, _p, _i, _d, _i, _i, _i,
                                 _i, _p, C.POINTER(_i)]
        L.oracle_pcg_rhs.argtypes = [_i, _i, _i, _i, _p, _p, _p, _i]
        L.oracle_true_residual.restype = _d
        L.oracle_true_residual.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _p, _p, _i,
                                           C.POINTER(_d)]
        L.oracle_matvec.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _p, _p, _i]
        L.oracle_correct_velocity.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _p, _d, _p,
                                              _p, _p]
        L.oracle_divergence_rhs.argtypes = [_i, _i, _i, _i, _d, _d, _d, _p, _p, _p, _p, _d,
                                            _p]
        L.oracle_static_rhs_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _p]
        L.oracle_pcg_var_2d.restype = _i
        L.oracle_pcg_var_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _p, _p, _p, _i, _d, _i, _i,
                                        _i, _p, C.POINTER(_i)]
        L.oracle_matvec_var_2d.argtypes = [_i, _i, _p, _p, _p, _p, _p, _p]
        L.oracle_true_residual_var_2d.restype = _d
        L.oracle_true_residual_var_2d.argtypes = [_i, _i, _p, _p, _p, _p, _p, _p, C.POINTER(_d)]
        L.oracle_smooth_cylinder_2d.argtypes = [_i, _i, _d, _d, _d, _d, _d, _d, _i, _p, _p, _p,
                                                _p]
    return _lib


def have_ref() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        if not have_ref():
            raise FileNotFoundError(f"{_REF} missing: run `make -C oracle ref` where the "
                                    "reference tree is present")
        _ref = _load(_REF)
        R = _ref
        R.ref_vcycle_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p]
        R.ref_vcycle_3d.argtypes = [_i, _i, _i, _d, _d, _d, _p, _p, _p]
        R.ref_pcg_2d.restype = _i
        R.ref_pcg_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _i, _d, _i]
        R.ref_pcg_3d.restype = _i
        R.ref_pcg_3d.argtypes = [_i, _i, _i, _d, _d, _d, _p, _p, _p, _i, _d, _i]
        R.ref_project_2d.restype = _i
        R.ref_project_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _d, _i, _d, _p]
        R.ref_static_rhs_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _p]
        R.ref_pcg_var_2d.restype = _i
        R.ref_pcg_var_2d.argtypes = [_i, _i, _d, _d, _p, _p, _p, _p, _p, _p, _i, _d, _i]
        R.ref_smooth_cylinder_2d.argtypes = [_i, _i, _d, _d, _d, _d, _d, _d, _p, _p, _p, _p]
        R.ref_project_3d.restype = _i
        R.ref_project_3d.argtypes = [_i, _i, _i, _d, _d, _d, _p, _p, _p, _p, _d, _i, _d, _p]
    return _ref


# ---------------------------------------------------------------------------
# helpers


def padded_shape(dim, nx, ny, nz=1):
    return (nz + 2, ny + 2, nx + 2) if dim == 3 else (ny + 2, nx + 2)


def _c8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def _cd(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dims(shape):
    if len(shape) == 3:
        return 3, shape[2] - 2, shape[1] - 2, shape[0] - 2
    return 2, shape[1] - 2, shape[0] - 2, 0


class Hierarchy:
    """The restated UAAMG hierarchy (masks, Galerkin coefficients) and V-cycle."""

    def __init__(self, solid, dx, dy, dz=1.0, dirichlet=False):
        self.solid = _c8(solid)
        self.dim, nx, ny, nz = _dims(self.solid.shape)
        self.h = lib().oh_create(self.dim, nx, ny, nz, dx, dy, dz, _ptr(self.solid),
                                 int(dirichlet))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oh_destroy(self.h)
            self.h = None

    @property
    def nlevels(self):
        return lib().oh_nlevels(self.h)

    def dims(self, l):
        a, b, c = _i(), _i(), _i()
        lib().oh_level_dims(self.h, l, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def _shape(self, l):
        nx, ny, nz = self.dims(l)
        return padded_shape(self.dim, nx, ny, nz)

    def level_solid(self, l):
        out = np.zeros(self._shape(l), np.uint8)
        lib().oh_level_solid(self.h, l, _ptr(out))
        return out

    def level_coeffs(self, l):
        sh = self._shape(l)
        cx, cy, cz, dg = (np.zeros(sh) for _ in range(4))
        lib().oh_level_coeffs(self.h, l, _ptr(cx), _ptr(cy), _ptr(cz), _ptr(dg))
        return cx, cy, cz, dg

    def vcycle(self, r):
        r = _cd(r)
        z = np.zeros_like(r)
        lib().oh_vcycle(self.h, _ptr(r), _ptr(z))
        return z


def pcg(solid, rhs, dx, dy, dz=1.0, max_iter=200, tol=1e-6, precond=True, tol_mode=1,
        x0=None, warm=False, dirichlet=False, hist=False):
    """Restated PCG (PCG::solve / PCG3D::solve).  tol_mode 0 = absolute like the
    reference, 1 = relative to ||r0||.  Returns (x, updates, status[, hist])."""
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    rhs = _cd(rhs)
    x = np.zeros_like(rhs) if x0 is None else _cd(x0).copy()
    h = np.zeros(max_iter + 1) if hist else None
    st = _i()
    n = lib().oracle_pcg(dim, nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(rhs), _ptr(x),
                         max_iter, tol, int(precond), tol_mode, int(warm), int(dirichlet),
                         _ptr(h), C.byref(st))
    if hist:
        return x, n, st.value, h[: n + 1]
    return x, n, st.value


def pcg_rhs(solid, rhs, dirichlet=False):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    rhs = _cd(rhs)
    b = np.zeros_like(rhs)
    lib().oracle_pcg_rhs(dim, nx, ny, nz, _ptr(solid), _ptr(rhs), _ptr(b), int(dirichlet))
    return b


def true_residual(solid, rhs, x, dx, dy, dz=1.0, dirichlet=False):
    """(||b - A x||, ||b||) over fluid cells, FP64."""
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    bn = _d()
    r = lib().oracle_true_residual(dim, nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(_cd(rhs)),
                                   _ptr(_cd(x)), int(dirichlet), C.byref(bn))
    return r, bn.value


def matvec(solid, x, dx, dy, dz=1.0, dirichlet=False):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    x = _cd(x)
    ax = np.zeros_like(x)
    lib().oracle_matvec(dim, nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(x), _ptr(ax),
                        int(dirichlet))
    return ax


def divergence_rhs(solid, u, v, w, dx, dy, dz, dt):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    rhs = np.zeros(solid.shape)
    lib().oracle_divergence_rhs(dim, nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(_cd(u)),
                                _ptr(_cd(v)), _ptr(_cd(w)) if w is not None else None, dt,
                                _ptr(rhs))
    return rhs


def correct_velocity(solid, p, dt, u, v, w, dx, dy, dz=1.0):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    u, v = _cd(u).copy(), _cd(v).copy()
    w = _cd(w).copy() if w is not None else None
    lib().oracle_correct_velocity(dim, nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(_cd(p)), dt,
                                  _ptr(u), _ptr(v), _ptr(w))
    return u, v, w


def pcg_var(solid, lap, rhs, dx, dy, max_iter=200, tol=1e-6, precond=True, tol_mode=1,
            x0=None, warm=False):
    """Restated 2D PCG with the variable-coefficient operator (pcg.cpp:35-46);
    lap = (lap_diag, lap_off_x, lap_off_y), padded.  Returns (x, updates, status)."""
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    ld, lx, ly = (_cd(a) for a in lap)
    rhs = _cd(rhs)
    x = np.zeros_like(rhs) if x0 is None else _cd(x0).copy()
    st = _i()
    n = lib().oracle_pcg_var_2d(nx, ny, dx, dy, _ptr(solid), _ptr(ld), _ptr(lx), _ptr(ly),
                                _ptr(rhs), _ptr(x), max_iter, tol, int(precond), tol_mode,
                                int(warm), None, C.byref(st))
    return x, n, st.value


def matvec_var(solid, lap, x):
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    ld, lx, ly = (_cd(a) for a in lap)
    x = _cd(x)
    ax = np.zeros_like(x)
    lib().oracle_matvec_var_2d(nx, ny, _ptr(solid), _ptr(ld), _ptr(lx), _ptr(ly), _ptr(x),
                               _ptr(ax))
    return ax


def true_residual_var(solid, lap, rhs, x):
    """(||b - A x||, ||b||) with the variable-coefficient operator, FP64."""
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    ld, lx, ly = (_cd(a) for a in lap)
    bn = _d()
    r = lib().oracle_true_residual_var_2d(nx, ny, _ptr(solid), _ptr(ld), _ptr(lx), _ptr(ly),
                                          _ptr(_cd(rhs)), _ptr(_cd(x)), C.byref(bn))
    return r, bn.value


def smooth_cylinder(solid, dx, dy, cx, cy, r, tw=0.0, inside=False):
    """Restated SmoothCylinder::applyToLaplacian: (solid', (diag, off_x, off_y))."""
    solid = _c8(solid).copy()
    _, nx, ny, _ = _dims(solid.shape)
    lap = tuple(np.zeros(solid.shape) for _ in range(3))
    lib().oracle_smooth_cylinder_2d(nx, ny, dx, dy, cx, cy, r, tw, int(inside), _ptr(solid),
                                    *(_ptr(a) for a in lap))
    return solid, lap


# --- the reference itself (compiled from its own sources) -------------------


def have_ref_gpu() -> bool:
    return os.path.exists(_REF_GPU)


_ref_gpu = None


def ref_gpu_pcg3d(solid, rhs, dx, dy, dz, max_iter=500, tol=1e-6, mode=0, reps=1):
    """The reference's CUDA CudaPCG3D on the current GPU: mode 0 solve_optimized (FP64),
    1 solve_mixed (FP32 V-cycle); stop ||r|| / ||r0|| < tol.  One untimed solve, then
    `reps` timed ones.  Returns (p, mean ms a solve, iterations, relative residual)."""
    global _ref_gpu
    if _ref_gpu is None:
        if not have_ref_gpu():
            raise FileNotFoundError(f"{_REF_GPU} missing: run `make -C oracle ref-gpu` where "
                                    "the reference tree is present")
        _ref_gpu = _load(_REF_GPU)
        _ref_gpu.ref_gpu_pcg3d.restype = _i
        _ref_gpu.ref_gpu_pcg3d.argtypes = [_i, _i, _i, _d, _d, _d, _p, _p, _p, _i, _d, _i, _i,
                                           C.POINTER(_d), C.POINTER(_i), C.POINTER(_d)]
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    if dim != 3:
        raise ValueError("ref_gpu_pcg3d takes a 3D problem")
    rhs = _cd(rhs)
    p = np.zeros_like(rhs)
    ms, it, rr = _d(), _i(), _d()
    e = _ref_gpu.ref_gpu_pcg3d(nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(rhs), _ptr(p), max_iter,
                               tol, mode, reps, C.byref(ms), C.byref(it), C.byref(rr))
    if e != 0:
        raise RuntimeError(f"reference GPU solve: CUDA error {e}")
    return p, ms.value, it.value, rr.value


def ref_pcg_var(solid, lap, rhs, dx, dy, max_iter=200, tol=1e-6, precond=True):
    """The reference's PCG::solve on a grid with init_variable_lap() and the given
    coefficients.  Returns (p, preconditioner applications)."""
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    ld, lx, ly = (_cd(a) for a in lap)
    rhs = _cd(rhs)
    p = np.zeros_like(rhs)
    n = ref().ref_pcg_var_2d(nx, ny, dx, dy, _ptr(solid), _ptr(ld), _ptr(lx), _ptr(ly),
                             _ptr(rhs), _ptr(p), max_iter, tol, int(precond))
    return p, n


def ref_smooth_cylinder(solid, dx, dy, cx, cy, r, tw=0.0):
    """SmoothCylinder(cx, cy, r, dx, dy, tw).applyToLaplacian as the reference
    runs it: (solid', (diag, off_x, off_y))."""
    solid = _c8(solid).copy()
    _, nx, ny, _ = _dims(solid.shape)
    lap = tuple(np.zeros(solid.shape) for _ in range(3))
    ref().ref_smooth_cylinder_2d(nx, ny, dx, dy, cx, cy, r, tw, _ptr(solid),
                                 *(_ptr(a) for a in lap))
    return solid, lap


def ref_vcycle(solid, r, dx, dy, dz=1.0):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    r = _cd(r)
    z = np.zeros_like(r)
    if dim == 3:
        ref().ref_vcycle_3d(nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(r), _ptr(z))
    else:
        ref().ref_vcycle_2d(nx, ny, dx, dy, _ptr(solid), _ptr(r), _ptr(z))
    return z


def ref_pcg(solid, rhs, dx, dy, dz=1.0, max_iter=200, tol=1e-6, precond=True):
    """The reference's PCG with its absolute stop sqrt(r.r) < tol.  Returns
    (p, preconditioner applications)."""
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    rhs = _cd(rhs)
    p = np.zeros_like(rhs)
    if dim == 3:
        n = ref().ref_pcg_3d(nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(rhs), _ptr(p), max_iter,
                             tol, int(precond))
    else:
        n = ref().ref_pcg_2d(nx, ny, dx, dy, _ptr(solid), _ptr(rhs), _ptr(p), max_iter, tol,
                             int(precond))
    return p, n


def static_rhs(solid, u, v, dx, dy):
    """RHS of recoverStaticPressure (pressure.cpp:35-66), 2D, padded."""
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    rhs = np.zeros(solid.shape)
    lib().oracle_static_rhs_2d(nx, ny, dx, dy, _ptr(solid), _ptr(_cd(u)), _ptr(_cd(v)), _ptr(rhs))
    return rhs


def ref_static_rhs(solid, u, v, dx, dy):
    """The same right-hand side as the reference's own recoverStaticPressure builds it."""
    solid = _c8(solid)
    _, nx, ny, _ = _dims(solid.shape)
    rhs = np.zeros(solid.shape)
    ref().ref_static_rhs_2d(nx, ny, dx, dy, _ptr(solid), _ptr(_cd(u)), _ptr(_cd(v)), _ptr(rhs))
    return rhs


def ref_project(solid, u, v, w, dx, dy, dz, dt, max_iter, tol):
    solid = _c8(solid)
    dim, nx, ny, nz = _dims(solid.shape)
    u, v = _cd(u).copy(), _cd(v).copy()
    p = np.zeros(solid.shape)
    if dim == 3:
        w = _cd(w).copy()
        n = ref().ref_project_3d(nx, ny, nz, dx, dy, dz, _ptr(solid), _ptr(u), _ptr(v), _ptr(w),
                                 dt, max_iter, tol, _ptr(p))
    else:
        n = ref().ref_project_2d(nx, ny, dx, dy, _ptr(solid), _ptr(u), _ptr(v), dt, max_iter,
                                 tol, _ptr(p))
    return u, v, w, p, n
