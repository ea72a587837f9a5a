"""Host-side mirror of the reference's pressure-solver surface over the C-ABI.

Mirrors (A-006/UAAMGPCG):
  Grid / Grid3D            include/core/grid.h:16-48, include/core/grid_3d.h:14-38
  Solver / Solver3D        include/solver/solver.h:18-34, include/solver/solver_3d.h:7-12
  Factory / Factory3D      src/solver/factory.cpp:16-25, src/solver/factory_3d.cpp:17-29
  PressureProjection[3D]   src/pressure/pressure.cpp:5-33, src/pressure/pressure_3d.cpp:5-40
  CudaPCGSolver[3D]        src/solver/cuda/cuda_pcg_solver{,_3d}.cu (the GPU adapter shape)

Arrays are numpy, ghost-padded, column-major with i fastest -- stored as C-order
arrays of shape (ny+2, nx+2) in 2D and (nz+2, ny+2, nx+2) in 3D, which is the
reference's memory order, so ``a.ravel()`` is the reference's flat vector.
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _capi


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# Grids


class Grid:
    """2D MAC grid: nx x ny cells, dx = lx/nx, dy = ly/ny; u (nx+1)(ny+2),
    v (nx+2)(ny+1), p and solid (nx+2)(ny+2), all padded and i-fastest."""

    dim = 2

    def __init__(self, nx, ny, lx, ly):
        self.nx, self.ny = int(nx), int(ny)
        self.dx, self.dy = lx / nx, ly / ny
        self.dz = 1.0
        self.u = np.zeros((ny + 2, nx + 1))
        self.v = np.zeros((ny + 1, nx + 2))
        self.p = np.zeros((ny + 2, nx + 2))
        self.solid = np.zeros((ny + 2, nx + 2), np.uint8)
        # variable-coefficient Laplacian (include/core/grid.h:23-31): empty until
        # init_variable_lap(); PCG::solve then uses them (pcg.cpp:35-46)
        self.lap_diag = np.zeros(0)
        self.lap_off_x = np.zeros(0)
        self.lap_off_y = np.zeros(0)

    def init_variable_lap(self):
        """Zero padded coefficient arrays (Grid::init_variable_lap, grid.cpp:12-17)."""
        self.lap_diag = np.zeros(self.p.shape)
        self.lap_off_x = np.zeros(self.p.shape)
        self.lap_off_y = np.zeros(self.p.shape)

    def has_variable_lap(self):
        return self.lap_diag.size != 0

    @property
    def nz(self):
        return 0

    def ip(self, i, j):
        return i + j * (self.nx + 2)

    def cell_shape(self):
        return self.p.shape


class Grid3D:
    """3D MAC grid (Grid3D): u (nx+1)(ny+2)(nz+2), v (nx+2)(ny+1)(nz+2),
    w (nx+2)(ny+2)(nz+1), p and solid (nx+2)(ny+2)(nz+2)."""

    dim = 3

    def __init__(self, nx, ny, nz, lx, ly, lz):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx, self.dy, self.dz = lx / nx, ly / ny, lz / nz
        self.u = np.zeros((nz + 2, ny + 2, nx + 1))
        self.v = np.zeros((nz + 2, ny + 1, nx + 2))
        self.w = np.zeros((nz + 1, ny + 2, nx + 2))
        self.p = np.zeros((nz + 2, ny + 2, nx + 2))
        self.solid = np.zeros((nz + 2, ny + 2, nx + 2), np.uint8)

    def ip(self, i, j, k):
        return i + j * (self.nx + 2) + k * (self.nx + 2) * (self.ny + 2)

    def cell_shape(self):
        return self.p.shape


# ---------------------------------------------------------------------------
# Handle


def set_tune_cache(path=None):
    """Process-wide JSON file that keeps the autotuner's choices (uaamg_set_tune_cache);
    None: memory only."""
    lib = _capi.load()
    st = lib.uaamg_set_tune_cache(None if path is None else str(path).encode())
    if st != _capi.OK:
        raise _capi.UaamgError(st, "set_tune_cache")


class Handle:
    """Owns one ``uaamg_handle`` (one GPU, one problem at a time)."""

    def __init__(self, device: int = 0):
        self.lib = _capi.load()
        h = C.c_void_p()
        st = self.lib.uaamg_create(C.byref(h), int(device))
        if st != _capi.OK:
            raise _capi.UaamgError(st, f"uaamg_create(device={device}) failed (no CUDA device?)")
        self.h = h
        self.dim = 0
        self.shape = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.uaamg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what, ok=(_capi.OK,)):
        if st not in ok:
            err = self.lib.uaamg_last_error(self.h).decode()
            raise _capi.UaamgError(st, f"{what}: {err}")
        return st

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.uaamg_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    def set_vcycle_kernels(self, mode):
        """0 / False: two fused z marches a level + the single-block small-level
        kernel (default); 1 / True: per-colour sweep kernels; 2: fused marches on every
        level; 3: four z marches a level + the small-level kernel; 4: four marches on
        every level."""
        self._check(self.lib.uaamg_set_vcycle_kernels(self.h, int(mode)), "vcycle")

    def set_batch_group(self, max_cells=0):
        """solve_batch: problems of at most max_cells padded cells share one CUDA graph
        per step (uaamg_set_batch_group; 0: one graph each)."""
        self._check(self.lib.uaamg_set_batch_group(self.h, int(max_cells)), "batch_group")

    def set_smoothing(self, sweeps_fine=1, sweeps_coarse=1):
        """Pre- and post-smoothing sweeps on the finest and the coarse levels
        (uaamg_set_smoothing; 1, 1 is the reference's V(1,1))."""
        self._check(self.lib.uaamg_set_smoothing(self.h, int(sweeps_fine), int(sweeps_coarse)),
                    "smoothing")

    def set_variable_laplacian(self, lap_diag=None, lap_off_x=None, lap_off_y=None):
        """The outer CG's variable-coefficient operator for the current 2D problem
        (uaamg_set_variable_laplacian); no arguments: back to the uniform one."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (lap_diag, lap_off_x, lap_off_y)]
        for a in arrs:
            if a is not None and self.shape is not None and a.shape != tuple(self.shape):
                raise ValueError(f"coefficient shape {a.shape} != padded grid {self.shape}")
        st = self.lib.uaamg_set_variable_laplacian(
            self.h, *(_ptr(a) if a is not None else None for a in arrs))
        self._check(st, "set_variable_laplacian")

    def set_dirichlet_walls(self, on: bool):
        self._check(self.lib.uaamg_set_dirichlet_walls(self.h, int(bool(on))), "dirichlet")

    def set_problem(self, solid: np.ndarray, dx: float, dy: float, dz: float = 1.0):
        solid = np.ascontiguousarray(solid, dtype=np.uint8)
        if solid.ndim == 3:
            nz, ny, nx = (s - 2 for s in solid.shape)
            st = self.lib.uaamg_set_problem_3d(self.h, nx, ny, nz, dx, dy, dz, _ptr(solid))
        elif solid.ndim == 2:
            ny, nx = (s - 2 for s in solid.shape)
            st = self.lib.uaamg_set_problem_2d(self.h, nx, ny, dx, dy, _ptr(solid))
        else:
            raise ValueError("solid must be a padded 2D or 3D array")
        self._check(st, "set_problem")
        self.dim = solid.ndim
        self.shape = solid.shape

    def set_problem_device(self, dim, nx, ny, nz, dx, dy, dz, d_solid_ptr: int):
        st = self.lib.uaamg_set_problem_device(self.h, dim, nx, ny, nz, dx, dy, dz,
                                               C.c_void_p(d_solid_ptr))
        self._check(st, "set_problem_device")
        self.dim = dim
        self.shape = (nz + 2, ny + 2, nx + 2) if dim == 3 else (ny + 2, nx + 2)

    @staticmethod
    def options(precision="fp64", tol=1e-6, max_iter=2000, tol_mode="abs", warm_start=False,
                replace_every=10, project_mean=False, preconditioner=True) -> _capi.Options:
        o = _capi.default_options()
        o.precision = _capi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        o.tol = float(tol)
        o.max_iter = int(max_iter)
        o.tol_mode = {"abs": _capi.TOL_ABS, "rel": _capi.TOL_REL}[tol_mode] \
            if isinstance(tol_mode, str) else int(tol_mode)
        o.warm_start = int(bool(warm_start))
        o.replace_every = int(replace_every)
        o.project_mean = int(bool(project_mean))
        o.preconditioner = int(bool(preconditioner))
        return o

    _SOLVE_OK = (_capi.OK, _capi.NOT_CONVERGED, _capi.BREAKDOWN)

    def solve(self, rhs: np.ndarray, p: np.ndarray, opts: _capi.Options | None = None,
              strict: bool = False):
        """Host-array solve (uaamg_solve); p is updated in place.  Returns stats."""
        if rhs.shape != self.shape or p.shape != self.shape:
            raise ValueError(f"arrays must have the padded shape {self.shape}")
        if p.dtype != np.float64 or not p.flags.c_contiguous:
            raise ValueError("p must be a C-contiguous float64 array")
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        st = _capi.Stats()
        s = self.lib.uaamg_solve(self.h, _ptr(rhs), _ptr(p), C.byref(opts or self.options()),
                                 C.byref(st))
        self._check(s, "solve", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def solve_device(self, d_rhs: int, d_p: int, opts: _capi.Options | None = None,
                     strict: bool = False):
        """Device-pointer solve (uaamg_solve_device).  Returns stats."""
        st = _capi.Stats()
        s = self.lib.uaamg_solve_device(self.h, C.c_void_p(d_rhs), C.c_void_p(d_p),
                                        C.byref(opts or self.options()), C.byref(st))
        self._check(s, "solve_device", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def face_shapes(self):
        """Shapes of the FP64 face-velocity arrays u, v[, w] of the current problem."""
        shp = self.shape
        if len(shp) == 2:
            ny2, nx2 = shp
            return [(ny2, nx2 - 1), (ny2 - 1, nx2)]
        nz2, ny2, nx2 = shp
        return [(nz2, ny2, nx2 - 1), (nz2, ny2 - 1, nx2), (nz2 - 1, ny2, nx2)]

    def project(self, u, v, w, p, dt: float, opts: _capi.Options | None = None,
                strict: bool = False):
        """Pressure projection with host arrays (uaamg_project): rhs = div(u)/dt,
        solve into p, u/v/w corrected in place.  Returns stats."""
        faces = [u, v] + ([w] if len(self.shape) == 3 else [])
        for a, shp in zip(faces + [p], self.face_shapes() + [self.shape]):
            if a.shape != shp or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(f"arrays must be C-contiguous float64 of shapes "
                                 f"{self.face_shapes()} and {self.shape}")
        st = _capi.Stats()
        s = self.lib.uaamg_project(self.h, float(dt), _ptr(u), _ptr(v),
                                   _ptr(w) if len(self.shape) == 3 else None, _ptr(p),
                                   C.byref(opts or self.options()), C.byref(st))
        self._check(s, "project", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def project_device(self, d_u: int, d_v: int, d_w: int, d_p: int, dt: float,
                       opts: _capi.Options | None = None, strict: bool = False):
        """Pressure projection with device pointers (uaamg_project_device)."""
        st = _capi.Stats()
        s = self.lib.uaamg_project_device(self.h, float(dt), C.c_void_p(d_u), C.c_void_p(d_v),
                                          C.c_void_p(d_w) if d_w else None, C.c_void_p(d_p),
                                          C.byref(opts or self.options()), C.byref(st))
        self._check(s, "project_device", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def static_pressure(self, u, v, p, opts: _capi.Options | None = None, strict: bool = False):
        """recoverStaticPressure on the GPU with host arrays (uaamg_static_pressure, 2D):
        p is overwritten with the static pressure.  Returns stats."""
        for a, shp in zip((u, v, p), self.face_shapes() + [self.shape]):
            if a.shape != shp or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("arrays must be C-contiguous float64 of the grid's shapes")
        st = _capi.Stats()
        s = self.lib.uaamg_static_pressure(self.h, _ptr(u), _ptr(v), _ptr(p),
                                           C.byref(opts or self.options()), C.byref(st))
        self._check(s, "static_pressure", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def static_pressure_device(self, d_u: int, d_v: int, d_p: int,
                               opts: _capi.Options | None = None, strict: bool = False):
        """recoverStaticPressure with device pointers (uaamg_static_pressure_device)."""
        st = _capi.Stats()
        s = self.lib.uaamg_static_pressure_device(self.h, C.c_void_p(d_u), C.c_void_p(d_v),
                                                  C.c_void_p(d_p), C.byref(opts or self.options()),
                                                  C.byref(st))
        self._check(s, "static_pressure_device", (_capi.OK,) if strict else self._SOLVE_OK)
        return st

    def profile_solve(self, d_rhs: int, d_p: int, opts: _capi.Options | None = None):
        """uaamg_profile_solve: (stats, [dict(name, level, launches, total_ms,
        bytes_per_launch)])."""
        st = _capi.Stats()
        cap = 256
        arr = (_capi.KernelTime * cap)()
        cnt = C.c_int()
        s = self.lib.uaamg_profile_solve(self.h, C.c_void_p(d_rhs), C.c_void_p(d_p),
                                         C.byref(opts or self.options()), C.byref(st), arr, cap,
                                         C.byref(cnt))
        self._check(s, "profile_solve", self._SOLVE_OK)
        rows = [dict(name=arr[q].name.decode(), level=arr[q].level, launches=arr[q].launches,
                     total_ms=arr[q].total_ms, bytes_per_launch=arr[q].bytes_per_launch)
                for q in range(min(cap, cnt.value))]
        return st, rows

    def precond_apply(self, r: np.ndarray, precision="fp64") -> np.ndarray:
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        prec = _capi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._check(self.lib.uaamg_precond_apply(self.h, prec, _ptr(r), _ptr(z)), "precond_apply")
        return z

    def residual_history(self, n: int) -> np.ndarray:
        out = np.zeros(n)
        self._check(self.lib.uaamg_residual_history(self.h, _ptr(out), n), "history")
        return out

    def num_levels(self) -> int:
        n = C.c_int()
        self._check(self.lib.uaamg_num_levels(self.h, C.byref(n)), "num_levels")
        return n.value

    def level_dims(self, l):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.uaamg_level_dims(self.h, l, C.byref(a), C.byref(b), C.byref(c)),
                    "level_dims")
        return a.value, b.value, c.value

    def copy_level(self, l, precision="fp64"):
        nx, ny, nz = self.level_dims(l)
        shape = (nz + 2, ny + 2, nx + 2) if self.dim == 3 else (ny + 2, nx + 2)
        solid = np.zeros(shape, np.uint8)
        cx, cy, cz = (np.zeros(shape) for _ in range(3))
        prec = _capi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._check(self.lib.uaamg_copy_level(self.h, prec, l, _ptr(solid), _ptr(cx), _ptr(cy),
                                              _ptr(cz)), "copy_level")
        return solid, cx, cy, cz

    def level_trim(self, l, precision="fp64"):
        """(boxes, trimmed boxes) of level l (uaamg_level_trim)."""
        a, b = C.c_int(), C.c_int()
        prec = _capi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self._check(self.lib.uaamg_level_trim(self.h, prec, l, C.byref(a), C.byref(b)),
                    "level_trim")
        return a.value, b.value

    def device_bytes(self) -> int:
        b = C.c_size_t()
        self._check(self.lib.uaamg_device_bytes(self.h, C.byref(b)), "device_bytes")
        return b.value

    def set_autotune(self, on: bool):
        self._check(self.lib.uaamg_set_autotune(self.h, int(bool(on))), "autotune")

    def solve_batch(self, problems, opts: _capi.Options | None = None, strict: bool = False):
        """uaamg_solve_batch over [(solid, rhs, p, dx, dy, dz), ...] (padded host
        arrays; each p updated in place).  Returns the list of per-problem stats."""
        keep, probs = [], (_capi.Problem * max(1, len(problems)))()
        for q, (solid, rhs, p, dx, dy, dz) in enumerate(problems):
            solid = np.ascontiguousarray(solid, dtype=np.uint8)
            rhs = np.ascontiguousarray(rhs, dtype=np.float64)
            if p.dtype != np.float64 or not p.flags.c_contiguous or p.shape != solid.shape \
                    or rhs.shape != solid.shape:
                raise ValueError(f"problem {q}: arrays must share the padded shape, p float64")
            keep += [solid, rhs]
            pr = probs[q]
            pr.dim = solid.ndim
            if solid.ndim == 3:
                pr.nz, pr.ny, pr.nx = (v - 2 for v in solid.shape)
            else:
                (pr.ny, pr.nx), pr.nz = (v - 2 for v in solid.shape), 0
            pr.dx, pr.dy, pr.dz = float(dx), float(dy), float(dz)
            pr.solid, pr.rhs, pr.p = solid.ctypes.data, rhs.ctypes.data, p.ctypes.data
        stats = (_capi.Stats * max(1, len(problems)))()
        s = self.lib.uaamg_solve_batch(self.h, len(problems), probs,
                                       C.byref(opts or self.options()), stats)
        self._check(s, "solve_batch", (_capi.OK,) if strict else self._SOLVE_OK)
        return [stats[q] for q in range(len(problems))]


class Server:
    """The serving loop (uaamg_server_*): submit requests of any size; each
    simulation id keeps its hierarchy and pressure on the device between requests."""

    def __init__(self, device=0, precision="mixed", tol=1e-6, max_iter=500, replace_every=10,
                 warm_start=True, max_active=16, hbm_budget_bytes=150 << 30):
        self.lib = _capi.load()
        cfg = _capi.ServerConfig()
        self.lib.uaamg_server_default_config(C.byref(cfg))
        cfg.device, cfg.precision = int(device), _capi.PRECISIONS[precision]
        cfg.tol, cfg.max_iter, cfg.replace_every = float(tol), int(max_iter), int(replace_every)
        cfg.warm_start, cfg.max_active = int(bool(warm_start)), int(max_active)
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        self.s = C.c_void_p()
        st = self.lib.uaamg_server_start(C.byref(self.s), C.byref(cfg))
        if st != _capi.OK:
            raise _capi.UaamgError(st, "server_start")
        self._keep = {}

    def submit(self, sim_id, solid, rhs, dx, dy, dz=1.0, p_out=None, borrow=False) -> int:
        """Queues one solve; p_out (padded float64, optional) receives the pressure.
        borrow: rhs and p_out are lent to the server (UAAMG_REQUEST_BORROW) -- keep them
        alive and rhs unchanged until the ticket is polled done; pinned arrays make the
        device copies asynchronous."""
        solid = np.ascontiguousarray(solid, dtype=np.uint8)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        q = _capi.Request()
        q.sim_id, q.dim = int(sim_id), solid.ndim
        if solid.ndim == 3:
            q.nz, q.ny, q.nx = (v - 2 for v in solid.shape)
        else:
            (q.ny, q.nx), q.nz = (v - 2 for v in solid.shape), 0
        q.dx, q.dy, q.dz = float(dx), float(dy), float(dz)
        q.solid, q.rhs = solid.ctypes.data, rhs.ctypes.data
        if p_out is not None:
            if p_out.dtype != np.float64 or not p_out.flags.c_contiguous or p_out.shape != solid.shape:
                raise ValueError("p_out must be a C-contiguous float64 array of the padded shape")
            q.p_out = p_out.ctypes.data
        q.flags = _capi.REQUEST_BORROW if borrow else 0
        t = C.c_longlong()
        st = self.lib.uaamg_server_submit(self.s, C.byref(q), C.byref(t))
        if st != _capi.OK:
            raise _capi.UaamgError(st, "server_submit")
        # the output buffer (and a lent right-hand side) must outlive the solve
        self._keep[t.value] = (p_out, rhs if borrow else None)
        return t.value

    def poll(self, ticket):
        """The result dict once the ticket finished (and releases it), else None."""
        res, done = _capi.Result(), C.c_int()
        st = self.lib.uaamg_server_poll(self.s, int(ticket), C.byref(res), C.byref(done))
        if st != _capi.OK:
            raise _capi.UaamgError(st, "server_poll")
        if not done.value:
            return None
        self._keep.pop(int(ticket), None)
        return res.as_dict()

    def drain(self):
        self.lib.uaamg_server_drain(self.s)

    def info(self):
        b, r, c = C.c_size_t(), C.c_int(), C.c_longlong()
        self.lib.uaamg_server_info(self.s, C.byref(b), C.byref(r), C.byref(c))
        return {"device_bytes": b.value, "resident": r.value, "completed": c.value}

    def stop(self):
        if self.s:
            self.lib.uaamg_server_stop(self.s)
            self.s = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Solver plug-ins


class Solver:
    """Abstract Poisson solver: solve lap(p) = rhs, writing g.p (solver.h:18-34)."""

    def solve(self, g, rhs, max_iter: int, tol: float):  # pragma: no cover - interface
        raise NotImplementedError

    def name(self) -> str:  # pragma: no cover - interface
        raise NotImplementedError


Solver3D = Solver


class GpuUAAMGPCG(Solver):
    """GPU UAAMG-preconditioned CG behind the reference's Solver interface: a
    drop-in for PCG(UAAMGPreconditioner) and CudaPCGSolver(true).

    precision: "fp64" (reference-exact), "fp32" (plain FP32 PCG) or "mixed"
    (FP32 CG with FP64 residual replacement).  tol_mode "abs" stops on
    sqrt(r.r) < tol exactly like PCG::solve; "rel" on sqrt(r.r) < tol*||b||.
    The solid mask is re-sent whenever it changes (the reference's adapter only
    re-sent it on a resize, cuda_pcg_solver.cu:45-49)."""

    def __init__(self, precision="fp64", tol_mode="abs", device=0, preconditioner=True,
                 replace_every=10, project_mean=False, warm_start=False):
        self.precision = precision
        self.tol_mode = tol_mode
        self.preconditioner = preconditioner
        self.replace_every = replace_every
        self.project_mean = project_mean
        self.warm_start = warm_start
        self.handle = Handle(device)
        self._key = None
        self._solid = None
        self._var = False
        self.last_stats = None

    def _sync_problem(self, g):
        key = (g.nx, g.ny, getattr(g, "nz", 0), g.dx, g.dy, getattr(g, "dz", 1.0))
        if key != self._key or self._solid is None or not np.array_equal(self._solid, g.solid):
            self.handle.set_problem(g.solid, g.dx, g.dy, getattr(g, "dz", 1.0))
            self._key = key
            self._solid = np.array(g.solid, dtype=np.uint8, copy=True)
            self._var = False
        # the grid's variable-coefficient Laplacian, sent on every call (the caller
        # may change the arrays in place), as PCG::solve reads them each time
        var = bool(getattr(g, "has_variable_lap", lambda: False)())
        if var:
            self.handle.set_variable_laplacian(g.lap_diag, g.lap_off_x, g.lap_off_y)
        elif self._var:
            self.handle.set_variable_laplacian()
        self._var = var

    def solve(self, g, rhs, max_iter, tol):
        self._sync_problem(g)
        rhs = np.asarray(rhs, dtype=np.float64).reshape(g.cell_shape())
        opts = Handle.options(self.precision, tol, max_iter, self.tol_mode, self.warm_start,
                              self.replace_every, self.project_mean, self.preconditioner)
        if g.p.dtype != np.float64 or not g.p.flags.c_contiguous:
            g.p = np.ascontiguousarray(g.p, dtype=np.float64)
        self.last_stats = self.handle.solve(rhs, g.p, opts)
        return self.last_stats

    def project(self, g, dt, max_iter, tol):
        """The whole pressure projection on the GPU (uaamg_project): divergence,
        solve and face correction; g.p and the face velocities are updated."""
        self._sync_problem(g)
        opts = Handle.options(self.precision, tol, max_iter, self.tol_mode, self.warm_start,
                              self.replace_every, self.project_mean, self.preconditioner)
        for name in ("p", "u", "v") + (("w",) if g.dim == 3 else ()):
            a = getattr(g, name)
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                setattr(g, name, np.ascontiguousarray(a, dtype=np.float64))
        self.last_stats = self.handle.project(g.u, g.v, g.w if g.dim == 3 else None, g.p, dt, opts)
        return self.last_stats

    def recover_static_pressure(self, g, max_iter, tol):
        """recoverStaticPressure on the GPU (uaamg_static_pressure): g.p receives the
        static pressure of the current velocity field (2D)."""
        self._sync_problem(g)
        opts = Handle.options(self.precision, tol, max_iter, self.tol_mode, False,
                              self.replace_every, self.project_mean, self.preconditioner)
        for name in ("p", "u", "v"):
            a = getattr(g, name)
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                setattr(g, name, np.ascontiguousarray(a, dtype=np.float64))
        self.last_stats = self.handle.static_pressure(g.u, g.v, g.p, opts)
        return self.last_stats

    def name(self):
        base = "PCG(CUDA-B200-UAAMG" if self.preconditioner else "CG(CUDA-B200"
        return f"{base},{self.precision})"


GpuUAAMGPCG3D = GpuUAAMGPCG


class SolverKind(enum.Enum):
    """Typed mirror of the Factory string keys (src/solver/factory.cpp:16-25) for
    the keys this library serves, plus the GPU keys it adds."""

    CG_GPU = "cg_gpu"
    PCG_UAAMG_GPU = "pcg_uaamg_gpu"
    PCG_UAAMG_GPU_FP32 = "pcg_uaamg_gpu_fp32"
    PCG_UAAMG_GPU_MIXED = "pcg_uaamg_gpu_mixed"


_KINDS = {
    SolverKind.CG_GPU: dict(precision="fp64", preconditioner=False),
    SolverKind.PCG_UAAMG_GPU: dict(precision="fp64"),
    SolverKind.PCG_UAAMG_GPU_FP32: dict(precision="fp32"),
    SolverKind.PCG_UAAMG_GPU_MIXED: dict(precision="mixed", tol_mode="rel"),
}


class Factory:
    """String-key factory for the GPU solvers (Factory::create).  Unlike the
    reference, an unknown key raises instead of silently returning Jacobi
    (factory.cpp:24): CPU-only solvers are not served by this library."""

    @staticmethod
    def create(name, device=0):
        kind = name if isinstance(name, SolverKind) else SolverKind(name)
        return GpuUAAMGPCG(device=device, **_KINDS[kind])


Factory3D = Factory


# ---------------------------------------------------------------------------
# Pressure projection (the caller of the path)


class PressureProjection:
    """PressureProjection::project (pressure.cpp:5-33; 3D: pressure_3d.cpp:5-40):
    rhs = div(u)/dt on fluid cells, p = 0, solve, u -= dt*grad p on faces between
    fluid cells."""

    @staticmethod
    def rhs(g, dt):
        nx, ny = g.nx, g.ny
        fluid = g.solid == 0
        if g.dim == 2:
            div = np.zeros(g.p.shape)
            div[1:-1, 1:-1] = ((g.u[1:-1, 1:] - g.u[1:-1, :-1]) / g.dx
                               + (g.v[1:, 1:-1] - g.v[:-1, 1:-1]) / g.dy)
            inner = np.zeros(g.p.shape, bool)
            inner[1:-1, 1:-1] = True
        else:
            div = np.zeros(g.p.shape)
            div[1:-1, 1:-1, 1:-1] = ((g.u[1:-1, 1:-1, 1:] - g.u[1:-1, 1:-1, :-1]) / g.dx
                                     + (g.v[1:-1, 1:, 1:-1] - g.v[1:-1, :-1, 1:-1]) / g.dy
                                     + (g.w[1:, 1:-1, 1:-1] - g.w[:-1, 1:-1, 1:-1]) / g.dz)
            inner = np.zeros(g.p.shape, bool)
            inner[1:-1, 1:-1, 1:-1] = True
        del nx, ny
        return np.where(inner & fluid, div / dt, 0.0)

    @staticmethod
    def correct(g, dt):
        s = g.solid != 0
        p = g.p
        if g.dim == 2:
            # u faces i = 1..nx-1 between cells i and i+1, rows j = 1..ny
            ok = ~(s[1:-1, 1:-2] | s[1:-1, 2:-1])
            g.u[1:-1, 1:-1] -= np.where(ok, dt * (p[1:-1, 2:-1] - p[1:-1, 1:-2]) / g.dx, 0.0)
            ok = ~(s[1:-2, 1:-1] | s[2:-1, 1:-1])
            g.v[1:-1, 1:-1] -= np.where(ok, dt * (p[2:-1, 1:-1] - p[1:-2, 1:-1]) / g.dy, 0.0)
        else:
            ok = ~(s[1:-1, 1:-1, 1:-2] | s[1:-1, 1:-1, 2:-1])
            g.u[1:-1, 1:-1, 1:-1] -= np.where(
                ok, dt * (p[1:-1, 1:-1, 2:-1] - p[1:-1, 1:-1, 1:-2]) / g.dx, 0.0)
            ok = ~(s[1:-1, 1:-2, 1:-1] | s[1:-1, 2:-1, 1:-1])
            g.v[1:-1, 1:-1, 1:-1] -= np.where(
                ok, dt * (p[1:-1, 2:-1, 1:-1] - p[1:-1, 1:-2, 1:-1]) / g.dy, 0.0)
            ok = ~(s[1:-2, 1:-1, 1:-1] | s[2:-1, 1:-1, 1:-1])
            g.w[1:-1, 1:-1, 1:-1] -= np.where(
                ok, dt * (p[2:-1, 1:-1, 1:-1] - p[1:-2, 1:-1, 1:-1]) / g.dz, 0.0)

    @staticmethod
    def recover_static_pressure(g, solver, max_iter, tol):
        """PressureProjection::recoverStaticPressure (pressure.cpp:35-66): the static
        pressure of the current velocities into g.p, its right-hand side built and
        solved on the GPU."""
        return solver.recover_static_pressure(g, max_iter, tol)

    @classmethod
    def project(cls, g, dt, solver, max_iter, tol, on_device=True):
        """A solver that can run the whole projection on the GPU does so (no
        host-side divergence or correction); any other solver gets the host steps."""
        if on_device and hasattr(solver, "project"):
            return solver.project(g, dt, max_iter, tol)
        rhs = cls.rhs(g, dt)
        g.p[...] = 0.0
        stats = solver.solve(g, rhs, max_iter, tol)
        cls.correct(g, dt)
        return stats


PressureProjection3D = PressureProjection
