"""The allocation-free residual check (uaamg_residual_noalloc) against the solver.

Callers that cannot allocate device memory -- code running under CUDA-graph
stream capture, host callbacks, or applications that own every allocation --
use uaamg_residual_noalloc to measure ||b - A p|| and ||b|| with no handle and no
cudaMalloc.  This test checks it, through the C-ABI, against the same two numbers
from the regular entry point (uaamg_solve_device with max_iter = 0 and a warm
start, whose exit statistics are the FP64 true residual of the given p) and against
the oracle's FP64 residual of the same p, on two calls in a row: the second call reuses the shared scratch the first one left.

This file is named to be collected last; it creates its own handle and buffers,
so it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import oracle as O
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # FP64 reductions in different orders


def _case(dim):
    from uaamg_b200 import workloads
    if dim == 3:
        solid, rhs = workloads.spheres_3d(40, 32, 24, nspheres=4, rmin=2.0, rmax=6.0, seed=9)
        sp = (1 / 40, 1 / 32, 1 / 24)
    else:
        solid, rhs = workloads.boxes(2, 96, 64, 0, 0.1, seed=9)
        sp = (1e-3, 1.5e-3, 1.0)
    return solid, rhs, sp


@pytest.mark.parametrize("dim", [3, 2])
def test_residual_noalloc_matches_solver(dim):
    import torch

    from uaamg_b200 import _capi
    from uaamg_b200.solver import Handle

    solid, rhs, sp = _case(dim)
    h = Handle(0)
    try:
        h.set_problem(solid, *sp)
        # a partly converged pressure, so the residual is far from zero
        p = np.zeros_like(rhs)
        h.solve(rhs, p, h.options("fp64", 1e-3, 3, "rel"))
        dev = torch.device("cuda:0")
        d_solid = torch.from_numpy(solid.copy()).to(dev)
        d_rhs = torch.from_numpy(rhs.copy()).to(dev)
        d_p = torch.from_numpy(p.copy()).to(dev)
        d_p_copy = d_p.clone()
        d_out = torch.zeros(2, dtype=torch.float64, device=dev)

        # the regular entry point: exit statistics of a zero-iteration warm start
        st = h.solve_device(d_rhs.data_ptr(), d_p_copy.data_ptr(),
                            h.options("fp64", 1e-6, 0, "rel", warm_start=True,
                                      preconditioner=False))
        ref = np.array([st.residual, st.rhs_norm])
        assert ref[0] > 1e-6 * ref[1]

        lib = _capi.load()
        nz = solid.shape[0] - 2 if dim == 3 else 0
        ny, nx = solid.shape[-2] - 2, solid.shape[-1] - 2
        stream = torch.cuda.current_stream(dev).cuda_stream
        for _ in range(2):
            d_out.fill_(-1.0)
            s = lib.uaamg_residual_noalloc(dim, nx, ny, nz, sp[0], sp[1], sp[2],
                                           C.c_void_p(d_solid.data_ptr()),
                                           C.c_void_p(d_rhs.data_ptr()),
                                           C.c_void_p(d_p.data_ptr()),
                                           C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
            assert s == _capi.OK
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            assert np.all(np.abs(got - ref) <= REL_TOL * np.abs(ref)), (got, ref)
        # and directly against the oracle's FP64 residual of the same p
        orc = np.array(O.true_residual(solid, rhs, p, *sp))
        assert np.all(np.abs(got - orc) <= REL_TOL * np.abs(orc)), (got, orc)
    finally:
        h.close()


def test_residual_noalloc_rejects_bad_sizes():
    from uaamg_b200 import _capi
    lib = _capi.load()
    null = C.c_void_p(0)
    # 1 interior cell along x, and a grid past 2^31 padded cells
    assert lib.uaamg_residual_noalloc(3, 1, 8, 8, 1.0, 1.0, 1.0, null, null, null, null,
                                      null) == _capi.INVALID_ARG
    assert lib.uaamg_residual_noalloc(3, 2048, 2048, 2048, 1.0, 1.0, 1.0, C.c_void_p(1),
                                      C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                      null) == _capi.INVALID_ARG
