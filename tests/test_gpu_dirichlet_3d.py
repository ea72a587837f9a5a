"""Dirichlet walls on a 3D problem with solid spheres and a different spacing per axis,
through the C-ABI on the GPU: the Dirichlet branches of the 3D search-direction march,
of the finest V-cycle level (the four-march form the engine runs when the finest level
has Dirichlet walls) and of the FP64 residual-replacement march of the mixed form,
checked against the oracle (the reference's operator with the wall channel,
pcg_3d.cpp:38-55; the wall share of the diagonal, uaamg_preconditioner_3d.cpp:50-66).
"""
import numpy as np
import pytest

from uaamg_b200 import workloads
from uaamg_b200.solver import Handle

import oracle as O

pytestmark = pytest.mark.gpu

SPACING = (1.0 / 40, 1.0 / 36, 1.0 / 44)


def _case():
    # 40 x 36 x 44 cells: two 32 x 16 column tiles along x, three along y, and odd
    # chunk remainders along z
    return workloads.spheres_3d(40, 36, 44, nspheres=4, rmin=3.0, rmax=6.0, seed=11,
                                sigma=2.0, trunc=8)


def _solve(solid, rhs, prec, tol, max_iter=400):
    hd = Handle(0)
    try:
        hd.set_dirichlet_walls(True)
        hd.set_problem(solid, *SPACING)
        p = np.zeros_like(rhs)
        st = hd.solve(rhs, p, hd.options(prec, tol, max_iter, "rel"))
    finally:
        hd.close()
    return p, st


def _rel_residual(solid, rhs, p):
    a, b = O.true_residual(solid, rhs, p, *SPACING, dirichlet=True)
    return a / b


def test_dirichlet_3d_fp64_matches_oracle():
    solid, rhs = _case()
    p, st = _solve(solid, rhs, "fp64", 1e-10)
    po, it, _ = O.pcg(solid, rhs, *SPACING, max_iter=400, tol=1e-10, tol_mode=1, dirichlet=True)
    assert st.status == 0
    assert abs(st.iterations - it) <= 1, (st.iterations, it)
    assert _rel_residual(solid, rhs, p) <= 1e-9
    assert np.abs(p - po).max() <= 1e-8 * np.abs(po).max()


def test_dirichlet_3d_mixed_reaches_tolerance():
    solid, rhs = _case()
    p64, _ = _solve(solid, rhs, "fp64", 1e-10)
    p, st = _solve(solid, rhs, "mixed", 1e-6)
    assert st.status == 0
    assert st.iterations > 10  # at least one FP64 residual replacement ran
    assert _rel_residual(solid, rhs, p) <= 1e-6
    fl = solid == 0
    assert np.linalg.norm((p - p64)[fl]) <= 1e-5 * np.linalg.norm(p64[fl])
