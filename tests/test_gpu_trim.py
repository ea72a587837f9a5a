"""Coarse-level trimming on the whole-tile box levels (the reference's tile trimming,
src/solver/cuda/cuda_uaamg_preconditioner_3d.cu:81-99 and :357-375): a box whose tile
and 2-cell ring are interior fluid with one diagonal and one coupling per axis runs
without loading its diagonals, couplings and codes.  The values it uses are the
stored ones, so every result is identical with and without trimming; the FP64
V-cycle stays bit-exact against the oracle on a problem where most coarse boxes are
trimmed."""
import os

import numpy as np
import pytest

from uaamg_b200 import workloads
from uaamg_b200.solver import Handle

import oracle as O

pytestmark = pytest.mark.gpu


def _case():
    # 96^3: level 1 (48^3), level 2 (24^3) and level 3 (12^3) run as boxes
    solid, rhs = workloads.spheres_3d(96, 96, 96, nspheres=3, rmin=4.0, rmax=8.0, seed=41)
    return solid, rhs, 1.0 / 96


def _handle(solid, h, trim):
    if not trim:
        os.environ["UAAMG_NO_TRIM"] = "1"
    try:
        hd = Handle(0)
        hd.set_problem(solid, h, h, h)
        for prec in ("fp64", "fp32", "mixed"):  # every precision's engine is built here
            hd.precond_apply(np.zeros_like(solid, dtype=np.float64), prec)
    finally:
        os.environ.pop("UAAMG_NO_TRIM", None)
    return hd


def test_trimmed_vcycle_fp64_bit_exact():
    solid, r, h = _case()
    hd = _handle(solid, h, True)
    try:
        boxes, trimmed = hd.level_trim(1, "fp64")
        assert boxes == 6 ** 3 and 0 < trimmed <= 4 ** 3, (boxes, trimmed)
        z = hd.precond_apply(r, "fp64")
    finally:
        hd.close()
    zr = O.Hierarchy(solid, h, h, h).vcycle(r)
    sl = (slice(1, -1),) * 3
    assert np.array_equal(z[sl], zr[sl])


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_trimming_changes_no_value(prec):
    solid, r, h = _case()
    on, off = _handle(solid, h, True), _handle(solid, h, False)
    try:
        assert on.level_trim(1, prec)[1] > 0 and off.level_trim(1, prec)[1] == 0
        assert np.array_equal(on.precond_apply(r, prec), off.precond_apply(r, prec))
        ps, its = [], []
        for hd in (on, off):
            p = np.zeros_like(r)
            st = hd.solve(r, p, hd.options(prec, 1e-6, 300, "rel"))
            ps.append(p)
            its.append(st.iterations)
        assert its[0] == its[1]
        assert np.array_equal(ps[0], ps[1])
    finally:
        on.close()
        off.close()
