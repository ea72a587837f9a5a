"""GPU checks of V-cycle mode 3 (every march level of a 2D problem as flat walks):
FP64 bit-exact against the reference's golden V-cycles and the oracle, and the PCG
with mode 3 against the default z marches in every precision."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture
def flat(handle):
    handle.set_vcycle_kernels(3)
    yield
    handle.set_vcycle_kernels(0)


@pytest.mark.parametrize("name", [n for n in golden_names("vcycle_") if "2d" in n])
def test_flat_vcycle_fp64_bit_exact(handle, flat, name):
    g = load_golden(name)
    handle.set_problem(g["solid"], g["dx"], g["dy"], g["dz"])
    z = handle.precond_apply(g["r"], "fp64")
    assert np.array_equal(z[1:-1, 1:-1], g["z"][1:-1, 1:-1])


@pytest.mark.parametrize("seed", range(4))
def test_flat_vcycle_random_vs_oracle(handle, flat, seed):
    from uaamg_b200 import workloads as W
    solid, rhs = W.boxes(2, 150 + 37 * seed, 97 + 11 * seed, 0, 0.1, seed=seed)
    sp = (1e-3, 1.5e-3)
    handle.set_problem(solid, *sp)
    z = handle.precond_apply(rhs, "fp64")
    zo = O.Hierarchy(solid, *sp).vcycle(rhs)
    assert np.array_equal(z[1:-1, 1:-1], zo[1:-1, 1:-1])


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_flat_pcg_matches_marches(handle, prec):
    from uaamg_b200 import workloads as W
    solid, rhs = W.boxes(2, 300, 200, 0, 0.1, seed=7)
    handle.set_problem(solid, 1e-3, 1.5e-3)
    opts = handle.options(prec, 1e-6, 400, "rel")
    p0 = np.zeros_like(rhs)
    s0 = handle.solve(rhs, p0, opts)
    handle.set_vcycle_kernels(3)
    try:
        p3 = np.zeros_like(rhs)
        s3 = handle.solve(rhs, p3, opts)
    finally:
        handle.set_vcycle_kernels(0)
    if prec == "fp64":
        # the V-cycle is bit-identical; the z sums are reduced in another order
        assert abs(s3.iterations - s0.iterations) <= 1
        assert np.abs(p3 - p0).max() <= 1e-6 * max(1.0, np.abs(p0).max())
    else:
        res, bn = O.true_residual(solid, rhs, p3, 1e-3, 1.5e-3)
        assert abs(s3.iterations - s0.iterations) <= 3
        if prec == "mixed":
            assert s3.status == 0 and res / bn <= 1e-6
