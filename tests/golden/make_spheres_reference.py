"""Runs the REFERENCE's own CPU solver (PCG3D + UAAMGPreconditioner3D, compiled
unchanged into oracle/_ref) on the 256^3 spheres workload to the relative
residual 1e-6 (absolute tol = 1e-6 * ||b||, b the PCG's normalised RHS) and
records its iteration count and wall time in spheres_256_reference.json, and
its pressure at 32768 seeded fluid cells (with the whole field's fluid mean and
mean-free L2 norm) in spheres_256_reference_p.npz.

The bench's reference arm and CPU baseline scale a one-iteration sample by this
count; GPU tests check that the FP64 GPU path needs the same count and that the
FP64 and mixed GPU pressures agree with the sampled reference pressure.

Run from the repository root after ``make -C oracle ref`` (takes minutes):
    python tests/golden/make_spheres_reference.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402
from uaamg_b200 import workloads  # noqa: E402


def main():
    solid, rhs, h = workloads.spheres_256()
    b = O.pcg_rhs(solid, rhs)
    bnorm = float(np.sqrt((b[solid == 0] ** 2).sum()))
    tol_abs = 1e-6 * bnorm
    t0 = time.perf_counter()
    p, applies = O.ref_pcg(solid, rhs, h, h, h, max_iter=500, tol=tol_abs)
    wall = time.perf_counter() - t0
    res, bn = O.true_residual(solid, rhs, p, h, h, h)
    out = {
        "workload": "spheres_256 (uaamg_b200.workloads.spheres_256)",
        "solver": "reference PCG3D(UAAMGPreconditioner3D), src/solver/pcg_3d.cpp",
        "tol_abs": tol_abs,
        "rhs_norm": bnorm,
        # the loop returns at its tolerance check, before that iteration's apply:
        # preconditioner applications = iterations (1 before the loop + iterations-1)
        "preconditioner_applications": applies,
        "iterations": applies,
        "true_rel_residual": res / bn,
        "wall_s_single_thread": round(wall, 1),
        "p_fluid_checksum": float(np.abs(p[solid == 0]).sum()),
    }
    # the reference pressure at seeded interior fluid cells (flat indices into the
    # padded array), for tests that compare whole-field-mean-free values
    inner = np.zeros(solid.shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    fl = np.flatnonzero((inner & (solid == 0)).reshape(-1))
    idx = np.sort(np.random.default_rng(20260303).choice(fl, 32768, replace=False))
    pf = p.reshape(-1)[fl]
    mean = float(pf.mean())
    l2 = float(np.sqrt(((pf - mean) ** 2).sum()))
    np.savez_compressed(os.path.join(HERE, "spheres_256_reference_p.npz"),
                        idx=idx.astype(np.int32), p=p.reshape(-1)[idx],
                        fluid_mean=np.float64(mean), fluid_l2=np.float64(l2))
    out["p_samples"] = "spheres_256_reference_p.npz"
    out["p_fluid_mean"] = mean
    out["p_fluid_meanfree_l2"] = l2
    with open(os.path.join(HERE, "spheres_256_reference.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
