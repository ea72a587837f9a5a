"""Command-line solve of the spheres workload: one GPU PCG solve of an n^3 Neumann
Poisson problem with seeded solid spheres and a smoothed-noise right-hand side
(the 256^3 benchmark problem at n = 256), through the C-ABI.  With
--workload obstacle_2d --project: one device-side pressure projection (divergence,
solve, face correction) of the 2048 x 1024 obstacle flow; --workload layered_2d: the
same grid solved with the variable-coefficient operator of a layered medium.

    python -m uaamg_b200.solve_case --n 256 --precision mixed --max-iter 90
    python -m uaamg_b200.solve_case --workload obstacle_2d --project
    python -m uaamg_b200.solve_case --workload layered_2d --max-iter 10

Prints one line with the status, iterations, FP64 true relative residual and the
wall time of the solve.  Used as the profiling target of the kernel summaries
(a short --max-iter gives a capture of a few launches of every kernel).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads
from .solver import Handle


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64"])
    ap.add_argument("--max-iter", type=int, default=500)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--workload", default="spheres",
                    choices=["spheres", "obstacle_2d", "layered_2d"])
    ap.add_argument("--project", action="store_true")
    ap.add_argument("--vcycle-kernels", type=int, default=0, choices=[0, 1, 2, 3, 4])
    a = ap.parse_args(argv)
    if a.workload in ("obstacle_2d", "layered_2d"):
        solid, u0, v0, rhs, dx, dy, dt = workloads.obstacle_2d()
        hd = Handle(0)
        hd.set_vcycle_kernels(a.vcycle_kernels)
        hd.set_problem(solid, dx, dy)
        if a.workload == "layered_2d":
            hd.set_variable_laplacian(*workloads.layered_lap_2d(solid, dx, dy, 0.5))
        opts = hd.options(a.precision, a.tol, a.max_iter, "rel")
        for _ in range(a.repeat):
            p = np.zeros_like(rhs)
            u, v = u0.copy(), v0.copy()
            t0 = time.perf_counter()
            st = hd.project(u, v, None, p, dt, opts) if a.project else hd.solve(rhs, p, opts)
            ms = (time.perf_counter() - t0) * 1e3
        print(json.dumps({"workload": a.workload, "project": a.project, "precision": a.precision,
                          "status": st.status, "iterations": st.iterations,
                          "true_rel_residual": st.rel_residual, "ms": round(ms, 3)}))
        hd.close()
        return
    if a.n == 256:
        solid, rhs, h = workloads.spheres_256()
    else:
        r = a.n / 256.0
        solid, rhs = workloads.spheres_3d(a.n, a.n, a.n, 32, 8.0 * r, 24.0 * r)
        h = 1.0 / a.n
    hd = Handle(0)
    hd.set_vcycle_kernels(a.vcycle_kernels)
    hd.set_problem(solid, h, h, h)
    opts = hd.options(a.precision, a.tol, a.max_iter, "rel")
    for _ in range(a.repeat):
        p = np.zeros_like(rhs)
        t0 = time.perf_counter()
        st = hd.solve(rhs, p, opts)
        ms = (time.perf_counter() - t0) * 1e3
    print(json.dumps({"n": a.n, "precision": a.precision, "status": st.status,
                      "iterations": st.iterations, "true_rel_residual": st.rel_residual,
                      "solve_ms": round(ms, 3), "kernel_launches": st.kernel_launches}))
    hd.close()


if __name__ == "__main__":
    main()
