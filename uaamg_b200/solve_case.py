"""Command-line solve of the spheres workload: one GPU PCG solve of an n^3 Neumann
Poisson problem with seeded solid spheres and a smoothed-noise right-hand side
(the 256^3 benchmark problem at n = 256), through the C-ABI.

    python -m uaamg_b200.solve_case --n 256 --precision mixed --max-iter 90

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
    a = ap.parse_args(argv)
    if a.n == 256:
        solid, rhs, h = workloads.spheres_256()
    else:
        r = a.n / 256.0
        solid, rhs = workloads.spheres_3d(a.n, a.n, a.n, 32, 8.0 * r, 24.0 * r)
        h = 1.0 / a.n
    hd = Handle(0)
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
