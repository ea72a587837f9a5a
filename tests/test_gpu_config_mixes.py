"""The batch and serving forms at the sizes of their benchmark workloads, through the
C-ABI on the GPU, checked with the oracle's FP64 residual:

* the full 96-problem uneven batch (64 2D problems of 64..1024 cells per axis, 32 3D
  problems of 32..128 per axis, solid boxes over 0-20 % of the cells) in ONE
  uaamg_solve_batch call in the mixed form: every problem reaches a true relative
  residual of 1e-6, and sampled problems equal their solve alone bit for bit;
* the first 40 simulation ids of the serving mix (70 % 2D n^2 with n lognormal around
  384, 30 % 3D n^3 around 96; obstacle flows whose right-hand side drifts from step to
  step) for two steps each, 16 solves in flight: every request reaches 1e-6, every
  second-step request warm-starts, and sampled requests equal the same id served
  alone.
"""
import numpy as np
import pytest

from uaamg_b200 import workloads
from uaamg_b200.solver import Handle, Server

import oracle as O

pytestmark = pytest.mark.gpu


def _rel(solid, rhs, p, dx, dy, dz):
    a, b = O.true_residual(solid, rhs, p, dx, dy, dz)
    return a / b


def test_batch96_mixed_reaches_tolerance_and_matches_alone():
    probs = workloads.batch96()
    hd = Handle(0)
    try:
        opts = hd.options("mixed", 1e-6, 1000, "rel")
        ps = [np.zeros_like(r) for _, r, *_ in probs]
        stats = hd.solve_batch([(s, r, p, dx, dy, dz) for (s, r, dx, dy, dz), p in zip(probs, ps)],
                               opts)
        assert len(stats) == 96
        for q, ((s, r, dx, dy, dz), p, st) in enumerate(zip(probs, ps, stats)):
            assert st.status == 0, (q, st.status)
            assert _rel(s, r, p, dx, dy, dz) <= 1e-6, q
        for q in (0, 37, 63, 64, 95):  # 2D and 3D, smallest and largest classes
            s, r, dx, dy, dz = probs[q]
            hd.set_problem(s, dx, dy, dz)
            p = np.zeros_like(r)
            st = hd.solve(r, p, opts)
            assert st.iterations == stats[q].iterations, q
            assert np.array_equal(p, ps[q]), q
    finally:
        hd.close()


def _fields(plan, sid):
    return workloads.serve_fields(*plan[sid][1:4])


def _serve(plan, ids, steps, max_active):
    srv = Server(0, "mixed", 1e-6, 500, max_active=max_active)
    fields = {sid: _fields(plan, sid) for sid in ids}
    tickets = []
    for t in range(steps):
        for sid in ids:
            solid, r0, r1 = fields[sid]
            rhs = r0 + (t / 20.0) * r1
            h = 1.0 / plan[sid][2]
            p = np.zeros_like(rhs)
            tk = srv.submit(sid, solid, rhs, h, h, h if solid.ndim == 3 else 1.0, p_out=p)
            tickets.append((tk, sid, t, p, solid, rhs, h))
            if max_active == 1:
                srv.drain()
    srv.drain()
    out = {}
    for tk, sid, t, p, solid, rhs, h in tickets:
        res = srv.poll(tk)
        assert res is not None and res["status"] == 0, (sid, t, res)
        out[(sid, t)] = (p, res, solid, rhs, h)
    srv.stop()
    return out


def test_serving_mix_slice_reaches_tolerance_and_matches_alone():
    plan = workloads.serve_plan(500, 20)
    ids = list(range(40))
    mixed = _serve(plan, ids, 2, 16)
    for (sid, t), (p, res, solid, rhs, h) in mixed.items():
        assert res["warm"] == (1 if t > 0 else 0), (sid, t)
        assert _rel(solid, rhs, p, h, h, h if solid.ndim == 3 else 1.0) <= 1e-6, (sid, t)
    sample = [0, 4, 21, 25]  # 3D 62^3, 3D 88^3, 2D 1386^2, 3D 115^3
    alone = _serve(plan, sample, 2, 1)
    for key, (p, res, *_rest) in alone.items():
        pm, rm = mixed[key][0], mixed[key][1]
        assert res["iterations"] == rm["iterations"], key
        assert np.array_equal(p, pm), key
