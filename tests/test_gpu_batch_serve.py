"""Batched uneven solves and the serving loop, through the C-ABI on the GPU: every
result equals the same problem solved alone (bit for bit: the kernels, their
order and their reductions do not depend on what runs beside them), served
requests warm-start from their simulation's previous pressure, and admission
under a small device budget evicts idle simulations."""
import numpy as np
import pytest

from uaamg_b200 import workloads
from uaamg_b200.solver import Handle, Server

import oracle as O

pytestmark = pytest.mark.gpu


def _problems():
    """Six uneven problems: (solid, rhs, dx, dy, dz)."""
    out = []
    for q, (dim, nx, ny, nz, cov) in enumerate([(2, 64, 128, 0, 0.1), (2, 96, 64, 0, 0.0),
                                                (3, 32, 48, 40, 0.15), (3, 24, 24, 24, 0.05),
                                                (2, 200, 56, 0, 0.2), (3, 40, 32, 16, 0.1)]):
        s, r = workloads.boxes(dim, nx, ny, nz, cov, seed=900 + q)
        h = 1.0 / max(nx, ny, nz)
        out.append((s, r, h, h, h if dim == 3 else 1.0))
    return out


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_batch_matches_solving_each_problem_alone(prec):
    probs = _problems()
    hd = Handle(0)
    opts = hd.options(prec, 1e-6, 400, "rel")
    alone = []
    for s, r, dx, dy, dz in probs:
        hd.set_problem(s, dx, dy, dz)
        p = np.zeros_like(r)
        st = hd.solve(r, p, opts)
        alone.append((p, st.iterations))
    for rep in range(2):  # the second call reuses the problem slots
        ps = [np.zeros_like(r) for _, r, *_ in probs]
        stats = hd.solve_batch([(s, r, p, dx, dy, dz) for (s, r, dx, dy, dz), p in zip(probs, ps)],
                               opts)
        for q, ((pa, ita), pb, st) in enumerate(zip(alone, ps, stats)):
            assert st.iterations == ita, (rep, q)
            assert np.array_equal(pa, pb), (rep, q)
            if prec == "mixed":
                s, r, dx, dy, dz = probs[q]
                res, bn = O.true_residual(s, r, pb, dx, dy, dz)
                assert res / bn <= 1e-6
    hd.close()


def _sims():
    """Four simulations (two 2D, two 3D obstacle flows): (sim_id, dx, dy, dz, rhs at step t)."""
    sims = []
    for sid, (dim, n) in enumerate([(2, 96), (2, 160), (3, 24), (3, 32)]):
        h = 1.0 / n
        if dim == 2:
            def gen(t, n=n, h=h, sid=sid):
                s, _, _, r = workloads.obstacle_flow_2d(n, n, h, h, 1e-3, 4, 700 + sid, t * 1e-3)
                return s, r
        else:
            def gen(t, n=n, h=h, sid=sid):
                s, _, _, _, r = workloads.obstacle_flow_3d(n, n, n, h, h, h, 1e-3, 3, 700 + sid,
                                                           t * 1e-3)
                return s, r
        sims.append((sid, h, h, h if dim == 3 else 1.0, gen))
    return sims


def _serve(max_active, order, steps=3, budget=150 << 30):
    srv = Server(0, "mixed", 1e-6, 500, max_active=max_active, hbm_budget_bytes=budget)
    sims = {sid: (dx, dy, dz, gen) for sid, dx, dy, dz, gen in _sims()}
    out, tickets = {}, []
    for sid, t in order(sims, steps):
        dx, dy, dz, gen = sims[sid]
        s, r = gen(t)
        p = np.zeros_like(r)
        tk = srv.submit(sid, s, r, dx, dy, dz, p_out=p)
        tickets.append((tk, sid, t, p, s, r))
        if max_active == 1:  # alone: every request runs by itself
            srv.drain()
    srv.drain()
    for tk, sid, t, p, s, r in tickets:
        res = srv.poll(tk)
        assert res is not None and res["status"] == 0, res
        out[(sid, t)] = (p, res, s, r)
    info = srv.info()
    srv.stop()
    return out, info


def _by_step(sims, steps):
    return [(sid, t) for t in range(steps) for sid in sims]


def test_served_results_are_the_same_alone_and_in_the_mix():
    alone, _ = _serve(1, _by_step)
    mixed, info = _serve(8, _by_step)
    assert info["completed"] == len(alone) and info["resident"] == 4
    for key, (p, res, s, r) in alone.items():
        pm, rm, _, _ = mixed[key]
        assert np.array_equal(p, pm), key
        assert res["iterations"] == rm["iterations"], key
        assert res["warm"] == rm["warm"] == (1 if key[1] > 0 else 0), key
        dx = dy = dz = 1.0 / (s.shape[-1] - 2)
        err, bn = O.true_residual(s, r, p, dx, dy, dz if s.ndim == 3 else 1.0)
        assert err / bn <= 1e-6, key


def test_warm_start_saves_iterations():
    out, _ = _serve(4, _by_step, steps=3)
    for sid in range(4):
        assert out[(sid, 2)][1]["iterations"] < out[(sid, 0)][1]["iterations"], sid


def test_small_budget_evicts_idle_simulations():
    # room for about one simulation: requests still finish, evicted ids restart cold
    out, info = _serve(2, _by_step, steps=2, budget=5 << 20)
    assert info["resident"] <= 2
    assert all(res["status"] == 0 for _, res, _, _ in out.values())
    assert any(res["warm"] == 0 for (sid, t), (_, res, _, _) in out.items() if t == 1)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_autotuned_chunks_give_identical_results(prec):
    """The z-chunk length changes only the blocks' shape: the preconditioner (every
    per-cell value) is bit-identical with autotuned chunks.  The solve's FP64 dot
    products are summed per block, so a different chunk length sums them in another
    order: the PCG iterates agree to rounding (FP64 1e-10, mixed 1e-6 relative) and
    the iteration counts to one."""
    s, r = workloads.spheres_3d(80, 64, 72, 12, 3.0, 9.0, seed=11)
    h = 1.0 / 80
    out, z = [], []
    for tune in (False, True):
        hd = Handle(0)
        hd.set_autotune(tune)
        hd.set_problem(s, h, h, h)
        z.append(hd.precond_apply(r, prec))
        p = np.zeros_like(r)
        st = hd.solve(r, p, hd.options(prec, 1e-6, 300, "rel"), strict=True)
        out.append((p, st.iterations))
        hd.close()
    assert np.array_equal(z[0], z[1])
    assert abs(out[0][1] - out[1][1]) <= 1
    d = np.abs(out[0][0] - out[1][0]).max() / np.abs(out[0][0]).max()
    assert d <= (1e-10 if prec == "fp64" else 1e-6), d


@pytest.mark.parametrize("prec", ["mixed", "fp32", "fp64"])
def test_smoothing_schedules_converge(prec):
    """V(nu, nu) cycles (uaamg_set_smoothing): more sweeps on the coarse levels, or on
    every level, still give a symmetric preconditioner -- PCG reaches the same
    tolerance (the mixed form's FP64 true residual 1e-6; FP64 and plain FP32 their
    recursive one) -- and needs no more iterations than the reference's V(1,1) (to
    within two)."""
    probs = _problems()[1:4]
    hd = Handle(0)
    for s, r, dx, dy, dz in probs:
        hd.set_problem(s, dx, dy, dz)
        its = {}
        for nu in [(1, 1), (1, 2), (2, 2)]:
            hd.set_smoothing(*nu)
            p = np.zeros_like(r)
            st = hd.solve(r, p, hd.options(prec, 1e-6, 400, "rel"))
            assert st.status == 0, (prec, nu, st.status)
            if prec == "mixed":
                res, bn = O.true_residual(s, r, p, dx, dy, dz)
                assert res / bn <= 1e-6, (nu, res / bn)
            its[nu] = st.iterations
        hd.set_smoothing(1, 1)
        assert its[(2, 2)] <= its[(1, 1)] + 2 and its[(1, 2)] <= its[(1, 1)] + 2, its
    hd.close()


def test_batch_autotune_schedules_and_cache_file(tmp_path):
    """With the autotuner on, a mixed batch picks a smoothing schedule and z-chunk
    lengths per problem class, stores them in the cache file, and a second batch call
    reuses them (identical results); every result meets the true residual 1e-6."""
    import json
    from uaamg_b200.solver import set_tune_cache
    path = tmp_path / "tune.json"
    set_tune_cache(str(path))
    try:
        probs = _problems()[:4]
        hd = Handle(0)
        hd.set_autotune(True)
        opts = hd.options("mixed", 1e-6, 400, "rel")
        runs = []
        for rep in range(2):
            ps = [np.zeros_like(r) for _, r, *_ in probs]
            hd.solve_batch([(s, r, p, dx, dy, dz) for (s, r, dx, dy, dz), p in zip(probs, ps)], opts)
            runs.append(ps)
            for (s, r, dx, dy, dz), p in zip(probs, ps):
                res, bn = O.true_residual(s, r, p, dx, dy, dz)
                assert res / bn <= 1e-6
        for a, b in zip(*runs):
            assert np.array_equal(a, b)
        entries = json.load(open(path))["entries"]
        assert sum(k.startswith("nu|") for k in entries) == len(probs)
        assert any(k.startswith("zc|") for k in entries)
        assert all(v in ([1, 1], [1, 2], [2, 2]) for k, v in entries.items() if k.startswith("nu|"))
        hd.close()
    finally:
        set_tune_cache(None)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_batch_group_graph_matches_per_problem_graphs(prec):
    """uaamg_set_batch_group: the small problems of a batch replayed as one CUDA graph
    per step give the same results, bit for bit, as one graph per problem (the same
    kernels in the same order on each problem's stream)."""
    probs = _problems()
    hd = Handle(0)
    opts = hd.options(prec, 1e-6, 400, "rel")
    out = {}
    for group in (0, 40000):
        hd.set_batch_group(group)
        ps = [np.zeros_like(r) for _, r, *_ in probs]
        stats = hd.solve_batch([(s, r, p, dx, dy, dz) for (s, r, dx, dy, dz), p in zip(probs, ps)],
                               opts)
        out[group] = (ps, [st.iterations for st in stats])
    hd.set_batch_group(0)
    assert out[0][1] == out[40000][1]
    for a, b in zip(out[0][0], out[40000][0]):
        assert np.array_equal(a, b)
    hd.close()


def test_borrowed_request_buffers_match_copies():
    """UAAMG_REQUEST_BORROW: a request that lends its right-hand side and output
    (no host copies; pinned here, so the device copies are asynchronous) gives the
    same pressure, bit for bit, as the copying submit."""
    import torch
    sims = _sims()
    out = {}
    for borrow in (False, True):
        srv = Server(0, "mixed", 1e-6, 500, max_active=4)
        tickets = []
        for sid, dx, dy, dz, gen in sims:
            s, r = gen(0)
            if borrow:
                rb = torch.empty(r.shape, dtype=torch.float64, pin_memory=True)
                pb = torch.zeros(r.shape, dtype=torch.float64, pin_memory=True)
                rb.numpy()[...] = r
                tk = srv.submit(sid, s, rb.numpy(), dx, dy, dz, p_out=pb.numpy(), borrow=True)
                tickets.append((tk, sid, pb, rb))
            else:
                p = np.zeros_like(r)
                tk = srv.submit(sid, s, r, dx, dy, dz, p_out=p)
                tickets.append((tk, sid, p, None))
        srv.drain()
        for tk, sid, p, _ in tickets:
            res = srv.poll(tk)
            assert res is not None and res["status"] == 0, res
            out[(borrow, sid)] = np.array(p.numpy() if borrow else p)
        srv.stop()
    for sid, *_ in sims:
        assert np.array_equal(out[(False, sid)], out[(True, sid)]), sid
