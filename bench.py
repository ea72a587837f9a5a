"""Benchmark: 256^3 UAAMG-preconditioned CG pressure solve on B200.

One step = one full pressure solve (7-point Neumann Poisson, 256^3 cells, 32 solid
spheres, smoothed-noise RHS) to FP64 true relative residual 1e-6 with the mixed
precision solver (FP32 CG + FP32 V-cycle, FP64 reductions, FP64 solution with
residual replacement every 10 iterations).  Inputs are resident in HBM for
`value`; `e2e` repeats the measurement through the host-array C-ABI call
(uaamg_solve) with the host<->device copies inside the timed region.

Multi-GPU (torchrun, one process per GPU): every rank solves its own replica of
the problem -- the solve does not shard -- so scaling is weak, `value` is the
whole-job time per solve (max-over-ranks time / solves of all ranks) and no
collective touches the data path.

--impl reference times the reference's own CPU solver (PCG3D + UAAMG3D, compiled
unchanged into oracle/_ref) on the same workload on the host cores: each step is a
bounded sample (one PCG iteration), scaled to a full solve by the reference's
iteration count for this workload (tests/golden/spheres_256_reference.json).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D 256^3 PCG solve ms (1e-6 rel. residual)"
WORKLOAD = ("spheres_256: 256^3 7-point Neumann Poisson, h=1/256, 32 seeded solid spheres "
            "r~U[8,24] cells, RHS = N(0,1) noise blurred sigma=4 cells, zero at solids, "
            "zero fluid mean (seed 20260303)")
REF_ITER_FIXTURE = os.path.join(ROOT, "tests", "golden", "spheres_256_reference.json")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _ref_iterations():
    with open(REF_ITER_FIXTURE) as f:
        return json.load(f)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q] == "Active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    """The reference's CPU PCG3D+UAAMG3D on the host cores (rank 0 only)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from uaamg_b200 import workloads

    kind = "reference" if O.have_ref() else "port"
    solid, rhs, h = workloads.spheres_256()
    fx = _ref_iterations()
    n_it = int(fx["iterations"])
    b = O.pcg_rhs(solid, rhs)
    tol_abs = 1e-6 * float((b[solid == 0] ** 2).sum()) ** 0.5
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_pcg(solid, rhs, h, h, h, max_iter=1, tol=tol_abs)
        else:
            O.pcg(solid, rhs, h, h, h, max_iter=1, tol=tol_abs, tol_mode=0)
        dt = (time.perf_counter() - t0) * 1e3
        if s >= args.warmup:
            times.append(dt)
    per_iter_sample = statistics.mean(times)
    value = per_iter_sample * n_it / 2.0
    sample = (f"one PCG iteration of the 256^3 solve (max_iter=1: 2 V-cycle applications "
              f"with their per-apply hierarchy rebuilds) per step, single thread; full solve = "
              f"sample x {n_it}/2 ({n_it} iterations to 1e-6, tests/golden/"
              f"spheres_256_reference.json)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(value, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64 (reference CPU)", "tol": 1e-6,
                   "iterations": n_it},
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": 1, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(solid, rhs, h, n_it):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    kind = "reference" if O.have_ref() else "port"
    b = O.pcg_rhs(solid, rhs)
    tol_abs = 1e-6 * float((b[solid == 0] ** 2).sum()) ** 0.5
    t0 = time.perf_counter()
    if kind == "reference":
        O.ref_pcg(solid, rhs, h, h, h, max_iter=1, tol=tol_abs)
    else:
        O.pcg(solid, rhs, h, h, h, max_iter=1, tol=tol_abs, tol_mode=0)
    t = (time.perf_counter() - t0) * 1e3
    return {"value": round(t * n_it / 2.0, 1), "unit": "ms", "cores": 1, "kind": kind,
            "sample": (f"one PCG iteration of the same 256^3 solve (2 V-cycle applications), "
                       f"single thread, {t / 1e3:.1f} s; full solve = sample x {n_it}/2")}


def run_ours(args):
    import numpy as np
    import torch

    ws, rank, local = _dist()
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)

    from uaamg_b200 import _capi, workloads
    from uaamg_b200.solver import Handle

    solid, rhs, h = workloads.spheres_256()
    hd = Handle(device)
    hd.set_problem(solid, h, h, h)
    opts = hd.options(args.precision, 1e-6, 500, "rel", replace_every=10)
    d_rhs = torch.from_numpy(rhs).to(f"cuda:{device}")
    d_p = torch.zeros_like(d_rhs)
    n_cells = rhs.size

    def step():
        d_p.zero_()
        return hd.solve_device(d_rhs.data_ptr(), d_p.data_ptr(), opts)

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    with ClockSampler(device) as clk:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launches = 0
        for _ in range(args.steps):
            st = step()
            launches += st.kernel_launches
        e1.record()
        torch.cuda.synchronize()
        barrier()
    elapsed = e0.elapsed_time(e1)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([elapsed], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    ms_per_step = elapsed / args.steps
    value = elapsed / (args.steps * ws)
    clocks = clk.summary()
    stats = st.as_dict()

    # e2e: the host-array C-ABI call, pinned host buffers, copies inside the timing
    h_rhs = torch.from_numpy(rhs).pin_memory()
    h_p = torch.zeros_like(h_rhs).pin_memory()
    rhs_np, p_np = h_rhs.numpy(), h_p.numpy()
    e2e_times = []
    for s in range(args.warmup + args.steps):
        p_np[...] = 0.0
        barrier()
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        hd.solve(rhs_np, p_np, opts)
        a1.record()
        torch.cuda.synchronize()
        if s >= args.warmup:
            e2e_times.append(a0.elapsed_time(a1))
    e2e_ms = sum(e2e_times) / len(e2e_times)
    if ws > 1:
        t = torch.tensor([e2e_ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_val = e2e_ms / ws

    # true residual of the e2e result, recomputed in FP64 on the host (oracle)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    res, bn = O.true_residual(solid, rhs, p_np, h, h, h)

    # in-situ per-kernel timing (one extra, unmeasured solve)
    d_p.zero_()
    _, rows = hd.profile_solve(d_rhs.data_ptr(), d_p.data_ptr(), opts)
    per_class = {}
    for r in rows:
        key = r["name"] if r["level"] == 0 else f"{r['name']}@L{r['level']}"
        per_class[key] = r
    total = sum(r["total_ms"] for r in rows)
    top = max(rows, key=lambda r: r["total_ms"])
    peak, peak_kind = _peaks()
    avg_ms = top["total_ms"] / top["launches"]
    achieved = top["bytes_per_launch"] / (avg_ms * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tfile):
        try:
            tk = json.load(open(tfile))
            key = f"{top['name']}@L{top['level']}"
            if key in tk:
                traffic = tk[key]
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": f"{top['name']} (level {top['level']})",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 3), "traffic": traffic,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": top["bytes_per_launch"],
                "avg_launch_us": round(avg_ms * 1e3, 2),
                "share_of_solve": round(top["total_ms"] / total, 3)}
    kernels = sorted(
        ({"kernel": k, "launches": v["launches"], "ms": round(v["total_ms"], 4),
          "share": round(v["total_ms"] / total, 4),
          "GB/s": round(v["bytes_per_launch"] * v["launches"] / (v["total_ms"] * 1e-3) / 1e9, 1)
          if v["total_ms"] > 0 and v["bytes_per_launch"] > 0 else None}
         for k, v in per_class.items()), key=lambda d: -d["ms"])[:12]

    # plain FP32 PCG and FP64 beside the headline (single solves, same inputs)
    beside = {}
    if rank == 0 and not args.no_beside:
        for prec in ("fp32", "fp64"):
            o2 = hd.options(prec, 1e-6, 500, "rel")
            d_p.zero_()
            torch.cuda.synchronize()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record()
            s2 = hd.solve_device(d_rhs.data_ptr(), d_p.data_ptr(), o2)
            b1.record()
            torch.cuda.synchronize()
            d_p.zero_()
            b0.record()
            s2 = hd.solve_device(d_rhs.data_ptr(), d_p.data_ptr(), o2)
            b1.record()
            torch.cuda.synchronize()
            beside[prec] = {"ms": round(b0.elapsed_time(b1), 3), "iterations": s2.iterations,
                            "true_rel_residual": s2.rel_residual,
                            "recursive_rel_residual": s2.recursive_residual / s2.rhs_norm}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        if os.path.exists(REF_ITER_FIXTURE):
            n_it = _ref_iterations()["iterations"]
        else:  # the FP64 GPU path runs the reference's iteration sequence
            n_it = beside.get("fp64", {}).get("iterations", stats["iterations"])
        cpu = cpu_baseline_sample(solid, rhs, h, n_it)

    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "ms", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 reductions and solution)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": args.precision, "tol": 1e-6,
                   "tol_rule": "FP64 true ||b-Ax||/||b||", "replace_every": 10,
                   "iterations": stats["iterations"],
                   "true_rel_residual": stats["rel_residual"],
                   "host_checked_rel_residual": res / bn,
                   "l2": "inputs larger than L2 (solve working set ~1.2 GB vs 126 MB L2)",
                   "parallelism": f"replicas x{ws}"},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_val, 3), "unit": "ms",
                "h2d_bytes_per_step": 2 * n_cells * 8, "d2h_bytes_per_step": n_cells * 8},
        "gpu_launches": launches,
        "clocks": clocks,
        "kernels": kernels,
        "beside": beside,
    }
    print(json.dumps(line), flush=True)
    hd.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-beside", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
