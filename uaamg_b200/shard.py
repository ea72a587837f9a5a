"""Spreading independent pressure problems over the GPUs of one node.

One process per GPU (the ranks of a torch.distributed job): each rank takes its own
share of the problems of a batch, or the simulation ids it owns in a serving mix, and
solves them on its own device.  The problems share no data, so nothing crosses ranks
on the data path; only scalars (times, worst residuals, rates) and per-request result
records are combined once at the end.  Work per GPU stays fixed as GPUs are added
(weak scaling).  Works with any backend: NCCL (tensors on the rank's GPU) or gloo
(tensors on the host).
"""
from __future__ import annotations


def shard(items, rank: int, world: int):
    """This rank's share of a list of independent problems (round-robin, so uneven
    problem sizes spread evenly)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    return list(items)[rank::world]


def owns(sim_id: int, rank: int, world: int) -> bool:
    """Whether this rank serves simulation id sim_id (every request of an id goes to
    the same rank, so its warm-start pressure stays on one GPU)."""
    return sim_id % world == rank


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _reduce(x: float, op) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x: float) -> float:
    """Maximum of x over the ranks (x itself without a process group)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX if dist.is_available() else None)


def reduce_sum(x: float) -> float:
    """Sum of x over the ranks (x itself without a process group)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM if dist.is_available() else None)


def gather(records: list) -> list:
    """Every rank's list of records, concatenated in rank order, on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(records)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(records))
    return [r for part in out for r in part]
