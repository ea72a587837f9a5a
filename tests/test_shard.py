"""Multi-GPU host logic on CPU: two gloo ranks split a batch and a serving mix with
uaamg_b200.shard, and combine their scalars and records exactly as bench.py does with
one process per GPU (no GPU needed: the collectives run on host tensors)."""
import datetime
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from uaamg_b200 import shard
        mine = shard.shard(list(range(11)), rank, world)
        everything = shard.gather(mine)
        worst = shard.reduce_max(0.25 + rank)
        total = shard.reduce_sum(1.0 + rank)
        ids = [i for i in range(9) if shard.owns(i, rank, world)]
        all_ids = shard.gather(ids)
        q.put((rank, mine, everything, worst, total, ids, all_ids))
    finally:
        dist.destroy_process_group()


def test_two_ranks_partition_the_work_and_combine_results():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            rank, *rest = q.get(timeout=120)
            out[rank] = rest
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    (m0, e0, w0, t0, i0, a0), (m1, e1, w1, t1, i1, a1) = out[0], out[1]
    assert not set(m0) & set(m1) and sorted(m0 + m1) == list(range(11))
    assert e0 == e1 and sorted(e0) == list(range(11))
    assert w0 == w1 == 1.25 and t0 == t1 == 3.0
    assert not set(i0) & set(i1) and sorted(a0) == list(range(9))


def test_single_process_falls_back_to_local_values():
    from uaamg_b200 import shard
    assert shard.shard([3, 1, 2], 0, 1) == [3, 1, 2]
    assert shard.reduce_max(2.5) == 2.5 and shard.reduce_sum(4.0) == 4.0
    assert shard.gather([1, 2]) == [1, 2]
    with pytest.raises(ValueError):
        shard.shard([1], 2, 2)
