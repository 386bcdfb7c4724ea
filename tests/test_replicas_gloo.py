"""The multi-GPU path on CPU: two gloo ranks shard rooms and combine the
timing exactly as bench.py does under torchrun (max over ranks)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ff-room_b200"))
    from ffrb.replicas import max_over_ranks, shard, sum_over_ranks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rooms = list(range(10))
    mine = shard(rooms, rank, world)
    t = 1.5 + rank            # a per-rank "device time"
    tmax = max_over_ranks(t, dist)
    cells = sum_over_ranks(sum(mine), dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, tmax, cells))


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, c0), (r1, m1, t1, c1) = res
    assert m0 == [0, 2, 4, 6, 8] and m1 == [1, 3, 5, 7, 9]
    assert t0 == t1 == 2.5
    assert c0 == c1 == 45


def test_shard_rejects_bad_rank():
    from ffrb.replicas import shard
    with pytest.raises(ValueError):
        shard([1, 2], 2, 2)
