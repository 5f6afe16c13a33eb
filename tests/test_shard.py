"""Ensemble sharding over ranks, checked with 2 gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from godar_b200.shard import lpt_partition


def test_lpt_partition_balanced_and_complete():
    from godar_b200 import generators as gen
    sizes = gen.ensemble_sizes(512)
    for k in (1, 2, 4, 8):
        parts = lpt_partition(sizes, k)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(np.sum(sizes[p])) for p in parts]
        assert max(loads) - min(loads) <= int(np.max(sizes))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from godar_b200 import generators as gen
    from godar_b200.shard import max_over_ranks, rank_share
    sizes = gen.ensemble_sizes(64)
    mine = rank_share(sizes, rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        q.put((got, t, [int(x) for x in sizes]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_disjoint_cover_and_max_time():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, t, sizes = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = set(got[0]), set(got[1])
    assert not (a & b) and (a | b) == set(range(len(sizes)))
    assert t == 2.0
