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


class _FakeBatch:
    """Stands in for godar_b200.lib.Batch on the CPU: records admissions and
    steps (no device)."""

    def __init__(self):
        self.fields, self.steps = [], 0

    def add_field(self, f):
        self.fields.append(f)
        return len(self.fields) - 1

    def step(self, k):
        self.steps += k

    def sync(self):
        return float(sum(f.n for f in self.fields)) * self.steps * 1e-6


def _bench_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from godar_b200.shard import max_over_ranks
    fields = bench.make_ensemble(12, rank, world, 1)
    b = _FakeBatch()
    for f in fields:
        b.add_field(f)
    b.step(5)
    ms = max_over_ranks(b.sync(), dist)
    got = [None] * world
    dist.all_gather_object(got, [(f.name, f.n, b.steps) for f in b.fields])
    if rank == 0:
        q.put((got, ms, [int(x) for x in bench.ensemble_sizes(12)]))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_ranks_step_disjoint_shares_of_one_ensemble():
    """bench.py under torchrun: each rank generates and steps only its LPT
    share of the one ensemble; together the ranks cover every field once,
    with the sizes the ensemble names."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, ms, sizes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    names = [n for part in got for n, _, _ in part]
    assert sorted(names) == sorted(f"ensemble[{i}]" for i in range(len(sizes)))
    for part in got:
        for name, n, steps in part:
            assert n == sizes[int(name.split("[")[1].rstrip("]"))]
            assert steps == 5
    loads = [sum(n for _, n, _ in part) for part in got]
    assert max(loads) - min(loads) <= max(sizes)
    assert ms == max(float(l) * 5 * 1e-6 for l in loads)
