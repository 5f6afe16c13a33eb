"""Serving: a request loop over one GPU with continuous batching.

Each request is a floe field to advance by a number of time steps (the
reference runs one field per job, utils/duplication.sh:551-588).  Requests
arrive over time; between chunks of steps the loop admits every request that
has arrived and fits the HBM budget (godar_batch_add refuses the rest, which
wait), advances all resident fields together in one batch, and retires the
fields that finished, so new work joins while earlier work is still on the
GPU.  A field's state stays on the device from admission to completion.

Latency of a request = completion time - arrival time (wall clock of the
loop).  Throughput = floe-steps of all requests / makespan.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .lib import Batch, GodarError
from .params import PREC_MIXED

GODAR_ERR_BUDGET = 8


@dataclass
class Request:
    rid: int
    arrival: float            # seconds after the start of the stream
    fld: object               # godar_b200.generators.Field
    nsteps: int
    admitted: float = -1.0
    done: float = -1.0
    result: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.fld.n


@dataclass
class ServeStats:
    completed: int
    makespan_s: float
    floe_steps: int
    throughput: float         # floe-steps/s over the makespan
    p50_s: float
    p99_s: float
    mean_queue_s: float
    max_resident: int
    gpu_ms: float

    def as_dict(self):
        return dict(self.__dict__)


def serve(requests, precision: int = PREC_MIXED, hbm_budget: int = 150 * 10**9, chunk: int = 50,
          keep: tuple = ("x", "y"), realtime: bool = True, on_complete=None,
          reserve: int = 16 << 30) -> ServeStats:
    """Runs the request stream to completion.  With realtime=False arrivals
    are admitted as soon as the loop reaches them (no waiting), which is how
    the tests replay a stream deterministically.  Before the first arrival
    the batch's memory pool is grown to min(reserve, hbm_budget) bytes."""
    b = Batch(precision, hbm_budget)
    try:
        if reserve > 0:
            b.reserve(min(reserve, hbm_budget) if hbm_budget else reserve)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting = deque()
        active = {}                # hid -> [request, steps left]
        t0 = time.perf_counter()
        gpu_ms = 0.0
        max_res = 0
        lat = []
        queue = []
        while pending or waiting or active:
            now = time.perf_counter() - t0
            while pending and (pending[0].arrival <= now or not realtime):
                waiting.append(pending.popleft())
            while waiting:
                rq = waiting[0]
                try:
                    hid = b.add_field(rq.fld)
                except GodarError as e:
                    if e.status == GODAR_ERR_BUDGET and active:
                        break
                    raise
                waiting.popleft()
                rq.admitted = time.perf_counter() - t0
                active[hid] = [rq, rq.nsteps]
            max_res = max(max_res, len(active))
            if not active:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.005)))
                continue
            k = min(chunk, min(v[1] for v in active.values()))
            b.step(k)
            gpu_ms += b.sync()
            finished = []
            for hid, v in active.items():
                v[1] -= k
                if v[1] == 0:
                    finished.append(hid)
            # read every finished field before removing any (a removal re-lays
            # the batch at the next step, not at once)
            for hid in finished:
                rq = active[hid][0]
                rq.result = {name: b.field(hid, name) for name in keep}
            for hid in finished:
                rq = active.pop(hid)[0]
                b.remove(hid)
                rq.done = time.perf_counter() - t0
                lat.append(rq.done - rq.arrival if realtime else rq.done - rq.admitted)
                queue.append(rq.admitted - rq.arrival if realtime else 0.0)
                if on_complete:
                    on_complete(rq)
        makespan = time.perf_counter() - t0
    finally:
        # the batch's device memory is returned on every exit, errors included
        b.close()
    fs = int(sum(r.n * r.nsteps for r in requests))
    lat_a = np.array(lat) if lat else np.zeros(1)
    return ServeStats(completed=len(lat), makespan_s=makespan, floe_steps=fs,
                      throughput=fs / makespan if makespan > 0 else 0.0,
                      p50_s=float(np.percentile(lat_a, 50)), p99_s=float(np.percentile(lat_a, 99)),
                      mean_queue_s=float(np.mean(queue)) if queue else 0.0, max_resident=max_res,
                      gpu_ms=gpu_ms)


def make_stream(count: int, rate: float = 20.0, seed: int = 5, lo: int = 512, hi: int = 65536,
                nsteps: int = 2000, procs: int = 1):
    """The served request stream of the benchmark's fifth configuration:
    Poisson arrivals at `rate` req/s, floe counts log-uniform in [lo, hi],
    bonded fields with their own seed and wind."""
    from . import generators as gen
    t, n = gen.served_arrivals(count, rate, seed, lo, hi)
    jobs = [(k, int(n[k]), nsteps) for k in range(count)]
    if procs > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(procs) as pool:
            fields = pool.map(_member, jobs, chunksize=1)
    else:
        fields = [_member(j) for j in jobs]
    return [Request(rid=k, arrival=float(t[k]), fld=fields[k], nsteps=nsteps) for k in range(count)]


def _member(job):
    from . import generators as gen
    k, n, nsteps = job
    return gen.served_member(k, n, nsteps=nsteps)
