#!/usr/bin/env python
"""Benchmark: floe-steps/s of the batched ensemble on B200.

Workload: the batched ensemble of 512 independent floe fields (floe counts
log-uniform in [256, 16384], bonded-field generator with seeds 10+i, 80%
target area fraction, uniform wind of random direction U[0,360) deg and speed
U[8,16] m/s), advanced with FP32 pair forces and FP64 integration, bond and
ridging state: per time step a candidate screen, the contact work list, the
bonds, the per-floe force sums and the floe update (forcing, integration),
replayed as CUDA graphs.  A "step" is one time step of every instance.  Under
torchrun each rank runs its share of the one ensemble (split by floe count):
strong scaling, no collective on the data path.

Reported beside it: the roofline of the dominant kernel and of each kernel
(HBM-bound), the plain FP64 single-instance GPU path on a sample of the same
ensemble and the FP64 method batched over the whole ensemble, the position
error of the mixed path against FP64, the end-to-end rate through the C ABI
with host buffers, the whole 1000-step run of the ensemble from admission,
the served request stream (1000 requests, 2000 steps each, both precisions)
with its latency, and the CPU oracle timed on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl godar|reference]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# steps of the engine's online autotuner (two samples of each of the screen's
# nine candidates) before a batch's launch configuration is fixed
TUNE_STEPS = 18
PHASE_EVERY = 16   # steps of the timed call whose kernels are timed one by one
METRIC = "floe-steps/s batched+served vs plain GPU at <=1e-5 rel err; p50/p99 latency"
UNIT = "floe-steps/s"


# ---------------------------------------------------------------- helpers
def _member(args):
    i, n = args
    from godar_b200 import generators as gen
    return gen.ensemble_member(i, int(n))


def ensemble_sizes(count: int):
    from godar_b200 import generators as gen
    return gen.ensemble_sizes(count, seed=4)


def make_ensemble(count: int, rank: int, nranks: int, procs: int):
    """The benchmark ensemble (512 fields, sizes log-uniform in [256, 16384],
    member i generated with seed 10+i), or this rank's share of it: fields
    are independent, so ranks split the one ensemble by floe count
    (longest-processing-time partition) and exchange nothing."""
    from godar_b200.shard import rank_share
    sizes = ensemble_sizes(count)
    mine = rank_share(sizes, rank, nranks) if nranks > 1 else list(range(count))
    jobs = [(i, int(sizes[i])) for i in mine]
    jobs.sort(key=lambda j: -j[1])
    if procs > 1 and len(jobs) > 1:
        with mp.get_context("spawn").Pool(min(procs, len(jobs))) as pool:
            fields = pool.map(_member, jobs, chunksize=1)
    else:
        fields = [_member(j) for j in jobs]
    fields.sort(key=lambda f: int(f.name.split("[")[1].rstrip("]")))
    return fields


def cpu_oracle_rate(fields, budget_s: float, procs: int):
    """The CPU oracle on a bounded sample of the ensemble, one process per
    core holding its fields: one time step of every sampled instance per step
    (about half a second), steps repeated for budget_s seconds after two
    warm-up steps.  Returns (median floe-steps/s, processes, description)."""
    sample = reference_sample(fields, 0.5, procs)
    rates, nproc = time_oracle(sample, procs, 2, 10 ** 6, max_seconds=budget_s)
    desc = (f"{len(sample)} of {len(fields)} ensemble instances ({sum(f.n for f in sample)} floes), one time "
            f"step of each per step, FP64 C oracle, {nproc} processes holding their fields; median over "
            f"{len(rates)} steps in {budget_s:g} s after 2 warm-up steps")
    return statistics.median(rates), nproc, desc


class ClockSampler:
    def __init__(self, index: int):
        self.path = os.path.join(tempfile.gettempdir(), f"godar_clocks_{os.getpid()}_{index}.csv")
        q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def mark(self):
        return time.time()

    def stop(self, t0: float, t1: float):
        if not self.p:
            return None
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                ts = time.mktime(time.strptime(parts[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                rows.append((ts, float(parts[1]), float(parts[2]), parts[5:9]))
            except Exception:
                continue
        if not rows:
            return None
        inside = [r for r in rows if t0 - 1.0 <= r[0] <= t1 + 1.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in inside), "sm_max_mhz": max(r[2] for r in inside),
                "reasons": reasons, "samples": len(inside)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- arms
def _ref_worker(conn, fields):
    """One host process of the reference arm: keeps its share of the sample
    as oracle fields and advances all of them by the number of time steps
    each command names; answers (floe-steps, seconds)."""
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as po
    oracles = [po.Oracle(f.params, f.x, f.y, f.r, f.h, field=f.forcing) for f in fields]
    nf = sum(f.n for f in fields)
    conn.send(nf)
    while True:
        k = conn.recv()
        if k is None:
            break
        t = time.perf_counter()
        for o in oracles:
            o.step(k)
        conn.send((nf * k, time.perf_counter() - t))
    for o in oracles:
        o.close()
    conn.close()


# per-core speed of the oracle on these fields, floe-steps/s (measured: about
# 4e5); a conservative figure sizes the sample
ORACLE_RATE_PER_CORE = 3.0e5
REFERENCE_ARM_SECONDS = 150.0


def reference_sample(fields, per_step: float, procs: int):
    """The instances of the ensemble (a prefix: instance sizes are drawn
    independently of their index) whose one time step takes about per_step
    seconds on procs cores; at least one instance."""
    target = per_step * ORACLE_RATE_PER_CORE * procs
    sample, tot = [], 0
    for f in fields:
        if sample and tot + f.n > target:
            break
        sample.append(f)
        tot += f.n
    return sample


def time_oracle(sample, procs: int, warmup: int, steps: int, max_seconds=None):
    """Advances the sample on min(procs, len(sample)) host processes, each
    holding its share (by floe count) for the whole call: warmup untimed
    steps, then up to `steps` timed ones (fewer once max_seconds of timed
    steps have passed).  A step is one time step of every instance, timed
    from the commands to the last answer.  Returns (floe-steps/s of each
    timed step, processes)."""
    from godar_b200.shard import lpt_partition
    parts = [p for p in lpt_partition([f.n for f in sample], min(procs, len(sample))) if p]
    ctx = mp.get_context("spawn")
    conns, workers = [], []
    try:
        for part in parts:
            a, b = ctx.Pipe()
            w = ctx.Process(target=_ref_worker, args=(b, [sample[i] for i in part]), daemon=True)
            w.start()
            b.close()
            conns.append(a)
            workers.append(w)
        for c in conns:
            c.recv()
        rates = []
        t_timed = 0.0
        for k in range(warmup + steps):
            t = time.perf_counter()
            for c in conns:
                c.send(1)
            work = sum(c.recv()[0] for c in conns)
            wall = time.perf_counter() - t
            if k >= warmup:
                rates.append(work / wall)
                t_timed += wall
                if max_seconds is not None and t_timed >= max_seconds:
                    break
    finally:
        for c in conns:
            try:
                c.send(None)
            except (BrokenPipeError, OSError):
                pass
        for w in workers:
            w.join(timeout=60)
    return rates, len(parts)


def run_reference(args, ws, rank):
    """The reference's CPU implementation of the path: the C oracle (the
    Fortran reference cannot be built here) on all host cores, one process per
    core holding its share of the sampled instances for the whole run.  The
    sample's step fits REFERENCE_ARM_SECONDS over all steps (0.05 to 2 s a
    step)."""
    if rank != 0:
        return
    procs = max(1, os.cpu_count() or 1)
    fields = make_ensemble(args.instances, 0, 1, procs)
    per_step = min(2.0, max(0.05, REFERENCE_ARM_SECONDS / max(1, args.steps + args.warmup)))
    sample = reference_sample(fields, per_step, procs)
    rates, nproc = time_oracle(sample, procs, args.warmup, args.steps)
    value = statistics.median(rates)
    nf = sum(f.n for f in fields)
    ns = sum(f.n for f in sample)
    desc = (f"{len(sample)} of {len(fields)} ensemble instances ({ns} of {nf} floes), one time step of each "
            f"per step, FP64 C oracle, {nproc} processes holding their fields for the whole run; "
            f"median over {args.steps} steps after {args.warmup} warm-up steps")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * nf / value,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(fields, ws, args.instances),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(fields, ws, count):
    nf = int(sum(f.n for f in fields))
    return {"workload": "batched ensemble: 512 fields, n log-uniform [256,16384], "
                        "80% area fraction target, bonded (gap < 0.05 (ri+rj)), wind 8-16 m/s",
            "instances": count, "instances_per_rank": len(fields), "floes_per_rank": nf,
            "global_floes": int(np.sum(ensemble_sizes(count))),
            "dt_s": float(fields[0].params.dt), "precision": "mixed (FP32 forces, FP64 integration)",
            "parallelism": f"ensemble split over {ws} rank(s) by floe count (LPT), no collective on the data path",
            "l2": "inputs larger than L2",
            "area_fraction": round(float(np.mean([f.meta["area_fraction"] for f in fields])), 3)}


def served_stream(args, procs):
    """The served request stream: Poisson arrivals at 20 req/s, floe counts
    log-uniform in [512, 65536], bonded fields with their own seed and wind,
    admitted by a 150 GB HBM budget with continuous batching; the same
    stream (fields generated once, before either run) in both precisions.
    Latency = completion - arrival (wall clock)."""
    from godar_b200.params import PREC_FP64, PREC_MIXED
    from godar_b200.serve import Request, make_stream, serve
    tg = time.perf_counter()
    base = make_stream(args.serve_requests, rate=20.0, seed=5, lo=512, hi=65536, nsteps=args.serve_steps,
                       procs=procs)
    gen_s = time.perf_counter() - tg
    full = args.serve_requests >= 1000 and args.serve_steps >= 2000
    out = {"requests": args.serve_requests, "steps_per_request": args.serve_steps, "rate_per_s": 20.0,
           "floes_per_request": "log-uniform [512, 65536]", "hbm_budget_bytes": 150 * 10**9,
           "floes_total": int(sum(r.n for r in base)), "generate_s": round(gen_s, 1),
           "sample": ("the whole stream" if full else
                      f"{args.serve_requests} requests of the 1000-request stream, {args.serve_steps} steps each")}
    for name, prec in (("mixed", PREC_MIXED), ("fp64", PREC_FP64)):
        reqs = [Request(rid=r.rid, arrival=r.arrival, fld=r.fld, nsteps=r.nsteps) for r in base]
        st = serve(reqs, precision=prec, hbm_budget=150 * 10**9, chunk=50, realtime=True)
        out[name] = {"throughput": st.throughput, "unit": UNIT, "p50_s": st.p50_s, "p99_s": st.p99_s,
                     "mean_queue_s": st.mean_queue_s, "makespan_s": st.makespan_s, "completed": st.completed,
                     "floe_steps": st.floe_steps, "max_resident": st.max_resident, "gpu_ms": st.gpu_ms}
    return out


def full_run(fields, steps: int):
    """Config 4 as configured: the ensemble admitted to a fresh batch and
    advanced `steps` time steps in one call sequence - set-up (upload, bond
    creation, neighbour rebuild), the autotuner's steps, every rebuild and
    a diagnostic last step included - timed by the host clock; then the
    device time of the last 100 steps on their own (the screen's
    displacement bound has grown by then)."""
    from godar_b200.lib import Batch
    from godar_b200.params import PREC_MIXED
    nf = sum(f.n for f in fields)
    late = min(100, steps // 2)
    b = Batch(PREC_MIXED)
    for f in fields:
        b.add_field(f)
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.step(steps - late)
    early_ms = b.sync()
    st0 = b.stats()
    b.step(late)
    late_ms = b.sync()
    wall = time.perf_counter() - t0
    st1 = b.stats()
    b.close()
    return {"steps": steps, "floes": nf, "wall_s": wall, "floe_steps_per_s": nf * steps / wall,
            "setup_and_rebuilds_s": wall - (early_ms + late_ms) / 1e3,
            "rebuilds": st1["rebuilds"], "rebuild_ms_total": st1["rebuild_ms"],
            "device_ms_first": early_ms, "first_steps": steps - late,
            "late_window": {"steps": f"{steps - late + 1}-{steps}", "device_ms": late_ms,
                            "ms_per_step": late_ms / late, "floe_steps_per_s": nf * late / (late_ms / 1e3),
                            "rebuilds_in_window": st1["rebuilds"] - st0["rebuilds"]},
            "timing": "wall: host clock around the whole sequence (set-up included); device_ms: CUDA events "
                      "of the step calls"}


def fp64_batched(fields, steps: int):
    """The FP64 plain method on the whole ensemble in one batch (every floe
    of every field per step, one thread per floe), device time."""
    from godar_b200.lib import Batch
    from godar_b200.params import PREC_FP64
    nf = sum(f.n for f in fields)
    b = Batch(PREC_FP64)
    for f in fields:
        b.add_field(f)
    b.step(TUNE_STEPS + 3)
    b.sync()
    b.prepare(steps)
    b.step(steps)
    ms = b.sync()
    b.close()
    return {"value": nf * steps / (ms / 1e3), "unit": UNIT, "steps": steps, "ms_per_step": ms / steps,
            "floes": nf, "timing": f"device time of {steps} steps after {TUNE_STEPS + 3} tuning/warm-up steps"}


def run_godar(args, ws, rank, local):
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from godar_b200.lib import Batch, Stepper
    from godar_b200.params import PREC_FP64, PREC_MIXED

    procs = max(1, (os.cpu_count() or 1) // ws)
    tg = time.perf_counter()
    fields = make_ensemble(args.instances, rank, ws, procs)
    gen_s = time.perf_counter() - tg
    nf = sum(f.n for f in fields)
    # the whole job's floes: the ensemble, split over the ranks
    gnf = int(np.sum(ensemble_sizes(args.instances)))

    b = Batch(PREC_MIXED)
    for f in fields:
        b.add_field(f)
    tc = time.perf_counter()
    # the online autotuner picks each kernel's block size and tile over the
    # first TUNE_STEPS steps (the simulation advances normally; no candidate
    # changes a result)
    b.step(TUNE_STEPS)
    b.step(args.warmup)
    b.sync()
    # every 16th step of the timed call times its kernels one by one with CUDA
    # events (an event between two kernels of a graph costs several
    # microseconds, so the other steps run without); the timed call's CUDA
    # graphs are captured before the clock starts
    b.set_phase_timing(PHASE_EVERY)
    b.prepare(args.steps)
    warm_s = time.perf_counter() - tc
    st0 = b.stats()

    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.time()
    b.step(args.steps)
    ms = b.sync()
    t1 = time.time()
    st1 = b.stats()
    clk = clocks.stop(t0, t1)
    if dist:
        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = gnf * args.steps / (ms / 1e3)

    # roofline of the dominant kernel: algorithmic bytes per launch over the
    # kernel's mean CUDA-event duration in the timed region.  Per kernel:
    # pair screen 36 B/floe own state + 4 B per candidate pair (CSR read);
    # pair work list 40 B per contact (history read+write); bonds 128 B per
    # bond; floe sums 20 B/floe; floe update 132 B/floe
    launches = st1["launches"] - st0["launches"]
    klaunch = st1["kernel_launches"] - st0["kernel_launches"]
    timed = st1["timed_steps"] - st0["timed_steps"]
    ph_ms = [(a - b) / max(1, timed) for a, b in zip(st1["phase_ms"], st0["phase_ms"])]
    step_ms = (st1["kernel_ms"] - st0["kernel_ms"]) / max(1, timed)
    P, C, B = st1["candidates"], st1["contacts"], st1["bonds"]
    names = ["k_pairs_screen (candidate screening)",
             "k_pairs_mixed (contact forces, ridging events, sheltering)",
             "k_bonds_mixed (bond forces and breaking)",
             "k_floe_sums (pair and bond record sums)",
             "k_floes_mixed (walls, ridging, drag, Coriolis, integration)"]
    algos = [36 * nf + 4 * P, 40 * C, 128 * B, 20 * nf, 132 * nf]
    peak, kind = peaks()
    phases = []
    for q in range(len(names)):
        ach = algos[q] / (ph_ms[q] / 1e3) / 1e9 if ph_ms[q] > 0 else 0.0
        phases.append({"kernel": names[q], "ms_per_launch": ph_ms[q], "algorithmic_bytes": algos[q],
                       "achieved_gbs": ach, "frac": ach / peak})
    dom = int(np.argmax(ph_ms))
    kms = ph_ms[dom]
    algo = algos[dom]
    achieved = algo / (kms / 1e3) / 1e9
    # DRAM traffic of the dominant kernel: the committed ncu capture's bytes
    # per unit (floe, candidate, contact or bond) scaled to this launch
    traffic = None
    tp = os.path.join(ROOT, "profiles", "step_mixed_traffic.json")
    if os.path.exists(tp):
        t = json.load(open(tp)).get(names[dom].split()[0])
        if t:
            units = {"floes": nf, "candidates": P, "contacts": C, "bonds": B}[t["per"]]
            traffic = t["bytes"] / t["units"] * units

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32 forces / f64 integration",
            "data": "synthetic", "config": workload_config(fields, ws, args.instances),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": kind,
                         "kernel": names[dom], "kernel_ms_per_launch": kms,
                         "algorithmic_bytes_per_launch": algo, "kernels": phases,
                         "step_ms": step_ms, "step_algorithmic_bytes": sum(algos),
                         "step_frac": sum(algos) / (step_ms / 1e3) / 1e9 / peak,
                         "timed_steps": timed,
                         "note": f"per-kernel figures of this rank, CUDA events around the kernels of every "
                                 f"{PHASE_EVERY}th step of the timed call ({timed} steps); step_ms is such a "
                                 f"step's device time from its first to its last kernel"},
            "launch_config": {"blocks": st1["blocks"], "variants": st1["variants"],
                              "variant_meaning": "screen items per lane 0=8 1=4 2=16; bonds 1=tiles streamed "
                                                 "through shared memory by bulk copies",
                              "cuda_graphs": st1["graphs"],
                              "graph_launches": st1["graph_launches"] - st0["graph_launches"]},
            "gpu_launches": int(klaunch + 24 * (st1["rebuilds"] - st0["rebuilds"])),
            "rebuilds_in_timed_region": st1["rebuilds"] - st0["rebuilds"],
            # the neighbour search (cell keys, radix sort, Verlet superset,
            # contact list, bond lists) of the set-up: host wall time per
            # rebuild, each to its end on the device
            "neighbour_rebuild": {"ms_per_rebuild": st0["rebuild_ms"] / max(1, st0["rebuilds"]),
                                  "rebuilds": st0["rebuilds"], "pairs": st0["pairs"],
                                  "contact_list": st0["contact_list"]},
            "counts_last_step": {k: st1[k] for k in ("candidates", "contacts", "bonds", "plastic")},
            "clocks": clk, "setup_s": {"generate": round(gen_s, 1), "admit_tune_warmup": round(warm_s, 1)},
            "untimed_steps_before_warmup": TUNE_STEPS}

    # end to end through the C ABI with host buffers, every step: upload the
    # step's uniform forcing of every instance, step, and read the step's
    # result back - a per-field summary (momentum, kinetic energy, largest
    # speed: the monitoring metric of a run, as a loss is of a training step)
    # and, in a second loop, every floe's position; every rank its share,
    # the slowest rank's time
    import torch as _t
    ke = max(1, min(args.steps, 50))
    nin = len(fields)
    uvw = _t.empty(4 * nin, dtype=_t.float64).pin_memory().numpy()
    for k, f in enumerate(fields):
        uvw[4 * k:4 * k + 4] = (f.params.ua, f.params.va, f.params.uw, f.params.vw)
    # two pinned buffers of each kind: the read-backs of consecutive steps
    # are in flight together
    osum = [_t.empty(4 * nin, dtype=_t.float64).pin_memory().numpy() for _ in range(2)]
    ox = [_t.empty(nf, dtype=_t.float64).pin_memory().numpy() for _ in range(2)]
    oy = [_t.empty(nf, dtype=_t.float64).pin_memory().numpy() for _ in range(2)]
    # the loops read no forces or stresses: no diagnostic steps
    b.set_diagnostics(False)
    for _ in range(4):      # single-step graphs of both sides captured
        b.step(1)
    b.sync()

    def e2e_loop(read):
        if dist:
            dist.barrier()
        te = time.perf_counter()
        for k in range(ke):
            # step k is queued behind step k-1 (checked once k is queued)
            # while the read-back of step k-1 is still copying
            b.set_uniform_forcing(uvw)
            b.step_async(1)
            read(k)
        b.wait()
        t = time.perf_counter() - te
        if dist:
            et = torch.tensor([t], device="cuda", dtype=torch.float64)
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
            t = float(et.item())
        return t

    sum_s = e2e_loop(lambda k: b.summary_async(osum[k & 1]))
    pos_s = e2e_loop(lambda k: b.get_all_async(["x", "y"], [ox[k & 1], oy[k & 1]]))
    b.set_diagnostics(True)
    line["e2e"] = {"value": gnf * ke / sum_s, "unit": UNIT, "h2d_bytes_per_step": 32 * args.instances,
                   "d2h_bytes_per_step": 32 * args.instances, "steps": ke,
                   "path": "godar_batch_set_uniform_forcing + godar_batch_step_async + godar_batch_summary_async "
                           "(per field: momentum, kinetic energy, largest speed; step k+1 queued behind step k, "
                           "the read-back of step k overlaps step k+1) + godar_batch_wait, diagnostics off"}
    line["e2e_positions"] = {"value": gnf * ke / pos_s, "unit": UNIT, "h2d_bytes_per_step": 32 * args.instances,
                             "d2h_bytes_per_step": 16 * gnf, "steps": ke,
                             "path": "godar_batch_set_uniform_forcing + godar_batch_step_async + "
                                     "godar_batch_get_all_async(x,y) (every floe's position; step k+1 queued behind "
                                     "step k, read-back of step k overlaps step k+1, two in flight) + godar_batch_wait, "
                                     "diagnostics off"}
    b.close()

    if rank == 0 and ws == 1:
        # plain FP64 single-instance GPU path on a sample of the same ensemble
        idx = np.linspace(0, len(fields) - 1, min(24, len(fields))).astype(int)
        tot_ms, tot_fs = 0.0, 0
        sp = 20
        for i in idx:
            f = fields[i]
            s = Stepper(f.params, f.n, PREC_FP64)
            s.upload(f.x, f.y, f.r, f.h)
            # autotune, warm up, and run the timed schedule once untimed so
            # that its CUDA graphs exist
            s.step(1, 0, TUNE_STEPS + 5)
            s.step(TUNE_STEPS + 6, 0, sp)
            t = time.perf_counter()
            s.step(TUNE_STEPS + 6 + sp, 0, sp)
            tot_ms += (time.perf_counter() - t) * 1e3
            tot_fs += f.n * sp
            s.close()
        plain_rate = tot_fs / (tot_ms / 1e3)
        line["plain_fp64_single_instance"] = {
            "value": plain_rate, "unit": UNIT,
            "sample": f"{len(idx)} instances run one at a time, {sp} steps each, wall time",
            "batched_mixed_over_plain": value / plain_rate}
        # the same plain FP64 method batched over the whole ensemble: the
        # precision-matched GPU figure beside the FP64 CPU arm
        if args.fp64_batched_steps > 0:
            line["fp64_batched"] = fp64_batched(fields, args.fp64_batched_steps)
            line["fp64_batched"]["batched_mixed_over_batched_fp64"] = value / line["fp64_batched"]["value"]

        # accuracy of the mixed path against FP64 on the largest instance
        # over 1000 steps (or warmup + timed steps if more)
        f = fields[int(np.argmax([g.n for g in fields]))]
        nst = max(1000, args.warmup + args.steps)
        s64 = Stepper(f.params, f.n, PREC_FP64)
        s32 = Stepper(f.params, f.n, PREC_MIXED)
        for s in (s64, s32):
            s.upload(f.x, f.y, f.r, f.h)
            s.step(1, 0, nst)
        L = max(f.params.nx, f.params.ny)

        def wrapped(d, Ld):
            return d - Ld * np.round(d / Ld)       # the ensemble's fields are doubly periodic

        ex = wrapped(s32.field("x") - s64.field("x"), f.params.nx)
        ey = wrapped(s32.field("y") - s64.field("y"), f.params.ny)
        perr = float(np.max(np.hypot(ex, ey)))
        disp = float(np.max(np.hypot(wrapped(s64.field("x") - f.x, f.params.nx),
                                     wrapped(s64.field("y") - f.y, f.params.ny))))

        def rel(k):
            ref = s64.field(k)
            scale = float(np.max(np.abs(ref))) or 1.0
            return float(np.max(np.abs(s32.field(k) - ref))) / scale

        line["mixed_vs_fp64"] = {"instance_floes": f.n, "steps": nst, "max_pos_err_m": perr,
                                 "max_displacement_m": disp, "max_pos_err_over_displacement": perr / disp,
                                 "max_pos_err_over_domain": perr / L,
                                 "max_vel_err_over_max_speed": max(rel("u"), rel("v")),
                                 "max_force_err_over_max_force": max(rel("tfx"), rel("tfy")),
                                 "max_torque_err_over_max_torque": rel("m")}
        # the output step (sea_ice_post's 25 text files) of that field
        with tempfile.TemporaryDirectory() as td:
            t = time.perf_counter()
            s64.write_posts(td, "01", nst, 1.0)
            out_ms = (time.perf_counter() - t) * 1e3
            out_bytes = sum(os.path.getsize(os.path.join(td, x)) for x in os.listdir(td))
        line["output_step"] = {"floes": f.n, "ms": out_ms, "bytes": out_bytes,
                               "path": "godar_gpu_write_posts (download, sparse bond/contact lists, "
                                       "list-directed records on host threads, 25 files appended)"}
        s64.close()
        s32.close()

        # config 4 as configured: 1000 steps from admission, set-up included
        if args.full_steps > 0:
            line["full_run"] = full_run(fields, args.full_steps)

        line["cpu_baseline"] = None
        if not args.no_cpu:
            rate, cores, desc = cpu_oracle_rate(fields, args.cpu_seconds, max(1, os.cpu_count() or 1))
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                    "sample": desc}
    if rank == 0 and ws == 1 and args.serve_requests > 0:
        line["served"] = served_stream(args, procs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="godar", choices=["godar", "reference"])
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--serve-steps", type=int, default=2000)
    ap.add_argument("--full-steps", type=int, default=1000)
    ap.add_argument("--fp64-batched-steps", type=int, default=20)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_godar(args, ws, rank, local)


if __name__ == "__main__":
    main()
