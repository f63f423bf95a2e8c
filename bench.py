#!/usr/bin/env python
"""Benchmark: synaptic events/s of the grid-mode simulation step on B200.

Workload (the scatter-bound roofline case): 1,000,000 LIF neurons (80 % E /
20 % I), fixed out-degree 1,000 with targets uniform over all neurons
(1e9 synapses: uint32 target + fp32 weight + uint8 delay, 9 GB), delays
U{1..16} steps, dt = 0.1 ms, per-neuron 20 Hz Poisson drive (~10 Hz mean
firing), no STDP, seeded synthetic network.  One bench step = 1,000 grid
steps = 100 ms simulated; the default 10 timed steps simulate 1 s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one network per GPU, no collective on
the data path: weak scaling), launched with torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "synaptic events/s"
UNIT = "events/s"
BYTES_PER_EVENT = 9  # uint32 target + fp32 weight + uint8 delay


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--neurons", type=int, default=1_000_000)
    ap.add_argument("--degree", type=int, default=1000)
    ap.add_argument("--chunk", type=int, default=1000, help="grid steps per bench step")
    ap.add_argument("--profile-steps", type=int, default=2000)
    ap.add_argument("--cpu-steps", type=int, default=300, help="timed grid steps of the CPU sample")
    ap.add_argument("--cpu-warmup", type=int, default=300)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served forms")
    ap.add_argument("--batch-members", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=20000, help="grid steps per member (2 s)")
    ap.add_argument("--served-jobs", type=int, default=2000)
    ap.add_argument("--plain-sample", type=int, default=16, help="jobs run one at a time for the plain arm")
    ap.add_argument("--det-steps", type=int, default=2000, help="timed grid steps of the deterministic plain run")
    ap.add_argument("--step-kernel", default="split", choices=["split", "two_barrier"],
                    help="persistent step kernel of the plain runs")
    ap.add_argument("--no-det", action="store_true", help="skip the deterministic-mode measurements")
    ap.add_argument("--no-bins", action="store_true", help="skip the binned-aggregation comparison")
    ap.add_argument("--no-probe", action="store_true", help="skip the device probe (ceilings)")
    ap.add_argument("--tuning", default="", help='launch geometry of the plain runs as JSON, e.g. {"blocks_per_sm": 1}')
    ap.add_argument("--bins-steps", type=int, default=2000, help="timed grid steps per binning trial")
    ap.add_argument("--no-saturated", action="store_true", help="skip the served form's saturation run")
    return ap.parse_args()


def workload(args, seed=1):
    from naer_b200 import spec as S
    s = S.scatter_outdegree(n=args.neurons, k=args.degree, seed=seed)
    # room for every spike of warm-up + timed + e2e + profile passes
    s.raster_capacity = 1 << 26
    return s


def workload_config(args, synapses):
    return {
        "workload": f"scatter_outdegree: {args.neurons} LIF (80/20), fixed out-degree {args.degree}, "
                    f"delays 1-16 steps, 20 Hz Poisson drive, no STDP",
        "neurons": args.neurons,
        "synapses": synapses,
        "dt_ms": 0.1,
        "step": f"{args.chunk} grid steps = {args.chunk * 0.1:.0f} ms simulated",
        "aggregation": "atomic",
        "l2": "inputs larger than L2 (9 B x synapses streamed; 126 MB L2)",
        "parallelism": "replicas",
        "tuning": args.tuning or "default",
    }


class Clocks:
    """nvidia-smi sampling in the background during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def reduce_max_sum(world, tmax, esum):
    """Max of the ranks' times and sum of their events (every rank gets both):
    the job's time is its slowest replica's, its work the sum of all."""
    if world == 1:
        return tmax, esum
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([tmax], dtype=torch.float64, device=dev)
    e = torch.tensor([esum], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(args, spec, steps, warm):
    """The oracle (multithreaded restatement of the reference's step) on the
    host cores: `warm` untimed grid steps, then `steps` timed ones."""
    from oracle import oracle as O
    threads = O.max_threads()
    o = O.OracleNet(spec, threads=threads, deterministic=False)
    o.run(warm)
    e0 = o.events
    t0 = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t0
    ev = o.events - e0
    o.close()
    return {"value": ev / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} grid steps ({steps * 0.1:.0f} ms simulated) of the same network after "
                      f"{warm} warm-up steps; {ev} events in {dt:.2f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    spec = workload(args)
    from oracle import oracle as O
    threads = O.max_threads()
    o = O.OracleNet(spec, threads=threads, deterministic=False)
    o.run(args.cpu_warmup)
    # one bench step is the same work as on the GPU arm: args.chunk grid
    # steps (100 ms simulated), so ms_per_step compares like with like
    per_step = args.chunk
    for _ in range(args.warmup):
        o.run(max(1, per_step // 10))
    e0 = o.events
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.run(per_step)
    dt = time.perf_counter() - t0
    ev = o.events - e0
    value = ev / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(args, int(o.S)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step {per_step} grid steps ({per_step * 0.1:.0f} ms simulated) of the same "
                                   f"network on the host cores, as one step of the GPU arm (the reference's OpenCL "
                                   f"kernels cannot run here: no OpenCL runtime)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def plain_runs(specs_steps, local, rasters=False):
    """Each job alone with the plain form, one after another: build, run,
    read the raster back.  Returns per-job seconds (run only, with build)
    and, with rasters=True, each job's (steps, ids)."""
    from naer_b200 import spec as S
    run_s, all_s, out = [], [], []
    for spec, steps in specs_steps:
        t0 = time.perf_counter()
        net = S.build(spec, device=local)
        t1 = time.perf_counter()
        net.run(steps)
        net.finish()
        r = net.read_spikes()
        t2 = time.perf_counter()
        net.close()
        run_s.append(t2 - t1)
        all_s.append(t2 - t0)
        out.append(r)
    return (run_s, all_s, out) if rasters else (run_s, all_s)


def same_raster(a, b):
    import numpy as np
    return len(a[1]) == len(b[1]) and bool(np.array_equal(a[0], b[0])) and bool(np.array_equal(a[1], b[1]))


def bench_plastic(args, local, stream_of):
    """The plastic workload: 100k LIF (80 % STDP-excitatory), fixed
    in-degree 1,000 (1e8 synapses), delays 1-20 steps, 10 Hz drive, pair STDP
    on E->E; 1 s simulated after 0.1 s of warm-up, CUDA events."""
    import torch
    from naer_b200 import spec as S
    spec = S.plastic_indegree(n=100_000, k=1000)
    spec.raster_capacity = 1 << 24
    net = S.build(spec, device=local)
    stream = stream_of(net)
    net.run(1000)
    net.finish()
    st0 = net.stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    net.run(10_000)
    e1.record(stream)
    e1.synchronize()
    st1 = net.stats()
    ms = e0.elapsed_time(e1)
    net.close()
    ev = st1["events"] - st0["events"]
    return {"workload": "plastic_indegree: 100000 LIF (80/20), fixed in-degree 1000, delays 1-20, 10 Hz drive, "
                        "pair STDP on E->E; 1 s simulated",
            "events_per_s": ev / (ms / 1e3), "ms_per_simulated_s": ms, "synapses": int(st1["synapses"]),
            "spikes_per_s_sim": (st1["spikes"] - st0["spikes"]) / 1.0 / 100_000,
            "stdp_history_overflows": int(st1["stdp_hist_overflow"])}


def bench_batched(args, local, deterministic=False, exact=False):
    """Batched form: independent networks of uneven sizes (log-uniform 2k-50k
    neurons, in-degree 100-1000, own seeds, Poisson 5-30 Hz, STDP on half)
    packed into one engine, autotuned, CUDA-graph step loop, 2 s simulated
    each; against one-at-a-time plain runs of a seeded sample of the same
    members (deterministic mode: the sample's rasters must equal their
    members' rasters in the batch, bit for bit)."""
    import numpy as np
    from naer_b200 import spec as S
    from naer_b200.forms import Batch
    members = [m.with_(deterministic=deterministic, exact=exact)
               for m in S.batch_members(count=args.batch_members, seed=1)]
    for m in members:
        m.raster_capacity = 1 << 22
    steps = args.batch_steps
    t0 = time.perf_counter()
    b = Batch(members, device=local, deterministic=deterministic, exact=exact, raster_capacity=1 << 27).compile()
    t1 = time.perf_counter()
    st0 = b.stats()
    t2 = time.perf_counter()
    tune = b.autotune(64)  # its trial steps are part of the members' simulated time
    done = b.stats()["step"]
    ph0 = b.phases()
    b.run(steps - done)
    b.finish()
    t3 = time.perf_counter()
    st1 = b.stats()
    ph1 = b.phases()
    ph = {k: ph1[k] - ph0[k] for k in ph1 if k != "reserved"}
    ph_tot = sum(ph.values()) or 1.0
    rng = np.random.default_rng(7)
    pick = rng.choice(len(members), min(args.plain_sample, len(members)), replace=False)
    identical = None
    if deterministic or exact:
        sp = b.read_spikes()
        run_s, all_s, alone = plain_runs([(members[int(i)], steps) for i in pick], local, rasters=True)
        identical = all(same_raster(b.member_spikes(int(i), sp), a) for i, a in zip(pick, alone))
    else:
        run_s, all_s = plain_runs([(members[int(i)], steps) for i in pick], local)
    b.close()
    sim_s = t3 - t2
    plain_rate = 1.0 / float(np.mean(run_s))
    sem = float(np.std(run_s, ddof=1) / np.sqrt(len(run_s))) if len(run_s) > 1 else 0.0
    return {
        "workload": f"{len(members)} networks, {st0['neurons']} neurons, {st0['synapses']} synapses in total; "
                    f"{steps} grid steps (2 s) each",
        "aggregation": "exact" if exact else "deterministic" if deterministic else "atomic",
        "sims_per_s": len(members) / sim_s,
        "sims_per_s_with_build": len(members) / (sim_s + t1 - t0),
        "events_per_s": (st1["events"] - st0["events"]) / sim_s,
        "us_per_step": sim_s / steps * 1e6,
        "phase_split": {k: round(v / ph_tot, 3) for k, v in ph.items()},
        "build_s": t1 - t0,
        "autotune": {k: tune[k] for k in ("blocks_per_sm", "launch_steps", "scatter_split", "graph_launches",
                                          "step_kernel", "best_us_per_step", "default_us_per_step", "trials")},
        "plain_sims_per_s": plain_rate,
        "plain_sims_per_s_with_build": 1.0 / float(np.mean(all_s)),
        "plain_sample": f"{len(pick)} members run alone one after another (mean {np.mean(run_s):.3f} s each, "
                        f"standard error {sem:.3f} s)",
        "speedup_vs_plain": (len(members) / sim_s) / plain_rate,
        "rasters_identical_to_alone": identical,
        "raster_records": int(st1["spikes"]),
    }


def bench_served(args, local, deterministic=False, saturate=False, exact=False):
    """Served form: a seeded Poisson stream of jobs (50/s; 1k-200k neurons
    log-uniform, in-degree 100-1000, 100 ms - 2 s, 30 % STDP) submitted on
    schedule to the continuous-batching server (150 GB budget); p50/p99
    latency from submission to raster delivered; against the same jobs' plain
    one-at-a-time runs (a seeded sample).  saturate=True submits every job
    at once: sims/s is then the server's capacity, not the arrival rate.
    Deterministic mode: the sample's rasters must equal their jobs' rasters
    in the mix, bit for bit."""
    import numpy as np
    from naer_b200 import spec as S
    from naer_b200.forms import Server
    from naer_b200 import _capi as capi_
    jobs = S.served_jobs(count=args.served_jobs, seed=1)
    jobs = [(ta, spec.with_(deterministic=deterministic, exact=exact), steps) for ta, spec, steps in jobs]
    srv = Server(device=local, budget_bytes=150 * 10**9, chunk_steps=256, deterministic=deterministic, exact=exact)
    ids = []
    t0 = time.perf_counter()
    for ta, spec, steps in jobs:
        now = time.perf_counter() - t0
        if not saturate and ta > now:
            time.sleep(ta - now)
        ids.append(srv.submit(spec, steps))
    ok = srv.drain(1800.0)
    wall = time.perf_counter() - t0
    st = srv.stats()
    errors = sorted({srv.error(j) for j in ids if srv.info(j)["state"] == capi_.JOB_FAILED})[:3]
    rng = np.random.default_rng(11)
    pick = rng.choice(len(jobs), min(args.plain_sample, len(jobs)), replace=False)
    identical = None
    if deterministic or exact:
        run_s, all_s, alone = plain_runs([(jobs[int(i)][1], jobs[int(i)][2]) for i in pick], local, rasters=True)
        identical = all(same_raster(srv.spikes(ids[int(i)]), a) for i, a in zip(pick, alone))
    else:
        run_s, all_s = plain_runs([(jobs[int(i)][1], jobs[int(i)][2]) for i in pick], local)
    srv.close()
    return {
        "workload": f"{len(jobs)} jobs, " + ("all submitted at once" if saturate else
                                            f"Poisson arrivals at 50/s over {jobs[-1][0]:.1f} s"),
        "aggregation": "exact" if exact else "deterministic" if deterministic else "atomic",
        "sims_per_s": st["sims_per_s"],
        "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
        "drained": ok, "wall_s": wall, "done": st["done"], "failed": st["failed"], "failure_messages": errors,
        "peak_device_gb": st["peak_bytes"] / 1e9, "chunks": st["chunks"], "raster_dropped": st["raster_dropped"],
        "thread_s": {k: round(st[k], 2) for k in ("build_s", "install_s", "step_s", "drain_s")},
        "plain_sims_per_s": 1.0 / float(np.mean(all_s)),
        "plain_latency_ms_mean": 1e3 * float(np.mean(all_s)),
        "plain_sample": f"{len(pick)} jobs run alone one after another (build + run + raster read)",
        "speedup_vs_plain": st["sims_per_s"] * float(np.mean(all_s)),
        "rasters_identical_to_alone": identical,
    }


def bench_bins(args, local, stream_of):
    """Shared-memory binning of the ring reductions (tuning `bins`) against
    direct L2 reductions, device time per grid step: on the roofline
    workload (uniform random targets: nothing to fold) and on a convergent
    one (every neuron also drives a 64-neuron readout: each step's readout
    events hit 64 ring cells)."""
    import torch
    from naer_b200 import spec as S
    out = {}
    for name, spec in [("roofline workload", workload(args)),
                       ("hub readout 200k + 64", S.hub_readout(n=200_000, k=100, readout=64))]:
        spec.raster_capacity = 1 << 24
        net = S.build(spec, device=local)
        stream = stream_of(net)
        row = {"synapses": int(net.getSynapses())}
        for bins in (0, 2048):
            net.set_tuning(bins=bins)
            net.run(256)
            net.finish()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ev0 = net.stats()["events"]
            e0.record(stream)
            net.run(args.bins_steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            ev = net.stats()["events"] - ev0
            row[f"bins_{bins}"] = {"us_per_step": 1e3 * ms / args.bins_steps, "events_per_s": ev / (ms / 1e3)}
        row["speedup_binned"] = row["bins_0"]["us_per_step"] / row["bins_2048"]["us_per_step"]
        net.close()
        out[name] = row
    return out


def bench_exact(args, local, stream_of):
    """The roofline workload in exact-sum aggregation (fixed-point weights,
    integer ring sums: bit-reproducible rasters from the atomic kernel):
    events/s over the timed steps, CUDA events on its stream, and whether a
    second run reproduces the first's raster."""
    import numpy as np
    import torch
    from naer_b200 import spec as S
    spec = workload(args).with_(exact=True)
    spec.raster_capacity = 1 << 24
    rasters = []
    out = {}
    for rep in range(2):
        net = S.build(spec, device=local)
        stream = stream_of(net)
        net.run(256)
        net.finish()
        st0 = net.stats()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        net.run(args.det_steps)
        e1.record(stream)
        e1.synchronize()
        st1 = net.stats()
        ms = e0.elapsed_time(e1)
        rasters.append(net.read_spikes())
        net.close()
        if rep == 0:
            ev = st1["events"] - st0["events"]
            out = {"workload": workload_config(args, int(st1["synapses"]))["workload"], "aggregation": "exact",
                   "steps": args.det_steps, "ms": ms, "events_per_s": ev / (ms / 1e3),
                   "ms_per_simulated_s": ms * 1e4 / args.det_steps}
    out["second_run_identical"] = bool(np.array_equal(rasters[0][0], rasters[1][0])
                                       and np.array_equal(rasters[0][1], rasters[1][1]))
    return out


def bench_deterministic(args, local, stream_of):
    """The roofline workload in deterministic aggregation (bit-reproducible
    rasters): events/s over the timed steps, CUDA events on its stream."""
    import torch
    from naer_b200 import spec as S
    spec = workload(args).with_(deterministic=True)
    spec.raster_capacity = 1 << 24
    net = S.build(spec, device=local)
    stream = stream_of(net)
    net.run(256)
    net.finish()
    st0 = net.stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    net.run(args.det_steps)
    e1.record(stream)
    e1.synchronize()
    st1 = net.stats()
    ms = e0.elapsed_time(e1)
    # block 0's split of k_det_step (after the timed region): LIF + first
    # barrier, linking pass + second barrier, folding pass + third barrier
    net.set_profiling(True)
    net.run(min(args.det_steps, 512))
    net.finish()
    prof = net.profile()
    net.close()
    ph = prof["phases_ms"]
    split = {"lif_barrier": ph["lif"], "link_barrier": ph["scatter"], "fold_barrier": ph["scatter_wait"]}
    tot = sum(split.values()) or 1.0
    ev = st1["events"] - st0["events"]
    return {"workload": workload_config(args, int(st1["synapses"]))["workload"],
            "aggregation": "deterministic", "steps": args.det_steps, "ms": ms,
            "events_per_s": ev / (ms / 1e3), "ms_per_simulated_s": ms * 1e4 / args.det_steps,
            "kernel": "k_det_step", "step_kernel_ms": prof["step_kernel_ms"], "drive_kernel_ms": prof["drive_kernel_ms"],
            "profiled_steps": prof["steps"], "phase_split": {k: round(v / tot, 3) for k, v in split.items()}}


def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    from naer_b200 import spec as S

    spec = workload(args, seed=1 + rank)
    net = S.build(spec, device=local)
    from naer_b200 import _capi as capi_
    kern = capi_.KERNEL_SPLIT if args.step_kernel == "split" else capi_.KERNEL_TWO_BARRIER
    extra_tuning = json.loads(args.tuning) if args.tuning else {}
    if kern != capi_.KERNEL_SPLIT or extra_tuning:
        net.set_tuning(step_kernel=kern, **extra_tuning)
    stream = torch.cuda.ExternalStream(net.stream(), device=torch.device("cuda", local))
    chunk = args.chunk

    # warm-up
    for _ in range(args.warmup):
        net.run(chunk)
    net.finish()

    # timed region: device-resident inputs, CUDA events on the engine stream
    clocks = Clocks(local) if rank == 0 else None
    st0 = net.stats()
    barrier(world)
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        net.run(chunk)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop() if clocks else None
    ms = ev0.elapsed_time(ev1)
    st1 = net.stats()
    events = st1["events"] - st0["events"]
    spikes = st1["spikes"] - st0["spikes"]
    ms_max, events_all = reduce_max_sum(world, ms, float(events))
    value = events_all / (ms_max / 1e3)

    # roofline: CUDA events around every launch on the engine stream; the
    # dominant kernel is the persistent step kernel k_run (LIF + scatter of
    # up to 64 grid steps per launch), timed against 9 B per delivered event
    net.set_profiling(True)
    p0 = net.stats()["events"]
    net.run(args.profile_steps)
    net.finish()
    prof = net.profile()
    net.set_profiling(False)
    pev = net.stats()["events"] - p0
    kern_s = prof["step_kernel_ms"] / 1e3
    launches = max(1, prof["step_kernel_launches"])
    peak = None
    peak_src = "fallback"
    try:
        peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
        peak_src = "measured"
    except Exception:
        peak = 6650.0
    achieved = BYTES_PER_EVENT * pev / kern_s / 1e9 if kern_s > 0 else 0.0
    ph = prof["phases_ms"]
    ph_tot = sum(ph.values()) or 1.0
    traffic = None
    kname = "k_step" if args.step_kernel == "split" else "k_run"
    tfile = ROOT / "profiles" / f"{kname}_traffic.json"
    if tfile.exists():
        try:
            t = json.loads(tfile.read_text())
            traffic = t["bytes_per_event"] * pev / launches
        except Exception:
            traffic = None

    # the device's own ceilings for this path (naer_probe_device): random
    # fp32 reductions into a ring-sized buffer (one per event), random
    # stores, streaming read, one grid barrier
    probe = None
    try:
        if args.no_probe:
            raise RuntimeError("skipped (--no-probe)")
        from naer_b200 import _capi as capi
        st_ = net.stats()
        probe = capi.probe_device(local, ring_cells=st_["ring_slots"] * args.neurons,
                                  small_cells=3 * args.neurons)
    except Exception as e:  # reported, never fatal to the bench line
        probe = {"error": str(e)}
    # The scatter window of the step kernel (block 0's %globaltimer split):
    # k_step delivers while it waits at both grid barriers and between them,
    # so its window is the step minus the LIF phase; k_run scatters only
    # between its two barriers.  The figure the ring-accumulation and HBM
    # ceilings bound.
    if args.step_kernel == "split":
        sc_ms = ph.get("lif_wait", 0.0) + ph.get("scatter", 0.0) + ph.get("scatter_wait", 0.0)
        sc_what = "step kernel minus its LIF phase (deliveries overlap both barriers)"
    else:
        sc_ms = ph.get("scatter", 0.0)
        sc_what = "between the two grid barriers"
    scatter_phase = None
    if sc_ms > 0:
        sc_rate = pev / (sc_ms / 1e3)
        scatter_phase = {"ms": sc_ms, "window": sc_what, "events_per_s": sc_rate,
                         "achieved_gbs": BYTES_PER_EVENT * sc_rate / 1e9,
                         "frac_hbm": BYTES_PER_EVENT * sc_rate / 1e9 / peak if peak else None,
                         "frac_of_red_ceiling": (sc_rate / probe["red_ring_per_s"]
                                                 if probe and probe.get("red_ring_per_s") else None)}

    # end to end through the C ABI: step calls + raster readback into pinned host memory
    e2e = None
    if not args.no_e2e:
        cap = max(1, int(spikes / max(1, args.steps) * 4) + 100_000)
        host = torch.empty((cap, 2), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        net.clear_spikes()
        barrier(world)
        e0 = net.stats()["events"]
        t0 = time.perf_counter()
        read = 0
        d2h = 0
        for _ in range(args.steps):
            net.run(chunk)
            n = net.read_raster(host, first=read)
            read += n
            d2h += n * 8
        t1 = time.perf_counter()
        e_ev = net.stats()["events"] - e0
        e_s, e_all = reduce_max_sum(world, t1 - t0, float(e_ev))
        e2e = {"value": e_all / e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
               "d2h_bytes_per_step": int(d2h / args.steps),
               "note": "naer_net_step + naer_net_read_raster per step; the network and its Poisson drive "
                       "are device-resident, as in the reference, so no input crosses host->device"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        net.close()
        cpu = cpu_sample(args, spec, args.cpu_steps, args.cpu_warmup)
    else:
        net.close()

    forms = {}
    if rank == 0 and world == 1 and not args.no_forms:
        forms["plastic"] = bench_plastic(
            args, local, lambda n: torch.cuda.ExternalStream(n.stream(), device=torch.device("cuda", local)))
        forms["batched"] = bench_batched(args, local)
        forms["served"] = bench_served(args, local)
        if not args.no_saturated:
            forms["served_saturated"] = bench_served(args, local, saturate=True)
        if not args.no_det:
            forms["batched_deterministic"] = bench_batched(args, local, deterministic=True)
            forms["served_deterministic"] = bench_served(args, local, deterministic=True, saturate=True)
            forms["batched_exact"] = bench_batched(args, local, exact=True)
            forms["served_exact"] = bench_served(args, local, exact=True, saturate=True)
    if rank == 0 and world == 1 and not args.no_bins:
        forms["binned_aggregation"] = bench_bins(
            args, local, lambda n: torch.cuda.ExternalStream(n.stream(), device=torch.device("cuda", local)))
    if rank == 0 and world == 1 and not args.no_det:
        forms["deterministic"] = bench_deterministic(
            args, local, lambda n: torch.cuda.ExternalStream(n.stream(), device=torch.device("cuda", local)))
        forms["exact"] = bench_exact(
            args, local, lambda n: torch.cuda.ExternalStream(n.stream(), device=torch.device("cuda", local)))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, int(st1["synapses"])),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "kernel": kname + " (persistent step kernel: LIF + scatter)",
                         "peak_source": peak_src,
                         "note": f"{BYTES_PER_EVENT} B x {pev} events over {launches} {kname} launches "
                                 f"({args.profile_steps} grid steps), {prof['step_kernel_ms']:.2f} ms of the step kernel "
                                 f"(CUDA events); Poisson-draw kernel {prof['drive_kernel_ms']:.2f} ms; "
                                 f"phase split of {kname} (block 0): "
                                 + ", ".join(f"{k} {v / ph_tot:.0%}" for k, v in ph.items())},
            "scatter_phase": scatter_phase,
            "device_probe": probe,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(st1["kernel_launches"] - st0["kernel_launches"]),
            "clocks": clk,
            "spikes_per_s_sim": spikes / (args.steps * chunk * 1e-4) / args.neurons,
        }
        line.update(forms)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
