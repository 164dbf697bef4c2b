#!/usr/bin/env python3
"""Benchmark of the B200 MPM time step (particle-steps/s).

Workload: the 2048x2048 mudflow (hx = 0.5 m, seeded bumpy slope, ~4.02M
particles, Bingham + Voellmy, adaptive CFL 0.4), plain FP64.  A step is one
pass of the reference loop body over all particles.  The particle state
(11 x 8 B x Np = 354 MB) is larger than the 126 MB L2, so no flush is done
between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload ensemble [--scenarios 512] [--steps 1000]
    python bench.py --workload serving [--requests 300] [--rate 100] [--budget-gb 150]

One JSON line on rank 0.  Multi-GPU runs are independent replicas (one
scenario, or one ensemble, per GPU, weak scaling): the step has no exchange.

The ensemble workload runs 512 independent scenarios (side log-uniform in
[64, 512] cells, h = 1 m, bumpy slope, release ellipse of 2-10 % of the area
at 4 particles per cell, rheology drawn per scenario, dt = 0.02 s, 1000
passes) as one batch and reports scenarios/s, beside the same scenarios run
one at a time through the single-scenario path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
WORKLOAD = "mudflow 2048x2048 cells, hx=0.5 m, ~4.02M particles, Bingham+Voellmy, CFL 0.4"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_profile():
    """dram bytes per launch from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"dampm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = max(mx, float(parts[2]))
                except ValueError:
                    continue
                for k, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(k)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def _allreduce(x: float, world: int, op: str = "max") -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _touched_nodes(d, key_cells: np.ndarray) -> int:
    """Nodes written by P2G's active strips: corners of occupied cells."""
    nrows = int(d.scalars["Ney"])
    cells = np.unique(key_cells)
    r = cells % nrows
    c = cells // nrows
    nodes = set()
    NR = nrows + 1
    for dr in (0, 1):
        for dc in (0, 1):
            nodes.update(((r + dr) + (c + dc) * NR).tolist())
    return len(nodes)


def cpu_baseline_port(d, seconds: float = 15.0):
    """The CPU restatement of optim_par (OpenMP, all host cores) on a bounded
    sample of the same workload: as many steps as fit in ~`seconds`."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    o = Oracle(d, threads=threads)
    o.run(1)  # warm-up (first-touch of the nodal arrays)
    n = 0
    t0 = time.perf_counter()
    while n < 1 or (time.perf_counter() - t0 < seconds and n < 50):
        o.run(1)
        n += 1
    el = time.perf_counter() - t0
    np_ = o.np
    o.close()
    return {"value": np_ * n / el, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{n} steps of the full workload ({np_} particles) after 1 warm-up step, "
                      f"{el:.1f} s"}


REF_MAX_STEPS = 30
LATE_IT = 1000  # the `late` window of the mudflow line starts here
LATE_STEPS = 20


def run_reference(args, world, rank):
    """--impl reference: the reference's own CPU solver on the host cores.

    oracle/_ref/optim_par is the reference's unmodified main/optim_par.cpp
    (built against stand-ins for its absent submodules); it reads DATA.json
    for the same 4.02M-particle mudflow and prints its own PERF line, timed
    with std::chrono after its 5 warm-up steps.  Its parallel STL runs serial
    without TBB, so it uses one core.  The reference's adaptive first step
    reads an uninitialised dt (main/optim_par.cpp:284,303), so the sample runs
    at a fixed dt equal to the workload's first CFL step; the per-step work is
    the same apart from the host CFL max/min scan it skips.  Without the
    build, the oracle restatement runs instead (kind "port").
    """
    if rank != 0:
        return 0
    import re
    import shutil
    import tempfile
    from amsc_b200 import scenarios
    from amsc_b200.data import to_json
    from oracle import refrun
    d = scenarios.mudflow(N=2048)
    np_ = d.np
    # a bounded sample: the reference takes seconds per step of this workload
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    if refrun.available():
        d.scalars.update({"DT_FIXED": 0.0145, "NSTEPS": 5 + steps})
        wd = tempfile.mkdtemp(prefix="dampm_refarm_")
        try:
            to_json(d, os.path.join(wd, "DATA.json"))
            out = subprocess.run([refrun.OPTIM_PAR], cwd=wd, capture_output=True, text=True,
                                 check=True)
        finally:
            shutil.rmtree(wd, ignore_errors=True)
        m = re.search(r"PERF np=(\d+) counted_steps=(\d+) tot_s=([0-9.eE+-]+)", out.stdout)
        n, counted, tot = int(m.group(1)), int(m.group(2)), float(m.group(3))
        v = n * counted / tot
        kind, cores = "reference", 1
        sample = (f"reference main/optim_par.cpp PERF line: {counted} steps of the full "
                  f"workload ({n} particles) after its 5 warm-up steps, {tot:.1f} s")
        ms_per_step = 1e3 * tot / counted
    else:
        from oracle.oracle import Oracle
        cores = os.cpu_count() or 1
        o = Oracle(d, threads=cores)
        for _ in range(max(min(args.warmup, 3), 1)):
            o.run(1)
        t0 = time.perf_counter()
        for _ in range(steps):
            o.run(1)
        tot = time.perf_counter() - t0
        v = o.np * steps / tot
        kind = "port"
        sample = f"oracle restatement, {steps} steps of the full workload after warm-up"
        ms_per_step = 1e3 * tot / steps
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": mudflow_config(np_, None, 1, args.merge_split,
                                     dt_mode=("fixed dt 0.0145 s, the workload's first CFL "
                                              "step: the reference's adaptive first step "
                                              "reads an uninitialised dt "
                                              "(main/optim_par.cpp:284,303)")
                                     if kind == "reference" else "adaptive CFL 0.4",
                                     launch="host program, one core" if kind == "reference"
                                     else "host program, OpenMP"),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def mudflow_config(np_, np_end, world, merge_split, dt_mode="adaptive CFL 0.4",
                   launch="CUDA graphs of 16 passes"):
    """The config object of the mudflow lines (this library's and the
    reference arm's carry the same keys)."""
    return {"workload": WORKLOAD + (", merge/split every 10 steps" if merge_split else ""),
            "particles": np_, "particles_end": np_end, "grid": "2048x2048",
            "precision": "fp64", "parallelism": f"replicas{world}",
            "l2": "state 354 MB > 126 MB L2, no flush", "launch": launch,
            "dt": dt_mode, "seed": 12345}


def cpu_baseline_scenarios(ds, passes, seconds: float = 15.0):
    """The CPU restatement (OpenMP, all host cores) on a bounded sample of the
    same scenarios, one at a time: each sampled scenario runs some of its
    passes and its time is scaled to `passes` (passes per scenario, a list
    or one count).  Returns scenarios/s."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    per = passes if isinstance(passes, (list, tuple)) else [passes] * len(ds)
    t_used, t_est, m = 0.0, 0.0, 0
    for d, n in zip(ds, per):
        if m and t_used > seconds:
            break
        o = Oracle(d, threads=threads)
        k = 0
        t0 = time.perf_counter()
        while k < n and (k < 2 or time.perf_counter() - t0 < seconds / 4):
            o.run(1)
            k += 1
        el = time.perf_counter() - t0
        o.close()
        t_used += el
        t_est += el / k * n
        m += 1
    return {"value": m / t_est, "unit": "scenarios/s", "cores": threads, "kind": "port",
            "sample": f"{m} scenarios one at a time, each timed over up to its first passes "
                      f"and scaled to its full run; {t_used:.1f} s of CPU time"}


def run_ensemble(args, world, rank, local):
    """--workload ensemble: scenarios/s of a batch of independent scenarios."""
    import torch
    torch.cuda.set_device(local)
    from amsc_b200 import scenarios
    from amsc_b200.batch import Batch
    from amsc_b200.dampm import Solver

    K = args.steps
    W = args.warmup
    n = args.scenarios
    seeds = [100000 * rank + k for k in range(n)]
    ds = [scenarios.ensemble_member(sd, nsteps=K + W) for sd in seeds]
    P = sum(d.np for d in ds)
    N = sum(d.nnodes for d in ds)
    stream = torch.cuda.Stream()  # a real stream: handle 0 would make the library create its own
    h2d = sum(8 * (10 * d.np + d.nnodes) for d in ds)
    d2h = sum(8 * d.np for d in ds)
    # end to end: host arrays in, all passes, final depths out
    _barrier(world)
    t0 = time.perf_counter()
    b = Batch(P + 1024, N + 1024, n + 1, stream=stream.cuda_stream, precision=args.precision)
    hs = [b.add(d) for d in ds]
    b.step(W)
    b.sync()
    # timed region: K passes of every scenario, CUDA events on the batch stream
    # (with --autotune, the tuner's passes are the first of the K)
    sampler = ClockSampler(local)
    sampler.start()
    ts0 = time.perf_counter()
    time.sleep(0.3)
    slept = time.perf_counter() - ts0  # the sampler's start, not part of the job
    l0 = b.usage()["launches"]
    _barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile_timed:
        torch.cuda.profiler.start()
    e0.record(stream)
    tuned = None
    if args.autotune:
        tuned = b.autotune(passes=16)
        b.step(K - tuned["passes"])
    else:
        b.step(K)
    e1.record(stream)
    torch.cuda.synchronize()
    if args.profile_timed:
        torch.cuda.profiler.stop()
    clocks = sampler.stop()
    el_ms = _allreduce(e0.elapsed_time(e1), world)
    launches = b.usage()["launches"] - l0
    # a scenario whose state goes non-finite is stopped by its status word
    # (fixed dt = 0.02 s is above the CFL limit of some members); it counts as
    # failed, not as a finished scenario
    st = b.states()
    failed = [k for k, h in enumerate(hs) if st[h]["failed"]]
    done = sum(1 for h in hs if not st[h]["running"] and not st[h]["failed"])
    outs = [b.download(h, "hp") for h in hs if not st[h]["failed"]]
    e2e_s = _allreduce(time.perf_counter() - t0 - slept, world)
    b.close()
    total = _allreduce(float(done), world, "sum")
    value = total / (el_ms * 1e-3)
    # the plain path: the same scenarios one at a time through dampm_ctx
    m = min(args.plain_sample, n)
    plain_ms = 0.0
    for d in ds[:m]:
        with Solver(d, stream=stream.cuda_stream) as s:
            s.step(W)
            s.sync()
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            s.step(K)
            a1.record(stream)
            torch.cuda.synchronize()
            plain_ms += a0.elapsed_time(a1)
    plain_value = m / (plain_ms * 1e-3) if m else None
    peak, peak_kind = _peaks()
    # algorithmic bytes of one pass: sort (~28 B), P2G (108 B) and G2P (184 B)
    # per particle
    achieved = 320.0 * P / (el_ms / K * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": "ensemble scenarios/s", "value": value, "unit": "scenarios/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": el_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": f"ensemble of {n} scenarios: side logU[64,512] cells, h=1 m, "
                                   "4 ppc, Bingham+Voellmy, dt=0.02 s",
                       "scenarios": n, "particles": P, "nodes": N, "passes": K,
                       "precision": args.precision,
                       "parallelism": f"batch; replicas{world}",
                       "l2": f"state {P * 188 / 1e6:.0f} MB > 126 MB L2, no flush"},
            "particle_steps_per_s": P * K / (el_ms * 1e-3) * world,
            "plain_path": {"value": plain_value, "unit": "scenarios/s",
                           "sample": f"first {m} scenarios alone through dampm_ctx, "
                                     f"{K} passes each, device time"},
            "batch_vs_plain": (value / world) / plain_value if plain_value else None,
            "finished": done,
            "failed": {"count": len(failed), "seeds": [seeds[k] for k in failed][:16],
                       "note": "stopped by the status word (non-finite state); not counted"},
            "autotune": tuned,
            "roofline": {"bound": "hbm", "kernel": "whole pass", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes_per_launch": 320.0 * P},
            "e2e": {"value": total / e2e_s, "unit": "scenarios/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "per ensemble: upload of every scenario, all passes, final hp back"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": (cpu_baseline_scenarios(ds, K) if world == 1 and
                             not args.no_cpu_baseline else None),
            "checksum_hp": float(sum(float(o.sum()) for o in outs)),
        }
        print(json.dumps(line), flush=True)
    _barrier(world)
    return 0


def run_mudflow_fp32(args, world, rank, local):
    """The mudflow in the FP32 form: a batch holding the one scenario."""
    import torch
    torch.cuda.set_device(local)
    from amsc_b200 import scenarios
    from amsc_b200.batch import Batch
    d = scenarios.mudflow(N=2048, seed=12345 + rank)
    stream = torch.cuda.Stream()
    b = Batch(d.np + 1024, d.nnodes + 1024, 2, stream=stream.cuda_stream, precision="fp32")
    h = b.add(d)
    b.step(args.warmup)
    b.sync()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    l0 = b.usage()["launches"]
    _barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    el_ms = _allreduce(e0.elapsed_time(e1), world)
    launches = b.usage()["launches"] - l0
    q = b.query(h)
    total = _allreduce(float(d.np), world, "sum")
    value = total * args.steps / (el_ms * 1e-3)
    peak, peak_kind = _peaks()
    # FP32 algorithmic bytes of a pass: sort ~28 B, P2G 56 B (13 x 4 B record
    # + index), G2P 96 B per particle
    per_pass = 180.0 * d.np
    achieved = per_pass / (el_ms / args.steps * 1e-3) / 1e9
    b.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(d)
        cpu["sample"] += " (the FP64 restatement: the reference has no FP32 form)"
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + ", FP32 form (a batch of one scenario)",
                       "particles": d.np, "grid": "2048x2048", "precision": "fp32",
                       "parallelism": f"replicas{world}",
                       "l2": "state 181 MB > 126 MB L2, no flush", "seed": 12345},
            "roofline": {"bound": "hbm", "kernel": "whole pass", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes_per_launch": per_pass},
            "e2e": None, "gpu_launches": int(launches), "clocks": clocks,
            "cpu_baseline": cpu, "state": {"it": q["it"], "t": q["t"], "dt": q["dt"]},
        }), flush=True)
    _barrier(world)
    return 0


def run_serving(args, world, rank, local):
    """--workload serving: requests arriving as a Poisson stream, served by
    continuous batching; scenarios/s and time-to-result percentiles."""
    import torch
    torch.cuda.set_device(local)
    from amsc_b200 import scenarios
    from amsc_b200.dampm import Solver
    from amsc_b200.serving import Request, Server, latency_summary, poisson_arrivals

    n = args.requests
    arr = poisson_arrivals(n, args.rate, seed=777 + rank)
    reqs = [Request(k, scenarios.serving_request(200000 * rank + k, t_end=args.t_end),
                    float(arr[k])) for k in range(n)]
    free, _ = torch.cuda.mem_get_info()
    budget = min(args.budget_gb * 1e9, 0.8 * free)
    stream = torch.cuda.Stream()
    srv = Server(budget, max_scenarios=args.max_scenarios, tick=args.tick,
                 stream=stream.cuda_stream, precision=args.precision,
                 graphs=not args.no_graphs)
    # warm-up: one short request through the same server
    warm = scenarios.serving_request(999999, t_end=0.2)
    srv.run([Request(-1, warm, 0.0)])
    l0 = srv.b.usage()["launches"]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    _barrier(world)
    t0 = time.perf_counter()
    srv.run(reqs)
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    launches = srv.b.usage()["launches"] - l0
    occupancy = srv.occupancy[:]
    srv.close()
    makespan = _allreduce(max(r.finished for r in reqs), world)
    total = _allreduce(float(n), world, "sum")
    value = total / makespan
    lat = latency_summary(reqs)
    passes = sum(r.passes for r in reqs)
    particle_steps = sum(r.passes * r.data.np for r in reqs)
    # the plain path: a sample of the same requests one at a time, host in to
    # host out, through dampm_ctx
    m = min(args.plain_sample, n)
    tp = time.perf_counter()
    for r in reqs[:m]:
        with Solver(r.data, stream=stream.cuda_stream) as s:
            s.run()
            for f in ("x", "y", "hp"):
                s.download(f)
    plain = m / (time.perf_counter() - tp) if m else None
    h2d = sum(8 * (10 * r.data.np + r.data.nnodes) for r in reqs)
    d2h = sum(8 * 3 * r.data.np for r in reqs)
    # time-to-result below and above capacity: the same requests at other
    # arrival rates, through a fresh server each
    sweep = []
    for rate in ([float(x) for x in args.rates.split(",")] if args.rates else []):
        arr_r = poisson_arrivals(n, rate, seed=777 + rank)
        rr = [Request(k, reqs[k].data, float(arr_r[k])) for k in range(n)]
        sv = Server(budget, max_scenarios=args.max_scenarios, tick=args.tick,
                    stream=stream.cuda_stream, precision=args.precision,
                    graphs=not args.no_graphs)
        sv.run([Request(-1, warm, 0.0)])
        sv.run(rr)
        sv.close()
        mk = max(r.finished for r in rr)
        sweep.append({"rate_per_s": rate, "scenarios_per_s": n / mk,
                      "latency": latency_summary(rr)})
    if rank == 0:
        line = {
            "metric": "serving scenarios/s", "value": value, "unit": "scenarios/s",
            "n_gpus": world, "steps": int(passes), "warmup": 1,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": f"serving: {n} requests, Poisson {args.rate}/s, side "
                                   "logU[64,1024] cells, h=1 m, CFL 0.4 to t=60 s",
                       "requests": n, "rate_per_s": args.rate, "t_end_s": args.t_end,
                       "budget_gb": round(budget / 1e9, 1), "tick_passes": args.tick,
                       "precision": args.precision, "cuda_graphs": not args.no_graphs,
                       "parallelism": f"continuous batching; replicas{world}",
                       "l2": "state > 126 MB L2 at full occupancy, no flush"},
            "latency": lat,
            "makespan_s": makespan, "wall_s": wall,
            "particle_steps_per_s": particle_steps / makespan,
            "mean_live_scenarios": float(np.mean(occupancy)) if occupancy else 0.0,
            "max_live_scenarios": int(max(occupancy)) if occupancy else 0,
            "compactions": srv.compactions,
            "plain_path": {"value": plain, "unit": "scenarios/s",
                           "sample": f"first {m} requests alone through dampm_ctx, upload "
                                     "to results on the host"},
            "serving_vs_plain": (value / world) / plain if plain else None,
            "e2e": {"value": value, "unit": "scenarios/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": "time-to-result runs from arrival to results on the host"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": (cpu_baseline_scenarios([r.data for r in reqs[:m]],
                                                    [r.passes for r in reqs[:m]])
                             if world == 1 and not args.no_cpu_baseline and m else None),
            "rate_sweep": sweep,
        }
        print(json.dumps(line), flush=True)
    _barrier(world)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="mudflow",
                    choices=["mudflow", "ensemble", "serving"])
    ap.add_argument("--requests", type=int, default=300)
    ap.add_argument("--rate", type=float, default=100.0)
    ap.add_argument("--rates", default="",
                    help="serving workload: also run these arrival rates (comma list)")
    ap.add_argument("--t-end", type=float, default=60.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-scenarios", type=int, default=1024)
    ap.add_argument("--tick", type=int, default=16)
    ap.add_argument("--merge-split", action="store_true",
                    help="mudflow workload: merge/split every 10 steps")
    ap.add_argument("--no-graphs", action="store_true",
                    help="serving workload: enqueue each pass instead of replaying graphs")
    ap.add_argument("--autotune", action="store_true",
                    help="ensemble workload: tune the unit plan during the timed passes")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp32 runs the FP32 form (mudflow: as a batch of one)")
    ap.add_argument("--scenarios", type=int, default=512)
    ap.add_argument("--plain-sample", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-timed", action="store_true",
                    help="ensemble: bracket the timed passes with cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-late", dest="late", action="store_false",
                    help="mudflow workload: skip the window at step 1000")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.steps is None:
        args.steps = 1000 if args.workload == "ensemble" else 400
    world, rank, local = _dist_init()
    if args.workload == "serving":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no request loop; its per-scenario CPU "
                                  "time is the mudflow reference arm"}))
            _barrier(world)
            return 0
        return run_serving(args, world, rank, local)
    if args.workload == "ensemble":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference runs one scenario per process; its "
                                  "per-scenario CPU time is the mudflow reference arm"}))
            _barrier(world)
            return 0
        rc = run_ensemble(args, world, rank, local)
        return rc
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        _barrier(world)
        return rc

    import torch
    torch.cuda.set_device(local)
    from amsc_b200 import scenarios
    from amsc_b200.dampm import STATE_FIELDS, Solver

    if args.precision == "fp32":
        return run_mudflow_fp32(args, world, rank, local)
    d = scenarios.mudflow(N=2048, seed=12345 + rank, merge_split=args.merge_split)
    np_ = d.np
    ts = torch.cuda.Stream()
    s = Solver(d, merge_split=args.merge_split, stream=ts.cuda_stream)
    # warm-up (the first call also captures the CUDA graph of the passes)
    s.step(args.warmup)
    s.sync()
    # timed region: K steps, device-timed with CUDA events on the library
    # stream; passes run as they do for a user (16 at a time from a graph)
    sampler = ClockSampler(local)
    _barrier(world)
    s.sync()
    sampler.start()
    time.sleep(0.3)  # let the sampler start before the timed region
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ts)
    s.step(args.steps)
    e1.record(ts)
    ts.synchronize()
    clocks = sampler.stop()
    launches = s.last_launch_count()
    el_ms = _allreduce(e0.elapsed_time(e1), world)
    total_particles = _allreduce(float(np_), world, "sum")
    value = total_particles * args.steps / (el_ms * 1e-3)
    ms_per_step = el_ms / args.steps
    st = s.status()

    # the same rate later in the run: advance to step LATE_IT (the flow has
    # spread and piled up), then time LATE_STEPS more
    late = None
    if not args.merge_split and args.late:
        s.step(max(0, LATE_IT - st["it"]))
        s.sync()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(ts)
        s.step(LATE_STEPS)
        l1.record(ts)
        ts.synchronize()
        lms = _allreduce(l0.elapsed_time(l1), world)
        sl = s.status()
        late = {"from_it": sl["it"] - LATE_STEPS, "steps": LATE_STEPS,
                "ms_per_step": lms / LATE_STEPS,
                "value": total_particles * LATE_STEPS / (lms * 1e-3), "unit": METRIC,
                "t": sl["t"]}

    # roofline of the dominant kernel.  `achieved` uses the algorithmic bytes
    # of the scope table: P2G reads 11 f64 fields of each particle and its
    # sorted index (92 B) and writes 5 f64 sums and reads Z per touched node
    # (48 B); G2P reads x, y, hp, Mp, Vp, H and the index (52 B) and writes
    # x, y, vpx, vpy, hp, F11, F12, F22 (64 B) per particle and reads vvxL,
    # vvyL, Z per touched node (24 B).  `design_bytes_per_launch` is what
    # this implementation moves: P2G gathers the 13-value f64 record and the
    # slot (108 B) and writes vvxL, vvyL (16 B per node); G2P reads the slot,
    # key, index and x, y, hp, H, Mp, Vp (60 B) and writes the 11 state
    # fields, key, index, sort slot and the 8-value record (164 B), and reads
    # vvxL, vvyL, Z (24 B per node).
    # The per-kernel times: the same warm-up and K steps once more, from the
    # same initial state, with CUDA events between the kernel classes (those
    # passes are launched one by one).
    with Solver(d, merge_split=args.merge_split, stream=ts.cuda_stream) as sk:
        sk.step(args.warmup)
        sk.sync()
        sk.timings(True)
        sk.step(args.steps)
        sk.sync()
        tm = sk.timings(False)
        x = sk.download("x")
        y = sk.download("y")
        np_now = sk.status()["np"]
    h = float(d.scalars["hx"])
    nrows = int(d.scalars["Ney"])
    kc = (np.clip(np.floor(y / h), 0, nrows - 1).astype(np.int64) +
          np.clip(np.floor(x / h), 0, int(d.scalars["Nex"]) - 1).astype(np.int64) * nrows)
    n_nodes = _touched_nodes(d, kc)
    alg = {"p2g": 92 * np_now + 48 * n_nodes, "g2p": 116 * np_now + 24 * n_nodes}
    design = {"p2g": 108 * np_now + 16 * n_nodes, "g2p": 224 * np_now + 24 * n_nodes}
    kms = {"p2g": tm[1] / args.steps, "g2p": tm[2] / args.steps}
    peak, peak_kind = _peaks()
    dom = "p2g" if kms["p2g"] >= kms["g2p"] else "g2p"
    achieved = alg[dom] / (kms[dom] * 1e-3) / 1e9
    traffic = _traffic_profile().get(dom)
    per_kernel = {k: {"algorithmic_bytes": alg[k], "design_bytes": design[k],
                      "ms": kms[k], "achieved_gbs": alg[k] / (kms[k] * 1e-3) / 1e9,
                      "frac": alg[k] / (kms[k] * 1e-3) / 1e9 / peak,
                      "design_gbs": design[k] / (kms[k] * 1e-3) / 1e9}
                  for k in ("p2g", "g2p")}

    # end to end through the C ABI with host buffers: per step the persistent
    # state goes host->device from pinned memory (dampm_set_state), the step
    # runs, and the state comes back (dampm_get_state)
    pin = {k: torch.empty(np_now, dtype=torch.float64, pin_memory=True).numpy()
           for k in STATE_FIELDS}
    s.get_state(pin)
    e2e_steps = max(args.e2e_steps, 1)
    _barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.set_state(pin)
        s.step(1)
        s.get_state(pin)
    e2e_s = _allreduce(time.perf_counter() - t0, world)
    e2e_value = total_particles * e2e_steps / e2e_s
    state_bytes = 8 * len(STATE_FIELDS) * np_now

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_port(d)
        except Exception as e:  # reported, not fatal
            cpu = {"error": str(e)}
    s.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": mudflow_config(np_, st["np"], world, args.merge_split,
                                     launch=("one pass at a time outside the merge/split "
                                             "cycle graphs" if args.merge_split
                                             else "CUDA graphs of 16 passes")),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg[dom],
                         "design_bytes_per_launch": design[dom],
                         "kernel_ms": kms[dom],
                         "kernel_ms_from": "the same warm-up and steps run again from the "
                                           "same state with CUDA events between kernel "
                                           "classes"},
            "kernels": per_kernel,
            "kernels_ms_per_step": {"sort": tm[0] / args.steps, "p2g": kms["p2g"],
                                    "g2p": kms["g2p"], "other": tm[3] / args.steps},
            "late": late,
            "e2e": {"value": e2e_value, "unit": METRIC,
                    "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "state": {"it": st["it"], "t": st["t"], "dt": st["dt"]},
        }
        print(json.dumps(line), flush=True)
    _barrier(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
