#!/usr/bin/env python3
"""Benchmark of the batched XPBD Cosserat-rod step on B200.

Default workload: the uneven batch -- 16384 rods of U{16..512} segments
(0.2 m per 32 segments), coiled, 1-4 primitives each, self-collision on,
dt 1/60 with 50 substeps -- run by the persistent batched kernel (one kernel
per step), with the plain one-rod-per-CTA kernel timed on the same batch for
the batched-vs-plain ratio. Metric: segment-substeps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload uneven|grid]
  python bench.py --impl reference ...     # the reference's CPU solver, host cores

Under torchrun, rank r of N simulates shard r of one seeded uneven batch of
N x 16384 rods on its own GPU (rods are independent: weak scaling, no
data-path collective); the other workloads run as replicas. The time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Floating-point operations (add, sub, mul, div, sqrt) per segment-substep of
# the reference's step, counted by the op-counting oracle build
# (liboracle_count.so; tests/test_oracle.py recomputes every value):
#   uneven      32 sampled rods of the uneven batch (seed 0), steps 25-44 -- the
#               window a 5-warm-up, 20-step run times -- with their primitives
#               and self-collision (contacts and self-contacts included)
#   hook        16 placements spread over the hook sweep, steps 23-42 (the
#               window the shape timing measures), bar, floor, self-collision
#   grid        a pinned 64-segment rod over the floor plane
#   cantilever  a pinned 64-segment rod, no contacts
FLOPS_PER_SEG_SUBSTEP = {"uneven": 1696.2, "hook": 1446.1, "grid": 890.5, "cantilever": 880.5}
# Algorithmic HBM bytes per segment per step: state read once and written once
# (x, v, force, kinematic velocity per particle; q, omega, torque per frame;
# float4 rows): read 4 x 16 + 3 x 16, written 2 x 16 + 2 x 16.
BYTES_PER_SEG_STEP = 7 * 16 + 4 * 16
# Measured DRAM bytes (read + write) per segment-step of the batched step,
# from one ncu capture of a 4096-rod uneven batch (state beyond L2, so the
# figure scales with segments: 246.0 MB over 1 084 256 segments).
DRAM_BYTES_PER_SEG_STEP = {"uneven": 226.9}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def build_workload(name: str, rods: int, seed: int, shard=None):
    from ropephysics_b200 import workloads
    if name == "uneven":
        return workloads.uneven(rods or 16384, seed=seed, shard=shard)
    if name == "grid":
        return workloads.grid(rods or 4096, seed=seed)
    if name == "cantilever":
        return workloads.cantilever()
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------------------- CPU reference


def load_synth():
    """ropephysics_b200/synth.py loaded by its path: the workload's seeded
    draws without importing the package, so a CPU-only process never maps the
    library."""
    import importlib.util
    name = "ropephysics_b200_synth"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "ropephysics_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


WORKLOAD_PARAMS = {"uneven": (1.0 / 60, 50), "grid": (1.0 / 60, 20), "cantilever": (1.0 / 60, 20)}


def workload_config(name: str, rods: int, seed: int) -> dict:
    """The workload's description, computed from the draws alone, identical in
    both arms' JSON lines."""
    S = load_synth()
    dt, substeps = WORKLOAD_PARAMS[name]
    if name == "uneven":
        n = rods or 16384
        segs = sum(d.segments for d in S.uneven(n, seed))
        wname = f"uneven-{n}x[16,512]"
    elif name == "grid":
        n = rods or 4096
        segs, wname = 64 * n, f"grid-{n}x64"
    else:
        n, segs, wname = 1, 64, "cantilever-1x64"
    state_bytes = BYTES_PER_SEG_STEP * segs
    return {"workload": wname, "rods": n, "segments": int(segs), "substeps": substeps, "dt": dt,
            "l2": "inputs larger than L2" if state_bytes > 126e6 else "L2-resident state"}


class ReferenceSample:
    """A bounded sample of the workload built by the reference's own builders
    (makeRodFromCenterline / makeStraightRod, src/core/rod.cpp) and stepped
    by its own FP64 CPU solver (crs::step, src/core/solver.cpp:269-290) in the
    GPU colour order, both compiled from the reference's sources into
    oracle/_ref/libcrs_ref.so. Rods are spread over host threads in contiguous
    ranges, as the reference's throughput case does
    (src/validation/scaling_cases.cpp:404-459). The rods come from the same
    seeded draws as the GPU arm's (ropephysics_b200/synth.py)."""

    def __init__(self, name: str, rods: int, seed: int, sample_rods: int):
        import oracle as orc
        S = load_synth()
        self.ref = ref = orc.Reference(gpu=False)
        self.handles, self.worlds = [], []
        mat = dict(youngs=S.YOUNGS, poisson=S.POISSON, density=S.DENSITY, radius=S.RADIUS)
        rng = np.random.default_rng(123)
        if name == "uneven":
            draws = S.uneven(rods or 16384, seed)
            idx = rng.choice(len(draws), size=min(sample_rods, len(draws)), replace=False)
            for i in idx:
                d = draws[i]
                h = ref.centerline(d.points, frame_seed=(0.0, 0.0, 1.0), **mat)
                rr = ref.export(h)
                rr.bRestD[:] = 0.0  # straight rest shape: the coil is loaded
                ref.import_state(h, rr)
                self.handles.append(h)
                self.worlds.append(ref.world(orc.World([orc.Primitive(*q) for q in d.prims], True, d.friction,
                                                       2, d.hash_table_size, 0.25)))
            self.segments = int(sum(draws[i].segments for i in idx))
            total = len(draws)
        elif name == "grid":
            g = S.grid(rods or 4096, seed)
            idx = rng.choice(len(g.youngs_scale), size=min(sample_rods, len(g.youngs_scale)), replace=False)
            for i in idx:
                m = dict(mat, youngs=S.YOUNGS * float(g.youngs_scale[i]))
                h = ref.straight(64, 1.0, origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, -1.0), **m)
                rr = ref.export(h)
                rr.invMass[0] = 0.0  # pinned top, moving at its drive's t = 0 velocity
                w = 2 * math.pi * g.frequency[i]
                rr.kinVel[0] = (0.0, 0.0, g.amplitude[i] * w * math.cos(g.phase[i]))
                ref.import_state(h, rr)
                self.handles.append(h)
                mu = 0.5 * float(g.friction_scale[i])
                self.worlds.append(ref.world(orc.World([orc.Primitive(*S.plane((0.0, 0.0, -1.2),
                                                                               (0.0, 0.0, 1.0), mu))])))
            self.segments = 64 * len(idx)
            total = len(g.youngs_scale)
        else:
            h = ref.straight(64, 1.0, **mat)
            ref.lib.ref_rod_clamp(h, 0)
            rr = ref.export(h)
            rr.extForce[rr.nP - 1] = (0.0, 0.0, -0.05)
            ref.import_state(h, rr)
            self.handles.append(h)
            self.worlds.append(None)
            self.segments, total, idx = 64, 1, [0]
        dt, self.substeps = WORKLOAD_PARAMS[name]
        f32 = lambda v: float(np.float32(v))
        self.params = orc.Params(dt=f32(dt), substeps=self.substeps, iterations=1,
                                 gravity=(0.0, 0.0, f32(-9.81)))
        self.desc = f"{len(idx)} of {total} rods ({self.segments} segments)"

    def run(self, steps: int, threads: int) -> float:
        """Wall seconds of `steps` steps of every sampled rod."""
        p = self.params
        H = (C.c_void_p * len(self.handles))(*self.handles)
        W = (C.c_void_p * len(self.worlds))(*self.worlds)
        g = (C.c_double * 3)(*p.gravity)
        return self.ref.lib.ref_step_many(H, W, len(self.handles), p.dt, p.substeps, p.iterations, g, 0.0, 0.0,
                                          1, steps, threads)

    def close(self):
        for h in self.handles:
            self.ref.free(h)
        self.handles = []


def cpu_reference_rate(name: str, rods: int, seed: int, sample_rods: int, budget_s: float, threads: int,
                       advance: int):
    """The reference's FP64 CPU step on a bounded sample of the workload, over
    `threads` host threads, timed from step `advance` (the step the GPU's
    timed region starts at: a coil's contact work changes as it relaxes).
    Returns (rate, kind, sample description, threads)."""
    sample = ReferenceSample(name, rods, seed, sample_rods)
    if advance > 1:
        sample.run(advance - 1, threads)
    t1 = sample.run(1, threads)
    steps = max(1, min(200, int(budget_s / max(t1, 1e-3))))
    t = sample.run(steps, threads)
    sample.close()
    rate = sample.segments * sample.substeps * steps / t
    desc = (f"{sample.desc} x {steps} steps x {sample.substeps} substeps from step {advance}, "
            f"{t:.1f} s")
    return rate, "reference", desc, threads


# ----------------------------------------------------------------------------- served stream


def run_served(capacity: float, seconds: float, seed: int, load: float, budget_gb: float,
               drain_s: float = 240.0):
    """The served rollout stream: Poisson arrivals of requests with the
    served-config shapes (1-1024 rods log-uniform, 32-512 segments, horizon
    100-2000 steps, random features, grid materials), submitted in real time
    to a continuous-batching server with an HBM admission budget. The spec's
    200 requests/s offer far more work than one GPU executes, so the arrival
    rate is set to `load` x the measured capacity and the spec's load factor is
    reported beside it. Latency = completion - submission, per request."""
    import threading

    import ropephysics_b200 as rp
    from ropephysics_b200 import workloads as W

    params = rp.StepParams(dt=1.0 / 60, substeps=20, iterations=1)
    rng = np.random.default_rng(seed)
    probe = [W.served_request(np.random.default_rng(seed + 1000 + i)) for i in range(32)]
    mean_work = float(np.mean([r.segment_substeps(params.substeps) for r in probe]))
    spec_rate = 200.0
    rate = max(0.05, load * capacity / mean_work)
    import torch

    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    # the arenas are the budget; leave room for the context and streams
    budget = min(int(budget_gb * (1 << 30)), int(0.85 * free))
    server = rp.Server(budget, params)
    ids, errors = [], []

    def submitter():
        t_next = time.perf_counter()
        t_end = t_next + seconds
        while True:
            t_next += rng.exponential(1.0 / rate)
            if t_next > t_end:
                break
            req = W.served_request(rng)
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            try:
                ids.append(server.submit(req.rods, req.steps, req.worlds, [0] * len(req.rods),
                                         req.drives, req.youngs_scale, req.friction_scale))
            except rp.RopeError as e:
                errors.append(str(e))

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    try:
        server.drain(drain_s)
        drained = True
    except rp.RopeError:
        drained = False
    st = server.stats()
    infos = [server.info(i) for i in ids]
    done = [i for i in infos if i["state"] == 2]
    lat = sorted(i["done_s"] - i["submit_s"] for i in done)
    work = sum(i["segment_substeps"] for i in done)
    span = (max(i["done_s"] for i in done) - min(i["submit_s"] for i in infos)) if done else 0.0
    server.close()
    pct = lambda v, p: float(np.percentile(v, p)) if v else None
    wait = sorted(i["admit_s"] - i["submit_s"] for i in done)  # queued behind the budget
    steps_per_s = [i["segment_substeps"] / max(i["done_s"] - i["admit_s"], 1e-9) for i in done]
    return {
        "requests": len(ids), "completed": len(done), "drained": drained, "rejected": len(errors),
        "p50_latency_s": pct(lat, 50), "p99_latency_s": pct(lat, 99),
        "mean_latency_s": float(np.mean(lat)) if lat else None,
        "p50_queue_wait_s": pct(wait, 50), "p99_queue_wait_s": pct(wait, 99),
        "p50_request_rate": pct(steps_per_s, 50),
        "sustained": work / span if span > 0 else None, "unit": "segment-substeps/s",
        "busy_s": st["busy_s"], "arrival_rate_req_s": rate, "window_s": seconds,
        "load_vs_capacity": load, "spec_rate_req_s": spec_rate,
        "spec_offered": spec_rate * mean_work, "spec_load_factor": spec_rate * mean_work / capacity,
        "budget_bytes": st["budget_bytes"], "peak_resident_bytes": st["peak_resident_bytes"],
        "steps_launched": st["steps_launched"],
    }


# ----------------------------------------------------------------------------- GPU arm


def measure_shapes(stream, fp32_peak: float) -> dict:
    """The other named shapes, batched (autotuned: for one short rod the tuner
    picks one rod per CTA) and plain, short timed runs on the same GPU: the
    clamped 64-segment cantilever with a tip load (latency of one rod), the
    4096 x 64 driven grid over a floor, and the 3600-cable hook sweep in mixed
    precision (compensated positions and frames, FP64 cone and verdicts).
    Device time with CUDA events after 3 warm-up steps."""
    import torch

    import ropephysics_b200 as rp
    from ropephysics_b200 import workloads as W

    mixed = rp.Precision.COMPENSATED | rp.Precision.FP64_CONE | rp.Precision.FP64_VERDICT
    out = {}
    for key, wl, prec, steps in (("cantilever", W.cantilever(), rp.Precision.REFERENCE, 200),
                                 ("grid", W.grid(4096), rp.Precision.REFERENCE, 20),
                                 ("hook", W.hook(), mixed, 20)):
        seg_sub = wl.segment_substeps_per_step()
        rates = {}
        tuning = None
        for label, strat in (("batched", rp.Strategy.BATCHED), ("plain", rp.Strategy.FUSED)):
            b = wl.make_batch(strat)
            b.set_precision(int(prec))
            b.set_stream(stream.cuda_stream)
            if strat == rp.Strategy.BATCHED:  # as a user's batch would run: autotuned
                tuning = b.autotune(wl.params, max_steps_per_launch=4)
            b.set_graph(True)
            b.step_many(wl.params, 3)
            b.step_many(wl.params, steps)
            b.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step_many(wl.params, steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            rates[label] = (seg_sub / (ms / 1e3), ms)
            b.close()
        flops = FLOPS_PER_SEG_SUBSTEP.get(key, 890.5)
        out[key] = {"workload": wl.name, "precision": int(prec), "unit": "segment-substeps/s", "tuning": tuning,
                    "batched": rates["batched"][0], "plain": rates["plain"][0],
                    "speedup": rates["batched"][0] / rates["plain"][0],
                    "ms_per_step_batched": rates["batched"][1], "ms_per_step_plain": rates["plain"][1],
                    "fp32_frac_batched": rates["batched"][0] * flops / 1e12 / fp32_peak}
    out["harness"] = measure_harness(stream)
    return out


def measure_harness(stream, attempts: int = 1024, steps: int = 630) -> dict:
    """One learning iteration's attempt batch of the harness-routing task:
    1024 motions on random cables (120 segments, 4 substeps x 4 sweeps, five
    primitives), each gripper an on-device waypoint schedule. A tenth of the
    6300-step schedule is timed, batched (autotuned) and plain, with CUDA
    events; `s_per_iteration` scales it to the whole schedule."""
    import numpy as np
    import torch

    import ropephysics_b200 as rp
    from ropephysics_b200 import harness as H

    t = H.HarnessTask()
    rng = np.random.default_rng(0)
    pols = [t.to_policy(t.hand_written_policy().reshape(-1) + 0.08 * rng.standard_normal(10))
            for _ in range(attempts)]
    youngs, friction = H.random_cables(rng, attempts)
    p = t.params()
    res = {"workload": f"harness-{attempts}x{t.segments}", "unit": "segment-substeps/s"}
    seg_sub = attempts * t.segments * p.substeps
    for label, strat in (("batched", rp.Strategy.BATCHED), ("plain", rp.Strategy.FUSED)):
        b = rp.Batch.create(t.build(), attempts, strat, t.world())
        b.set_stream(stream.cuda_stream)
        b.set_material_scales(youngs, friction)
        if strat == rp.Strategy.BATCHED:
            b.autotune(p, max_steps_per_launch=4)
        b.set_waypoint_drives([t.drive(q) for q in pols])
        b.set_graph(True)
        b.step_many(p, 20)
        b.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step_many(p, steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[label] = seg_sub / (ms / 1e3)
        res[f"ms_per_step_{label}"] = ms
        res[f"s_per_iteration_{label}"] = ms * t.steps() / 1e3
        b.close()
    res["speedup"] = res["batched"] / res["plain"]
    return res


def run_ours(args):
    world_size, rank, local = dist_setup(args)
    import torch
    torch.cuda.set_device(local)
    import ropephysics_b200 as rp

    # N ranks: shards of one seeded batch of N x rods (every rank the same
    # spread of lengths; weak scaling), else independent replicas
    shard = (rank, world_size) if world_size > 1 and args.workload == "uneven" else None
    wl = build_workload(args.workload, args.rods, seed=args.seed if shard else args.seed + rank, shard=shard)
    config = workload_config(args.workload, args.rods, args.seed)
    config["parallelism"] = f"shards{world_size}" if shard else f"replicas{world_size}"
    if world_size == 1:
        assert config["segments"] == int(wl.segments.sum()) and config["workload"] == wl.name
    seg_sub = wl.segment_substeps_per_step()
    p = wl.params
    # the roofline denominator, measured on this device before anything else runs
    fp32_peak = rp.measure_fp32_peak(8192)

    batch = wl.make_batch(rp.Strategy.BATCHED)
    stream = torch.cuda.Stream()
    batch.set_stream(stream.cuda_stream)
    batch.set_graph(True)
    # rods per CTA, threads per rod and steps per launch, timed on this batch
    # (its state is restored afterwards)
    tuning = batch.autotune(p, max_steps_per_launch=4) if not args.no_tune else batch.tuning

    # warm-up: first launches pay module load; the graph is captured here
    for _ in range(args.warmup):
        batch.step_many(p, 1)
    batch.step_many(p, args.steps)
    batch.synchronize()
    # the end-to-end twin: the same rods, advanced to the state the timed
    # region starts from (every launch shape gives bitwise the same steps)
    twins = []
    if not args.no_e2e:
        for _ in range(2):  # pipelined and serial end-to-end runs
            twin = wl.make_batch(rp.Strategy.BATCHED)
            twin.set_stream(stream.cuda_stream)
            twin.set_tuning(tuning["cta_threads"], tuning["pairs_per_thread"], 1)
            twin.step_many(p, args.warmup + args.steps)
            twin.synchronize()
            twins.append(twin)

    # ---- device-resident throughput (value) ----
    barrier(world_size)
    torch.cuda.synchronize()
    launches0 = batch.kernel_launches
    with ClockSampler(local) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.step_many(p, args.steps)
        e1.record(stream)
        e1.synchronize()
    launches = batch.kernel_launches - launches0
    torch.cuda.synchronize()
    barrier(world_size)
    ms = max_over_ranks(e0.elapsed_time(e1), world_size)
    value = seg_sub * args.steps * world_size / (ms / 1e3)

    # ---- end to end through the public API with pinned host buffers ----
    # Every step: the kinematic velocities in (host -> device), one step, the
    # positions, frames and contact states out (device -> host). Same rods and
    # same starting state as the timed region (twin batches). Two ways:
    #   pipelined  the copies ride a second stream (the overlapped copy calls)
    #              and the host takes step k's results while step k+1 runs;
    #              input and output host buffers are double-buffered
    #   serial     copies on the batch's stream and a host synchronize after
    #              every step; per-phase event times
    e2e = None
    if twins:
        nbytes = {k: twins[0].state_bytes(k) for k in (twins[0].POSITIONS, twins[0].FRAMES, twins[0].CONTACTS)}
        h2d = 16 * twins[0].total_particles
        d2h = int(sum(nbytes.values()))
        kin = [torch.zeros(twins[0].total_particles * 4, dtype=torch.float32).pin_memory() for _ in range(2)]
        outs = [{k: torch.empty(max(1, n), dtype=torch.uint8).pin_memory() for k, n in nbytes.items()}
                for _ in range(2)]
        # pipelined
        tw = twins[0]
        copy = torch.cuda.Stream()
        tw.set_copy_stream(copy.cuda_stream)
        done = [torch.cuda.Event() for _ in range(args.steps)]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world_size)
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(args.steps):
            tw.write_state_overlapped(tw.KINEMATIC, kin[k % 2].data_ptr(), h2d)
            tw.step(p)
            for what, n in nbytes.items():
                if n:
                    tw.read_state_overlapped(what, outs[k % 2][what].data_ptr(), n)
            done[k].record(copy)
            if k >= 1:
                done[k - 1].synchronize()  # step k-1's results are in host memory
        t1.record(copy)
        t1.synchronize()
        pipe_s = max_over_ranks(t0.elapsed_time(t1) / 1e3, world_size)
        tw.close()
        # serial
        tw = twins[1]
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
        barrier(world_size)
        torch.cuda.synchronize()
        for k in range(args.steps):
            ev[k][0].record(stream)
            tw.write_state_async(tw.KINEMATIC, kin[0].data_ptr(), h2d)
            ev[k][1].record(stream)
            tw.step(p)
            ev[k][2].record(stream)
            for what, n in nbytes.items():
                if n:
                    tw.read_state_async(what, outs[0][what].data_ptr(), n)
            ev[k][3].record(stream)
            tw.synchronize()
        phase = [sum(ev[k][i].elapsed_time(ev[k][i + 1]) for k in range(args.steps)) / args.steps
                 for i in range(3)]
        serial_s = max_over_ranks(ev[0][0].elapsed_time(ev[-1][3]) / 1e3, world_size)
        tw.close()
        e2e = {"value": seg_sub * args.steps * world_size / pipe_s, "unit": "segment-substeps/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": pipe_s * 1e3 / args.steps,
               "how": "pipelined: inputs and outputs of every step over the host link on a copy stream "
                      "(rp_batch_*_state_overlapped), results of step k taken by the host while step k+1 runs",
               "serial": {"value": seg_sub * args.steps * world_size / serial_s,
                          "ms_per_step": serial_s * 1e3 / args.steps, "h2d_ms": phase[0], "step_ms": phase[1],
                          "d2h_ms": phase[2], "h2d_gbs": h2d / phase[0] / 1e6, "d2h_gbs": d2h / phase[2] / 1e6},
               "start": "the timed region's starting state (twin batches)"}

    # ---- plain one-rod-per-CTA step on the same batch (batched vs plain) ----
    plain_rate = None
    if not args.no_plain:
        try:
            plain = wl.make_batch(rp.Strategy.FUSED)
            plain.set_stream(stream.cuda_stream)
            plain.step(p)
            plain.synchronize()
            ps = max(1, min(args.steps, 3))
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            for _ in range(ps):
                plain.step(p)
            q1.record(stream)
            q1.synchronize()
            plain_rate = seg_sub * ps / (q0.elapsed_time(q1) / 1e3)
            plain.close()
        except rp.RopeError as e:
            plain_rate = f"unavailable: {e}"

    peaks = measured_peaks()
    per_launch_s = (ms / 1e3) / max(1, launches)
    steps_per_launch = args.steps / max(1, launches)
    fps = FLOPS_PER_SEG_SUBSTEP.get(args.workload, 880.5)
    flops_launch = fps * seg_sub * steps_per_launch
    bytes_launch = BYTES_PER_SEG_STEP * config["segments"] * steps_per_launch
    traffic = (DRAM_BYTES_PER_SEG_STEP[args.workload] * config["segments"] * steps_per_launch
               if args.workload in DRAM_BYTES_PER_SEG_STEP else None)
    clk = clocks.summary()
    line = {
        "metric": "segment-substeps/s",
        "value": value,
        "unit": "segment-substeps/s",
        "n_gpus": world_size,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": config,
        "launch": {"strategy": "batched", "tuning": tuning, "graph": True,
                   "steps_per_launch": steps_per_launch},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "plain": {"value": plain_rate, "unit": "segment-substeps/s",
                  "speedup": (value / world_size / plain_rate) if isinstance(plain_rate, float) else None},
        "roofline": {"bound": "fp32", "achieved": flops_launch / per_launch_s / 1e12,
                     "peak": fp32_peak["tflops"], "unit": "TFLOP/s",
                     "frac": flops_launch / per_launch_s / 1e12 / fp32_peak["tflops"],
                     "traffic": traffic,
                     "flops_per_segment_substep": fps,
                     "note": "of measured: peak = FP32 FMA microkernel on this GPU (rp_measure_fp32_peak); "
                             "FLOPs = the reference step's add/sub/mul/div/sqrt count on this workload "
                             "(op-counting oracle, contacts and self-collision included); traffic = DRAM "
                             "bytes per launch from ncu on 4096 rods, scaled by segments"},
        "hbm": {"achieved": bytes_launch / per_launch_s / 1e9, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": bytes_launch / per_launch_s / 1e9 / peaks.get("hbm_gbs", 6650.0),
                "bytes_per_segment_step": BYTES_PER_SEG_STEP,
                "peak_source": "fallback" if peaks.get("fallback") else "measured"},
        "clocks": clk,
    }
    if world_size == 1 and not args.no_shapes:
        line["shapes"] = measure_shapes(stream, fp32_peak["tflops"])
    if world_size == 1 and not args.no_served:
        batch.close()
        line["served"] = run_served(value, args.served_seconds, args.seed + 7,
                                    args.served_load, args.served_budget_gb)
    if rank == 0 and world_size == 1 and not args.no_cpu:
        rate, kind, sample, threads = cpu_reference_rate(args.workload, args.rods, args.seed, args.cpu_rods,
                                                          args.cpu_seconds, os.cpu_count() or 1,
                                                          args.warmup + args.steps)
        line["cpu_baseline"] = {"value": rate, "unit": "segment-substeps/s", "cores": threads,
                                "kind": kind, "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reference_gpu_rates(seed: int) -> dict:
    """The reference's own FP32 GPU batch (src/gpu/gpu_solver.cu and
    gpu_batch.cpp, built for sm_100a into oracle/_ref/libcrs_ref_gpu.so) on
    the shapes its API can express, driven the way its API drives them:
    one Batch::step per step, kinematic velocities uploaded from the host
    every step, wall time over the steps with a device synchronise at the
    end (the reference's calls are synchronous).
      grid              the 4096 x 64 driven grid in full: one fused batch,
                        per-rod stiffness and friction scales, floor
      uneven_by_length  the uneven batch grouped by length (its Batch holds
                        one prototype and one world): 8 lengths spread over
                        16..512, every rod of that length as one batch with
                        self-collision on and no primitives; fused where its
                        shared memory allows, else its multi-kernel path"""
    import oracle as orc
    S = load_synth()
    try:
        R = orc.Reference(gpu=True)
    except Exception as e:  # the reference GPU build is absent
        return {"unavailable": f"reference GPU library: {e}"}
    if not R.lib.refgpu_available():
        return {"unavailable": "no CUDA device"}
    FP = C.POINTER(C.c_float)
    mat = dict(youngs=S.YOUNGS, poisson=S.POISSON, density=S.DENSITY, radius=S.RADIUS)
    out = {"unit": "segment-substeps/s", "timing": "wall clock, synchronised, reference API call pattern"}
    # ---- grid ----
    dt, sub = WORKLOAD_PARAMS["grid"]
    g = S.grid(4096, seed)
    h = R.straight(64, 1.0, origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, -1.0), **mat)
    rr = R.export(h)
    rr.invMass[0] = 0.0
    R.import_state(h, rr)
    wh = R.world(orc.World([orc.Primitive(*S.plane((0.0, 0.0, -1.2), (0.0, 0.0, 1.0), 0.5))]))
    rb = R.lib.refgpu_create(h, 4096, 1, wh)
    grav = (C.c_double * 3)(0.0, 0.0, float(np.float32(-9.81)))
    ys = np.ascontiguousarray(g.youngs_scale, np.float32)
    fs = np.ascontiguousarray(g.friction_scale, np.float32)
    R.lib.refgpu_set_material_scales(rb, ys.ctypes.data_as(FP), fs.ctypes.data_as(FP), 4096)
    kin = np.zeros((4096, 65, 3), np.float32)
    w = 2 * math.pi * g.frequency

    def grid_step(s):
        kin[:, 0, 2] = g.amplitude * w * np.cos(w * s * dt + g.phase)
        R.lib.refgpu_set_kinematic(rb, kin.ctypes.data_as(FP), 4096 * 65)
        R.lib.refgpu_step(rb, dt, sub, 1, grav, 0.0, 0.0, 1, 1)

    for s in range(3):
        grid_step(s)
    R.lib.refgpu_sync(rb)
    steps = 20
    t0 = time.perf_counter()
    for s in range(steps):
        grid_step(3 + s)
    R.lib.refgpu_sync(rb)
    t = time.perf_counter() - t0
    out["grid"] = {"workload": "grid-4096x64", "rate": 4096 * 64 * sub * steps / t,
                   "ms_per_step": t * 1e3 / steps, "strategy": "fused"}
    R.lib.refgpu_free(rb)
    R.free(h)
    # ---- uneven batch, grouped by length ----
    dt, sub = WORKLOAD_PARAMS["uneven"]
    draws = S.uneven(16384, seed)
    by_len = {}
    for d in draws:
        by_len.setdefault(d.segments, []).append(d)
    lengths = sorted(by_len)
    pick = [lengths[int(round(i * (len(lengths) - 1) / 7))] for i in range(8)]
    total_work, total_t, groups = 0, 0.0, []
    for n in pick:
        rods = by_len[n]
        hs = []
        for d in rods:
            hh = R.centerline(d.points, frame_seed=(0.0, 0.0, 1.0), **mat)
            q = R.export(hh)
            q.bRestD[:] = 0.0
            R.import_state(hh, q)
            hs.append(hh)
        wh = R.world(orc.World([], True, rods[0].friction, 2, rods[0].hash_table_size, 0.25))
        fused = 1
        rb = R.lib.refgpu_create(hs[0], len(hs), 1, wh)
        if not rb:
            fused = 0
            rb = R.lib.refgpu_create(hs[0], len(hs), 0, wh)
        for i, hh in enumerate(hs):
            R.lib.refgpu_upload_rod(rb, i, hh)
        R.lib.refgpu_step(rb, dt, sub, 1, grav, 0.0, 0.0, 1, 1)
        R.lib.refgpu_sync(rb)
        k = 3
        t0 = time.perf_counter()
        R.lib.refgpu_step(rb, dt, sub, 1, grav, 0.0, 0.0, 1, k)
        R.lib.refgpu_sync(rb)
        t = time.perf_counter() - t0
        total_work += len(hs) * n * sub * k
        total_t += t
        groups.append({"segments": n, "rods": len(hs), "strategy": "fused" if fused else "multi-kernel",
                       "ms_per_step": t * 1e3 / k})
        R.lib.refgpu_free(rb)
        for hh in hs:
            R.free(hh)
    out["uneven_by_length"] = {"rate": total_work / total_t, "groups": groups,
                               "sample": "8 lengths over 16..512, every rod of each length, self-collision, "
                                         "no primitives, 3 steps each"}
    return out


def run_reference(args):
    """The reference's own FP64 CPU step on this box's host cores, on the
    workload's seeded draws: this process never imports ropephysics_b200.
    Each timed step is one run of the bounded sample."""
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    config = workload_config(args.workload, args.rods, args.seed)
    config["parallelism"] = f"replicas{world_size}"
    threads = os.cpu_count() or 1
    sample = ReferenceSample(args.workload, args.rods, args.seed, args.cpu_rods)
    # warm-up: advance the sample to the step the GPU arm's timed region
    # starts at (its warm-up steps plus its graph warm-up of `steps` steps)
    sample.run(max(1, args.warmup + args.steps), threads)
    steps = max(1, args.steps)
    # steps of the sample per timed step, so the whole run takes ~cpu_seconds
    t1 = sample.run(1, threads)
    per = max(1, min(200, int(args.cpu_seconds / steps / max(t1, 1e-3))))
    times = [sample.run(per, threads) for _ in range(steps)]
    sample.close()
    total = sum(times)
    value = sample.segments * sample.substeps * per * steps / total
    desc = (f"{sample.desc} x {per} steps x {sample.substeps} substeps per timed step, "
            f"{steps} timed steps from step {args.warmup + args.steps}, {total:.1f} s")
    line = {"metric": "segment-substeps/s", "value": value, "unit": "segment-substeps/s",
            "n_gpus": world_size, "steps": steps, "warmup": args.warmup,
            "ms_per_step": total * 1e3 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": "segment-substeps/s", "cores": threads,
                             "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": "segment-substeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_rates(args.seed)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["uneven", "grid", "cantilever"], default="uneven")
    ap.add_argument("--rods", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-shapes", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--cpu-rods", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-seconds", type=float, default=60.0)
    ap.add_argument("--served-load", type=float, default=0.7)
    ap.add_argument("--served-budget-gb", type=float, default=150.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
