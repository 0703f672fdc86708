#!/usr/bin/env python3
"""Benchmark of the batched XPBD Cosserat-rod step on B200.

Default workload: the uneven batch -- 16384 rods of U{16..512} segments
(0.2 m per 32 segments), coiled, 1-4 primitives each, self-collision on,
dt 1/60 with 50 substeps -- run by the persistent batched kernel (one kernel
per step), with the plain one-rod-per-CTA kernel timed on the same batch for
the batched-vs-plain ratio. Metric: segment-substeps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload uneven|grid]
  python bench.py --impl reference ...     # the reference's CPU solver, host cores

Under torchrun every rank simulates its own seeded workload on its own GPU
(rods are independent: weak scaling, no data-path collective); the time is the
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

# Floating-point operations per segment-substep of the plain step (add, sub,
# mul, div, sqrt), counted exactly by the op-counting oracle build
# (liboracle_count.so; tests/test_oracle.py pins these values). Contacts add
# ~10 per (particle, primitive) slot.
FLOPS_PER_SEG_SUBSTEP = {"grid": 890.5, "uneven": 880.5, "cantilever": 880.5, "hook": 890.5}
# Algorithmic HBM bytes per segment per step: state read once and written once
# (x, v, force, kinematic velocity per particle; q, omega, torque per frame;
# float4 rows): read 4 x 16 + 3 x 16, written 2 x 16 + 2 x 16.
BYTES_PER_SEG_STEP = 7 * 16 + 4 * 16
# Measured DRAM bytes (read + write) per segment-step of the batched step,
# from one ncu capture of a 4096-rod uneven batch (state beyond L2, so the
# figure scales with segments: 265.9 MB over 1 084 256 segments).
DRAM_BYTES_PER_SEG_STEP = {"uneven": 232.0}


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


def build_workload(name: str, rods: int, seed: int):
    from ropephysics_b200 import workloads
    if name == "uneven":
        return workloads.uneven(rods or 16384, seed=seed)
    if name == "grid":
        return workloads.grid(rods or 4096, seed=seed)
    if name == "cantilever":
        return workloads.cantilever()
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------------------- CPU reference


def cpu_reference_rate(wl, sample_rods: int, budget_s: float, threads: int):
    """The reference's own FP64 CPU step (src/core/solver.cpp, compiled from its
    sources into oracle/_ref) on a bounded sample of the same workload, rods
    spread over host threads as its throughput case does
    (src/validation/scaling_cases.cpp:404-459). Falls back to this
    repository's restatement (oracle/liboracle_f64.so) when the reference
    library is absent. Returns (rate, kind, sample description, threads)."""
    import oracle as orc
    kind = "reference"
    try:
        ref = orc.Reference(gpu=False)
    except FileNotFoundError:
        ref = None
        kind = "port"
    rng = np.random.default_rng(123)
    idx = rng.choice(len(wl.rods), size=min(sample_rods, len(wl.rods)), replace=False)
    p = wl.params
    f32 = lambda v: float(np.float32(v))
    params = orc.Params(dt=f32(p.dt), substeps=p.substeps, iterations=p.iterations,
                        gravity=tuple(f32(g) for g in p.gravity))
    segs = sum(wl.rods[i].num_stretch for i in idx)
    if ref is not None:
        handles, worlds = [], []
        for i in idx:
            r = wl.rods[i]
            h = ref.centerline(r.x, youngs=r.material.youngs, poisson=r.material.poisson,
                               density=r.material.density, radius=r.material.radius)
            rr = ref.export(h)
            n = r.num_particles
            rr.x[:n] = r.x
            rr.invMass[:n] = r.inv_mass
            rr.q[: r.num_frames] = r.q
            rr.bRestD[: r.num_bend] = r.b_rest_darboux
            rr.kinVel[:n] = r.kin_velocity
            rr.extForce[:n] = r.ext_force
            ref.import_state(h, rr)
            handles.append(h)
            w = wl.worlds[wl.world_of_rod[i]] if wl.worlds else None
            worlds.append(ref.world(orc.World([orc.Primitive(q.type, q.a, q.b, q.normal, q.half_extents,
                                                             q.rotation, q.radius, q.friction)
                                               for q in w.primitives], w.self_collision,
                                              w.self_friction, w.self_skip, w.hash_table_size,
                                              w.contact_margin_radii)) if w else None)
        H = (C.c_void_p * len(handles))(*handles)
        W = (C.c_void_p * len(worlds))(*worlds)
        g = (C.c_double * 3)(*params.gravity)

        def run(steps):
            return ref.lib.ref_step_many(H, W, len(handles), params.dt, params.substeps,
                                         params.iterations, g, 0.0, 0.0, 1, steps, threads)
        t1 = run(1)
        steps = max(1, min(200, int(budget_s / max(t1, 1e-3))))
        t = run(steps)
        for h in handles:
            ref.free(h)
    else:
        o = orc.Oracle("f64")
        rods = [orc.Rod(wl.rods[i].num_particles) for i in idx]
        raise SystemExit("reference CPU library missing and port path not wired")
    rate = segs * p.substeps * steps / t
    sample = (f"{len(idx)} of {len(wl.rods)} rods ({segs} segments) x {steps} steps x "
              f"{p.substeps} substeps, {t:.1f} s")
    return rate, kind, sample, threads


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
    """The other named shapes, batched and plain, short timed runs on the same
    GPU: the clamped 64-segment cantilever with a tip load (latency of one
    rod), the 4096 x 64 driven grid over a floor, and the 3600-cable hook
    sweep in mixed precision (compensated positions and frames, FP64 cone and
    verdicts). Device time with CUDA events after 3 warm-up steps."""
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
        for label, strat in (("batched", rp.Strategy.BATCHED), ("plain", rp.Strategy.FUSED)):
            b = wl.make_batch(strat)
            b.set_precision(int(prec))
            b.set_stream(stream.cuda_stream)
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
        out[key] = {"workload": wl.name, "precision": int(prec), "unit": "segment-substeps/s",
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

    wl = build_workload(args.workload, args.rods, seed=args.seed + rank)
    seg_sub = wl.segment_substeps_per_step()
    batch = wl.make_batch(rp.Strategy.BATCHED)
    stream = torch.cuda.Stream()
    batch.set_stream(stream.cuda_stream)
    batch.set_graph(True)
    p = wl.params
    # rods per CTA, threads per rod and steps per launch, timed on this batch
    # (its state is restored afterwards)
    tuning = batch.autotune(p, max_steps_per_launch=4) if not args.no_tune else batch.tuning

    # warm-up: first launches pay module load; the graph is captured here
    for _ in range(args.warmup):
        batch.step_many(p, 1)
    batch.step_many(p, args.steps)
    batch.synchronize()

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
    nbytes = {k: batch.state_bytes(k) for k in (batch.POSITIONS, batch.FRAMES, batch.CONTACTS)}
    kin = torch.zeros(batch.total_particles * 4, dtype=torch.float32).pin_memory()
    outs = {k: torch.empty(max(1, n), dtype=torch.uint8).pin_memory() for k, n in nbytes.items()}
    e2e_steps = max(3, args.steps // 2)
    batch.set_graph(False)

    def e2e_step():
        batch.write_state_async(batch.KINEMATIC, kin.data_ptr(), 16 * batch.total_particles)
        batch.step(p)
        for k, n in nbytes.items():
            if n:
                batch.read_state_async(k, outs[k].data_ptr(), n)
        batch.synchronize()
    e2e_step()
    barrier(world_size)
    torch.cuda.synchronize()
    # events on the batch's stream bracket the copies and the steps; every
    # step ends in a host synchronize, so the span includes the host round trips
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    f1.record(stream)
    f1.synchronize()
    e2e_s = max_over_ranks(f0.elapsed_time(f1) / 1e3, world_size)
    e2e = seg_sub * e2e_steps * world_size / e2e_s

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
    per_launch_s = (ms / 1e3) / args.steps
    flops = FLOPS_PER_SEG_SUBSTEP.get(args.workload, 880.5) * seg_sub
    bytes_alg = BYTES_PER_SEG_STEP * int(wl.segments.sum())
    clk = clocks.summary()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = sms * 128 * 2 * (clk.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
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
        "config": {"workload": wl.name, "rods": len(wl.rods), "segments": int(wl.segments.sum()),
                   "substeps": p.substeps, "dt": p.dt, "strategy": "batched", "tuning": tuning,
                   "graph": True, "l2": "inputs larger than L2" if bytes_alg > 126e6 else "L2-resident state",
                   "parallelism": f"replicas{world_size}"},
        "e2e": {"value": e2e, "unit": "segment-substeps/s", "h2d_bytes_per_step": 16 * batch.total_particles,
                "d2h_bytes_per_step": int(sum(nbytes.values()))},
        "gpu_launches": int(launches),
        "plain": {"value": plain_rate, "unit": "segment-substeps/s",
                  "speedup": (value / world_size / plain_rate) if isinstance(plain_rate, float) else None},
        "roofline": {"bound": "hbm", "achieved": bytes_alg / per_launch_s / 1e9,
                     "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": bytes_alg / per_launch_s / 1e9 / peaks.get("hbm_gbs", 6650.0),
                     "traffic": (DRAM_BYTES_PER_SEG_STEP[args.workload] * int(wl.segments.sum())
                                 if args.workload in DRAM_BYTES_PER_SEG_STEP else None),
                     "note": "of measured; traffic per launch from ncu on 4096 rods scaled by segments; "
                             "the step is FP32-latency bound, see fp32"},
        "fp32": {"achieved": flops / per_launch_s / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
                 "frac": flops / per_launch_s / 1e12 / fp32_peak,
                 "flops_per_segment_substep": FLOPS_PER_SEG_SUBSTEP.get(args.workload, 880.5)},
        "clocks": clk,
    }
    if not args.no_shapes:
        line["shapes"] = measure_shapes(stream, fp32_peak)
    if not args.no_served:
        batch.close()
        line["served"] = run_served(value / world_size, args.served_seconds, args.seed + 7 + rank,
                                    args.served_load, args.served_budget_gb)
    if rank == 0 and world_size == 1 and not args.no_cpu:
        rate, kind, sample, threads = cpu_reference_rate(wl, args.cpu_rods, args.cpu_seconds,
                                                          os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": rate, "unit": "segment-substeps/s", "cores": threads,
                                "kind": kind, "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = build_workload(args.workload, args.rods, seed=args.seed)
    threads = os.cpu_count() or 1
    rates = []
    samples = []
    for _ in range(args.warmup):
        cpu_reference_rate(wl, args.cpu_rods, 1.0, threads)
    for _ in range(max(1, args.steps)):
        r, kind, sample, _ = cpu_reference_rate(wl, args.cpu_rods, args.cpu_seconds / max(1, args.steps),
                                                threads)
        rates.append(r)
        samples.append(sample)
    value = statistics.median(rates)
    line = {"metric": "segment-substeps/s", "value": value, "unit": "segment-substeps/s",
            "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": wl.name, "rods": len(wl.rods), "segments": int(wl.segments.sum()),
                       "substeps": wl.params.substeps, "dt": wl.params.dt,
                       "parallelism": f"replicas{world_size}", "sample": "bounded CPU sample per step"},
            "cpu_baseline": {"value": value, "unit": "segment-substeps/s", "cores": threads,
                             "kind": kind, "sample": samples[-1]},
            "e2e": {"value": value, "unit": "segment-substeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
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
    ap.add_argument("--cpu-rods", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-seconds", type=float, default=20.0)
    ap.add_argument("--served-load", type=float, default=0.7)
    ap.add_argument("--served-budget-gb", type=float, default=150.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
