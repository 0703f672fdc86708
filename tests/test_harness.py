"""The harness-routing task and its on-device pieces, checked on the CPU.

* The task mirror (ropephysics_b200.harness) equals the reference's
  HarnessTask: schedule length, hand-written motion, and the cable it builds
  (every descriptor double, src/apps/harness_routing.cpp:19-27).
* The waypoint-schedule arithmetic the kernels run (rp_step_common.cuh:
  waypointAt, waypointVelocity), transcribed operation for operation, gives
  the reference's HarnessTask::gripperVelocity bit for bit on random motions
  at every step of the schedule. Python floats are IEEE doubles rounded per
  operation, as the kernel's __d*_rn intrinsics are.
* The evaluation the kernel runs (rp_harness.cu), transcribed with its
  lane-strided partition and warp reductions, equals the reference's
  HarnessTask::evaluate on random and adversarial cables (ties between
  crossings, segments parallel to a peg line, cables above the clip).
"""
import math

import numpy as np
import pytest

from ropephysics_b200 import harness as H
from tests.test_host import _same


# ---- transcriptions of the device code (test-only) ----

def waypoint_at(d, t):
    fx, fy, t0 = d.start[0], d.start[1], 0.0
    for k in range(len(d.waypoints)):
        t1 = t0 + d.legs[k]
        if t < t1:
            u = (t - t0) / d.legs[k]
            u = (u * u) * (3.0 - 2.0 * u)
            return fx + (d.waypoints[k][0] - fx) * u, fy + (d.waypoints[k][1] - fy) * u
        fx, fy, t0 = d.waypoints[k][0], d.waypoints[k][1], t1
    return fx, fy


def waypoint_velocity(d, step):
    period = d.dt * float(d.steps_per_control)
    tick = step // d.steps_per_control
    ax, ay = waypoint_at(d, float(tick + 1) * period)
    bx, by = waypoint_at(d, float(tick) * period)
    inv = 1.0 / period
    return np.float32((ax - bx) * inv), np.float32((ay - by) * inv), np.float32((d.height - d.height) * inv)


def evaluate_like_kernel(xyz, b):
    x = np.asarray(xyz, np.float32).astype(np.float64)
    n = len(x)

    def crossing(px, qx, at):
        if (px - at) * (qx - at) > 0.0:
            return None
        return (at - px) / (qx - px) if abs(qx - px) > 1e-9 else 0.0

    lanes = []
    for lane in range(32):
        va = vb = miss = 1e9
        ia = ib = 2 ** 31 - 1
        sa = sb = 0.0
        for i in range(lane, n - 1, 32):
            p, q = x[i], x[i + 1]
            u = crossing(p[0], q[0], b.peg_a[0])
            if u is not None:
                y = p[1] + (q[1] - p[1]) * u
                if abs(y - b.peg_a[1]) < va:
                    va, ia, sa = abs(y - b.peg_a[1]), i, y - b.peg_a[1]
            u = crossing(p[0], q[0], b.peg_b[0])
            if u is not None:
                y = p[1] + (q[1] - p[1]) * u
                if abs(y - b.peg_b[1]) < vb:
                    vb, ib, sb = abs(y - b.peg_b[1]), i, y - b.peg_b[1]
            u = crossing(p[0], q[0], b.clip[0])
            if u is not None:
                cy = p[1] + (q[1] - p[1]) * u
                cz = p[2] + (q[2] - p[2]) * u
                if not cz > b.clip_height and abs(cy - b.clip[1]) < miss:
                    miss = abs(cy - b.clip[1])
        lanes.append((va, ia, sa, vb, ib, sb, miss))

    def argmin(vals):  # butterfly over 32 lanes, lowest index among equals
        vals = list(vals)
        o = 16
        while o:
            nxt = []
            for l in range(32):
                v, i, s = vals[l]
                ov, oi, os_ = vals[l ^ o]
                nxt.append((ov, oi, os_) if (ov < v or (ov == v and oi < i)) else (v, i, s))
            vals = nxt
            o >>= 1
        return vals[0]

    va, _, sa = argmin([(l[0], l[1], l[2]) for l in lanes])
    vb, _, sb = argmin([(l[3], l[4], l[5]) for l in lanes])
    miss = min(l[6] for l in lanes)
    a = sa if va < 1e9 else 0.0
    bb = sb if vb < 1e9 else 0.0
    reach = (b.peg_radius + b.cable_radius) + b.lay_slack
    below = a < 0.0 and -a <= reach
    above = bb > 0.0 and bb <= reach
    through = miss < b.clip_half_gap

    def clamp01(v):
        m = v if v < 1.0 else 1.0
        return m if 0.0 < m else 0.0

    def peg(off):
        return 0.0 if off <= 0.0 else 1.0 - 0.5 * clamp01((off - reach) / 0.1)

    clip_score = 1.0 if through else clamp01(1.0 - (miss - b.clip_half_gap) / 0.1)
    return dict(score=(peg(-a) + peg(bb)) + clip_score, side_a=a, side_b=bb, clip_miss=miss, below_a=below,
                above_b=above, through_clip=through, success=below and above and through)


# ---- tests ----

def test_task_mirror_equals_reference(reference):
    t = H.HarnessTask()
    assert t.steps() == reference.lib.ref_harness_steps() == 6300
    assert np.array_equal(t.hand_written_policy(), reference.harness_hand_policy())
    for scale in (1.0, 0.4, 3.7):
        h = reference.lib.ref_harness_build(scale)
        try:
            _same(t.build(scale), reference.export(h))
        finally:
            reference.free(h)


def random_policy(rng, t):
    return t.to_policy(t.hand_written_policy().reshape(-1) + 0.08 * rng.standard_normal(10))


def test_schedule_arithmetic_equals_reference_velocity(reference):
    t = H.HarnessTask()
    rng = np.random.default_rng(4)
    steps = list(range(0, 40)) + list(range(2380, 2420)) + list(range(3080, 3120)) + \
        list(range(4500, 4520)) + list(range(5280, 5320)) + [6290, 6299, 6300, 7000]
    for _ in range(12):
        pol = random_policy(rng, t)
        d = t.drive(pol)
        for s in steps:
            ref = reference.harness_velocity(pol, s).astype(np.float32)
            got = np.array(waypoint_velocity(d, s), np.float32)
            assert np.array_equal(got, ref), (s, got, ref)


def test_evaluation_equals_reference(reference):
    t = H.HarnessTask()
    b = t.board()
    rng = np.random.default_rng(9)
    cables = []
    n = t.segments + 1
    s = np.linspace(0.0, 1.0, n)
    for _ in range(40):  # smooth random routes across the board
        k = rng.uniform(-0.12, 0.12, 4)
        y = k[0] * np.sin(math.pi * s * 2) + k[1] * np.sin(math.pi * s * 3) + k[2] * s
        z = np.abs(k[3]) * rng.uniform(0, 1) * np.sin(math.pi * s) + 0.004
        cables.append(np.stack([1.1 * s - 0.05, y, z], 1))
    straight = np.stack([np.zeros(n), -1.2 * s, np.full(n, 0.004)], 1)  # never crosses a peg line
    cables.append(straight)
    zig = np.stack([np.where(np.arange(n) % 2, 0.26, 0.24), np.linspace(-0.1, 0.1, n), np.full(n, 0.004)], 1)
    cables.append(zig)  # many crossings of x = peg A, some at equal distance
    tie = np.stack([np.where(np.arange(n) % 2, 0.26, 0.24), np.full(n, -0.07), np.full(n, 0.004)], 1)
    cables.append(tie)  # every crossing at the same |y - peg|: the earliest segment wins
    vertical = straight.copy()
    vertical[:, 0] = 0.55  # lies along x = peg B: u = 0 branch
    cables.append(vertical)
    high = cables[0].copy()
    high[:, 2] = 0.5  # above the clip everywhere
    cables.append(high)
    for c in cables:
        ref = reference.harness_evaluate(c)
        got = evaluate_like_kernel(c, b)
        for key, v in ref.items():
            assert got[key] == v, (key, got[key], v)
