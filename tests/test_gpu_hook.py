"""Hook sweep: hold/slide verdicts of 3600 draped cables against the FP64 CPU.

3600 cables of 120 segments (1.2 m, r 4 mm) draped over a capsule bar
(r 2 cm) at 60 leg ratios 1:1..4:1 x 30 friction values in [0.05, 0.6] x 2
stiffnesses (1e8, 3e8 Pa), floor, self-collision, 8 s at dt 1/60 with 20
substeps, run as one batched launch per step with compensated positions, the
FP64 friction-cone test and FP64 verdicts. The verdict is the reference's
HangOutcome (apps/cable_hanging.h:68-77): the short end is sampled every 3
steps (50 ms) and at the end; held <=> max rise <= 0.05 m.

The 200 placements nearest the capstan boundary mu = ln(ratio) / pi are
re-run on the reference's own FP64 CPU solver (compiled from its sources,
colour-ordered, observed by its own HangOutcome). These are the placements
where single precision is known to flip verdicts; the agreement is asserted
and printed for both this library's mixed-precision mode and its
reference-order FP32 mode.
"""
import math
import os

import numpy as np
import pytest

import ropephysics_b200 as rp
from oracle import Params, Primitive as OP, World as OW
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS, INTERVAL = 480, 3


def gpu_verdicts(wl, precision):
    b = wl.make_batch(rp.Strategy.BATCHED)
    b.set_precision(precision)
    b.arm_hold_observer([0] * len(wl.rods), interval=INTERVAL, tolerance=0.05)
    b.set_graph(True)
    b.step_many(wl.params, STEPS)
    rise, held, near = b.read_hold_verdicts()
    assert b.error_count() == 0
    b.close()
    return rise, held, near


def test_hook_sweep_verdicts_vs_fp64_cpu(reference):
    wl = W.hook()
    assert len(wl.rods) == 3600
    ratios = np.array(wl.info["ratios"])
    mus = np.array(wl.info["frictions"])
    Es = wl.info["stiffnesses"]
    # rod index = (e * 30 + m) * 60 + i
    idx = np.arange(3600)
    e_i, m_i, r_i = idx // 1800, (idx // 60) % 30, idx % 60
    boundary = np.abs(mus[m_i] - np.log(ratios[r_i]) / math.pi)
    nearest = np.argsort(boundary, kind="stable")[:200]

    mixed = rp.Precision.COMPENSATED | rp.Precision.FP64_CONE | rp.Precision.FP64_VERDICT
    rise_m, held_m, near_m = gpu_verdicts(wl, mixed)
    rise_f, held_f, _ = gpu_verdicts(wl, rp.Precision.REFERENCE)

    handles, worlds = [], []
    for r in nearest:
        mu = float(mus[m_i[r]])
        handles.append(reference.hanging(float(ratios[r_i[r]]), float(Es[e_i[r]]), length=1.2,
                                         segments=120, bar_radius=0.02, bar_height=0.8))
        # the reference's drape builder (straight rest shape) at the sweep's
        # geometry; the product builds the same doubles (host tests)
        worlds.append(reference.world(OW([OP.capsule((0, -0.3, 0.8), (0, 0.3, 0.8), 0.02, mu),
                                          OP.plane((0, 0, 0), (0, 0, 1), mu)],
                                         self_collision=True, self_friction=mu, hash_table_size=256)))
    p = Params(dt=float(np.float32(1.0 / 60)), substeps=20, iterations=1,
               gravity=(0.0, 0.0, float(np.float32(-9.81))))
    rise_c, held_c = reference.hold_many(handles, worlds, p, STEPS, INTERVAL, os.cpu_count() or 1)
    for h in handles:
        reference.free(h)
    agree_m = int(np.sum(held_m[nearest] == held_c))
    agree_f = int(np.sum(held_f[nearest] == held_c))
    print(f"\nhook sweep: held {held_m.sum()}/3600 (mixed) {held_f.sum()}/3600 (FP32); "
          f"200 nearest the capstan boundary: mixed agrees {agree_m}/200, FP32 {agree_f}/200, "
          f"near-boundary flags {int(near_m[nearest].sum())}")
    assert agree_m >= 180
    # the sweep is not degenerate: both outcomes occur
    assert 0 < held_m.sum() < 3600
