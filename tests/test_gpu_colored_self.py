"""The opt-in coloured self-contact projection (RP_PRECISION_COLORED_SELF).

The reference lists colouring each rod's self contacts as its next GPU
speed-up (REMAINING.md:14-17: the self-contact projection is sequential
within a rod) with one condition: its self-collision parity checks must still
pass within float rounding. Checked here:

* the self-collision restart (gpu_cases.cpp:421-546): one step from the
  coiled restart state in coloured order stays within the reference's
  tolerance of the FP64 CPU solver (3e-5 m, with an effect at least 10x
  larger), as the exact order does;
* on tightly coiled, loaded rods with dozens of contacts each (violent
  motion: the two orders part by centimetres within a step), the coloured
  order is deterministic, and after one step it is about as close to the
  FP64 CPU solver as the exact FP32 order is; it is timed against the exact
  level order;
* the fused strategy ignores the flag (it keeps the reference's serial
  order).
"""

import numpy as np
import pytest

import ropephysics_b200 as rp
from oracle import Context
from tests.helpers import max_dx, oparams, product_rod
from tests.test_oracle import rope_restart_rod

pytestmark = pytest.mark.gpu

COLORED = rp.Precision.COLORED_SELF


def test_colored_restart_within_reference_tolerance(oracle64):
    rope, world, params, g = rope_restart_rod(oracle64)
    proto = product_rod(rope)
    pw = rp.World([rp.Primitive.plane((0, 0, 0), (0, 0, 1), 0.6)], self_collision=True,
                  self_friction=0.3, hash_table_size=256)
    sp = rp.StepParams(dt=1e-3, substeps=16, iterations=4, linear_damping=1.0, angular_damping=1.0)
    cpu = rope.copy()
    oracle64.step(cpu, oparams(sp), world=world, ctx=Context())
    from oracle import World as OW
    nos = rope.copy()
    oracle64.step(nos, oparams(sp), world=OW(world.primitives, False), ctx=Context())
    effect = max_dx(cpu.x, nos.x)
    out = {}
    for flags in (0, COLORED):
        b = rp.Batch.create(proto, 1, rp.Strategy.BATCHED, pw)
        b.set_precision(int(flags))
        b.step(sp)
        r = product_rod(rope)
        b.download(0, r)
        out[flags] = r.x.copy()
        assert b.self_contact_overflow() == 0
        b.close()
    err_exact = max_dx(out[0], cpu.x)
    err_col = max_dx(out[COLORED], cpu.x)
    print(f"\nrestart, one step vs FP64 CPU: exact order {err_exact:.2e} m, coloured {err_col:.2e} m, "
          f"effect of self-collision {effect:.2e} m")
    assert err_col <= 3e-5
    assert effect / 3e-5 >= 10


def coiled(count, seed=11):
    from ropephysics_b200 import workloads as W
    rng = np.random.default_rng(seed)
    rods, worlds = [], []
    mat = rp.Material(1e8, 0.3, 1100.0, 5e-3)
    for _ in range(count):
        n = int(rng.integers(40, 260))
        pts = W.helix(n, 0.2 * n / 32, float(rng.uniform(0.03, 0.08)), pitch=1.97 * mat.radius)
        r = rp.Rod.centerline(pts, mat)
        r.b_rest_darboux[:] = 0.0
        rods.append(r)
        lo = pts.min(0)
        worlds.append(rp.World([rp.Primitive.plane((0, 0, lo[2] - 0.004), (0, 0, 1), 0.6)],
                               self_collision=True, self_friction=0.4, hash_table_size=W.table_for(n)))
    return rods, worlds


def test_colored_on_contact_heavy_coils(oracle64):
    from oracle import Context as Ctx
    from tests.helpers import oracle_world
    from ropephysics_b200 import workloads as W
    rods, worlds = coiled(64)
    p = rp.StepParams(dt=1.0 / 60, substeps=20, iterations=2)
    out = {}
    for key, flags in (("exact", 0), ("colored", COLORED), ("colored2", COLORED)):
        b = rp.Batch.create_mixed(rods, worlds, list(range(len(rods))), rp.Strategy.BATCHED)
        b.set_precision(int(flags))
        b.step(p)
        first = b.download_positions()
        pools = [len(b.read_self_contacts(i)) for i in range(len(rods))]
        for _ in range(3):
            b.step(p)
        out[key] = (first, b.download_positions(), pools)
        assert b.error_count() == 0
        b.close()
    assert np.array_equal(out["colored"][1], out["colored2"][1])  # deterministic
    assert max(out["exact"][2]) >= 10
    assert np.all(np.isfinite(out["colored"][1]))
    # one step of the first 8 rods on the FP64 CPU solver
    off = np.concatenate([[0], np.cumsum([r.num_particles for r in rods])])
    err = {"exact": 0.0, "colored": 0.0}
    for i in range(8):
        o = oracle64.centerline(np.asarray(rods[i].x, np.float64), youngs=1e8, poisson=0.3, density=1100.0,
                                radius=5e-3, frame_seed=(0, 0, 1))
        o.bRestD[:] = 0.0
        oracle64.step(o, oparams(p), world=oracle_world(worlds[i]), ctx=Ctx())
        for key in err:
            err[key] = max(err[key], max_dx(out[key][0][off[i]:off[i + 1]], o.x[: o.nP]))
    d1 = float(np.max(np.abs(out["colored"][0] - out["exact"][0])))
    print(f"\ncoils: contacts per rod up to {max(out['exact'][2])}; coloured vs exact order after 1 step "
          f"{d1:.2e} m; vs FP64 CPU after 1 step (8 rods): exact {err['exact']:.2e} m, coloured "
          f"{err['colored']:.2e} m")
    assert err["colored"] <= 5 * err["exact"] + 1e-3


def test_colored_speed_on_coils():
    import torch
    rods, worlds = coiled(2048, seed=3)
    p = rp.StepParams(dt=1.0 / 60, substeps=20, iterations=2)
    s = torch.cuda.Stream()
    ms = {}
    for key, flags in (("exact", 0), ("colored", COLORED)):
        b = rp.Batch.create_mixed(rods, worlds, list(range(len(rods))), rp.Strategy.BATCHED)
        b.set_precision(int(flags))
        b.set_stream(s.cuda_stream)
        b.set_graph(True)
        b.step_many(p, 3)
        b.step_many(p, 10)
        b.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        b.step_many(p, 10)
        e1.record(s)
        e1.synchronize()
        ms[key] = e0.elapsed_time(e1) / 10
        b.close()
    print(f"\n2048 tightly coiled rods: exact level order {ms['exact']:.3f} ms per step, coloured "
          f"{ms['colored']:.3f} ms ({ms['exact'] / ms['colored']:.2f}x)")
    assert ms["colored"] < 1.2 * ms["exact"]


def test_fused_ignores_the_flag():
    rods, worlds = coiled(8, seed=5)
    p = rp.StepParams(dt=1.0 / 60, substeps=20, iterations=2)
    xs = []
    for flags in (0, COLORED):
        b = rp.Batch.create_mixed(rods, worlds, list(range(len(rods))), rp.Strategy.FUSED)
        b.set_precision(int(flags))
        for _ in range(2):
            b.step(p)
        xs.append(b.download_positions())
        b.close()
    assert np.array_equal(xs[0], xs[1])
