"""The oracle is pinned before it is trusted (CPU only).

1. Against the reference's published golden vector docs/data/crosscheck.csv,
   reproduced here as tests/golden/crosscheck.csv: byte for byte.
2. Against the reference compiled from its sources (oracle/_ref): builders,
   colourings, self-collision index gaps, contact lists and whole trajectories
   with world contacts and self-collision, bit for bit.
3. Against the other committed fixtures (colourings, parity trajectories, the
   coiled-rope restart state), which the reference itself produced.
"""
import math
import os

import numpy as np
import pytest

from oracle import Context, Params, Primitive, World
from tests.helpers import REF_MAT, benchmark_rod

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
# the reference's source tree: $RP_REFERENCE, else a checkout beside the repo
REFERENCE = os.environ.get("RP_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(
    os.path.dirname(os.path.abspath(__file__)))), "reference"))


def _fmt(v):
    return "%.12g" % v


def test_crosscheck_golden_byte_exact(oracle64):
    """runCrossCheck (src/validation/cases.cpp:772-806) vs the published CSV."""
    rod = oracle64.straight(16, 1.0, **REF_MAT)
    oracle64.clamp(rod, False)
    oracle64.step(rod, Params(dt=1e-3, substeps=4, iterations=1), colored=False, steps=200)
    lines = ["index,x,y,z,qw,qx,qy,qz"]
    for i in range(rod.nP):
        q = rod.q[i] if i < rod.nS else (1.0, 0.0, 0.0, 0.0)
        lines.append(",".join([str(i)] + [_fmt(v) for v in list(rod.x[i]) + list(q)]))
    golden = open(os.path.join(GOLDEN, "crosscheck.csv")).read().splitlines()
    assert lines == golden


def test_golden_matches_published_reference_data():
    """The fixture equals the reference's own docs/data/crosscheck.csv."""
    pub = os.path.join(REFERENCE, "docs", "data", "crosscheck.csv")
    if not os.path.exists(pub):
        pytest.skip("reference tree not present")
    assert open(pub).read().split() == open(os.path.join(GOLDEN, "crosscheck.csv")).read().split()


@pytest.mark.parametrize("n", [8, 32, 128, 512])
def test_coloring_golden(oracle64, n):
    """2 + 2 colours, order colour-major then index (docs/data/coloring.csv)."""
    g = np.load(os.path.join(GOLDEN, "coloring.npz"))
    rod = benchmark_rod(oracle64, n)
    for bend in (False, True):
        c = oracle64.coloring(rod, bend)
        key = f"{'bend' if bend else 'stretch'}_{n}"
        assert np.array_equal(c.order, g[key + "_order"])
        assert np.array_equal(c.color_start, g[key + "_start"])
        assert c.num_colors == 2


def test_parity_trajectories_golden(oracle64):
    """Colour-ordered FP64 trajectories equal the reference's, bit for bit."""
    from tests.helpers import contact_world, oracle_world, twist_root
    g = np.load(os.path.join(GOLDEN, "parity_cpu.npz"))
    p = Params(dt=1e-3, substeps=8, iterations=1)
    world = oracle_world(contact_world())
    for scen in ("gravity", "loaded", "contact"):
        for n in (16, 48):
            rod = benchmark_rod(oracle64, n)
            root = rod.nS - 1
            rest = rod.q[root].copy()
            if scen == "loaded":
                rod.extForce[rod.nP - 1] = (0.0, 0.02, 0.05)
                rod.extTorque[n // 2] = (2e-3, 0.0, -1e-3)
                rod.kinVel[0] = (0.0, 0.05, 0.1)
            ctx = Context()
            done = 0
            for cp in (1, 10, 50):
                while done < cp:
                    if scen == "loaded":
                        twist_root(rod, root, rest, done)
                    oracle64.step(rod, p, world=world if scen == "contact" else None, ctx=ctx)
                    done += 1
                assert np.array_equal(rod.x[: rod.nP], g[f"{scen}_{n}_{cp}_x"]), (scen, n, cp)
                assert np.array_equal(rod.q[: rod.nS], g[f"{scen}_{n}_{cp}_q"]), (scen, n, cp)


def rope_restart_rod(oracle):
    """The coiled rope of gpu_cases.cpp:437-484 at its committed restart state."""
    g = np.load(os.path.join(GOLDEN, "rope_restart.npz"))
    d = [0.08, 0.03, 1.0]
    s = 1.0 / math.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
    rope = oracle.straight(150, 1.2, youngs=2e6, poisson=0.35, density=1000.0, radius=5e-3,
                           origin=(0, 0, 0.02), direction=[c * s for c in d])
    rope.x[:, 2] = 1.2 + 0.05 - rope.x[:, 2]
    rope.xPrev[...] = rope.x
    oracle.set_rest_from_current(rope)
    assert np.array_equal(rope.sRest[: rope.nSt], g["s_rest"])
    assert np.array_equal(rope.bRestD[: rope.nB], g["b_rest_darboux"])
    rope.x[: rope.nP] = g["x"]
    rope.v[: rope.nP] = g["v"]
    rope.q[: rope.nS] = g["q"]
    rope.omega[: rope.nS] = g["omega"]
    world = World([Primitive.plane((0, 0, 0), (0, 0, 1), 0.6)], self_collision=True,
                  self_friction=0.3, hash_table_size=256)
    params = Params(dt=1e-3, substeps=16, iterations=4, linear_damping=1.0, angular_damping=1.0)
    return rope, world, params, g


def test_rope_restart_golden(oracle64):
    """Self-collision contact list and one step from the restart, bit for bit."""
    rope, world, params, g = rope_restart_rod(oracle64)
    ctx = oracle64.generate_contacts(rope, world)
    cs = ctx.contacts()
    assert len(cs) == len(g["contact_idx"])
    for c, idx in zip(cs, g["contact_idx"]):
        assert c["idx"] == tuple(int(i) for i in idx[: c["count"]])
    assert sum(c["count"] == 4 for c in cs) >= 5
    oracle64.step(rope, params, world=world, ctx=Context())
    assert np.array_equal(rope.x[: rope.nP], g["x1"])
    assert np.array_equal(rope.q[: rope.nS], g["q1"])


# ---- live comparisons with the reference built from source (skips if absent) ----

@pytest.mark.parametrize("n", [4, 16, 63, 150])
def test_builders_match_reference(oracle64, reference, n):
    fields = ("x", "q", "invMass", "mass", "inertia", "invInertia", "sRest", "sComp", "bRest",
              "bComp", "bRestD", "bA", "bB", "sP0", "sP1", "sSeg")
    for tip in (False, True):
        rod = oracle64.straight(n, 0.7, **REF_MAT, direction=(0.3, -0.2, 0.9))
        oracle64.clamp(rod, tip)
        h = reference.straight(n, 0.7, **REF_MAT, direction=(0.3, -0.2, 0.9))
        reference.lib.ref_rod_clamp(h, int(tip))
        rr = reference.export(h)
        for f in fields:
            assert np.array_equal(getattr(rod, f), getattr(rr, f)), f
        reference.free(h)
    t = np.linspace(0, 3 * math.pi, n + 1)
    pts = np.stack([0.1 * np.cos(t), 0.1 * np.sin(t), 0.02 * t], 1)
    rod = oracle64.centerline(pts, **REF_MAT, frame_seed=(0, 1, 0), twist_per_length=0.7)
    h = reference.centerline(pts, **REF_MAT, frame_seed=(0, 1, 0), twist_per_length=0.7)
    rr = reference.export(h)
    for f in fields:
        assert np.array_equal(getattr(rod, f), getattr(rr, f)), f
    reference.free(h)


def test_world_and_self_trajectory_match_reference(oracle64, reference):
    """All four primitive types plus self-collision, 300 coloured steps."""
    n = 120
    t = np.linspace(0, 6 * math.pi, n + 1)
    pts = np.stack([0.08 * np.cos(t), 0.08 * np.sin(t), 0.3 + 0.012 * t], 1)
    rod = oracle64.centerline(pts, youngs=2e6, radius=5e-3)
    rod.bRestD[:] = 0.0
    h = reference.centerline(pts, youngs=2e6, radius=5e-3)
    rr = reference.export(h)
    rr.bRestD[:] = 0.0
    reference.import_state(h, rr)
    w = World([Primitive.plane((0, 0, 0), (0, 0, 1), 0.6),
               Primitive.sphere((0.05, 0, 0.15), 0.05, 0.3),
               Primitive.capsule((-0.1, -0.2, 0.2), (-0.1, 0.2, 0.2), 0.02, 0.4),
               Primitive.box((0.0, 0.08, 0.25), (0.05, 0.02, 0.04), (0.9238795, 0, 0.3826834, 0), 0.5)],
              self_collision=True, self_friction=0.3, hash_table_size=256)
    wh = reference.world(w)
    assert oracle64.self_gap(rod, w) == reference.lib.ref_self_gap(h, wh)
    p = Params(dt=1e-3, substeps=16, iterations=2, linear_damping=1, angular_damping=1)
    ctx = Context()
    for _ in range(300):
        oracle64.step(rod, p, world=w, ctx=ctx)
        reference.step(h, p, world_handle=wh)
    rr = reference.export(h)
    assert np.array_equal(rod.x, rr.x) and np.array_equal(rod.q, rr.q)
    assert sum(c["count"] == 4 for c in ctx.contacts()) >= 1
    ci, cw, cn, co = reference.contacts(h)
    ours = ctx.contacts()
    assert len(ours) == len(ci)
    for c, idx, off in zip(ours, ci, co):
        assert c["idx"] == tuple(int(i) for i in idx[: c["count"]])
        assert c["offset"] == off


def test_float_oracle_tracks_double(oracle64, oracle32):
    """The float build (the reference's CRS_REAL_FLOAT tie-breaker) stays within
    the reference's documented float envelope: 5e-9 m after 1 step and at most
    ~3e-4 m after 200 (src/gpu/gpu_cases.cpp:137-147)."""
    for n in (16, 48):
        rd = benchmark_rod(oracle64, n)
        rf = benchmark_rod(oracle32, n)
        p = Params(dt=1e-3, substeps=8, iterations=1)
        oracle64.step(rd, p, steps=1)
        oracle32.step(rf, p, steps=1)
        assert np.max(np.abs(rd.x - rf.x)) < 1e-7  # gpu_cases.cpp:285
        oracle64.step(rd, p, steps=199)
        oracle32.step(rf, p, steps=199)
        assert np.max(np.abs(rd.x - rf.x)) < 1e-3


def test_op_count_oracle_reproduces_double():
    """The op-counting build computes the same numbers as the double build."""
    from oracle import Oracle
    oc, od = Oracle("count"), Oracle("f64")
    a, b = benchmark_rod(oc, 16), benchmark_rod(od, 16)
    p = Params(dt=1e-3, substeps=8, iterations=1)
    oc.op_reset()
    oc.step(a, p, steps=3)
    od.step(b, p, steps=3)
    assert np.array_equal(a.x, b.x)
    ops = oc.op_counts()
    assert ops["add"] > 0 and ops["mul"] > 0 and ops["div"] > 0 and ops["sqrt"] > 0


def test_flops_per_segment_substep_match_bench():
    """The bench's algorithmic FLOPs per segment-substep (add, sub, mul, div,
    sqrt) are the op-counting oracle's count for a pinned 64-segment rod at
    dt 1/60 with 20 substeps, free (the cantilever) and with a floor plane
    (the grid)."""
    import bench
    from oracle import Context, Oracle, Primitive as OP, World as OW
    oc = Oracle("count")
    p = Params(dt=1 / 60, substeps=20, iterations=1)

    def per_seg_substep(world):
        r = oc.straight(64, 1.0, youngs=1e8, poisson=0.3, density=1100, radius=5e-3, direction=(0, 0, -1))
        oc.pin(r, 0)
        ctx = Context(dtype=np.float64) if world else None
        oc.step(r, p, world=world, ctx=ctx, steps=1)
        oc.op_reset()
        oc.step(r, p, world=world, ctx=ctx, steps=1)
        c = oc.op_counts()
        return sum(c[k] for k in ("add", "mul", "div", "sqrt")) / (64 * 20)

    # the bench quotes them to one decimal
    assert per_seg_substep(None) == pytest.approx(bench.FLOPS_PER_SEG_SUBSTEP["cantilever"], abs=0.05)
    floor = OW([OP.plane((0, 0, -1.2), (0, 0, 1), 0.5)])
    assert per_seg_substep(floor) == pytest.approx(bench.FLOPS_PER_SEG_SUBSTEP["grid"], abs=0.05)


def _counted_window(oc, rods, params, skip, count):
    """FLOPs per segment-substep of `count` steps after `skip` steps of the
    (rod, world, context, segments) tuples."""
    for r, w, ctx, _ in rods:
        oc.step(r, params, world=w, ctx=ctx, steps=skip)
    oc.op_reset()
    for r, w, ctx, _ in rods:
        oc.step(r, params, world=w, ctx=ctx, steps=count)
    c = oc.op_counts()
    segs = sum(s for *_, s in rods)
    return sum(c[k] for k in ("add", "mul", "div", "sqrt")) / (segs * params.substeps * count)


def test_flops_per_segment_substep_uneven_batch():
    """The uneven batch's count includes its contacts and self-collision:
    32 rods sampled as the bench's CPU leg samples them (seed 123) from the
    seed-0 draws, built by the oracle's builders, counted over steps 25-44."""
    import bench
    from oracle import Context, Oracle, Primitive as OP, World as OW
    from ropephysics_b200 import synth
    oc = Oracle("count")
    draws = synth.uneven(16384, 0)
    idx = np.random.default_rng(123).choice(len(draws), size=32, replace=False)
    f32 = lambda v: float(np.float32(v))
    p = Params(dt=f32(1 / 60), substeps=50, iterations=1, gravity=(0.0, 0.0, f32(-9.81)))
    rods = []
    for i in idx:
        d = draws[i]
        r = oc.centerline(d.points, youngs=synth.YOUNGS, poisson=synth.POISSON, density=synth.DENSITY,
                          radius=synth.RADIUS, frame_seed=(0, 0, 1))
        r.bRestD[:] = 0.0
        w = OW([OP(*q) for q in d.prims], True, d.friction, 2, d.hash_table_size, 0.25)
        rods.append((r, w, Context(dtype=np.float64), d.segments))
    assert _counted_window(oc, rods, p, 25, 20) == pytest.approx(bench.FLOPS_PER_SEG_SUBSTEP["uneven"],
                                                                 abs=0.05)


def test_flops_per_segment_substep_hook_sweep():
    """The hook sweep's count: 16 placements spread over the sweep (leg ratio,
    friction, stiffness), on the bar and floor with self-collision, counted
    over steps 23-42 (the window the bench's shape timing measures)."""
    import bench
    from oracle import Context, Oracle, Primitive as OP, World as OW
    from ropephysics_b200 import workloads as W
    oc = Oracle("count")
    f32 = lambda v: float(np.float32(v))
    p = Params(dt=f32(1 / 60), substeps=20, iterations=1, gravity=(0.0, 0.0, f32(-9.81)))
    rods = []
    for k in range(16):
        ratio, mu, youngs = 1.0 + 3.0 * k / 15, 0.05 + 0.55 * ((7 * k) % 16) / 15, (1e8, 3e8)[k % 2]
        r = oc.centerline(W.hanging_cable_points(ratio), youngs=youngs, frame_seed=(0, 1, 0),
                          **W.HOOK_MATERIAL)
        r.bRestD[:] = 0.0
        w = OW([OP.capsule((0.0, -0.3, 0.8), (0.0, 0.3, 0.8), 0.02, mu), OP.plane((0, 0, W.HOOK_FLOOR_Z), (0, 0, 1), mu)],
               True, mu, 2, 256, 0.25)
        rods.append((r, w, Context(dtype=np.float64), 120))
    assert _counted_window(oc, rods, p, 23, 20) == pytest.approx(bench.FLOPS_PER_SEG_SUBSTEP["hook"], abs=0.05)
