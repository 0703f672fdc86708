"""Parity with the reference's own FP32 GPU path.

The reference's CUDA batch (src/gpu/gpu_solver.cu + gpu_batch.cpp), compiled
from its sources for sm_100a into oracle/_ref/libcrs_ref_gpu.so, runs the
same scenarios beside this library on the same B200. Positions and frames
must agree within 1e-5 relative to the rod length at the horizons where the
comparison means anything: the reference's float path is itself chaotic at
~1e-4 m after 200 steps (its float-vs-double drift), so beyond ~50 steps any
difference in FMA contraction grows like that drift. The measured errors at
every horizon are printed for the record.
"""
import ctypes

import numpy as np
import pytest

import ropephysics_b200 as rp
from oracle import Params
from tests.helpers import REF_MAT, contact_world, max_dq, max_dx, oracle_world, twisted_root

pytestmark = pytest.mark.gpu

BENCH = rp.StepParams(dt=1e-3, substeps=8, iterations=1)
OPAR = Params(dt=1e-3, substeps=8, iterations=1)
STRATS = (rp.Strategy.MULTI_KERNEL, rp.Strategy.FUSED, rp.Strategy.BATCHED)


def _ref_from(R, orod):
    """A reference Rod handle holding the oracle rod's topology and state."""
    h = R.from_rod(orod)
    rr = R.export(h)
    assert np.array_equal(rr.x, orod.x) and np.array_equal(rr.sComp, orod.sComp)
    return h


def _one_substep(p):
    return rp.StepParams(dt=float(np.float32(p.dt)) / p.substeps, substeps=1, iterations=p.iterations,
                         gravity=p.gravity, linear_damping=p.linear_damping,
                         angular_damping=p.angular_damping)


def test_self_pairs_bit_exact_vs_reference_gpu(reference_gpu, oracle64):
    """Self-contact pair lists -- membership and order -- equal the reference
    FP32 GPU kernel's from identical input state: the coiled rope restart of
    gpu_cases.cpp:437-484 and tightly coiled rods with dozens of contacts,
    at several hash-table sizes, including coils dense enough to overflow the
    pool (equal truncation and equal overflow counts)."""
    R = reference_gpu
    if not R.lib.refgpu_available():
        pytest.skip("no device for the reference GPU path")
    from tests.test_oracle import rope_restart_rod
    from ropephysics_b200 import workloads as W
    cases = []
    rope, world, params, _ = rope_restart_rod(oracle64)
    cases.append((rope, world))
    rng = np.random.default_rng(5)
    from oracle import World as OW, Primitive as OP
    for table in (64, 256, 1024):
        n = int(rng.integers(60, 250))
        pts = W.helix(n, 0.2 * n / 32, float(rng.uniform(0.03, 0.08)), pitch=1.97 * 5e-3)
        o = oracle64.centerline(pts, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
        o.bRestD[:] = 0.0
        cases.append((o, OW([OP.plane((0, 0, pts[:, 2].min() - 0.004), (0, 0, 1), 0.6)],
                            self_collision=True, self_friction=0.4, hash_table_size=table)))
    # denser coils: adjacent turns pressed together, so the contacts exceed
    # the pool's capacity max(16, nSt / 2) and both paths must truncate alike
    for table in (128, 512):
        n = int(rng.integers(120, 220))
        pts = W.helix(n, 0.2 * n / 32, float(rng.uniform(0.02, 0.03)), pitch=1.6 * 5e-3)
        o = oracle64.centerline(pts, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
        o.bRestD[:] = 0.0
        cases.append((o, OW([], self_collision=True, self_friction=0.4, hash_table_size=table)))
    from tests.helpers import product_rod
    total = 0
    overflowed = 0
    for orod, ow in cases:
        h = _ref_from(R, orod)
        wh = R.world(ow)
        rb = R.lib.refgpu_create(h, 1, 0, wh)  # multi-kernel: pool in global memory
        assert rb
        one = _one_substep(rp.StepParams(dt=1e-3, substeps=16, iterations=2))
        g = (ctypes.c_double * 3)(*one.gravity)
        R.lib.refgpu_step(rb, one.dt, 1, one.iterations, g, 0.0, 0.0, 1, 1)
        R.lib.refgpu_sync(rb)
        expect = R.gpu_self_pairs(rb)
        ref_overflow = int(R.lib.refgpu_overflow(rb))
        overflowed += ref_overflow > 0
        pw = rp.World([rp.Primitive(p.type, p.a, p.b, p.normal, p.half_extents, p.rotation,
                                    p.radius, p.friction) for p in ow.primitives],
                      self_collision=True, self_friction=ow.self_friction,
                      hash_table_size=ow.hash_table_size)
        proto = product_rod(orod)
        for s in STRATS:
            b = rp.Batch.create(proto, 1, s, pw)
            b.step(one)
            got = [tuple(int(v) for v in p) for p in b.read_self_contacts(0)]
            assert got == expect, (s, ow.hash_table_size, len(got), len(expect))
            assert b.self_contact_overflow() == ref_overflow, (s, ref_overflow)
            b.close()
        total += len(expect)
        R.lib.refgpu_free(rb)
        R.free(h)
    assert total >= 40
    assert overflowed >= 1  # the truncation path was exercised


def test_contact_active_sets_vs_reference_gpu(reference_gpu, oracle64):
    """World-contact active flags per (particle, primitive) equal the
    reference FP32 GPU kernel's from identical input state, for all four
    primitive types."""
    R = reference_gpu
    if not R.lib.refgpu_available():
        pytest.skip("no device for the reference GPU path")
    from oracle import World as OW, Primitive as OP
    from tests.helpers import product_rod
    n = 120
    t = np.linspace(0, 4 * np.pi, n + 1)
    pts = np.stack([0.1 * np.cos(t), 0.1 * np.sin(t), 0.3 + 0.01 * t], 1)
    o = oracle64.centerline(pts, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
    # each primitive overlaps the coil somewhere (the sphere touches the first
    # particle, the capsule crosses the coil at y = -0.1, the box at y = 0.1)
    prims = [OP.plane((0, 0, 0.3 - 0.003), (0, 0, 1), 0.5), OP.sphere((0.1165, 0.0, 0.3), 0.012, 0.3),
             OP.capsule((-0.2, -0.1, 0.34), (0.2, -0.1, 0.34), 0.006, 0.4),
             OP.box((0.0, 0.1, 0.36), (0.05, 0.004, 0.02), (0.9238795, 0, 0, 0.3826834), 0.6)]
    ow = OW(prims)
    h = _ref_from(R, o)
    rb = R.lib.refgpu_create(h, 1, 0, R.world(ow))
    one = _one_substep(rp.StepParams(dt=1e-3, substeps=8, iterations=1))
    g = (ctypes.c_double * 3)(*one.gravity)
    R.lib.refgpu_step(rb, one.dt, 1, 1, g, 0.0, 0.0, 1, 1)
    R.lib.refgpu_sync(rb)
    expect = R.gpu_contact_active(rb, 0, o.nP, len(prims))
    pw = rp.World([rp.Primitive(p.type, p.a, p.b, p.normal, p.half_extents, p.rotation, p.radius,
                                p.friction) for p in prims])
    for s in STRATS:
        b = rp.Batch.create(product_rod(o), 1, s, pw)
        b.step(one)
        got = (b.read_contact_states().reshape(o.nP, len(prims)) != 0).astype(np.int32)
        assert np.array_equal(got, expect), s
        b.close()
    assert expect.sum(axis=0).min() >= 1  # every primitive type made contact
    R.lib.refgpu_free(rb)
    R.free(h)


def _ref_rod(reference, n):
    h = reference.straight(n, 1.0, **REF_MAT)
    reference.lib.ref_rod_clamp(h, 0)
    return h


@pytest.mark.parametrize("scen", ["gravity", "loaded", "contact"])
@pytest.mark.parametrize("n", [16, 48, 128])
def test_positions_match_reference_gpu(reference_gpu, scen, n):
    R = reference_gpu
    if not R.lib.refgpu_available():
        pytest.skip("no device for the reference GPU path")
    h = _ref_rod(R, n)
    rod = R.export(h)
    root = rod.nS - 1
    rest = rod.q[root].copy()
    if scen == "loaded":
        rod.extForce[rod.nP - 1] = (0.0, 0.02, 0.05)
        rod.extTorque[n // 2] = (2e-3, 0.0, -1e-3)
        rod.kinVel[0] = (0.0, 0.05, 0.1)
        R.import_state(h, rod)
    world = contact_world() if scen == "contact" else None
    wh = R.world(oracle_world(world)) if world else None
    rb = R.lib.refgpu_create(h, 1, 1, wh)
    assert rb, "reference batch could not be created"
    from tests.helpers import product_rod
    proto = product_rod(rod)
    mine = {s: rp.Batch.create(proto, 1, s, world) for s in STRATS}
    g = (ctypes.c_double * 3)(*BENCH.gravity)
    report = {}
    done = 0
    for cp in (1, 10, 50, 200):
        while done < cp:
            if scen == "loaded":
                rod.q[root] = twisted_root(done, rest)
                R.import_state(h, rod)
                R.lib.refgpu_set_loads(rb, 0, h)
                proto.q[root] = rod.q[root]
                for b in mine.values():
                    b.set_loads(0, proto)
            R.lib.refgpu_step(rb, BENCH.dt, BENCH.substeps, BENCH.iterations, g, 0.0, 0.0, 1, 1)
            for b in mine.values():
                b.step(BENCH)
            done += 1
        R.lib.refgpu_sync(rb)
        R.lib.refgpu_download(rb, 0, h)
        ref = R.export(h)
        for s, b in mine.items():
            out = product_rod(ref)
            b.download(0, out)
            dx = max_dx(out.x, ref.x[: ref.nP])
            dq = max_dq(out.q, ref.q[: ref.nS])
            report[(cp, s.name)] = (dx, dq)
        # the reference's download overwrote the host rod's state; restore loads
        rod = R.export(h)
        if scen == "loaded":
            rod.extForce[rod.nP - 1] = (0.0, 0.02, 0.05)
            rod.extTorque[n // 2] = (2e-3, 0.0, -1e-3)
            rod.kinVel[0] = (0.0, 0.05, 0.1)
    print(f"\n{scen} n={n}:", {k: f"dx={v[0]:.2e} dq={v[1]:.2e}" for k, v in report.items()})
    for (cp, s), (dx, dq) in report.items():
        if cp <= 10:
            assert dx / 1.0 <= 1e-5, (cp, s, dx)
            assert dq <= 1e-5, (cp, s, dq)
        assert dx <= 1e-3, (cp, s, dx)
    R.lib.refgpu_free(rb)
    R.free(h)
    for b in mine.values():
        b.close()
