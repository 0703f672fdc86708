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
