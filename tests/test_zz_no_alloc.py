"""rp_batch_step_static_scratch: the batched step with its scratch in a fixed
static device array, allocating nothing.

Two identical batches are stepped side by side, one by rp_batch_step and one
by rp_batch_step_static_scratch, called through the C ABI; after each of two
calls in a row the positions, frames and contact states must agree within
the tolerance stated here: exact (0), since the kernel and its arithmetic are
the same and only the scratch addresses differ. A batch whose scratch exceeds
RP_STATIC_SCRATCH_BYTES is rejected with a message, and nothing is launched.
The file is named to be collected last, and the tests also pass alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu

STATIC_SCRATCH_BYTES = 32 << 20
TOL = 0.0


def static_step(batch, params):
    p = params.to_c()
    return rp.lib().rp_batch_step_static_scratch(batch._h, C.byref(p))


def test_static_scratch_step_equals_step_twice():
    wl = W.uneven(24, seed=3)
    assert any(w.self_collision for w in wl.worlds) and any(len(w.primitives) for w in wl.worlds)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    for call in range(2):
        a.step(wl.params)
        assert static_step(b, wl.params) == 0, rp.lib().rp_last_error()
        a.synchronize()
        b.synchronize()
        xa, xb = a.download_positions(), b.download_positions()
        qa, qb = a.download_frames(), b.download_frames()
        assert np.all(np.isfinite(xb))
        assert np.max(np.abs(xa - xb)) <= TOL, call
        assert np.max(np.abs(qa - qb)) <= TOL, call
        assert np.array_equal(a.read_contact_states(), b.read_contact_states()), call
    assert b.error_count() == 0
    a.close()
    b.close()


def test_static_scratch_rejects_oversized_batch():
    # 512 rods x 512 segments x 4 primitives: 16 B x 262144 frames + 32 B x
    # 1050624 contact slots = 37.8 MB of scratch > 32 MiB
    rod = rp.Rod.straight(512, 1.0, W.GRID_MATERIAL)
    prims = [rp.Primitive.plane((0, 0, -2), (0, 0, 1), 0.5),
             rp.Primitive.sphere((0.5, 0, 0.3), 0.1, 0.5),
             rp.Primitive.capsule((0, -0.2, 0.2), (0, 0.2, 0.2), 0.02, 0.5),
             rp.Primitive.box((0.8, 0, 0), (0.1, 0.1, 0.1), (1, 0, 0, 0), 0.5)]
    batch = rp.Batch.create_mixed([rod] * 512, [rp.World(prims)], [0] * 512, rp.Strategy.BATCHED)
    before = batch.kernel_launches
    st = static_step(batch, rp.StepParams(dt=1.0 / 60, substeps=4))
    msg = rp.lib().rp_last_error().decode()
    assert st == 1  # RP_ERR_INVALID
    assert str(STATIC_SCRATCH_BYTES) in msg and "rp_batch_step" in msg
    assert batch.kernel_launches == before
    batch.close()


def test_static_scratch_needs_batched_strategy():
    rod = rp.Rod.straight(32, 0.5, W.GRID_MATERIAL)
    batch = rp.Batch.create(rod, 2, rp.Strategy.FUSED)
    assert static_step(batch, rp.StepParams()) == 1
    batch.close()
