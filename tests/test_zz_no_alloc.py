"""rp_batch_step_static_scratch: the batched step with its scratch in a fixed
static device array, allocating nothing.

Two identical batches are stepped side by side, one by rp_batch_step and one
by rp_batch_step_static_scratch, called through the C ABI; after each of two
calls in a row the positions, frames and contact states must agree within
the tolerance stated here: exact (0), since the kernel and its arithmetic are
the same and only the scratch addresses differ. The cases cover every
section of the array: reference precision (start-of-substep frames in shared
memory) and compensated precision (those frames in the array), a mixed batch
whose contact slots fit in shared memory and one of long rods with four
primitives each, whose slots live in the array, both with self-collision on
(the self-contact pool in the array). A batch whose scratch exceeds
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


def long_rods_four_primitives(count=6, segments=500):
    """Coiled rods of 500 segments over a floor, each beside a sphere, a
    capsule and a box: 32 B x 501 particles x 4 primitives = 64 KB of contact
    slots per rod, which the plan leaves in global memory."""
    rods, worlds = [], []
    for i in range(count):
        pts = W.helix(segments, 0.2 * segments / 32, 0.08 + 0.01 * i, 4.0 * W.GRID_MATERIAL.radius)
        rod = rp.Rod.centerline(pts, W.GRID_MATERIAL)
        rod.b_rest_darboux[:] = 0.0
        rods.append(rod)
        top = float(pts[:, 2].max())
        worlds.append(rp.World([rp.Primitive.plane((0, 0, -0.006), (0, 0, 1), 0.5),
                                rp.Primitive.sphere((0.0, 0.0, top + 0.06), 0.05, 0.4),
                                rp.Primitive.capsule((-0.3, 0.0, 0.3), (0.3, 0.0, 0.3), 0.02, 0.6),
                                rp.Primitive.box((0.25, 0.0, 0.5), (0.05, 0.05, 0.05), (1, 0, 0, 0), 0.3)],
                               self_collision=True, self_friction=0.4, hash_table_size=W.table_for(segments)))
    return W.Workload("long4", rods, worlds, list(range(count)), rp.StepParams(dt=1.0 / 60, substeps=20))


MIXED = int(rp.Precision.COMPENSATED | rp.Precision.FP64_CONE)


@pytest.mark.parametrize("precision", [0, MIXED], ids=["reference", "compensated"])
@pytest.mark.parametrize("shape", ["uneven24", "long4"])
def test_static_scratch_step_equals_step_twice(shape, precision):
    wl = W.uneven(24, seed=3) if shape == "uneven24" else long_rods_four_primitives()
    assert any(w.self_collision for w in wl.worlds) and any(len(w.primitives) for w in wl.worlds)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    a.set_precision(precision)
    b.set_precision(precision)
    if shape == "long4":
        # one 500-segment rod per CTA; with its 64 KB of slots the group would
        # need well over 140 KB, so the plan keeps them in global memory
        assert b.shared_bytes_per_block < 140_000
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
        if shape == "long4":
            assert np.any(a.read_contact_states() >= 2), "the floor must push"
    assert b.error_count() == 0
    a.close()
    b.close()


def test_static_scratch_rejects_oversized_batch():
    # 640 rods x 513 particles x 8 primitives x 32 B = 84.0 MB of contact
    # slots in global memory (with them in shared memory a 512-segment rod's
    # group would fit one CTA per SM instead of two) > 32 MiB
    rod = rp.Rod.straight(512, 1.0, W.GRID_MATERIAL)
    prims = [rp.Primitive.plane((0, 0, -2), (0, 0, 1), 0.5)]
    for k in range(7):
        prims.append(rp.Primitive.sphere((0.5, 0.1 * k, 0.3), 0.1, 0.5))
    batch = rp.Batch.create_mixed([rod] * 640, [rp.World(prims)], [0] * 640, rp.Strategy.BATCHED)
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
