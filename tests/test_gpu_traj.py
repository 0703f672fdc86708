"""The .rodtraj writer: frames written from device buffers while stepping.

Rods lying on a floor (so world contacts push), stepped and appended frame by
frame; after closing, the file parses as the reference's format
(src/validation/scenes.cpp:13-20) and every frame's positions equal the
batch's downloaded positions at that step, bit for bit (tolerance: exact), and
its contact points are the positions of the particles whose slots pushed. A
file declared longer than written gets its frame count corrected.
"""
import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu


def floor_batch(n_rods=8, segments=24, precision=rp.Precision.REFERENCE):
    rod = rp.Rod.straight(segments, 0.5, W.GRID_MATERIAL, origin=(0.0, 0.0, 0.005), direction=(1.0, 0.0, 0.0))
    world = rp.World([rp.Primitive.plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.6)])
    b = rp.Batch.create(rod, n_rods, rp.Strategy.BATCHED, world)
    b.set_precision(precision)
    return b, rod.num_particles


@pytest.mark.parametrize("precision", [rp.Precision.REFERENCE, rp.Precision.COMPENSATED])
def test_frames_equal_downloads(tmp_path, precision):
    b, nP = floor_batch(precision=precision)
    p = rp.StepParams(dt=1.0 / 60, substeps=10)
    path = tmp_path / "floor.rodtraj"
    t = rp.Trajectory(path, 10, b, radius=W.GRID_MATERIAL.radius, fps=60.0)
    expect_x, expect_c = [], []
    for f in range(4):
        b.step(p)
        t.append(seconds=0.01 * f)
        x = b.download_positions().reshape(8, nP, 3)
        states = b.read_contact_states().reshape(8, nP, 1)
        pushing = (states == rp.ContactState.STICK) | (states == rp.ContactState.SLIP)
        expect_x.append(x)
        expect_c.append(x[pushing[..., 0]])
    assert t.close() == 4
    tr = rp.read_rodtraj(path)
    assert (tr["num_frames"], tr["num_rods"], tr["num_particles"]) == (4, 8, nP)
    assert tr["fps"] == 60.0 and tr["radius"] == np.float32(W.GRID_MATERIAL.radius)
    for f in range(4):
        assert tr["seconds"][f] == np.float32(0.01 * f)
        assert np.array_equal(tr["positions"][f], expect_x[f])
        assert np.array_equal(tr["contacts"][f], expect_c[f])
    assert sum(len(c) for c in tr["contacts"]) > 0  # the floor pushed
    b.close()


def test_rejects_mixed_lengths_and_foreign_batches(tmp_path):
    rods = [rp.Rod.straight(n, 0.3, W.GRID_MATERIAL) for n in (16, 24)]
    mixed = rp.Batch.create_mixed(rods, [], [0, 0], rp.Strategy.BATCHED)
    with pytest.raises(rp.RopeError) as e:
        rp.Trajectory(tmp_path / "m.rodtraj", 1, mixed, 0.005, 60.0)
    assert e.value.status == 1
    a, _ = floor_batch(2, 8)
    b, _ = floor_batch(2, 8)
    t = rp.Trajectory(tmp_path / "a.rodtraj", 1, a, 0.005, 60.0)
    assert rp.lib().rp_traj_append(t._h, b._h, 0.0) == 1
    assert t.close() == 0
    mixed.close()
    a.close()
    b.close()
