"""Edge cases of size: the shortest rods, the longest, the most primitives.

* Rods of 2, 3 and 4 segments (the fewest the builders accept; no self pair beyond the
  index gap) with self-collision and a floor on: every strategy gives the same
  state bit for bit, and the FP64 oracle agrees to 1e-5 of the rod length
  after a few steps.
* A 3000-segment rod fits the batched kernel's shared memory and steps
  bitwise equal to the multi-kernel strategy; a 4000-segment rod exceeds it:
  the batched strategy refuses it with RP_ERR_SHARED_MEMORY and a message, the
  multi-kernel strategy (state in global memory) steps it and agrees with the
  FP64 oracle.
* A world with 64 primitives (the maximum) steps identically under every
  strategy.
* A precision change whose layout no longer fits is refused and leaves the
  batch's plan untouched.
"""
import numpy as np
import pytest

import ropephysics_b200 as rp
from oracle import Params, Primitive as OP, World as OW
from ropephysics_b200 import workloads as W
from tests.helpers import max_dx, product_rod

pytestmark = pytest.mark.gpu

STRATS = (rp.Strategy.MULTI_KERNEL, rp.Strategy.FUSED, rp.Strategy.BATCHED)
P = rp.StepParams(dt=1e-3, substeps=8, iterations=1)
OPAR = Params(dt=float(np.float32(1e-3)), substeps=8, iterations=1, gravity=(0.0, 0.0, float(np.float32(-9.81))))


def run_all(proto, world, steps, n=3):
    out = {}
    for s in STRATS:
        b = rp.Batch.create(proto, n, s, world)
        b.step_many(P, steps)
        out[s] = (b.download_positions(), b.download_frames())
        b.close()
    return out


@pytest.mark.parametrize("segments", [2, 3, 4])
def test_shortest_rods(oracle64, segments):
    o = oracle64.straight(segments, 0.02 * segments, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3,
                          origin=(0, 0, 0.004), direction=(1, 0, 0))
    ow = OW([OP.plane((0, 0, 0), (0, 0, 1), 0.5)], self_collision=True, self_friction=0.3, hash_table_size=64)
    world = rp.World([rp.Primitive.plane((0, 0, 0), (0, 0, 1), 0.5)], self_collision=True, self_friction=0.3,
                     hash_table_size=64)
    res = run_all(product_rod(o), world, 5)
    ref = res[rp.Strategy.MULTI_KERNEL]
    for s in STRATS:
        assert np.array_equal(res[s][0], ref[0]) and np.array_equal(res[s][1], ref[1]), s
        assert np.all(np.isfinite(res[s][0]))
    oracle64.step(o, OPAR, world=ow, steps=5)
    got = ref[0].reshape(3, -1, 3)[0]
    assert np.max(np.abs(got - o.x[: o.nP])) <= 1e-5 * 0.02 * segments + 1e-7


def test_longest_rods(oracle64):
    # 3000 segments: the batched kernel's lean layout (positions and frames
    # with their start-of-substep copies, 64 bytes a segment without
    # self-collision) fits one CTA's shared memory; its 256-thread team
    # projects several constraints of a colour per lane, in pairs
    n = 3000
    o = oracle64.straight(n, 3.0, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
    oracle64.clamp(o, False)
    proto = product_rod(o)
    out = {}
    for s in (rp.Strategy.BATCHED, rp.Strategy.MULTI_KERNEL):
        b = rp.Batch.create(proto, 1, s)
        b.step_many(P, 3)
        out[s] = (b.download_positions().reshape(-1, 3), b.download_frames())
        b.close()
    assert np.array_equal(out[rp.Strategy.BATCHED][0], out[rp.Strategy.MULTI_KERNEL][0])
    assert np.array_equal(out[rp.Strategy.BATCHED][1], out[rp.Strategy.MULTI_KERNEL][1])
    oracle64.step(o, OPAR, steps=3)
    assert np.max(np.abs(out[rp.Strategy.MULTI_KERNEL][0] - o.x[: o.nP])) <= 1e-5 * 3.0
    # 4000 segments exceed it: the batched strategy refuses the rod, the
    # multi-kernel strategy (state in global memory) steps it
    n = 4000
    o = oracle64.straight(n, 4.0, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
    oracle64.clamp(o, False)
    proto = product_rod(o)
    with pytest.raises(rp.RopeError) as e:
        rp.Batch.create(proto, 1, rp.Strategy.BATCHED)
    assert e.value.status == 3 and "shared memory" in str(e.value)
    b = rp.Batch.create(proto, 1, rp.Strategy.MULTI_KERNEL)
    b.step_many(P, 3)
    x = b.download_positions().reshape(-1, 3)
    b.close()
    oracle64.step(o, OPAR, steps=3)
    assert np.max(np.abs(x - o.x[: o.nP])) <= 1e-5 * 4.0


def test_sixty_four_primitives():
    rng = np.random.default_rng(11)
    prims = [rp.Primitive.plane((0, 0, -0.4), (0, 0, 1), 0.5)]
    while len(prims) < 64:
        c = rng.uniform(-0.3, 0.3, 3) + (0.25, 0, -0.3)
        prims.append(rp.Primitive.sphere(tuple(c), float(rng.uniform(0.01, 0.04)), float(rng.uniform(0.2, 0.9))))
    world = rp.World(prims, self_collision=True, self_friction=0.4, hash_table_size=256)
    rod = rp.Rod.centerline(W.helix(96, 0.6, 0.05, 0.02, origin=(0.25, 0.0, -0.1)), W.GRID_MATERIAL)
    res = run_all(rod, world, 20, n=4)
    ref = res[rp.Strategy.MULTI_KERNEL]
    for s in STRATS:
        assert np.array_equal(res[s][0], ref[0]), s
    assert np.all(np.isfinite(ref[0]))


def test_refused_precision_change_keeps_the_plan(oracle64):
    """A clamped rod long enough to fit the batched kernel's shared memory in
    reference precision but not compensated (its layout adds the Kahan
    compensation rows of positions and frames): switching it to compensated
    precision must fail with RP_ERR_SHARED_MEMORY and leave the batch's plan
    as it was -- same shared memory per CTA, and steps bitwise equal to a
    batch that never tried. The length is the first of a ladder that splits
    the two layouts on this device."""
    proto = b = smem = None
    for n in range(2000, 4001, 100):
        o = oracle64.straight(n, n / 1000.0, youngs=1e8, poisson=0.3, density=1100.0, radius=5e-3)
        oracle64.clamp(o, False)
        cand = product_rod(o)
        try:
            trial = rp.Batch.create(cand, 2, rp.Strategy.BATCHED)
        except rp.RopeError:
            break  # too long even for reference precision
        smem = trial.shared_bytes_per_block
        try:
            trial.set_precision(int(rp.Precision.COMPENSATED))
        except rp.RopeError as e:
            assert e.status == 3 and "shared memory" in str(e)
            proto, b = cand, trial
            break
        trial.close()
    assert b is not None, "no rod length splits the reference and compensated layouts"
    assert b.shared_bytes_per_block == smem
    with pytest.raises(rp.RopeError) as e:
        b.set_precision(int(rp.Precision.COMPENSATED))
    assert e.value.status == 3 and "shared memory" in str(e.value)
    assert b.shared_bytes_per_block == smem
    b.step_many(P, 3)
    fresh = rp.Batch.create(proto, 2, rp.Strategy.BATCHED)
    fresh.step_many(P, 3)
    assert np.array_equal(b.download_positions(), fresh.download_positions())
    assert np.array_equal(b.download_frames(), fresh.download_frames())
    b.close()
    fresh.close()
