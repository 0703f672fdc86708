"""Launch shapes of the batched strategy change speed, never results.

CTA size (rods per CTA), pairs per thread (threads per rod) and whole steps
per launch are picked by rp_batch_autotune; every choice must give the same
positions, frames, contact states, self-contact lists, hold verdicts and
drive times as the default shape, bit for bit (tolerance: exact), including a
step count that is not a multiple of the steps per launch. That includes one
rod per CTA (cta_threads 0: the plain kernel stepping a batched batch).
Autotuning itself leaves the batch's state untouched, and on one short rod it
picks whichever of the batched team and one rod per CTA it timed faster.
"""
import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu


def same_state(a, b):
    assert np.array_equal(a.download_positions(), b.download_positions())
    assert np.array_equal(a.download_frames(), b.download_frames())
    assert np.array_equal(a.read_contact_states(), b.read_contact_states())


@pytest.mark.parametrize("shape,steps,graph", [((128, 2, 4), 10, True), ((256, 2, 3), 7, False),
                                               ((128, 1, 2), 5, True)])
def test_shapes_give_identical_results_grid(shape, steps, graph):
    wl = W.grid(64, seed=2)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    b.set_tuning(*shape)
    assert b.tuning == dict(zip(("cta_threads", "pairs_per_thread", "steps_per_launch"), shape))
    b.set_graph(graph)
    for bt in (a, b):
        bt.arm_hold_observer([0] * len(wl.rods), interval=3, tolerance=0.05)
    a.step_many(wl.params, steps)
    b.step_many(wl.params, steps)
    same_state(a, b)
    ra, ha, _ = a.read_hold_verdicts()
    rb, hb, _ = b.read_hold_verdicts()
    assert np.array_equal(ra, rb) and np.array_equal(ha, hb)
    a.close()
    b.close()


@pytest.mark.parametrize("shape", [(256, 2, 4), (128, 1, 3)])
def test_shapes_give_identical_results_self_collision(shape):
    wl = W.uneven(48, seed=4)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    b.set_tuning(*shape)
    a.step_many(wl.params, 7)
    b.step_many(wl.params, 7)
    same_state(a, b)
    for r in range(len(wl.rods)):
        assert np.array_equal(a.read_self_contacts(r), b.read_self_contacts(r))
    assert a.self_contact_overflow() == b.self_contact_overflow()
    assert a.error_count() == 0 and b.error_count() == 0
    a.close()
    b.close()


def test_autotune_keeps_state_and_results():
    wl = W.uneven(96, seed=6)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    a.step_many(wl.params, 2)
    b.step_many(wl.params, 2)
    x0 = b.download_positions()
    launches = b.kernel_launches
    tuning = b.autotune(wl.params, max_steps_per_launch=4)
    assert tuning["cta_threads"] in (0, 128, 256) and tuning["pairs_per_thread"] in (1, 2)
    assert 1 <= tuning["steps_per_launch"] <= 4
    assert np.array_equal(b.download_positions(), x0)
    assert b.kernel_launches == launches
    same_state(a, b)
    a.step_many(wl.params, 6)
    b.step_many(wl.params, 6)
    same_state(a, b)
    a.close()
    b.close()


@pytest.mark.parametrize("graph", [False, True])
def test_one_rod_per_cta_gives_identical_results(graph):
    """The batched batch stepped by the plain kernel: mixed rods with
    contacts, self-collision and drives, equal to the default batched shape."""
    wl = W.uneven(24, seed=9)
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    b.set_tuning(0, 1, 1)
    assert b.tuning == {"cta_threads": 0, "pairs_per_thread": 1, "steps_per_launch": 1}
    b.set_graph(graph)
    a.step_many(wl.params, 5)
    b.step_many(wl.params, 5)
    same_state(a, b)
    for r in range(len(wl.rods)):
        assert np.array_equal(a.read_self_contacts(r), b.read_self_contacts(r))
    # and back to a batched shape mid-run
    b.set_tuning(128, 1, 2)
    a.step_many(wl.params, 3)
    b.step_many(wl.params, 3)
    same_state(a, b)
    a.close()
    b.close()


def test_autotune_single_short_rod():
    wl = W.cantilever()
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.FUSED)
    tuning = a.autotune(wl.params, max_steps_per_launch=4)
    assert tuning["cta_threads"] in (0, 128, 256)
    a.step_many(wl.params, 20)
    b.step_many(wl.params, 20)
    same_state(a, b)
    a.close()
    b.close()
