"""Overlapped state copies (rp_batch_set_copy_stream and the
rp_batch_*_state_overlapped calls) against the stream-ordered ones.

Two batches of the same driven grid step side by side: one uploads each
step's kinematic velocities and reads back positions, frames and contact
states with the stream-ordered copies and a synchronize per step; the other
does the same through the overlapped calls on a copy stream, reading step
k's results while step k+1 runs, with double-buffered host memory. Every
output read back and the final state must be equal byte for byte.
"""
import math

import numpy as np
import pytest
import torch

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 6


def kinematics(wl, s):
    """Rows of 4 floats per particle: the drives' top velocity at step s."""
    n_p = wl.rods[0].num_particles
    v = np.zeros((len(wl.rods), n_p, 4), np.float32)
    for r, d in enumerate(wl.drives):
        w = 2 * math.pi * d.frequency
        v[r, d.particle, 2] = d.amplitude * w * math.cos(w * s * wl.params.dt + d.phase)
    return torch.from_numpy(v.reshape(-1)).pin_memory()


def test_overlapped_copies_equal_stream_ordered():
    wl = W.grid(256, seed=4)
    wl.drives = None  # velocities come from the uploads
    a = wl.make_batch(rp.Strategy.BATCHED)
    b = wl.make_batch(rp.Strategy.BATCHED)
    copy = torch.cuda.Stream()
    b.set_copy_stream(copy.cuda_stream)
    whats = (a.POSITIONS, a.FRAMES, a.CONTACTS)
    sizes = {w: a.state_bytes(w) for w in whats}
    h2d = 16 * a.total_particles
    ref_out, got_out = [], []
    bufs = [{w: torch.empty(sizes[w], dtype=torch.uint8).pin_memory() for w in whats} for _ in range(2)]
    kin = [kinematics(W.grid(256, seed=4), s) for s in range(STEPS)]
    events = [torch.cuda.Event() for _ in range(STEPS)]
    for s in range(STEPS):
        # stream-ordered
        a.write_state_async(a.KINEMATIC, kin[s].data_ptr(), h2d)
        a.step(wl.params)
        out = {w: torch.empty(sizes[w], dtype=torch.uint8).pin_memory() for w in whats}
        for w in whats:
            a.read_state_async(w, out[w].data_ptr(), sizes[w])
        a.synchronize()
        ref_out.append({w: out[w].numpy().copy() for w in whats})
        # overlapped, one step behind on the host
        b.write_state_overlapped(b.KINEMATIC, kin[s].data_ptr(), h2d)
        b.step(wl.params)
        for w in whats:
            b.read_state_overlapped(w, bufs[s % 2][w].data_ptr(), sizes[w])
        events[s].record(copy)
        if s >= 1:
            events[s - 1].synchronize()
            got_out.append({w: bufs[(s - 1) % 2][w].numpy().copy() for w in whats})
    events[-1].synchronize()
    got_out.append({w: bufs[(STEPS - 1) % 2][w].numpy().copy() for w in whats})
    for s in range(STEPS):
        for w in whats:
            assert np.array_equal(ref_out[s][w], got_out[s][w]), (s, w)
    b.synchronize()
    assert np.array_equal(a.download_positions(), b.download_positions())
    assert np.array_equal(a.download_frames(), b.download_frames())
    # the tops really moved with the uploaded velocities
    assert not np.array_equal(ref_out[0][a.POSITIONS], ref_out[-1][a.POSITIONS])
    a.close()
    b.close()


def test_overlapped_copies_need_a_copy_stream():
    wl = W.grid(8, seed=1)
    b = wl.make_batch(rp.Strategy.BATCHED)
    dst = torch.empty(b.state_bytes(b.POSITIONS), dtype=torch.uint8).pin_memory()
    with pytest.raises(rp.RopeError) as e:
        b.read_state_overlapped(b.POSITIONS, dst.data_ptr(), dst.numel())
    assert "copy stream" in str(e.value)
    b.close()
