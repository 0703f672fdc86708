"""This library against the reference's own GPU batch on the same B200.

The plain batched grid (4096 rods of 64 segments, top particle pinned and
driven sinusoidally, per-rod stiffness and friction scales, floor plane, dt
1/60 with 20 substeps) is the one named shape the reference's batch can
express. Both run it the way the reference's API runs it: one step call per
step with the drives' kinematic velocities uploaded from the host each step
(the reference's Batch::setKinematicVelocities). This library also runs it
with on-device drives replayed from a CUDA graph. Wall time over 50 steps
with a synchronisation at the end; the library must be faster than the
reference's fused kernel on the same GPU, and the ratios are printed.
"""
import math
import time

import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 50


def drive_velocities(wl, t):
    """Kinematic velocity of every particle at time t (rod-major): the pinned
    top moves along z at A 2 pi f cos(2 pi f t + phase), the rest is zero."""
    n_rods, n_p = len(wl.rods), wl.rods[0].num_particles
    v = np.zeros((n_rods, n_p, 3), np.float32)
    for r, d in enumerate(wl.drives):
        w = 2 * math.pi * d.frequency
        v[r, d.particle, 2] = d.amplitude * w * math.cos(w * t + d.phase)
    return v.reshape(-1)


def test_faster_than_the_reference_gpu_batch_on_the_grid(reference_gpu, oracle64):
    R = reference_gpu
    if not R.lib.refgpu_available():
        pytest.skip("no device for the reference GPU path")
    import ctypes as C
    from oracle import Primitive as OP, World as OW
    wl = W.grid(4096)
    n_rods = len(wl.rods)
    p = wl.params
    kin = [drive_velocities(wl, s * p.dt) for s in range(STEPS + 3)]

    # the reference: fused batch, kinematic velocities uploaded every step
    o = oracle64.straight(64, 1.0, youngs=W.GRID_MATERIAL.youngs, poisson=W.GRID_MATERIAL.poisson,
                          density=W.GRID_MATERIAL.density, radius=W.GRID_MATERIAL.radius,
                          direction=(0, 0, -1))
    oracle64.pin(o, 0)
    h = R.from_rod(o)
    wh = R.world(OW([OP.plane((0, 0, -1.2), (0, 0, 1), 0.5)]))
    rb = R.lib.refgpu_create(h, n_rods, 1, wh)
    assert rb
    ys = np.ascontiguousarray(wl.youngs_scale, np.float32)
    fs = np.ascontiguousarray(wl.friction_scale, np.float32)
    fp = C.POINTER(C.c_float)
    R.lib.refgpu_set_material_scales(rb, ys.ctypes.data_as(fp), fs.ctypes.data_as(fp), n_rods)
    g = (C.c_double * 3)(*p.gravity)

    def ref_step(s):
        R.lib.refgpu_set_kinematic(rb, kin[s].ctypes.data_as(fp), len(kin[s]) // 3)
        R.lib.refgpu_step(rb, p.dt, p.substeps, p.iterations, g, 0.0, 0.0, 1, 1)

    for s in range(3):
        ref_step(s)
    R.lib.refgpu_sync(rb)
    t0 = time.perf_counter()
    for s in range(STEPS):
        ref_step(3 + s)
    R.lib.refgpu_sync(rb)
    t_ref = time.perf_counter() - t0
    R.lib.refgpu_free(rb)
    R.free(h)

    # this library, the same API pattern (host kinematic upload per step)
    b = rp.Batch.create(wl.rods[0], n_rods, rp.Strategy.BATCHED, wl.worlds[0])
    b.set_material_scales(wl.youngs_scale, wl.friction_scale)
    k4 = [np.concatenate([k.reshape(-1, 3), np.zeros((len(k) // 3, 1), np.float32)], axis=1).copy()
          for k in kin]

    def our_step(s):
        b.write_state_async(b.KINEMATIC, k4[s].ctypes.data, k4[s].nbytes)
        b.step(p)
        b.synchronize()  # the host buffer of this step must outlive its copy

    for s in range(3):
        our_step(s)
    t0 = time.perf_counter()
    for s in range(STEPS):
        our_step(3 + s)
    t_ours = time.perf_counter() - t0
    b.close()

    # this library's own form: on-device drives, graph replay
    d = wl.make_batch(rp.Strategy.BATCHED)
    d.set_graph(True)
    d.step_many(p, 3)
    d.step_many(p, STEPS)
    d.synchronize()
    t0 = time.perf_counter()
    d.step_many(p, STEPS)
    d.synchronize()
    t_graph = time.perf_counter() - t0
    d.close()

    seg_sub = wl.segment_substeps_per_step() * STEPS
    print(f"\ngrid 4096x64, {STEPS} steps: reference fused {seg_sub / t_ref:.3e}, this library "
          f"(same API pattern) {seg_sub / t_ours:.3e} ({t_ref / t_ours:.2f}x), on-device drives + graph "
          f"{seg_sub / t_graph:.3e} ({t_ref / t_graph:.2f}x) segment-substeps/s")
    assert t_ours < t_ref
    assert t_graph < t_ref
