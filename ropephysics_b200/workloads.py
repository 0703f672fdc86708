"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No external data: every rod, material draw, drive and primitive comes from a
numpy Generator seeded by the caller. The uneven batch and the grid take their
draws from ``synth`` (numpy only), which the CPU reference timing shares, so
both sides simulate the same rods.

  cantilever   1 clamped rod, 64 segments, 1 m, r 5 mm, E 1e8, nu 0.3,
               rho 1100, gravity plus a 0.05 N tip load; dt 1/60, 20 substeps
  grid         N rods of 64 segments hanging from a pinned, sinusoidally
               driven top particle; E 1e8 x U(0.4, 4), mu 0.5 x U(0.6, 1.4);
               floor at z = -1.2; dt 1/60, 20 substeps
  uneven       N rods, segments U{16..512}, length 0.2 m per 32 segments,
               initial helix coil (radius U(0.05, 0.2) m) with a straight rest
               shape, 1-4 primitives per rod (sphere r U(0.02, 0.2), capsule
               r U(0.01, 0.05) len U(0.1, 0.5), box half-extents
               U(0.05, 0.3)) within 1 m of the rod, mu U(0.2, 1.0),
               self-collision on; dt 1/60, 50 substeps
  hook         cables of 120 segments, 1.2 m, r 4 mm draped over a capsule
               bar (r 2 cm) at leg ratios 1:1..4:1, mu in [0.05, 0.6], E 1e8
               or 3e8; floor; self-collision on; dt 1/60, 20 substeps
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import Batch, Drive, Material, Primitive, Rod, StepParams, Strategy, World
from . import synth
from .synth import helix, table_for  # noqa: F401  (re-exported for callers)

GRID_MATERIAL = Material(youngs=synth.YOUNGS, poisson=synth.POISSON, density=synth.DENSITY,
                         radius=synth.RADIUS)


def primitive(spec) -> Primitive:
    """A Primitive from a synth spec tuple."""
    t, a, b, n, h, r, radius, mu = spec
    return Primitive(int(t), a=tuple(a), b=tuple(b), normal=tuple(n), half_extents=tuple(h),
                     rotation=tuple(r), radius=float(radius), friction=float(mu))


@dataclass
class Workload:
    name: str
    rods: List[Rod]
    worlds: List[World]
    world_of_rod: List[int]
    params: StepParams
    youngs_scale: Optional[np.ndarray] = None
    friction_scale: Optional[np.ndarray] = None
    drives: Optional[List[Drive]] = None
    steps: int = 1
    info: dict = field(default_factory=dict)

    @property
    def segments(self) -> np.ndarray:
        return np.array([r.num_stretch for r in self.rods], np.int64)

    def segment_substeps_per_step(self) -> int:
        return int(self.segments.sum()) * self.params.substeps

    def make_batch(self, strategy: Strategy = Strategy.BATCHED) -> Batch:
        if len({id(r) for r in self.rods}) == 1 and len(self.worlds) <= 1:
            b = Batch.create(self.rods[0], len(self.rods), strategy,
                             self.worlds[0] if self.worlds else None)
        else:
            b = Batch.create_mixed(self.rods, self.worlds, self.world_of_rod, strategy)
        if self.youngs_scale is not None or self.friction_scale is not None:
            b.set_material_scales(self.youngs_scale, self.friction_scale)
        if self.drives is not None:
            b.set_drives(self.drives)
        return b


def cantilever() -> Workload:
    """Plain method, small: a clamped 64-segment cantilever with a tip load."""
    rod = Rod.straight(64, 1.0, GRID_MATERIAL)
    rod.clamp_end(tip=False)
    rod.ext_force[-1] = (0.0, 0.0, -0.05)
    return Workload("cantilever-1x64", [rod], [], [0],
                    StepParams(dt=1.0 / 60, substeps=20, iterations=1), steps=2000)


def grid(num_rods: int = 4096, seed: int = 0) -> Workload:
    """Plain batched grid: hanging rods, per-rod stiffness/friction, driven tops."""
    d = synth.grid(num_rods, seed)
    rod = Rod.straight(64, 1.0, GRID_MATERIAL, origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, -1.0))
    rod.pin_particle(0)
    world = World([Primitive.plane((0.0, 0.0, -1.2), (0.0, 0.0, 1.0), 0.5)])
    ys, fs = d.youngs_scale, d.friction_scale
    drives = [Drive(0, (0.0, 0.0, 1.0), float(a), float(f), float(p))
              for a, f, p in zip(d.amplitude, d.frequency, d.phase)]
    return Workload(f"grid-{num_rods}x64", [rod] * num_rods, [world], [0] * num_rods,
                    StepParams(dt=1.0 / 60, substeps=20, iterations=1), ys, fs, drives, steps=1000,
                    info=dict(seed=seed))


def _random_primitive(rng, centre, mu, lo, hi, clearance=0.02, tries=64) -> Primitive:
    """synth.random_primitive as a Primitive."""
    return primitive(synth.random_primitive(rng, centre, mu, lo, hi, clearance, tries))


def uneven(num_rods: int = 16384, seed: int = 0, min_seg: int = 16, max_seg: int = 512,
           substeps: int = 50, hash_table_size: int = 0, shard=None) -> Workload:
    """Uneven batch: rods of 16..512 segments, coiled, each with its own world.
    hash_table_size 0 sizes each rod's table with table_for(). shard=(k, n):
    the k-th of n shards of a batch of n x num_rods rods drawn from `seed`
    (synth.shard: length-sorted, every n-th rod)."""
    rods, worlds = [], []
    draws = synth.uneven(num_rods * (shard[1] if shard else 1), seed, min_seg, max_seg, hash_table_size)
    if shard:
        draws = synth.shard(draws, *shard)
    for d in draws:
        rod = Rod.centerline(d.points, GRID_MATERIAL, frame_seed=(0.0, 0.0, 1.0))
        rod.b_rest_darboux[:] = 0.0  # straight rest shape: the coil is loaded
        rods.append(rod)
        worlds.append(World([primitive(q) for q in d.prims], self_collision=True, self_friction=d.friction,
                            hash_table_size=d.hash_table_size))
    return Workload(f"uneven-{len(rods)}x[{min_seg},{max_seg}]", rods, worlds, list(range(len(rods))),
                    StepParams(dt=1.0 / 60, substeps=substeps, iterations=1), steps=500,
                    info=dict(seed=seed, hash_table_size=hash_table_size or "2n, pow2, 64..1024"))


@dataclass
class ServedRequest:
    rods: List[Rod]
    steps: int
    worlds: List[World]
    drives: Optional[List[Drive]]
    youngs_scale: np.ndarray
    friction_scale: np.ndarray
    features: dict

    def segment_substeps(self, substeps: int) -> int:
        return int(sum(r.num_stretch for r in self.rods)) * substeps * self.steps


def served_request(rng, max_rods: int = 1024, min_seg: int = 32, max_seg: int = 512,
                   min_steps: int = 100, max_steps: int = 2000) -> ServedRequest:
    """One request of the served stream: 1..max_rods rods (log-uniform) of one
    shape with U{min_seg..max_seg} segments hanging from a pinned top, a
    horizon U{min_steps..max_steps}, each feature -- floor, primitives, driven
    top, self-collision -- present with probability 1/2, and per-rod material
    as in the grid (E x U(0.4, 4), mu x U(0.6, 1.4))."""
    count = int(round(math.exp(rng.uniform(0.0, math.log(max_rods)))))
    count = max(1, min(max_rods, count))
    n = int(rng.integers(min_seg, max_seg + 1))
    steps = int(rng.integers(min_steps, max_steps + 1))
    feats = {k: bool(rng.random() < 0.5) for k in ("floor", "primitives", "driven", "self")}
    length = n / 64.0
    rod = Rod.straight(n, length, GRID_MATERIAL, origin=(0.0, 0.0, 0.0), direction=(0.0, 0.0, -1.0))
    rod.pin_particle(0)
    mu = 0.5
    prims = []
    if feats["floor"]:
        prims.append(Primitive.plane((0.0, 0.0, -length - 0.05), (0.0, 0.0, 1.0), mu))
    if feats["primitives"]:
        lo, hi = np.array([0.0, 0.0, -length]), np.array([0.0, 0.0, 0.0])
        for _ in range(int(rng.integers(1, 5))):
            prims.append(_random_primitive(rng, (0.0, 0.0, -length / 2), mu, lo, hi))
    world = World(prims, self_collision=feats["self"], self_friction=mu, hash_table_size=table_for(n))
    drives = None
    if feats["driven"]:
        drives = [Drive(0, (0.0, 0.0, 1.0), float(a), float(f), float(p))
                  for a, f, p in zip(rng.uniform(0.0, 0.1, count), rng.uniform(0.5, 2.0, count),
                                     rng.uniform(0.0, 2 * math.pi, count))]
    ys = rng.uniform(0.4, 4.0, count).astype(np.float32)
    fs = rng.uniform(0.6, 1.4, count).astype(np.float32)
    return ServedRequest([rod] * count, steps, [world], drives, ys, fs, feats)


def hanging_cable_points(leg_ratio: float, length=1.2, segments=120, bar_radius=0.02,
                         bar_height=0.8, cable_radius=0.004):
    """Drape over a horizontal bar (the geometry of the reference's cable
    task, src/apps/cable_hanging.cpp:18-47): short leg on -x, half a turn over
    the top, long leg on +x with long/short = leg_ratio."""
    wrap = bar_radius + cable_radius
    arc = math.pi * wrap
    legs = length - arc
    long_leg = legs * leg_ratio / (1.0 + leg_ratio)
    short_leg = legs - long_leg
    top = bar_height
    pts = []
    h = length / segments
    for i in range(segments + 1):
        s = h * i
        if s < short_leg:
            p = (-wrap, 0.0, top - (short_leg - s))
        elif s < short_leg + arc:
            phi = (s - short_leg) / wrap
            p = (-wrap * math.cos(phi), 0.0, top + wrap * math.sin(phi))
        else:
            p = (wrap, 0.0, top - (s - short_leg - arc))
        pts.append(p)
    return np.array(pts)


HOOK_MATERIAL = dict(poisson=0.35, density=1100.0, radius=0.004)
# The floor of the hook sweep, below the lowest point of every drape: a
# 1.2 m cable over the bar at 0.8 m reaches 0.1 m below z = 0 at the 4:1
# ratio, so a floor at 0 would start those placements inside it.
HOOK_FLOOR_Z = -0.25


def hook(ratios: int = 60, frictions: int = 30, stiffnesses=(1e8, 3e8)) -> Workload:
    """Mixed-precision hook sweep: leg ratio x friction x stiffness placements."""
    rods, worlds, wor = [], [], []
    rs = np.linspace(1.0, 4.0, ratios)
    mus = np.linspace(0.05, 0.6, frictions)
    for E in stiffnesses:
        for mu in mus:
            w = World([Primitive.capsule((0.0, -0.3, 0.8), (0.0, 0.3, 0.8), 0.02, float(mu)),
                       Primitive.plane((0.0, 0.0, HOOK_FLOOR_Z), (0.0, 0.0, 1.0), float(mu))],
                      self_collision=True, self_friction=float(mu), hash_table_size=256)
            worlds.append(w)
            for r in rs:
                rod = Rod.centerline(hanging_cable_points(float(r)),
                                     Material(youngs=float(E), **HOOK_MATERIAL), frame_seed=(0.0, 1.0, 0.0))
                rod.b_rest_darboux[:] = 0.0
                rods.append(rod)
                wor.append(len(worlds) - 1)
    return Workload(f"hook-{len(rods)}x120", rods, worlds, wor,
                    StepParams(dt=1.0 / 60, substeps=20, iterations=1), steps=480,
                    info=dict(ratios=rs.tolist(), frictions=mus.tolist(), stiffnesses=list(stiffnesses)))
