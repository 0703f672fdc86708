"""Seeded draws of the benchmark workloads, in numpy only.

This module imports nothing from the package, so a process can draw a
workload without loading the native library: the CPU reference timing builds
its rods from these draws with the reference's own builders, while
``workloads.py`` builds the library's rods from the very same draws. Every
number comes from a numpy Generator seeded by the caller; the order of the
draws fixes the workload, so it must not change.

Primitive specs are tuples ``(type, a, b, normal, half_extents, rotation,
radius, friction)`` with the reference's type codes (``TPrimitive::Type``,
src/core/geometry.h:19): 0 plane, 1 sphere, 2 capsule, 3 box.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

# the rod section of every benchmark workload but the hook sweep
YOUNGS, POISSON, DENSITY, RADIUS = 1e8, 0.3, 1100.0, 5e-3

PLANE, SPHERE, CAPSULE, BOX = 0, 1, 2, 3


def plane(point, normal, friction):
    n = np.asarray(normal, float)
    n = n * (1.0 / np.sqrt(n @ n))
    return (PLANE, tuple(point), (0.0, 0.0, 0.0), tuple(n), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0, 0.0), 0.0,
            friction)


def sphere(centre, radius, friction):
    return (SPHERE, tuple(centre), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0, 0.0),
            radius, friction)


def capsule(a, b, radius, friction):
    return (CAPSULE, tuple(a), tuple(b), (0.0, 0.0, 1.0), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0, 0.0), radius,
            friction)


def box(centre, half_extents, rotation, friction):
    return (BOX, tuple(centre), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), tuple(half_extents), tuple(rotation), 0.0,
            friction)


def helix(n: int, length: float, coil_radius: float, pitch: float, origin=(0.0, 0.0, 0.0)):
    """n+1 points of arc length `length` on a vertical helix."""
    turn = math.sqrt((2 * math.pi * coil_radius) ** 2 + pitch ** 2)
    total = 2 * math.pi * length / turn
    t = np.linspace(0.0, total, n + 1)
    o = np.asarray(origin, float)
    return np.stack([o[0] + coil_radius * np.cos(t), o[1] + coil_radius * np.sin(t),
                     o[2] + pitch * t / (2 * math.pi)], axis=1)


def random_quat(rng):
    q = rng.normal(size=4)
    return tuple(q / np.linalg.norm(q))


def random_primitive(rng, centre, mu, lo, hi, clearance=0.02, tries=64):
    """A sphere, capsule or box centred within 1 m of `centre` whose bounding
    sphere keeps `clearance` from the rod's box [lo, hi] (no rod starts inside
    a primitive)."""
    for _ in range(tries):
        kind = int(rng.integers(1, 4))  # sphere, capsule, box
        d = rng.normal(size=3)
        d = d / np.linalg.norm(d) * rng.uniform(0.0, 1.0) ** (1.0 / 3.0)
        c = np.asarray(centre) + d
        if kind == 1:
            r = float(rng.uniform(0.02, 0.2))
            prim, bound = sphere(tuple(c), r, mu), r
        elif kind == 2:
            axis = rng.normal(size=3)
            half = rng.uniform(0.1, 0.5) * 0.5
            axis = axis / np.linalg.norm(axis) * half
            r = float(rng.uniform(0.01, 0.05))
            prim = capsule(tuple(c - axis), tuple(c + axis), r, mu)
            bound = half + r
        else:
            h = rng.uniform(0.05, 0.3, 3)
            prim, bound = box(tuple(c), tuple(h), random_quat(rng), mu), float(np.linalg.norm(h))
        gap = np.linalg.norm(np.maximum(np.abs(c - (lo + hi) / 2) - (hi - lo) / 2, 0.0)) - bound
        if gap >= clearance:
            return prim
    return prim


def table_for(segments: int, lo: int = 64, hi: int = 1024) -> int:
    """Spatial-hash table size for a rod: the power of two >= 2 x segments,
    clamped to [lo, hi] (few bucket collisions, bounded shared memory)."""
    t = lo
    while t < 2 * segments and t < hi:
        t *= 2
    return t


@dataclass
class UnevenRod:
    """One rod of the uneven batch: a coiled centre line (frames seeded with
    +z, straight rest shape) and its own world."""
    points: np.ndarray
    prims: List[Tuple]
    friction: float
    hash_table_size: int

    @property
    def segments(self) -> int:
        return len(self.points) - 1


def uneven(num_rods: int = 16384, seed: int = 0, min_seg: int = 16, max_seg: int = 512,
           hash_table_size: int = 0) -> List[UnevenRod]:
    """The uneven batch: rods of U{min_seg..max_seg} segments, 0.2 m per 32
    segments, on a helix of radius U(0.05, 0.2) m and pitch 4 r, each with
    1-4 primitives within 1 m, mu U(0.2, 1.0), self-collision on.
    hash_table_size 0 sizes each rod's table with table_for()."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num_rods):
        n = int(rng.integers(min_seg, max_seg + 1))
        length = 0.2 * n / 32.0
        rc = float(rng.uniform(0.05, 0.2))
        pts = helix(n, length, rc, pitch=4.0 * RADIUS, origin=(0.0, 0.0, 0.0))
        mu = float(rng.uniform(0.2, 1.0))
        centre = pts.mean(axis=0)
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        prims = [random_primitive(rng, centre, mu, lo, hi) for _ in range(int(rng.integers(1, 5)))]
        out.append(UnevenRod(pts, prims, mu, hash_table_size or table_for(n)))
    return out


def shard(draws: List[UnevenRod], k: int, n: int) -> List[UnevenRod]:
    """The k-th of n shards of a batch: rods sorted by length (stable), every
    n-th from position k, so each shard holds the same spread of lengths and
    the shards of one batch are disjoint and cover it. No rod of one shard
    interacts with another's (rods are independent), so shards step on
    separate GPUs with no exchange."""
    order = sorted(range(len(draws)), key=lambda i: -draws[i].segments)
    return [draws[i] for i in order[k::n]]


@dataclass
class GridDraws:
    youngs_scale: np.ndarray  # float32, per rod
    friction_scale: np.ndarray
    amplitude: np.ndarray     # [m]
    frequency: np.ndarray     # [Hz]
    phase: np.ndarray         # [rad]


def grid(num_rods: int = 4096, seed: int = 0) -> GridDraws:
    """Per-rod draws of the driven grid: E x U(0.4, 4), mu x U(0.6, 1.4),
    top drive A U(0, 0.1) m, f U(0.5, 2) Hz, phase U(0, 2 pi)."""
    rng = np.random.default_rng(seed)
    ys = rng.uniform(0.4, 4.0, num_rods).astype(np.float32)
    fs = rng.uniform(0.6, 1.4, num_rods).astype(np.float32)
    amp = rng.uniform(0.0, 0.1, num_rods)
    freq = rng.uniform(0.5, 2.0, num_rods)
    phase = rng.uniform(0.0, 2 * math.pi, num_rods)
    return GridDraws(ys, fs, amp, freq, phase)
