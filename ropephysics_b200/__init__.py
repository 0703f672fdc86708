"""ropephysics_b200 -- B200-native batched XPBD Cosserat-rod step.

Python host mirror of the C ABI in ``include/ropephysics_b200.h``, shaped like
the reference's batch API (``crs::gpu::Batch``, src/gpu/gpu_solver.h:66-145):

    rod = Rod.straight(64, 1.0, Material(1e7, 0.35, 1000, 5e-3))
    rod.clamp_end(tip=False)
    batch = Batch.create(rod, num_rods=4096, strategy=Strategy.BATCHED, world=world)
    batch.step(StepParams(dt=1/60, substeps=20))
    x = batch.download_positions()

Every call goes through ``librp_b200.so``; there is no CPU fallback. A
failing call raises ``RopeError`` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi

__all__ = ["RopeError", "Strategy", "Precision", "ContactState", "Material", "Primitive", "World",
           "StepParams", "Drive", "Rod", "Batch", "Server", "cuda_available", "device_name",
           "diagnostic", "max_fused_segments", "measure_fp32_peak", "coloring", "self_collision_index_gap", "lib", "Trajectory",
           "read_rodtraj", "WaypointDrive", "HarnessBoard", "HARNESS_OUTCOME"]


def lib():
    return _abi.load()


class RopeError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def _check(status: int):
    if status != 0:
        raise RopeError(status, lib().rp_last_error().decode(errors="replace"))


class Strategy(enum.IntEnum):
    MULTI_KERNEL = 0
    FUSED = 1
    BATCHED = 2


class Precision(enum.IntFlag):
    REFERENCE = 0
    COMPENSATED = 1
    FP64_CONE = 2
    FP64_VERDICT = 4
    COLORED_SELF = 8


class ContactState(enum.IntEnum):
    NONE = 0
    SEPARATED = 1
    STICK = 2
    SLIP = 3


@dataclass
class Material:
    youngs: float = 1e7
    poisson: float = 0.35
    density: float = 1000.0
    radius: float = 5e-3

    def to_c(self) -> _abi.Material:
        return _abi.Material(self.youngs, self.poisson, self.density, self.radius)


@dataclass
class Primitive:
    """Analytic collision primitive (reference src/core/geometry.h:17-65)."""
    type: int
    a: Sequence[float] = (0.0, 0.0, 0.0)
    b: Sequence[float] = (0.0, 0.0, 0.0)
    normal: Sequence[float] = (0.0, 0.0, 1.0)
    half_extents: Sequence[float] = (0.0, 0.0, 0.0)
    rotation: Sequence[float] = (1.0, 0.0, 0.0, 0.0)
    radius: float = 0.0
    friction: float = 0.0

    @staticmethod
    def plane(point, normal, friction):
        n = np.asarray(normal, float)
        n = n * (1.0 / np.sqrt(n @ n))
        return Primitive(0, a=tuple(point), normal=tuple(n), friction=friction)

    @staticmethod
    def sphere(centre, radius, friction):
        return Primitive(1, a=tuple(centre), radius=radius, friction=friction)

    @staticmethod
    def capsule(a, b, radius, friction):
        return Primitive(2, a=tuple(a), b=tuple(b), radius=radius, friction=friction)

    @staticmethod
    def box(centre, half_extents, rotation, friction):
        return Primitive(3, a=tuple(centre), half_extents=tuple(half_extents),
                         rotation=tuple(rotation), friction=friction)

    def to_c(self) -> _abi.Primitive:
        p = _abi.Primitive()
        p.type = int(self.type)
        p.a[:] = [float(v) for v in self.a]
        p.b[:] = [float(v) for v in self.b]
        p.normal[:] = [float(v) for v in self.normal]
        p.half_extents[:] = [float(v) for v in self.half_extents]
        p.rotation[:] = [float(v) for v in self.rotation]
        p.radius = float(self.radius)
        p.friction = float(self.friction)
        return p


@dataclass
class World:
    """Collision world (reference src/core/collision.h:83-106)."""
    primitives: list = field(default_factory=list)
    self_collision: bool = False
    self_friction: float = 0.0
    self_skip: int = 2
    hash_table_size: int = 4096
    contact_margin_radii: float = 0.25

    def to_c(self) -> _abi.World:
        arr = (_abi.Primitive * max(1, len(self.primitives)))(*[p.to_c() for p in self.primitives])
        w = _abi.World()
        w.primitives = C.cast(arr, C.POINTER(_abi.Primitive))
        w.num_primitives = len(self.primitives)
        w.self_collision = int(self.self_collision)
        w.self_friction = float(self.self_friction)
        w.self_skip = int(self.self_skip)
        w.hash_table_size = int(self.hash_table_size)
        w.contact_margin_radii = float(self.contact_margin_radii)
        w._keep = arr
        return w


@dataclass
class StepParams:
    """Reference BatchParams (src/gpu/gpu_solver.h:52-60)."""
    dt: float = 1e-3
    substeps: int = 8
    iterations: int = 1
    gravity: Sequence[float] = (0.0, 0.0, -9.81)
    linear_damping: float = 0.0
    angular_damping: float = 0.0
    contact_interval: int = 1

    def to_c(self) -> _abi.StepParams:
        p = _abi.StepParams()
        p.dt = self.dt
        p.substeps = self.substeps
        p.iterations = self.iterations
        p.gravity[:] = [float(v) for v in self.gravity]
        p.linear_damping = self.linear_damping
        p.angular_damping = self.angular_damping
        p.contact_interval = self.contact_interval
        return p


@dataclass
class Drive:
    """On-device sinusoidal drive of one pinned particle."""
    particle: int = -1
    axis: Sequence[float] = (0.0, 0.0, 1.0)
    amplitude: float = 0.0
    frequency: float = 0.0
    phase: float = 0.0


@dataclass
class WaypointDrive:
    """On-device waypoint schedule of one pinned particle (a gripper motion):
    from `start` through `waypoints` (x, y), `legs` seconds each with a
    smoothstep, at `height`, the velocity held for `steps_per_control`
    steps of `dt` (rp_waypoint_drive)."""
    particle: int
    start: Sequence[float]
    waypoints: Sequence[Sequence[float]]
    legs: Sequence[float]
    height: float = 0.0
    dt: float = 1e-3
    steps_per_control: int = 1


@dataclass
class HarnessBoard:
    """A routing board: the cable passes below peg A, above peg B and
    through the clip (rp_harness_board)."""
    peg_a: Sequence[float]
    peg_b: Sequence[float]
    clip: Sequence[float]
    peg_radius: float
    clip_half_gap: float
    clip_height: float
    cable_radius: float
    lay_slack: float = 0.015


HARNESS_OUTCOME = np.dtype([("score", "<f8"), ("side_a", "<f8"), ("side_b", "<f8"), ("clip_miss", "<f8"),
                            ("below_a", "u1"), ("above_b", "u1"), ("through_clip", "u1"), ("success", "u1"),
                            ("reserved", "u1", 4)])

_F64 = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)


def _np(ptr, n, dtype, shape):
    if n == 0 or not ptr:
        return np.zeros(shape, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).view(dtype).reshape(shape)


class Rod:
    """Host rod descriptor owned by the library (reference ``crs::Rod``).

    Arrays are numpy views of the library's storage, so writing
    ``rod.ext_force[-1] = (0, 0, -0.05)`` changes the descriptor in place."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        self._refresh()

    def __del__(self):
        try:
            if self._h:
                lib().rp_rod_destroy(self._h)
        except Exception:
            pass

    def _refresh(self):
        d = _abi.RodDesc()
        _check(lib().rp_rod_view(self._h, C.byref(d)))
        self.desc = d
        nP, nS, nSt, nB = d.num_particles, d.num_frames, d.num_stretch, d.num_bend
        f, i = np.float64, np.int32
        self.x = _np(d.x, 3 * nP, f, (nP, 3))
        self.v = _np(d.v, 3 * nP, f, (nP, 3))
        self.inv_mass = _np(d.inv_mass, nP, f, (nP,))
        self.mass = _np(d.mass, nP, f, (nP,))
        self.ext_force = _np(d.ext_force, 3 * nP, f, (nP, 3))
        self.kin_velocity = _np(d.kin_velocity, 3 * nP, f, (nP, 3))
        self.q = _np(d.q, 4 * nS, f, (nS, 4))
        self.omega = _np(d.omega, 3 * nS, f, (nS, 3))
        self.inertia = _np(d.inertia, 3 * nS, f, (nS, 3))
        self.inv_inertia = _np(d.inv_inertia, 3 * nS, f, (nS, 3))
        self.ext_torque = _np(d.ext_torque, 3 * nS, f, (nS, 3))
        self.s_p0 = _np(d.s_p0, nSt, i, (nSt,))
        self.s_p1 = _np(d.s_p1, nSt, i, (nSt,))
        self.s_seg = _np(d.s_seg, nSt, i, (nSt,))
        self.s_rest = _np(d.s_rest, nSt, f, (nSt,))
        self.s_compliance = _np(d.s_compliance, 3 * nSt, f, (nSt, 3))
        self.b_a = _np(d.b_a, nB, i, (nB,))
        self.b_b = _np(d.b_b, nB, i, (nB,))
        self.b_rest = _np(d.b_rest, nB, f, (nB,))
        self.b_compliance = _np(d.b_compliance, 3 * nB, f, (nB, 3))
        self.b_rest_darboux = _np(d.b_rest_darboux, 3 * nB, f, (nB, 3))

    num_particles = property(lambda s: s.desc.num_particles)
    num_frames = property(lambda s: s.desc.num_frames)
    num_stretch = property(lambda s: s.desc.num_stretch)
    num_bend = property(lambda s: s.desc.num_bend)
    material = property(lambda s: Material(s.desc.material.youngs, s.desc.material.poisson,
                                           s.desc.material.density, s.desc.material.radius))

    # ---- builders (reference src/core/rod.h:126-167) ----
    @classmethod
    def straight(cls, segments: int, length: float, material: Material = Material(),
                 origin=(0.0, 0.0, 0.0), direction=(1.0, 0.0, 0.0)) -> "Rod":
        h = C.c_void_p()
        m = material.to_c()
        _check(lib().rp_rod_create_straight(segments, length, C.byref(m),
                                            (C.c_double * 3)(*origin), (C.c_double * 3)(*direction),
                                            C.byref(h)))
        return cls(h.value)

    @classmethod
    def centerline(cls, points, material: Material = Material(), frame_seed=(0.0, 0.0, 1.0),
                   twist_per_length: float = 0.0) -> "Rod":
        pts = np.ascontiguousarray(points, np.float64)
        h = C.c_void_p()
        m = material.to_c()
        _check(lib().rp_rod_create_centerline(pts.ctypes.data_as(_F64), len(pts), C.byref(m),
                                              (C.c_double * 3)(*frame_seed), float(twist_per_length),
                                              C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, material: Material, **a) -> "Rod":
        """Deep copy of caller arrays: x, v, inv_mass, q, inertia, inv_inertia,
        s_p0, s_p1, s_seg, s_rest, s_compliance, b_a, b_b, b_rest,
        b_compliance, b_rest_darboux (+ optional mass, ext_force,
        kin_velocity, omega, ext_torque)."""
        keep = {}

        def arr(name, dtype):
            if name not in a or a[name] is None:
                return None
            v = np.ascontiguousarray(a[name], dtype)
            keep[name] = v
            return v.ctypes.data_as(C.POINTER(C.c_double if dtype == np.float64 else C.c_int32))

        d = _abi.RodDesc()
        d.num_particles = len(a["x"])
        d.num_frames = len(a["q"])
        d.num_stretch = len(a["s_p0"])
        d.num_bend = len(a["b_a"])
        d.material = material.to_c()
        for n in ("x", "v", "inv_mass", "mass", "ext_force", "kin_velocity", "q", "omega", "inertia",
                  "inv_inertia", "ext_torque", "s_rest", "s_compliance", "b_rest", "b_compliance",
                  "b_rest_darboux"):
            p = arr(n, np.float64)
            if p is not None:
                setattr(d, n, p)
        for n in ("s_p0", "s_p1", "s_seg", "b_a", "b_b"):
            p = arr(n, np.int32)
            if p is not None:
                setattr(d, n, p)
        h = C.c_void_p()
        _check(lib().rp_rod_create_from_desc(C.byref(d), C.byref(h)))
        return cls(h.value)

    def clamp_end(self, tip: bool = False) -> int:
        g = C.c_int32()
        _check(lib().rp_rod_clamp_end(self._h, int(tip), C.byref(g)))
        self._refresh()
        return g.value

    def pin_particle(self, i: int):
        _check(lib().rp_rod_pin_particle(self._h, i))

    def set_rest_from_current(self):
        _check(lib().rp_rod_set_rest_from_current(self._h))

    def coloring(self, bend: bool):
        n = self.num_bend if bend else self.num_stretch
        order = np.zeros(max(n, 1), np.int32)
        starts = np.zeros(n + 2, np.int32)
        nc = C.c_int32()
        _check(lib().rp_rod_coloring(C.byref(self.desc), int(bend), order.ctypes.data_as(_I32),
                                     starts.ctypes.data_as(_I32), C.byref(nc)))
        return order[:n].copy(), starts[: nc.value + 1].copy()


def coloring(rod: Rod, bend: bool):
    return rod.coloring(bend)


def self_collision_index_gap(rod: Rod, world: World) -> int:
    g = C.c_int32()
    w = world.to_c()
    _check(lib().rp_self_collision_index_gap(C.byref(rod.desc), C.byref(w), C.byref(g)))
    return g.value


def cuda_available() -> bool:
    return bool(lib().rp_cuda_available())


def measure_fp32_peak(trips: int = 4096) -> dict:
    """The current device's FP32 FMA throughput, measured on every SM
    (rp_measure_fp32_peak): {"tflops": ..., "ms": ...}."""
    t, ms = C.c_double(), C.c_double()
    _check(lib().rp_measure_fp32_peak(int(trips), C.byref(t), C.byref(ms)))
    return {"tflops": t.value, "ms": ms.value}


def device_name() -> str:
    buf = C.create_string_buffer(512)
    lib().rp_device_name(buf, 512)
    return buf.value.decode()


def diagnostic() -> str:
    buf = C.create_string_buffer(1024)
    lib().rp_diagnostic(buf, 1024)
    return buf.value.decode()


def max_fused_segments() -> int:
    return lib().rp_max_fused_segments()


class Batch:
    """A device-resident batch of rods (reference ``crs::gpu::Batch``)."""

    def __init__(self, handle, rods, worlds):
        self._h = C.c_void_p(handle)
        self._keep = (rods, worlds)
        L = lib()
        self.num_rods = L.rp_batch_num_rods(self._h)
        self.particles = np.array([L.rp_batch_num_particles(self._h, r) for r in range(self.num_rods)],
                                  np.int64)
        self.offsets = np.array([L.rp_batch_particle_offset(self._h, r) for r in range(self.num_rods)],
                                np.int64)
        self.total_particles = int(self.particles.sum())
        self.frames = np.array([L.rp_batch_num_frames(self._h, r) for r in range(self.num_rods)],
                               np.int64)
        self.frame_offsets = np.array([L.rp_batch_frame_offset(self._h, r)
                                       for r in range(self.num_rods)], np.int64)
        self.total_frames = int(self.frames.sum())

    def close(self):
        if self._h:
            lib().rp_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @classmethod
    def create(cls, prototype: Rod, num_rods: int, strategy: Strategy = Strategy.FUSED,
               world: Optional[World] = None) -> "Batch":
        h = C.c_void_p()
        w = world.to_c() if world is not None else None
        _check(lib().rp_batch_create(C.byref(prototype.desc), num_rods, int(strategy),
                                     C.byref(w) if w is not None else None, C.byref(h)))
        return cls(h.value, [prototype], w)

    @classmethod
    def create_mixed(cls, rods: Sequence[Rod], worlds: Sequence[World] = (),
                     world_of_rod: Optional[Sequence[int]] = None,
                     strategy: Strategy = Strategy.BATCHED) -> "Batch":
        descs = (C.POINTER(_abi.RodDesc) * len(rods))(*[C.pointer(r.desc) for r in rods])
        cw = [w.to_c() for w in worlds]
        warr = (_abi.World * max(1, len(cw)))(*cw) if cw else None
        wor = np.ascontiguousarray(world_of_rod, np.int32) if world_of_rod is not None else None
        h = C.c_void_p()
        _check(lib().rp_batch_create_mixed(descs, len(rods), warr, len(cw),
                                           wor.ctypes.data_as(_I32) if wor is not None else None,
                                           int(strategy), C.byref(h)))
        return cls(h.value, list(rods), (cw, warr, wor))

    # ---- stepping ----
    def step(self, params: StepParams):
        p = params.to_c()
        _check(lib().rp_batch_step(self._h, C.byref(p)))

    def step_many(self, params: StepParams, steps: int):
        p = params.to_c()
        _check(lib().rp_batch_step_many(self._h, C.byref(p), steps))

    def synchronize(self):
        _check(lib().rp_batch_synchronize(self._h))

    def set_stream(self, stream_ptr: int):
        _check(lib().rp_batch_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_precision(self, flags: int):
        _check(lib().rp_batch_set_precision(self._h, int(flags)))

    def set_graph(self, enabled: bool):
        _check(lib().rp_batch_set_graph(self._h, int(enabled)))

    def autotune(self, params: StepParams, max_steps_per_launch: int = 4) -> dict:
        """Time the batched launch shapes on this batch (state restored after)
        and keep the fastest; returns the chosen tuning."""
        p = params.to_c()
        _check(lib().rp_batch_autotune(self._h, C.byref(p), max_steps_per_launch))
        return self.tuning

    @property
    def tuning(self) -> dict:
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().rp_batch_get_tuning(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"cta_threads": a.value, "pairs_per_thread": b.value, "steps_per_launch": c.value}

    def set_tuning(self, cta_threads: int = 256, pairs_per_thread: int = 1, steps_per_launch: int = 1):
        _check(lib().rp_batch_set_tuning(self._h, cta_threads, pairs_per_thread, steps_per_launch))

    # ---- state transfer ----
    def download(self, rod_index: int, rod: Rod):
        _check(lib().rp_batch_download(self._h, rod_index, C.byref(rod.desc)))

    def download_positions(self) -> np.ndarray:
        out = np.zeros((self.total_particles, 3), np.float32)
        _check(lib().rp_batch_download_positions(self._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                 out.size))
        return out

    def positions_of(self, rod_index: int, positions: Optional[np.ndarray] = None) -> np.ndarray:
        pos = self.download_positions() if positions is None else positions
        o, n = int(self.offsets[rod_index]), int(self.particles[rod_index])
        return pos[o:o + n]

    def download_frames(self) -> np.ndarray:
        out = np.zeros((self.total_frames, 4), np.float32)
        _check(lib().rp_batch_download_frames(self._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                              out.size))
        return out

    def frames_of(self, rod_index: int, frames: Optional[np.ndarray] = None) -> np.ndarray:
        q = self.download_frames() if frames is None else frames
        o, n = int(self.frame_offsets[rod_index]), int(self.frames[rod_index])
        return q[o:o + n]

    def upload(self, rod: Rod):
        _check(lib().rp_batch_upload(self._h, C.byref(rod.desc)))

    def set_loads(self, rod_index: int, rod: Rod):
        _check(lib().rp_batch_set_loads(self._h, rod_index, C.byref(rod.desc)))

    def upload_rod(self, rod_index: int, rod: Rod):
        _check(lib().rp_batch_upload_rod(self._h, rod_index, C.byref(rod.desc)))

    def set_kinematic_velocities(self, rod_major_xyz):
        v = np.ascontiguousarray(rod_major_xyz, np.float32).reshape(-1, 3)
        _check(lib().rp_batch_set_kinematic_velocities(self._h, v.ctypes.data_as(C.POINTER(C.c_float)),
                                                       len(v)))

    def set_material_scales(self, youngs_scale=None, friction_scale=None):
        y = np.ascontiguousarray(youngs_scale, np.float32) if youngs_scale is not None else None
        f = np.ascontiguousarray(friction_scale, np.float32) if friction_scale is not None else None
        FP = C.POINTER(C.c_float)
        _check(lib().rp_batch_set_material_scales(self._h, y.ctypes.data_as(FP) if y is not None else None,
                                                  f.ctypes.data_as(FP) if f is not None else None,
                                                  self.num_rods))

    def set_waypoint_drives(self, drives: Optional[Sequence[Optional[WaypointDrive]]]):
        """One waypoint schedule per rod (None: undriven rod); replaces the
        sinusoidal drives and restarts the schedules' step count."""
        if drives is None:
            _check(lib().rp_batch_set_waypoint_drives(self._h, None, 0))
            return
        arr = (_abi.WaypointDrive * len(drives))()
        for i, d in enumerate(drives):
            if d is None:
                arr[i].particle = -1
                continue
            n = len(d.waypoints)
            if not 1 <= n <= _abi.MAX_WAYPOINTS or len(d.legs) != n:
                raise ValueError(f"1..{_abi.MAX_WAYPOINTS} waypoints, one leg each")
            arr[i].particle = d.particle
            arr[i].count = n
            arr[i].steps_per_control = d.steps_per_control
            arr[i].dt = d.dt
            arr[i].start[:] = [float(d.start[0]), float(d.start[1])]
            arr[i].height = d.height
            for k in range(n):
                arr[i].legs[k] = float(d.legs[k])
                arr[i].waypoints[k][0] = float(d.waypoints[k][0])
                arr[i].waypoints[k][1] = float(d.waypoints[k][1])
        _check(lib().rp_batch_set_waypoint_drives(self._h, arr, len(drives)))

    def evaluate_harness(self, board: HarnessBoard) -> np.ndarray:
        """Routing outcome of every rod's current centre line on `board`,
        computed on the device (structured array, HARNESS_OUTCOME)."""
        b = _abi.HarnessBoard()
        b.peg_a[:] = [float(v) for v in board.peg_a[:2]]
        b.peg_b[:] = [float(v) for v in board.peg_b[:2]]
        b.clip[:] = [float(v) for v in board.clip[:2]]
        b.peg_radius = board.peg_radius
        b.clip_half_gap = board.clip_half_gap
        b.clip_height = board.clip_height
        b.cable_radius = board.cable_radius
        b.lay_slack = board.lay_slack
        out = np.zeros(self.num_rods, HARNESS_OUTCOME)
        _check(lib().rp_batch_evaluate_harness(self._h, C.byref(b),
                                               out.ctypes.data_as(C.POINTER(_abi.HarnessOutcome)),
                                               self.num_rods))
        return out

    def set_drives(self, drives: Optional[Sequence[Drive]]):
        if drives is None:
            _check(lib().rp_batch_set_drives(self._h, None, 0))
            return
        arr = (_abi.Drive * len(drives))()
        for i, d in enumerate(drives):
            arr[i].particle = d.particle
            arr[i].axis[:] = [float(v) for v in d.axis]
            arr[i].amplitude = d.amplitude
            arr[i].frequency = d.frequency
            arr[i].phase = d.phase
        _check(lib().rp_batch_set_drives(self._h, arr, len(drives)))

    def set_time(self, t: float):
        _check(lib().rp_batch_set_time(self._h, float(t)))

    # ---- raw asynchronous copies (pinned buffers for streaming) ----
    POSITIONS, FRAMES, CONTACTS, KINEMATIC = 0, 1, 2, 3

    def state_bytes(self, what: int) -> int:
        if what in (self.POSITIONS, self.KINEMATIC):
            return 16 * self.total_particles
        if what == self.FRAMES:
            return 16 * self.total_frames
        n = C.c_int64()
        _check(lib().rp_batch_read_contact_states(self._h, None, 0, C.byref(n)))
        return n.value

    def read_state_async(self, what: int, dst_ptr: int, nbytes: int):
        _check(lib().rp_batch_read_state_async(self._h, what, C.c_void_p(dst_ptr), nbytes))

    def set_copy_stream(self, stream_ptr: int):
        _check(lib().rp_batch_set_copy_stream(self._h, C.c_void_p(stream_ptr)))

    def read_state_overlapped(self, what: int, dst_ptr: int, nbytes: int):
        _check(lib().rp_batch_read_state_overlapped(self._h, what, C.c_void_p(dst_ptr), nbytes))

    def write_state_overlapped(self, what: int, src_ptr: int, nbytes: int):
        _check(lib().rp_batch_write_state_overlapped(self._h, what, C.c_void_p(src_ptr), nbytes))

    def write_state_async(self, what: int, src_ptr: int, nbytes: int):
        _check(lib().rp_batch_write_state_async(self._h, what, C.c_void_p(src_ptr), nbytes))

    # ---- outputs ----
    def read_contact_states(self) -> np.ndarray:
        n = C.c_int64()
        _check(lib().rp_batch_read_contact_states(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.uint8)
        _check(lib().rp_batch_read_contact_states(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                  out.size, C.byref(n)))
        return out[: n.value]

    def read_self_contacts(self, rod_index: int) -> np.ndarray:
        n = C.c_int32()
        _check(lib().rp_batch_read_self_contacts(self._h, rod_index, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2), np.int32)
        _check(lib().rp_batch_read_self_contacts(self._h, rod_index, out.ctypes.data_as(_I32),
                                                 out.shape[0], C.byref(n)))
        return out[: n.value]

    def arm_hold_observer(self, particle_of_rod, interval: int = 50, tolerance: float = 0.05, start_z=None):
        """start_z: each rod's start height (e.g. the double the rod was built
        from); None reads it from the device."""
        p = np.ascontiguousarray(particle_of_rod, np.int32)
        if start_z is None:
            _check(lib().rp_batch_arm_hold_observer(self._h, p.ctypes.data_as(_I32), len(p), interval,
                                                    tolerance))
            return
        z = np.ascontiguousarray(start_z, np.float64)
        if len(z) != len(p):
            raise ValueError("start_z needs one height per rod")
        _check(lib().rp_batch_arm_hold_observer_at(self._h, p.ctypes.data_as(_I32), z.ctypes.data_as(_F64),
                                                   len(p), interval, tolerance))

    def read_hold_verdicts(self):
        n = self.num_rods
        rise = np.zeros(n)
        held = np.zeros(n, np.uint8)
        near = np.zeros(n, np.uint8)
        _check(lib().rp_batch_read_hold_verdicts(self._h, rise.ctypes.data_as(_F64),
                                                 held.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                 near.ctypes.data_as(C.POINTER(C.c_uint8)), n))
        return rise, held.astype(bool), near.astype(bool)

    # ---- accessors (reference gpu_solver.h:117-130) ----
    @property
    def strategy(self) -> Strategy:
        return Strategy(lib().rp_batch_strategy(self._h))

    @property
    def stretch_colors(self) -> int:
        return lib().rp_batch_stretch_colors(self._h)

    @property
    def bend_colors(self) -> int:
        return lib().rp_batch_bend_colors(self._h)

    @property
    def shared_bytes_per_block(self) -> int:
        return lib().rp_batch_shared_bytes_per_block(self._h)

    def launches_per_step(self, params: StepParams) -> int:
        p = params.to_c()
        return lib().rp_batch_launches_per_step(self._h, C.byref(p))

    def self_contact_overflow(self) -> int:
        return lib().rp_batch_self_contact_overflow(self._h)

    @property
    def kernel_launches(self) -> int:
        return lib().rp_batch_kernel_launches(self._h)

    def error_count(self) -> int:
        return lib().rp_batch_error_count(self._h)

    def num_segments(self, rod_index: int = 0) -> int:
        return lib().rp_batch_num_segments(self._h, rod_index)


class Server:
    """Continuous-batching server (rp_server_*): requests of rods with a
    horizon, admitted by an HBM budget, stepped together in one launch per
    step, retired when done."""

    def __init__(self, budget_bytes: int, params: StepParams, precision: int = 0):
        cfg = _abi.ServerConfig()
        cfg.hbm_budget_bytes = int(budget_bytes)
        cfg.params = params.to_c()
        cfg.precision = int(precision)
        cfg.max_steps_in_flight = 1
        h = C.c_void_p()
        _check(lib().rp_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if self._h:
            lib().rp_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, rods: Sequence[Rod], steps: int, worlds: Sequence[World] = (),
               world_of_rod=None, drives: Optional[Sequence[Drive]] = None, youngs_scale=None,
               friction_scale=None) -> int:
        req = _abi.Request()
        descs = (C.POINTER(_abi.RodDesc) * len(rods))(*[C.pointer(r.desc) for r in rods])
        req.rods = descs
        req.num_rods = len(rods)
        req.steps = int(steps)
        cw = [w.to_c() for w in worlds]
        warr = (_abi.World * max(1, len(cw)))(*cw) if cw else None
        req.worlds = warr
        req.num_worlds = len(cw)
        keep = [descs, cw, warr, rods]
        if world_of_rod is not None:
            wor = np.ascontiguousarray(world_of_rod, np.int32)
            req.world_of_rod = wor.ctypes.data_as(_I32)
            keep.append(wor)
        if drives is not None:
            arr = (_abi.Drive * len(drives))()
            for i, d in enumerate(drives):
                arr[i].particle = d.particle
                arr[i].axis[:] = [float(v) for v in d.axis]
                arr[i].amplitude = d.amplitude
                arr[i].frequency = d.frequency
                arr[i].phase = d.phase
            req.drives = arr
            keep.append(arr)
        FP = C.POINTER(C.c_float)
        for name, val in (("youngs_scale", youngs_scale), ("friction_scale", friction_scale)):
            if val is not None:
                a = np.ascontiguousarray(val, np.float32)
                setattr(req, name, a.ctypes.data_as(FP))
                keep.append(a)
        rid = C.c_uint64()
        _check(lib().rp_server_submit(self._h, C.byref(req), C.byref(rid)))
        return rid.value

    def info(self, rid: int) -> dict:
        i = _abi.RequestInfo()
        _check(lib().rp_server_info(self._h, rid, C.byref(i)))
        return {f: getattr(i, f) for f, _ in _abi.RequestInfo._fields_}

    def wait(self, rid: int, timeout: float = 600.0):
        _check(lib().rp_server_wait(self._h, rid, float(timeout)))

    def result(self, rid: int) -> np.ndarray:
        n = self.info(rid)["num_particles"]
        out = np.zeros((n, 3), np.float32)
        _check(lib().rp_server_result(self._h, rid, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def release(self, rid: int):
        _check(lib().rp_server_release(self._h, rid))

    def stats(self) -> dict:
        s = _abi.ServerStats()
        _check(lib().rp_server_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in _abi.ServerStats._fields_}

    def drain(self, timeout: float = 600.0):
        _check(lib().rp_server_drain(self._h, float(timeout)))


class Trajectory:
    """A .rodtraj file written from a batch's device buffers (the reference's
    demo-scene trajectory format, src/validation/scenes.cpp:13-20)."""

    def __init__(self, path: str, num_frames: int, batch: "Batch", radius: float, fps: float):
        h = C.c_void_p()
        _check(lib().rp_traj_open(str(path).encode(), num_frames, batch._h, radius, fps, C.byref(h)))
        self._h = h
        self._batch = batch

    def append(self, seconds: float = 0.0):
        """Queue the batch's current positions and contacts as the next frame."""
        _check(lib().rp_traj_append(self._h, self._batch._h, float(seconds)))

    def close(self) -> int:
        """Write the queued frames, close the file; returns the frame count."""
        if not self._h:
            return 0
        n = C.c_int32()
        h, self._h = self._h, None
        _check(lib().rp_traj_close(h, C.byref(n)))
        return n.value

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_rodtraj(path: str) -> dict:
    """Parse a .rodtraj file: header fields and per-frame seconds, positions
    (rods x particles x 3) and contact points (n x 3)."""
    data = open(path, "rb").read()
    if data[:8] != b"RODTRAJ1":
        raise ValueError("not a RODTRAJ1 file")
    frames, rods, particles = np.frombuffer(data, np.int32, 3, 8)
    radius, fps = np.frombuffer(data, np.float32, 2, 20)
    at = 28
    out = {"num_frames": int(frames), "num_rods": int(rods), "num_particles": int(particles),
           "radius": float(radius), "fps": float(fps), "seconds": [], "positions": [], "contacts": []}
    for _ in range(int(frames)):
        out["seconds"].append(float(np.frombuffer(data, np.float32, 1, at)[0]))
        at += 4
        n = int(rods) * int(particles) * 3
        out["positions"].append(np.frombuffer(data, np.float32, n, at).reshape(int(rods), int(particles), 3))
        at += 4 * n
        nc = int(np.frombuffer(data, np.int32, 1, at)[0])
        at += 4
        out["contacts"].append(np.frombuffer(data, np.float32, 3 * nc, at).reshape(nc, 3))
        at += 12 * nc
    if at != len(data):
        raise ValueError(f"{len(data) - at} trailing bytes")
    return out
