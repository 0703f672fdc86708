"""Oracle bindings -- TEST INFRASTRUCTURE ONLY.

The checker the GPU path is compared against. Only tests/, the smoke check in
``__graft_entry__.py`` and the CPU-baseline leg of ``bench.py`` import this
package; the shipped library (``ropephysics_b200``) never does.

Three native libraries are bound here, all built by ``oracle/Makefile``:

* ``liboracle_f64.so`` -- this repository's C++ restatement of the reference
  FP64 CPU solver (``rod_oracle.cpp``; each function cites the reference
  file:line it restates). ``liboracle_f32.so`` is the same source in single
  precision, ``liboracle_count.so`` the same source with an op-counting scalar.
* ``_ref/libcrs_ref.so`` -- the reference's own CPU solver compiled from its
  sources (``src/core``), reached through ``ref_shim.cpp``. It pins the
  restatement. ``_ref/libcrs_ref_gpu.so`` adds the reference's CUDA batch
  (``src/gpu``) built for sm_100a, for parity against its FP32 GPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_i32p = C.POINTER(C.c_int32)


def _rod_struct(real):
    rp = C.POINTER(real)

    class OrcRod(C.Structure):
        _fields_ = [
            ("nP", C.c_int32), ("nS", C.c_int32), ("nSt", C.c_int32), ("nB", C.c_int32),
            ("x", rp), ("xPrev", rp), ("v", rp), ("invMass", rp), ("mass", rp),
            ("extForce", rp), ("kinVel", rp),
            ("q", rp), ("qPrev", rp), ("omega", rp), ("invInertia", rp), ("inertia", rp),
            ("extTorque", rp),
            ("sP0", _i32p), ("sP1", _i32p), ("sSeg", _i32p),
            ("sRest", rp), ("sComp", rp), ("sLam", rp),
            ("bA", _i32p), ("bB", _i32p),
            ("bRest", rp), ("bRestD", rp), ("bComp", rp), ("bLam", rp),
            ("radius", real), ("youngs", real), ("poisson", real), ("density", real),
        ]
    return OrcRod


OrcRod64 = _rod_struct(C.c_double)
OrcRod32 = _rod_struct(C.c_float)


class OrcColoring(C.Structure):
    _fields_ = [("count", C.c_int32), ("numColors", C.c_int32),
                ("order", _i32p), ("colorStart", _i32p)]


class OrcPrim(C.Structure):
    _fields_ = [("type", C.c_int32), ("pad", C.c_int32),
                ("a", C.c_double * 3), ("b", C.c_double * 3), ("normal", C.c_double * 3),
                ("halfExtents", C.c_double * 3), ("rotation", C.c_double * 4),
                ("radius", C.c_double), ("friction", C.c_double)]


class OrcWorld(C.Structure):
    _fields_ = [("prims", C.POINTER(OrcPrim)), ("numPrims", C.c_int32),
                ("selfCollision", C.c_int32), ("selfFriction", C.c_double),
                ("selfSkip", C.c_int32), ("hashTableSize", C.c_int32),
                ("contactMarginRadii", C.c_double)]


def _contact_struct(real):
    class OrcContact(C.Structure):
        _fields_ = [("idx", C.c_int32 * 4), ("weight", real * 4), ("normal", real * 3),
                    ("offset", real), ("friction", real), ("lambdaN", real),
                    ("appliedTangential", real), ("count", C.c_int32),
                    ("frictionState", C.c_int32), ("prim", C.c_int32), ("pad", C.c_int32)]
    return OrcContact


OrcContact64 = _contact_struct(C.c_double)
OrcContact32 = _contact_struct(C.c_float)


class OrcParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("substeps", C.c_int32), ("iterations", C.c_int32),
                ("gravity", C.c_double * 3), ("linearDamping", C.c_double),
                ("angularDamping", C.c_double), ("contactInterval", C.c_int32),
                ("pad", C.c_int32), ("stretchColoring", C.POINTER(OrcColoring)),
                ("bendColoring", C.POINTER(OrcColoring))]


def _context_struct(contact):
    class OrcContext(C.Structure):
        _fields_ = [("contacts", C.POINTER(contact)), ("count", C.c_int32),
                    ("capacity", C.c_int32), ("overflow", C.c_int32), ("pad", C.c_int32)]
    return OrcContext


OrcContext64 = _context_struct(OrcContact64)
OrcContext32 = _context_struct(OrcContact32)

# ----------------------------------------------------------------------------- data


@dataclass
class Primitive:
    """A world primitive (reference src/core/geometry.h:17-65)."""
    type: int  # 0 plane, 1 sphere, 2 capsule, 3 box
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
        n = n * (1.0 / np.sqrt(n @ n))  # makePlane normalizes (geometry.h:30-37)
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

    def to_c(self) -> OrcPrim:
        p = OrcPrim()
        p.type = self.type
        p.a[:] = list(map(float, self.a))
        p.b[:] = list(map(float, self.b))
        p.normal[:] = list(map(float, self.normal))
        p.halfExtents[:] = list(map(float, self.half_extents))
        p.rotation[:] = list(map(float, self.rotation))
        p.radius = float(self.radius)
        p.friction = float(self.friction)
        return p


@dataclass
class World:
    """CollisionWorld (reference src/core/collision.h:83-106)."""
    primitives: list = field(default_factory=list)
    self_collision: bool = False
    self_friction: float = 0.0
    self_skip: int = 2
    hash_table_size: int = 4096
    contact_margin_radii: float = 0.25

    def to_c(self):
        arr = (OrcPrim * max(1, len(self.primitives)))(*[p.to_c() for p in self.primitives])
        w = OrcWorld()
        w.prims = C.cast(arr, C.POINTER(OrcPrim))
        w.numPrims = len(self.primitives)
        w.selfCollision = int(self.self_collision)
        w.selfFriction = float(self.self_friction)
        w.selfSkip = int(self.self_skip)
        w.hashTableSize = int(self.hash_table_size)
        w.contactMarginRadii = float(self.contact_margin_radii)
        w._keep = arr
        return w


@dataclass
class Params:
    """SolverParams (reference src/core/solver.h:15-37)."""
    dt: float = 1e-3
    substeps: int = 10
    iterations: int = 1
    gravity: Sequence[float] = (0.0, 0.0, -9.81)
    linear_damping: float = 0.0
    angular_damping: float = 0.0
    contact_interval: int = 1


class Rod:
    """A rod as numpy structure-of-arrays (reference src/core/rod.h:49-121),
    in float64 (or float32 for the float oracle). Capacity leaves room for two
    ghost frames and two ghost bends (clampEndExact at both ends)."""

    FIELDS_P = ("x", "xPrev", "v", "extForce", "kinVel")
    FIELDS_S = ("omega", "invInertia", "inertia", "extTorque")

    def __init__(self, nP: int, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        nS = nP - 1
        capS, capB = nS + 2, nS + 1
        z = lambda *shape: np.zeros(shape, self.dtype)
        self.x, self.xPrev, self.v = z(nP, 3), z(nP, 3), z(nP, 3)
        self.invMass, self.mass = z(nP), z(nP)
        self.extForce, self.kinVel = z(nP, 3), z(nP, 3)
        self.q, self.qPrev = z(capS, 4), z(capS, 4)
        self.omega, self.invInertia, self.inertia, self.extTorque = (z(capS, 3), z(capS, 3),
                                                                      z(capS, 3), z(capS, 3))
        self.sP0 = np.zeros(nS, np.int32)
        self.sP1 = np.zeros(nS, np.int32)
        self.sSeg = np.zeros(nS, np.int32)
        self.sRest, self.sComp, self.sLam = z(nS), z(nS, 3), z(nS, 3)
        self.bA = np.zeros(capB, np.int32)
        self.bB = np.zeros(capB, np.int32)
        self.bRest, self.bRestD, self.bComp, self.bLam = z(capB), z(capB, 3), z(capB, 3), z(capB, 3)
        S = OrcRod64 if self.dtype == np.float64 else OrcRod32
        self.c = S()
        self.c.nP, self.c.nS, self.c.nSt, self.c.nB = nP, nS, nS, nS - 1
        real = C.c_double if self.dtype == np.float64 else C.c_float
        for name, _ in S._fields_:
            arr = getattr(self, name, None)
            if isinstance(arr, np.ndarray):
                ct = C.c_int32 if arr.dtype == np.int32 else real
                setattr(self.c, name, arr.ctypes.data_as(C.POINTER(ct)))

    # sizes live in the C struct (builders and clamps update them)
    nP = property(lambda s: s.c.nP)
    nS = property(lambda s: s.c.nS)
    nSt = property(lambda s: s.c.nSt)
    nB = property(lambda s: s.c.nB)
    radius = property(lambda s: float(s.c.radius))

    def copy(self, dtype=None) -> "Rod":
        r = Rod(self.x.shape[0], dtype or self.dtype)
        for name, _ in OrcRod64._fields_:
            a = getattr(self, name, None)
            if isinstance(a, np.ndarray):
                getattr(r, name)[...] = a
        for f in ("nP", "nS", "nSt", "nB", "radius", "youngs", "poisson", "density"):
            setattr(r.c, f, getattr(self.c, f))
        return r

    def state(self):
        """Positions (nP,3), frames (nS,4) -- the compared outputs."""
        return self.x[: self.nP].copy(), self.q[: self.nS].copy()


class Coloring:
    def __init__(self, order: np.ndarray, color_start: np.ndarray):
        self.order = np.ascontiguousarray(order, np.int32)
        self.color_start = np.ascontiguousarray(color_start, np.int32)
        self.c = OrcColoring()
        self.c.count = len(self.order)
        self.c.numColors = len(self.color_start) - 1
        self.c.order = self.order.ctypes.data_as(_i32p)
        self.c.colorStart = self.color_start.ctypes.data_as(_i32p)

    @property
    def num_colors(self):
        return len(self.color_start) - 1


class Context:
    """Per-rod contact scratch (reference src/core/solver.h:41-44)."""

    def __init__(self, capacity: int = 4096, dtype=np.float64):
        ct = OrcContact64 if np.dtype(dtype) == np.float64 else OrcContact32
        cx = OrcContext64 if np.dtype(dtype) == np.float64 else OrcContext32
        self.buf = (ct * capacity)()
        self.c = cx()
        self.c.contacts = C.cast(self.buf, C.POINTER(ct))
        self.c.capacity = capacity

    def contacts(self):
        out = []
        for i in range(self.c.count):
            k = self.buf[i]
            out.append(dict(idx=tuple(k.idx[: k.count]), weight=tuple(k.weight[: k.count]),
                            normal=tuple(k.normal), offset=k.offset, friction=k.friction,
                            lambdaN=k.lambdaN, count=k.count, friction_state=k.frictionState,
                            prim=k.prim))
        return out


# ----------------------------------------------------------------------------- library


def _load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    return C.CDLL(path)


class Oracle:
    """This repository's CPU restatement (liboracle_{f64,f32,count}.so)."""

    def __init__(self, variant: str = "f64"):
        self.variant = variant
        self.dtype = np.float32 if variant == "f32" else np.float64
        self.lib = _load(f"liboracle_{variant}.so")
        L = self.lib
        RP = C.POINTER(OrcRod32 if variant == "f32" else OrcRod64)
        CX = C.POINTER(OrcContext32 if variant == "f32" else OrcContext64)
        d3 = C.POINTER(C.c_double)
        L.orc_build_straight.argtypes = [RP, C.c_int32, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_double, d3, d3]
        L.orc_build_centerline.argtypes = [RP, d3, C.c_int32, C.c_double, C.c_double, C.c_double,
                                           C.c_double, d3, C.c_double]
        L.orc_clamp_end.argtypes = [RP, C.c_int32]
        L.orc_set_rest_from_current.argtypes = [RP]
        L.orc_pin_particle.argtypes = [RP, C.c_int32]
        L.orc_color_stretch.argtypes = [RP, C.POINTER(OrcColoring)]
        L.orc_color_bend.argtypes = [RP, C.POINTER(OrcColoring)]
        L.orc_self_gap.argtypes = [RP, C.POINTER(OrcWorld)]
        L.orc_generate_contacts.argtypes = [RP, C.POINTER(OrcWorld), CX]
        L.orc_step.argtypes = [RP, C.POINTER(OrcParams)]
        L.orc_step_world.argtypes = [RP, C.POINTER(OrcParams), C.POINTER(OrcWorld), CX]
        L.orc_op_counts.argtypes = [C.POINTER(C.c_uint64)]
        self._RP = RP

    @staticmethod
    def _d3(v):
        return (C.c_double * 3)(*map(float, v))

    def straight(self, n, length, youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3,
                 origin=(0, 0, 0), direction=(1, 0, 0)) -> Rod:
        rod = Rod(n + 1, self.dtype)
        rc = self.lib.orc_build_straight(C.byref(rod.c), n, length, youngs, poisson, density,
                                         radius, self._d3(origin), self._d3(direction))
        assert rc == 0
        return rod

    def centerline(self, points, youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3,
                   frame_seed=(0, 0, 1), twist_per_length=0.0) -> Rod:
        pts = np.ascontiguousarray(points, np.float64)
        rod = Rod(len(pts), self.dtype)
        rc = self.lib.orc_build_centerline(C.byref(rod.c),
                                           pts.ctypes.data_as(C.POINTER(C.c_double)), len(pts),
                                           youngs, poisson, density, radius,
                                           self._d3(frame_seed), float(twist_per_length))
        assert rc == 0
        return rod

    def clamp(self, rod: Rod, tip: bool = False) -> int:
        return self.lib.orc_clamp_end(C.byref(rod.c), int(tip))

    def set_rest_from_current(self, rod: Rod):
        self.lib.orc_set_rest_from_current(C.byref(rod.c))

    def pin(self, rod: Rod, i: int):
        self.lib.orc_pin_particle(C.byref(rod.c), i)

    def coloring(self, rod: Rod, bend: bool) -> Coloring:
        n = rod.nB if bend else rod.nSt
        order = np.zeros(max(1, n), np.int32)
        starts = np.zeros(n + 2, np.int32)
        col = Coloring(order, starts)
        (self.lib.orc_color_bend if bend else self.lib.orc_color_stretch)(C.byref(rod.c),
                                                                          C.byref(col.c))
        return Coloring(order[:n], starts[: col.c.numColors + 1])

    def self_gap(self, rod: Rod, world: World) -> int:
        w = world.to_c()
        return self.lib.orc_self_gap(C.byref(rod.c), C.byref(w))

    def generate_contacts(self, rod: Rod, world: World, ctx: Optional[Context] = None):
        ctx = ctx or Context(dtype=self.dtype)
        w = world.to_c()
        self.lib.orc_generate_contacts(C.byref(rod.c), C.byref(w), C.byref(ctx.c))
        return ctx

    def params_c(self, p: Params, rod: Optional[Rod] = None, colored: bool = False):
        c = OrcParams()
        c.dt = p.dt
        c.substeps = p.substeps
        c.iterations = p.iterations
        c.gravity[:] = list(map(float, p.gravity))
        c.linearDamping = p.linear_damping
        c.angularDamping = p.angular_damping
        c.contactInterval = p.contact_interval
        keep = []
        if colored:
            sc, bc = self.coloring(rod, False), self.coloring(rod, True)
            c.stretchColoring = C.pointer(sc.c)
            c.bendColoring = C.pointer(bc.c)
            keep = [sc, bc]
        c._keep = keep
        return c

    def step(self, rod: Rod, p: Params, world: Optional[World] = None,
             ctx: Optional[Context] = None, colored: bool = True, steps: int = 1):
        """`colored` runs the sweep in the GPU's colour order (the reference's
        SolverParams::stretchColoring/bendColoring, solver.h:31-36)."""
        pc = self.params_c(p, rod, colored)
        if world is None:
            for _ in range(steps):
                self.lib.orc_step(C.byref(rod.c), C.byref(pc))
            return None
        ctx = ctx or Context(dtype=self.dtype)
        w = world.to_c()
        for _ in range(steps):
            self.lib.orc_step_world(C.byref(rod.c), C.byref(pc), C.byref(w), C.byref(ctx.c))
        return ctx

    def op_counts(self):
        out = (C.c_uint64 * 6)()
        self.lib.orc_op_counts(out)
        return dict(zip(("add", "mul", "div", "sqrt", "cmp", "other"), list(out)))

    def op_reset(self):
        self.lib.orc_op_reset()


class Reference:
    """The reference's own solver compiled from its sources (oracle/_ref)."""

    def __init__(self, gpu: bool = False):
        self.lib = _load(os.path.join("_ref", "libcrs_ref_gpu.so" if gpu else "libcrs_ref.so"))
        L = self.lib
        vp, d3 = C.c_void_p, C.POINTER(C.c_double)
        L.ref_rod_straight.restype = vp
        L.ref_rod_straight.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, d3, d3]
        L.ref_rod_centerline.restype = vp
        L.ref_rod_centerline.argtypes = [d3, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, d3, C.c_double]
        L.ref_rod_hanging.restype = vp
        L.ref_rod_hanging.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double]
        L.ref_rod_free.argtypes = [vp]
        L.ref_rod_from.restype = vp
        L.ref_rod_from.argtypes = [C.POINTER(OrcRod64)]
        L.ref_rod_clamp.argtypes = [vp, C.c_int]
        L.ref_rod_set_rest_from_current.argtypes = [vp]
        L.ref_rod_sizes.argtypes = [vp, C.POINTER(C.c_int)]
        L.ref_rod_export.argtypes = [vp, C.POINTER(OrcRod64)]
        L.ref_rod_import_state.argtypes = [vp, C.POINTER(OrcRod64)]
        L.ref_world_create.restype = vp
        L.ref_world_create.argtypes = [C.POINTER(OrcPrim), C.c_int, C.c_int, C.c_double, C.c_int,
                                       C.c_int, C.c_double]
        L.ref_world_free.argtypes = [vp]
        L.ref_self_gap.argtypes = [vp, vp]
        L.ref_coloring.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_step.argtypes = [vp, vp, C.c_double, C.c_int, C.c_int, d3, C.c_double, C.c_double,
                               C.c_int, C.c_int, C.c_int]
        L.ref_step_many.restype = C.c_double
        L.ref_step_many.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int, C.c_double, C.c_int,
                                    C.c_int, d3, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        L.ref_generate_contacts.argtypes = [vp, vp, C.POINTER(C.c_int), d3, d3, d3, C.c_int]
        L.ref_hold_many.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int, C.c_double, C.c_int, C.c_int,
                                    d3, C.c_int, C.c_int, C.c_int, d3, C.POINTER(C.c_int)]
        L.ref_contacts.argtypes = [vp, C.POINTER(C.c_int), d3, d3, d3, C.c_int]
        L.ref_harness_steps.restype = C.c_int
        L.ref_harness_hand_policy.argtypes = [d3]
        L.ref_harness_velocity.argtypes = [d3, C.c_int, d3]
        L.ref_harness_evaluate.argtypes = [C.POINTER(C.c_float), C.c_int, d3, C.POINTER(C.c_int)]
        L.ref_harness_build.restype = vp
        L.ref_harness_build.argtypes = [C.c_double]
        L.ref_harness_world.restype = vp
        L.ref_harness_world.argtypes = [C.c_double]
        L.ref_harness_attempt_cpu.argtypes = [d3, C.c_double, C.c_double, d3, C.POINTER(C.c_int), d3]
        self.gpu = gpu
        if gpu:
            L.refgpu_create.restype = vp
            L.refgpu_create.argtypes = [vp, C.c_int, C.c_int, vp]
            L.refgpu_free.argtypes = [vp]
            L.refgpu_step.argtypes = [vp, C.c_double, C.c_int, C.c_int, d3, C.c_double,
                                      C.c_double, C.c_int, C.c_int]
            L.refgpu_sync.argtypes = [vp]
            L.refgpu_download.argtypes = [vp, C.c_int, vp]
            L.refgpu_upload_rod.argtypes = [vp, C.c_int, vp]
            L.refgpu_set_loads.argtypes = [vp, C.c_int, vp]
            L.refgpu_set_kinematic.argtypes = [vp, C.POINTER(C.c_float), C.c_long]
            L.refgpu_set_material_scales.argtypes = [vp, C.POINTER(C.c_float),
                                                     C.POINTER(C.c_float), C.c_int]
            L.refgpu_download_positions.argtypes = [vp, C.POINTER(C.c_float)]
            L.refgpu_overflow.restype = C.c_longlong
            L.refgpu_overflow.argtypes = [vp]
            L.refgpu_self_pairs.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.c_int]
            L.refgpu_contact_active.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
            fp = C.POINTER(C.c_float)
            L.refgpu_download_state.argtypes = [vp, fp, fp, fp, fp]

    # ---- the harness-routing task (src/apps/harness_routing.h:27-97) ----
    @staticmethod
    def _outcome(d, f):
        return dict(score=d[0], side_a=d[1], side_b=d[2], clip_miss=d[3], below_a=bool(f[0]),
                    above_b=bool(f[1]), through_clip=bool(f[2]), success=bool(f[3]))

    def harness_hand_policy(self) -> np.ndarray:
        p = np.zeros(10)
        self.lib.ref_harness_hand_policy(p.ctypes.data_as(C.POINTER(C.c_double)))
        return p.reshape(5, 2)

    def harness_velocity(self, policy, step: int) -> np.ndarray:
        """HarnessTask::gripperVelocity in double."""
        p = np.ascontiguousarray(policy, np.float64).reshape(10)
        v = np.zeros(3)
        d3 = C.POINTER(C.c_double)
        self.lib.ref_harness_velocity(p.ctypes.data_as(d3), int(step), v.ctypes.data_as(d3))
        return v

    def harness_evaluate(self, xyz) -> dict:
        """HarnessTask::evaluate of one cable given as float positions."""
        x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        d = np.zeros(4)
        f = np.zeros(4, np.int32)
        self.lib.ref_harness_evaluate(x.ctypes.data_as(C.POINTER(C.c_float)), len(x),
                                      d.ctypes.data_as(C.POINTER(C.c_double)),
                                      f.ctypes.data_as(C.POINTER(C.c_int)))
        return self._outcome(d, f)

    def harness_attempt_cpu(self, policy, youngs_scale: float, friction_scale: float):
        """One attempt on the FP64 CPU solver (attemptOnCpu); (outcome, positions)."""
        p = np.ascontiguousarray(policy, np.float64).reshape(10)
        d = np.zeros(4)
        f = np.zeros(4, np.int32)
        x = np.zeros((121, 3))
        d3 = C.POINTER(C.c_double)
        self.lib.ref_harness_attempt_cpu(p.ctypes.data_as(d3), float(youngs_scale), float(friction_scale),
                                         d.ctypes.data_as(d3), f.ctypes.data_as(C.POINTER(C.c_int)),
                                         x.ctypes.data_as(d3))
        return self._outcome(d, f), x

    def gpu_self_pairs(self, batch, rod=0, cap=4096):
        """(j, k) pairs of the reference GPU's last self-contact regeneration
        (multi-kernel batches only)."""
        out = np.zeros((cap, 2), np.int32)
        n = self.lib.refgpu_self_pairs(batch, rod, out.ctypes.data_as(C.POINTER(C.c_int)), cap)
        assert n >= 0, "reference batch is not multi-kernel or has no self-collision"
        return [tuple(int(v) for v in p) for p in out[:n]]

    def gpu_state(self, batch, num_rods, num_particles, num_frames):
        """(x, v, q, omega) of every rod of a reference GPU batch, float32,
        shaped (rods, particles, 3) and (rods, frames, 4 | 3)."""
        x = np.zeros((num_rods, num_particles, 3), np.float32)
        v = np.zeros_like(x)
        q = np.zeros((num_rods, num_frames, 4), np.float32)
        w = np.zeros((num_rods, num_frames, 3), np.float32)
        fp = C.POINTER(C.c_float)
        self.lib.refgpu_download_state(batch, x.ctypes.data_as(fp), v.ctypes.data_as(fp), q.ctypes.data_as(fp),
                                       w.ctypes.data_as(fp))
        return x, v, q, w

    def gpu_contact_active(self, batch, rod, num_particles, num_prims):
        out = np.zeros(num_particles * num_prims, np.int32)
        n = self.lib.refgpu_contact_active(batch, rod, out.ctypes.data_as(C.POINTER(C.c_int)))
        assert n >= 0
        return out.reshape(num_particles, num_prims)

    # --- rods (handles to crs::Rod) ---
    def straight(self, n, length, youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3,
                 origin=(0, 0, 0), direction=(1, 0, 0)):
        return self.lib.ref_rod_straight(n, length, youngs, poisson, density, radius,
                                         Oracle._d3(origin), Oracle._d3(direction))

    def centerline(self, points, youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3,
                   frame_seed=(0, 0, 1), twist_per_length=0.0):
        pts = np.ascontiguousarray(points, np.float64)
        return self.lib.ref_rod_centerline(pts.ctypes.data_as(C.POINTER(C.c_double)), len(pts),
                                           youngs, poisson, density, radius,
                                           Oracle._d3(frame_seed), float(twist_per_length))

    def hanging(self, legRatio, youngs, length=1.0, segments=100, bar_radius=0.05, bar_height=0.8):
        """The cable of the reference's cable task (apps/cable_hanging.cpp:18-47)."""
        return self.lib.ref_rod_hanging(length, segments, bar_radius, bar_height, legRatio, youngs)

    def hold_many(self, handles, world_handles, p: Params, steps, interval, threads):
        """Reference HangOutcome verdicts (max rise of particle 0, held) per rod."""
        n = len(handles)
        H = (C.c_void_p * n)(*handles)
        W = (C.c_void_p * n)(*world_handles)
        rise = np.zeros(n)
        held = np.zeros(n, np.int32)
        self.lib.ref_hold_many(H, W, n, p.dt, p.substeps, p.iterations, Oracle._d3(p.gravity), steps,
                               interval, threads, rise.ctypes.data_as(C.POINTER(C.c_double)),
                               held.ctypes.data_as(C.POINTER(C.c_int)))
        return rise, held.astype(bool)

    def from_rod(self, rod: Rod):
        """A reference Rod handle holding exactly `rod`'s arrays."""
        return self.lib.ref_rod_from(C.byref(rod.c))

    def free(self, h):
        self.lib.ref_rod_free(h)

    def export(self, h) -> Rod:
        sizes = (C.c_int * 4)()
        self.lib.ref_rod_sizes(h, sizes)
        nP, nS, nSt, nB = list(sizes)
        rod = Rod(nP, np.float64)
        # the reference rod may carry up to two ghosts; Rod() has that capacity
        assert nS <= rod.q.shape[0] and nB <= rod.bA.shape[0]
        self.lib.ref_rod_export(h, C.byref(rod.c))
        return rod

    def import_state(self, h, rod: Rod):
        self.lib.ref_rod_import_state(h, C.byref(rod.c))

    def world(self, w: World):
        c = w.to_c()
        return self.lib.ref_world_create(c.prims, c.numPrims, c.selfCollision, c.selfFriction,
                                         c.selfSkip, c.hashTableSize, c.contactMarginRadii)

    def coloring(self, h, bend: bool) -> Coloring:
        sizes = (C.c_int * 4)()
        self.lib.ref_rod_sizes(h, sizes)
        n = sizes[3] if bend else sizes[2]
        order = np.zeros(max(n, 1), np.int32)
        starts = np.zeros(n + 2, np.int32)
        nc = self.lib.ref_coloring(h, int(bend), order.ctypes.data_as(C.POINTER(C.c_int)),
                                   starts.ctypes.data_as(C.POINTER(C.c_int)))
        return Coloring(order[:n], starts[: nc + 1])

    def step(self, h, p: Params, world_handle=None, colored=True, steps=1):
        self.lib.ref_step(h, world_handle, p.dt, p.substeps, p.iterations,
                          Oracle._d3(p.gravity), p.linear_damping, p.angular_damping,
                          p.contact_interval, int(colored), steps)

    def contacts(self, h, cap=8192):
        """The contact list the rod's last substep used (its SolverContext)."""
        idx = np.zeros((cap, 4), np.int32)
        w = np.zeros((cap, 4))
        n = np.zeros((cap, 3))
        off = np.zeros(cap)
        D = C.POINTER(C.c_double)
        cnt = self.lib.ref_contacts(h, idx.ctypes.data_as(C.POINTER(C.c_int)), w.ctypes.data_as(D),
                                    n.ctypes.data_as(D), off.ctypes.data_as(D), cap)
        return idx[:cnt], w[:cnt], n[:cnt], off[:cnt]

    def generate_contacts(self, h, world_handle, cap=8192):
        idx = np.zeros((cap, 4), np.int32)
        w = np.zeros((cap, 4))
        n = np.zeros((cap, 3))
        off = np.zeros(cap)
        D = C.POINTER(C.c_double)
        cnt = self.lib.ref_generate_contacts(h, world_handle, idx.ctypes.data_as(C.POINTER(C.c_int)),
                                             w.ctypes.data_as(D), n.ctypes.data_as(D),
                                             off.ctypes.data_as(D), cap)
        return idx[:cnt], w[:cnt], n[:cnt], off[:cnt]
