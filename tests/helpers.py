"""Shared builders and comparisons for the parity tests.

Scenarios follow the reference's own GPU parity cases (src/gpu/gpu_cases.cpp:
126-548): the benchmark cantilever (gpu_cases.cpp:28-33), its loaded variant
(tip force, mid torque, moving root, driven root twist) and its contact
variant (floor 0.1 mm below, sphere under the middle).
"""
from __future__ import annotations

import math

import numpy as np

import ropephysics_b200 as rp
from oracle import Params, Primitive as OPrim, World as OWorld

REF_MAT = dict(youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3)


def product_rod(orod) -> rp.Rod:
    """A product descriptor holding exactly the oracle rod's doubles."""
    n = orod.nP
    return rp.Rod.from_arrays(
        rp.Material(float(orod.c.youngs), float(orod.c.poisson), float(orod.c.density),
                    float(orod.c.radius)),
        x=orod.x[:n], v=orod.v[:n], inv_mass=orod.invMass[:n], mass=orod.mass[:n],
        ext_force=orod.extForce[:n], kin_velocity=orod.kinVel[:n],
        q=orod.q[: orod.nS], omega=orod.omega[: orod.nS], inertia=orod.inertia[: orod.nS],
        inv_inertia=orod.invInertia[: orod.nS], ext_torque=orod.extTorque[: orod.nS],
        s_p0=orod.sP0[: orod.nSt], s_p1=orod.sP1[: orod.nSt], s_seg=orod.sSeg[: orod.nSt],
        s_rest=orod.sRest[: orod.nSt], s_compliance=orod.sComp[: orod.nSt],
        b_a=orod.bA[: orod.nB], b_b=orod.bB[: orod.nB], b_rest=orod.bRest[: orod.nB],
        b_compliance=orod.bComp[: orod.nB], b_rest_darboux=orod.bRestD[: orod.nB])


def sync_loads(prod: rp.Rod, orod):
    """Copy the oracle rod's loads and fixed-frame orientations into `prod`."""
    n = orod.nP
    prod.ext_force[...] = orod.extForce[:n]
    prod.kin_velocity[...] = orod.kinVel[:n]
    prod.ext_torque[...] = orod.extTorque[: orod.nS]
    prod.q[...] = orod.q[: orod.nS]


def oracle_world(w: rp.World) -> OWorld:
    return OWorld([OPrim(p.type, p.a, p.b, p.normal, p.half_extents, p.rotation, p.radius, p.friction)
                   for p in w.primitives], w.self_collision, w.self_friction, w.self_skip,
                  w.hash_table_size, w.contact_margin_radii)


def oparams(p: rp.StepParams) -> Params:
    """Oracle params that run in the same precision as the float GPU params:
    dt, gravity and damping are the float32 values the device sees."""
    f = lambda v: float(np.float32(v))
    return Params(dt=f(p.dt), substeps=p.substeps, iterations=p.iterations,
                  gravity=tuple(f(g) for g in p.gravity), linear_damping=f(p.linear_damping),
                  angular_damping=f(p.angular_damping), contact_interval=p.contact_interval)


def benchmark_rod(oracle, n):
    """gpu_cases.cpp:28-33: 1 m along x, clamped root (ghost frame), E 1e7."""
    r = oracle.straight(n, 1.0, **REF_MAT)
    oracle.clamp(r, False)
    return r


def contact_world() -> rp.World:
    """gpu_cases.cpp:173-177: floor 0.1 mm under the rod, sphere under its middle."""
    return rp.World([rp.Primitive.plane((0, 0, -0.0051), (0, 0, 1), 0.5),
                     rp.Primitive.sphere((0.5, 0, -0.0851), 0.08, 0.3)])


def max_dx(a, b) -> float:
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    return float(np.max(np.linalg.norm(a - b, axis=1))) if len(a) else 0.0


def max_dq(a, b) -> float:
    """Largest quaternion difference on the same hemisphere (gpu_cases.cpp:44-53)."""
    a = np.asarray(a, np.float64).reshape(-1, 4)
    b = np.asarray(b, np.float64).reshape(-1, 4)
    s = np.where(np.sum(a * b, axis=1) < 0, -1.0, 1.0)[:, None]
    return float(np.max(np.linalg.norm(a - b * s, axis=1))) if len(a) else 0.0


def twist_root(orod, root_frame, rest_q, step_index):
    """The loaded scenario's driven root: 0.5 rad/s about x (gpu_cases.cpp:193-197)."""
    orod.q[root_frame] = twisted_root(step_index, rest_q)


def twisted_root(step_index, rest_q):
    """normalize(quatAxisAngle((1,0,0), 0.5e-3 (step+1)) * rest) in the
    reference's operation order (math3.h:245-346)."""
    angle = 0.5e-3 * (step_index + 1)
    h = angle * 0.5
    w, x, y, z = math.cos(h), math.sin(h), 0.0, 0.0
    rw, rx, ry, rz = (float(v) for v in rest_q)
    q = [w * rw - (x * rx + y * ry + z * rz), rx * w + x * rw + (y * rz - z * ry),
         ry * w + y * rw + (z * rx - x * rz), rz * w + z * rw + (x * ry - y * rx)]
    s = 1.0 / math.sqrt(((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]) + q[3] * q[3])
    return np.array([c * s for c in q])


def segment_distance(p1, q1, p2, q2) -> float:
    """Distance between the closest points of two segments (FP64, clamped
    parametric solution of geometry.h:170-207)."""
    p1, q1, p2, q2 = (np.asarray(v, np.float64) for v in (p1, q1, p2, q2))
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = d1 @ d1, d2 @ d2, d2 @ r
    c, b = d1 @ r, d1 @ d2
    denom = a * e - b * b
    s = min(max((b * f - c * e) / denom, 0.0), 1.0) if denom > 1e-30 else 0.0
    t = (b * s + f) / e
    if t < 0.0:
        t, s = 0.0, min(max(-c / a, 0.0), 1.0)
    elif t > 1.0:
        t, s = 1.0, min(max((b - c) / a, 0.0), 1.0)
    return float(np.linalg.norm((p1 + d1 * s) - (p2 + d2 * t)))


def helix_points(n, length, coil_radius, pitch_gap, radius, origin=(0.0, 0.0, 0.0)):
    """n+1 points on a helix of total arc length `length` whose turns are
    separated by `pitch_gap` + 2 radius along the axis."""
    pitch = pitch_gap + 2.0 * radius
    turn_len = math.sqrt((2 * math.pi * coil_radius) ** 2 + pitch ** 2)
    total_angle = 2 * math.pi * length / turn_len
    t = np.linspace(0.0, total_angle, n + 1)
    o = np.asarray(origin, float)
    return np.stack([o[0] + coil_radius * np.cos(t), o[1] + coil_radius * np.sin(t),
                     o[2] + pitch * t / (2 * math.pi)], axis=1)
