"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own CPU solver, compiled from its sources by
``make -C oracle ref`` into ``oracle/_ref/libcrs_ref.so``, on the reference's
own validation setups, and writes small fixtures that travel with the repo:

  crosscheck.csv     runCrossCheck (src/validation/cases.cpp:772-806): 16
                     segments, clamped root, dt 1e-3, 4 substeps, 200 steps,
                     index-order sweeps, written like the reference's Csv
                     (12 significant digits). Equal byte for byte to the
                     reference's published docs/data/crosscheck.csv.
  coloring.npz       stretch/bend colourings of the benchmark rod at n = 8, 32,
                     128, 512 (src/gpu/gpu_cases.cpp:88-121).
  parity_cpu.npz     the GPU parity scenarios (gpu_cases.cpp:162-239) run on the
                     colour-ordered FP64 CPU: states after 1, 10 and 50 steps.
  rope_restart.npz   the self-collision restart state of gpu_cases.cpp:437-484
                     (rope pre-stepped until it holds >= 5 self contacts), its
                     contact list, and the state one step later.

Usage: python tests/golden/make_golden.py   (needs the reference's sources --
$RP_REFERENCE, else a checkout beside the repository -- built into oracle/_ref
by ``make -C oracle ref``; the fixtures are committed, so the tests do not.)
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import Params, Primitive, Reference, World  # noqa: E402

MAT = dict(youngs=1e7, poisson=0.35, density=1000.0, radius=5e-3)


def fmt12(v: float) -> str:
    return "%.12g" % v


def crosscheck(ref: Reference):
    h = ref.straight(16, 1.0, **MAT)
    ref.lib.ref_rod_clamp(h, 0)
    ref.step(h, Params(dt=1e-3, substeps=4, iterations=1), colored=False, steps=200)
    rod = ref.export(h)
    lines = ["index,x,y,z,qw,qx,qy,qz"]
    for i in range(rod.nP):
        q = rod.q[i] if i < rod.nS else (1.0, 0.0, 0.0, 0.0)
        lines.append(",".join([str(i)] + [fmt12(v) for v in list(rod.x[i]) + list(q)]))
    ref.free(h)
    with open(os.path.join(HERE, "crosscheck.csv"), "w") as f:
        f.write("\n".join(lines) + "\n")


def coloring(ref: Reference):
    out = {}
    for n in (8, 32, 128, 512):
        h = ref.straight(n, 1.0, **MAT)
        ref.lib.ref_rod_clamp(h, 0)
        for bend in (False, True):
            c = ref.coloring(h, bend)
            key = f"{'bend' if bend else 'stretch'}_{n}"
            out[key + "_order"] = c.order
            out[key + "_start"] = c.color_start
        ref.free(h)
    np.savez_compressed(os.path.join(HERE, "coloring.npz"), **out)


def quat_axis_angle_mul(angle, rest):
    # normalize(quatAxisAngle((1,0,0), angle) * rest), reference op order
    h = angle * 0.5
    w, x, y, z = math.cos(h), math.sin(h), 0.0, 0.0
    rw, rx, ry, rz = rest
    q = [w * rw - (x * rx + y * ry + z * rz), rx * w + x * rw + (y * rz - z * ry),
         ry * w + y * rw + (z * rx - x * rz), rz * w + z * rw + (x * ry - y * rx)]
    n = math.sqrt(((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]) + q[3] * q[3])
    s = 1.0 / n
    return [c * s for c in q]


def parity(ref: Reference):
    world = World([Primitive.plane((0, 0, -0.0051), (0, 0, 1), 0.5),
                   Primitive.sphere((0.5, 0, -0.0851), 0.08, 0.3)])
    wh = ref.world(world)
    p = Params(dt=1e-3, substeps=8, iterations=1)
    out = {}
    for scen in ("gravity", "loaded", "contact"):
        for n in (16, 48):
            h = ref.straight(n, 1.0, **MAT)
            ref.lib.ref_rod_clamp(h, 0)
            rod = ref.export(h)
            root = rod.nS - 1
            rest = rod.q[root].copy()
            if scen == "loaded":
                rod.extForce[rod.nP - 1] = (0.0, 0.02, 0.05)
                rod.extTorque[n // 2] = (2e-3, 0.0, -1e-3)
                rod.kinVel[0] = (0.0, 0.05, 0.1)
                ref.import_state(h, rod)
            done = 0
            for cp in (1, 10, 50):
                while done < cp:
                    if scen == "loaded":
                        rod = ref.export(h)
                        rod.q[root] = quat_axis_angle_mul(0.5e-3 * (done + 1), rest)
                        ref.import_state(h, rod)
                    ref.step(h, p, world_handle=wh if scen == "contact" else None, colored=True)
                    done += 1
                rod = ref.export(h)
                out[f"{scen}_{n}_{cp}_x"] = rod.x[: rod.nP].copy()
                out[f"{scen}_{n}_{cp}_q"] = rod.q[: rod.nS].copy()
            ref.free(h)
    np.savez_compressed(os.path.join(HERE, "parity_cpu.npz"), **out)


def rope(ref: Reference):
    n, L = 150, 1.2
    d = [0.08, 0.03, 1.0]
    s = 1.0 / math.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
    d = [c * s for c in d]
    h = ref.straight(n, L, youngs=2e6, poisson=0.35, density=1000.0, radius=5e-3,
                     origin=(0, 0, 0.02), direction=d)
    rod = ref.export(h)
    rod.x[:, 2] = L + 0.05 - rod.x[:, 2]
    rod.xPrev[...] = rod.x
    ref.import_state(h, rod)
    ref.lib.ref_rod_set_rest_from_current(h)
    world = World([Primitive.plane((0, 0, 0), (0, 0, 1), 0.6)], self_collision=True,
                  self_friction=0.3, hash_table_size=256)
    wh = ref.world(world)
    p = Params(dt=1e-3, substeps=16, iterations=4, linear_damping=1.0, angular_damping=1.0)
    steps = 0
    while steps < 3000:
        ref.step(h, p, world_handle=wh, colored=True)
        steps += 1
        # the list of the step's last substep, as selfContactsIn(ctx) reads it
        idx = ref.contacts(h)[0]
        if int(np.sum(idx[:, 3] >= 0)) >= 5:
            break
    rod = ref.export(h)
    idx, w, nrm, off = ref.generate_contacts(h, wh)
    out = dict(steps=np.int32(steps), x=rod.x[: rod.nP].copy(), v=rod.v[: rod.nP].copy(),
               q=rod.q[: rod.nS].copy(), omega=rod.omega[: rod.nS].copy(),
               s_rest=rod.sRest[: rod.nSt].copy(), b_rest=rod.bRest[: rod.nB].copy(),
               b_rest_darboux=rod.bRestD[: rod.nB].copy(), contact_idx=idx, contact_weight=w)
    ref.step(h, p, world_handle=wh, colored=True)
    rod1 = ref.export(h)
    out["x1"] = rod1.x[: rod1.nP].copy()
    out["q1"] = rod1.q[: rod1.nS].copy()
    np.savez_compressed(os.path.join(HERE, "rope_restart.npz"), **out)
    ref.free(h)


if __name__ == "__main__":
    ref = Reference()
    crosscheck(ref)
    coloring(ref)
    parity(ref)
    rope(ref)
    print("fixtures written to", HERE)
