"""A robot routing a wire harness, learned on the device.

The task mirrors the reference's HarnessTask (src/apps/harness_routing.h:27-97,
harness_routing.cpp:10-154): a cable plugged into a connector at one end, its
other end held by a gripper that must lay it below peg A, above peg B and
through a clip, following a few waypoints on a fixed schedule; the cable's
stiffness and the board's friction vary from cable to cable.

The learning loop mirrors runHarnessLearning (src/validation/
application_cases.cpp:338-481): a cross-entropy method over the 10 waypoint
coordinates, each iteration trying `population` motions on random cables in one
batch and refitting to the best tenth. What changes is where the work runs.
The reference uploads every rod's gripper velocity from the host once per
control tick (attemptsOnGpu, application_cases.cpp:220-262: 630 uploads per
attempt batch) and downloads all positions to score them on the host. Here
each rod's motion is an on-device waypoint schedule (rp_waypoint_drive), the
whole attempt runs as graph replays with no host traffic, and the routing
outcome is computed on the device (rp_batch_evaluate_harness): only the
outcomes come back. The velocities and outcomes equal the reference's host
computations bit for bit, so an attempt batch here equals the reference's
upload-per-tick pattern run on this library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import (Batch, HarnessBoard, Material, Primitive, Rod, StepParams, Strategy, WaypointDrive, World)

WAYPOINTS = 5


@dataclass
class HarnessTask:
    """Board, cable and schedule (reference HarnessTask, harness_routing.h:27-76)."""
    connector: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    peg_a: Tuple[float, float, float] = (0.25, -0.06, 0.0)
    peg_b: Tuple[float, float, float] = (0.55, 0.06, 0.0)
    clip: Tuple[float, float, float] = (0.85, 0.0, 0.0)
    peg_radius: float = 0.012
    peg_height: float = 0.06
    clip_post_radius: float = 0.006
    clip_half_gap: float = 0.018
    clip_height: float = 0.04
    board_friction: float = 0.5
    cable_length: float = 1.2
    segments: int = 120
    cable_youngs: float = 5e6
    leg_seconds: Tuple[float, ...] = (2.4, 0.7, 0.7, 0.8, 0.7)
    hold_seconds: float = 1.0
    steps_per_control: int = 10

    # ---- the cable, the board, the solver (harness_routing.cpp:10-67) ----
    def material(self, youngs_scale: float = 1.0) -> Material:
        return Material(youngs=self.cable_youngs * youngs_scale, poisson=0.35, density=1100.0, radius=0.004)

    def build(self, youngs_scale: float = 1.0) -> Rod:
        """The cable off the board edge, from the connector towards -y; particle
        0 plugged in, the last held by the gripper (both pinned)."""
        m = self.material(youngs_scale)
        start = (self.connector[0], self.connector[1], self.connector[2] + m.radius)
        rod = Rod.straight(self.segments, self.cable_length, m, origin=start, direction=(0.0, -1.0, 0.0))
        rod.pin_particle(0)
        rod.pin_particle(self.segments)
        return rod

    def world(self, friction_scale: float = 1.0) -> World:
        mu = self.board_friction * friction_scale
        prims = [Primitive.plane((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), mu)]
        for peg in (self.peg_a, self.peg_b):
            prims.append(Primitive.capsule(peg, (peg[0], peg[1], peg[2] + self.peg_height), self.peg_radius, mu))
        for side in (-1.0, 1.0):
            post = (self.clip[0], self.clip[1] + side * self.clip_half_gap, self.clip[2])
            prims.append(Primitive.capsule(post, (post[0], post[1], post[2] + self.clip_height),
                                           self.clip_post_radius, mu))
        return World(prims)

    def params(self) -> StepParams:
        """4 substeps x 4 sweeps at dt 1 ms (harness_routing.cpp:44-57)."""
        return StepParams(dt=1e-3, substeps=4, iterations=4, gravity=(0.0, 0.0, -9.81))

    def steps(self) -> int:
        total = self.hold_seconds
        for s in self.leg_seconds:
            total += s
        return int(round(total / 1e-3))

    def hand_written_policy(self) -> np.ndarray:
        """Straight at the targets (harness_routing.cpp:69-75); (5, 2)."""
        return np.array([(self.peg_a[0], self.peg_a[1] - 0.08), (0.40, 0.0),
                         (self.peg_b[0], self.peg_b[1] + 0.08),
                         (self.clip[0] - 0.10, 0.0), (self.clip[0] + 0.18, 0.0)], np.float64)

    # ---- the gripper's motion as an on-device schedule ----
    def drive(self, policy) -> WaypointDrive:
        """The gripper following `policy` ((5, 2) waypoints), as the schedule
        HarnessTask::gripperVelocity samples (harness_routing.cpp:81-106)."""
        p = np.asarray(policy, np.float64).reshape(WAYPOINTS, 2)
        start = (self.connector[0], self.connector[1] - self.cable_length)
        return WaypointDrive(particle=self.segments, start=start, waypoints=[tuple(w) for w in p],
                             legs=list(self.leg_seconds), height=self.material().radius, dt=1e-3,
                             steps_per_control=self.steps_per_control)

    def board(self) -> HarnessBoard:
        return HarnessBoard(peg_a=self.peg_a[:2], peg_b=self.peg_b[:2], clip=self.clip[:2],
                            peg_radius=self.peg_radius, clip_half_gap=self.clip_half_gap,
                            clip_height=self.clip_height, cable_radius=self.material().radius,
                            lay_slack=0.015)

    # ---- the learner's parametrisation (application_cases.cpp:280-298) ----
    def to_policy(self, v) -> np.ndarray:
        """10 numbers to waypoints, each pulled back to within the cable's reach
        of the connector."""
        w = np.asarray(v, np.float64).reshape(WAYPOINTS, 2).copy()
        c = np.asarray(self.connector[:2], np.float64)
        for k in range(WAYPOINTS):
            d = w[k] - c
            reach = math.sqrt(d[0] * d[0] + d[1] * d[1])
            if reach > self.cable_length:
                w[k] = c + d * (self.cable_length / reach)
        return w


def random_cables(rng: np.random.Generator, n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Stiffness 0.4..4x log-uniform, friction 0.6..1.4x (application_cases.cpp:300-309)."""
    youngs = (0.4 * 10.0 ** rng.uniform(0.0, 1.0, n)).astype(np.float32)
    friction = (0.6 + 0.8 * rng.uniform(0.0, 1.0, n)).astype(np.float32)
    return youngs, friction


class Attempts:
    """One batch of attempts: rod r follows policies[r] on a cable with
    youngs[r], friction[r]. Reusable across CEM iterations of one size (the
    batch, its graph and its buffers stay on the device)."""

    def __init__(self, task: HarnessTask, count: int, strategy: Strategy = Strategy.BATCHED,
                 graph: bool = True, autotune: bool = True):
        self.task = task
        self.count = count
        self.proto = task.build()
        self.batch = Batch.create(self.proto, count, strategy, task.world())
        self._params = task.params()
        self._board = task.board()
        if autotune and strategy == Strategy.BATCHED:
            # the launch shape for this batch (the state is restored after)
            self.batch.autotune(self._params, max_steps_per_launch=4)
        self.batch.set_graph(graph)

    def run(self, policies, youngs, friction) -> np.ndarray:
        """Reset every cable, run the whole schedule, return the outcomes."""
        b = self.batch
        b.upload(self.proto)
        b.set_material_scales(youngs, friction)
        b.set_waypoint_drives([self.task.drive(p) for p in policies])
        b.step_many(self._params, self.task.steps())
        return b.evaluate_harness(self._board)

    def close(self):
        self.batch.close()


@dataclass
class LearningResult:
    mean: np.ndarray
    history: List[dict] = field(default_factory=list)
    learned_rate: float = 0.0
    hand_rate: float = 0.0
    seconds: float = 0.0
    # the final comparison: fresh cables and both motions' outcomes on them
    fresh_youngs: Optional[np.ndarray] = None
    fresh_friction: Optional[np.ndarray] = None
    learned_outcomes: Optional[np.ndarray] = None
    hand_outcomes: Optional[np.ndarray] = None


def learn(task: Optional[HarnessTask] = None, population: int = 1024, iterations: int = 10,
          seed: int = 20260917, sigma0: float = 0.08, sigma_floor: float = 0.003,
          strategy: Strategy = Strategy.BATCHED) -> LearningResult:
    """Cross-entropy method over the waypoints (runHarnessLearning,
    application_cases.cpp:352-447), then the learned and the hand-written
    motions on the same fresh random cables."""
    import time
    task = task or HarnessTask()
    rng = np.random.default_rng(seed)
    elites = population // 10
    mean = task.hand_written_policy().reshape(-1)
    sigma = np.full(mean.shape, sigma0)
    att = Attempts(task, population, strategy)
    res = LearningResult(mean=mean)
    try:
        for it in range(iterations):
            samples = np.stack([task.to_policy(mean + sigma * rng.standard_normal(mean.shape)).reshape(-1)
                                for _ in range(population)])
            youngs, friction = random_cables(rng, population)
            t0 = time.perf_counter()
            out = att.run(samples.reshape(population, WAYPOINTS, 2), youngs, friction)
            dt = time.perf_counter() - t0
            res.seconds += dt
            res.history.append(dict(iteration=it, success_rate=float(out["success"].mean()),
                                    mean_score=float(out["score"].mean()), seconds=dt))
            order = np.argsort(-out["score"], kind="stable")[:elites]
            e = samples[order]
            mean = e.mean(axis=0)
            sigma = np.maximum(np.sqrt(((e - mean) ** 2).mean(axis=0)), sigma_floor)
        res.mean = mean
        learned = task.to_policy(mean)
        youngs, friction = random_cables(rng, population)
        res.fresh_youngs, res.fresh_friction = youngs, friction
        res.learned_outcomes = att.run([learned] * population, youngs, friction)
        res.hand_outcomes = att.run([task.hand_written_policy()] * population, youngs, friction)
        res.learned_rate = float(res.learned_outcomes["success"].mean())
        res.hand_rate = float(res.hand_outcomes["success"].mean())
    finally:
        att.close()
    return res
