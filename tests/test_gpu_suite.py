"""The reference's own GPU validation suite, run through this library.

`oracle/_ref/rodsim_b200` is the reference's validation driver (src/main.cpp,
src/gpu/gpu_suite.cpp and the case files, compiled unchanged from the
reference's sources) linked against the crs::gpu::Batch binding over this
library; `oracle/_ref/rodsim_ref` is the same driver with the reference's own
CUDA batch built for sm_100a. Each scenario is written once against
gpu::Batch and run end to end (src/gpu/gpu_suite.cpp:836-954).

* In the reference's FP32 operation order this library prints the same
  measured numbers as the reference's own kernel (%.6g, tolerance: equal
  strings) on the contact, incline-2 and incline scenarios, and passes the
  suite's checks.
* With compensated positions and the FP64 friction cone
  (RP_B200_PRECISION=3) the incline at 8 substeps, which the reference marks
  as beyond float ("slip angle 13.5 %"), lands inside its bounds (slip angle
  5 %, effective mu while sliding 8 %): the contact constraint is measured on
  the compensated positions. The capstan agrees with the colour-ordered FP64
  CPU solver within the suite's agreement bound (0.01).
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
LINE = re.compile(r"^ {4}(\S.*?)\s+GPU (\S+)\s+CPU (\S+)\s+\(diff (\S+)\)$")
SCENARIO = re.compile(r"^  (\S+): \S+ s on the GPU")


def run_suite(binary, scenarios, precision=None, cpu=False, timeout=900):
    path = os.path.join(REF, binary)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (reference sources absent)")
    env = dict(os.environ, CRS_GPU_SUITE_ONLY=",".join(scenarios))
    if not cpu:
        env["CRS_GPU_SUITE_NO_CPU"] = "1"
    env.pop("RP_B200_PRECISION", None)
    if precision is not None:
        env["RP_B200_PRECISION"] = str(precision)
    r = subprocess.run([path, "gpu-suite", "--no-out"], env=env, capture_output=True, text=True,
                       timeout=timeout)
    values, scenario = {}, None
    for line in r.stdout.splitlines():
        h = SCENARIO.match(line)
        if h:
            scenario = h.group(1)
        m = LINE.match(line)
        if m:
            values[(scenario, m.group(1))] = (m.group(2), m.group(3), float(m.group(4)))
    return r.returncode, values, r.stdout


def test_reference_order_prints_the_reference_kernels_numbers():
    scenarios = ["contact", "incline-2", "incline"]
    rc, ours, out = run_suite("rodsim_b200", scenarios)
    rc_ref, ref, _ = run_suite("rodsim_ref", scenarios)
    assert rc == 0, out  # the suite's own checks
    assert len(ours) == 6 and set(ours) == set(ref)
    for name in ours:
        assert ours[name][0] == ref[name][0], (name, ours[name], ref[name])


def test_mixed_precision_incline_within_tolerance():
    _, fp32, _ = run_suite("rodsim_b200", ["incline"])
    _, mixed, out = run_suite("rodsim_b200", ["incline"], precision=3)
    slip = ("incline", "slip angle vs atan(mu) (relative)")
    mu = ("incline", "effective mu while sliding (relative)")
    print(f"\nincline at 8 substeps: FP32 slip {fp32[slip][0]} mu {fp32[mu][0]}; "
          f"mixed slip {mixed[slip][0]} mu {mixed[mu][0]}")
    assert float(fp32[slip][0]) > 0.05  # the float limit the reference reports
    # the reference's own bounds for the incline (src/gpu/gpu_suite.cpp:640-645)
    assert float(mixed[slip][0]) <= 0.05
    assert float(mixed[mu][0]) <= 0.08


def test_mixed_precision_capstan_agrees_with_fp64_cpu():
    _, vals, out = run_suite("rodsim_b200", ["capstan"], precision=3, cpu=True)
    assert len(vals) == 2, out
    for name, (gpu, cpu, diff) in vals.items():
        assert abs(diff) <= 0.01, (name, gpu, cpu)


@pytest.mark.parametrize("case", ["gpu-parity", "gpu-determinism"])
def test_reference_acceptance_cases_pass(case):
    """The reference's own GPU acceptance cases (src/gpu/gpu_cases.cpp:126-607)
    run unchanged against this library: GPU vs CPU after one and 200 steps,
    contact and material scales, self-collision restarts, strategies agreeing
    exactly, bitwise determinism across runs."""
    path = os.path.join(REF, "rodsim_b200")
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (reference sources absent)")
    env = dict(os.environ)
    env.pop("RP_B200_PRECISION", None)
    r = subprocess.run([path, case, "--no-out"], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "PASS: 0 failed check(s)" in r.stdout, r.stdout[-3000:]
    assert "[SKIP]" not in r.stdout


def test_mixed_precision_twist_buckling_converges_at_the_reference_order():
    """Twist buckling (Michell/Greenhill threshold from growth rates, n = 16,
    24, 32): the reference marks it beyond float ("a substep moves the rod
    ~1e-9 m, below float spacing") and its GPU path measures convergence
    order 0.31. With compensated positions and frames the thresholds meet the
    suite's bounds and the order lands in its range 1.7..2.3."""
    _, vals, out = run_suite("rodsim_b200", ["twist-buckling"], precision=3, timeout=1500)
    get = lambda q: float(vals[("twist-buckling", q)][0])
    order = get("buckling threshold convergence order")
    print(f"\ntwist buckling (mixed): thresholds {get('buckling threshold, n = 16'):.5g} "
          f"{get('buckling threshold, n = 24'):.5g} {get('buckling threshold, n = 32'):.5g}, order {order:.3f}")
    assert 1.7 <= order <= 2.3
    assert get("buckling threshold, n = 16") <= 0.02
    assert get("buckling threshold, n = 24") <= 0.02
    assert get("buckling threshold, n = 32") <= 0.01


def test_mixed_precision_cantilever_matches_the_analytic_tip():
    """Tip-load cantilever and elastica by XPBD relaxation: beyond float for
    the reference (tip vs Euler-Bernoulli 3.8 %); with compensated positions
    and frames inside the CPU case's tolerances (1 % and 0.5 % of L)."""
    _, vals, out = run_suite("rodsim_b200", ["tip-load"], precision=3)
    eb = float(vals[("tip-load", "cantilever tip vs Euler-Bernoulli")][0])
    ela = float(vals[("tip-load", "elastica tip vs exact, alpha 0.5-5 (/L)")][0])
    print(f"\ncantilever (mixed): tip vs Euler-Bernoulli {eb:.4g}, elastica {ela:.4g}")
    assert eb <= 0.01
    assert ela <= 0.005
