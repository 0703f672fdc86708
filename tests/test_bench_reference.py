"""The bench's reference arm on the CPU.

`bench.py --impl reference` times the reference's own FP64 CPU solver on a
bounded sample of the workload. Its rods must come from the reference's own
builders and the workload's seeded draws, never from this library: the
process must neither import ``ropephysics_b200`` nor map ``librp_b200.so``.
Both arms must also describe the same workload with the same config keys.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--rods", "64", "--steps", "1", "--warmup", "1",
            "--cpu-rods", "6", "--cpu-seconds", "0.5"]
runpy.run_path(sys.argv[0], run_name="__main__")
maps = open("/proc/self/maps").read()
print(json.dumps({"librp": "librp_b200" in maps, "package": "ropephysics_b200" in sys.modules,
                  "ref": "libcrs_ref.so" in maps}))
""".replace("import runpy, sys", "import json, runpy, sys")


def test_reference_arm_never_loads_the_library(reference):
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    line, maps = lines[0], lines[1]
    assert maps == {"librp": False, "package": False, "ref": True}
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["ms_per_step"] > 0 and line["steps"] == 1


def test_both_arms_describe_the_same_workload():
    import bench
    wl = bench.build_workload("uneven", 64, seed=0)
    cfg = bench.workload_config("uneven", 64, 0)
    assert cfg["workload"] == wl.name and cfg["segments"] == int(wl.segments.sum())
    assert cfg["rods"] == len(wl.rods) and cfg["substeps"] == wl.params.substeps
    assert cfg["dt"] == wl.params.dt
    for name, n in (("grid", 32), ("cantilever", 0)):
        wl = bench.build_workload(name, n, seed=0)
        cfg = bench.workload_config(name, n, 0)
        assert cfg["workload"] == wl.name and cfg["segments"] == int(wl.segments.sum())
