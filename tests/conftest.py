"""pytest configuration: the `gpu` marker and the oracle build.

Tests marked ``gpu`` need a CUDA device and run on the B200; everything else
runs on the CPU. The oracle libraries are test infrastructure and are built
on demand from ``oracle/Makefile`` (the reference part only where the
reference sources are present).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")
    oracle = os.path.join(ROOT, "oracle")
    if not all(os.path.exists(os.path.join(oracle, f"liboracle_{v}.so")) for v in ("f64", "f32", "count")):
        subprocess.run(["make", "-C", oracle, "all"], check=True, stdout=subprocess.DEVNULL)
    lib = os.path.join(ROOT, "ropephysics_b200", "librp_b200.so")
    if not os.path.exists(lib):
        from ropephysics_b200 import build
        build.build()


@pytest.fixture(scope="session")
def oracle64():
    from oracle import Oracle
    return Oracle("f64")


@pytest.fixture(scope="session")
def oracle32():
    from oracle import Oracle
    return Oracle("f32")


def _ref_lib(gpu):
    name = "libcrs_ref_gpu.so" if gpu else "libcrs_ref.so"
    path = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(path):
        return None
    from oracle import Reference
    return Reference(gpu=gpu)


@pytest.fixture(scope="session")
def reference():
    """The reference's CPU solver built from its sources, or skip."""
    r = _ref_lib(False)
    if r is None:
        pytest.skip("oracle/_ref/libcrs_ref.so not built (reference sources absent)")
    return r


@pytest.fixture(scope="session")
def reference_gpu():
    """The reference's CUDA batch built for sm_100a, or skip."""
    r = _ref_lib(True)
    if r is None:
        pytest.skip("oracle/_ref/libcrs_ref_gpu.so not built (reference sources absent)")
    return r
