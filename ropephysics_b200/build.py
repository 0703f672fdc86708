"""Build the native library ``ropephysics_b200/librp_b200.so`` in-tree.

CUDA sources are compiled by nvcc for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); host sources by g++. The CUDA runtime is
linked statically, so the library needs only the NVIDIA driver at run time.
Run ``python -m ropephysics_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librp_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc") if os.path.exists(os.path.join(CUDA_HOME, "bin", "nvcc")) \
    else (shutil.which("nvcc") or "nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", f"-I{os.path.join(CUDA_HOME, 'include')}"]
# --fmad=false: no multiply-add is fused unless the source says so (__fmaf_rn),
# so every kernel rounds the reference-order arithmetic identically
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "--fmad=false"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter"]

CU_SOURCES = ["rp_plain.cu", "rp_batched.cu", "rp_static_scratch.cu", "rp_traj.cu", "rp_harness.cu",
              "rp_peak.cu"]
CPP_SOURCES = ["rp_rod.cpp", "rp_hostutil.cpp", "rp_batch.cpp", "rp_batch_tune.cpp", "rp_batch_io.cpp",
               "rp_server.cpp", "rp_traj.cpp"]
HEADERS = ["rp_internal.h", "rp_layout.h", "rp_launch.h", "rp_math.cuh", "rp_step_common.cuh",
           "rp_host.h", "rp_batch_impl.h", "rp_bulk.cuh"]


def _newest_dep() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS]
    paths.append(os.path.join(ROOT, "include", "ropephysics_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _stale(target: str, source: str, dep: float) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return t < os.path.getmtime(source) or t < dep


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every source that changed and link the library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    dep = _newest_dep()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, s, dep):
            cmd = [NVCC] + NVCC_FLAGS + INCLUDES + (["-Xptxas", "-v"] if ptxas_info else []) + \
                ["-c", s, "-o", o]
            jobs.append(cmd)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, s, dep):
            jobs.append([CXX] + CXX_FLAGS + INCLUDES + ["-c", s, "-o", o])
    procs = [(cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
             for cmd in jobs]
    failed = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or ptxas_info or p.returncode != 0:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed.append(" ".join(cmd))
    if failed:
        raise RuntimeError("compilation failed:\n" + "\n".join(failed))
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, "-shared"] + ARCH + ["-Xlinker", "-soname=librp_b200.so", "-o", LIB] + objs + \
            ["-lpthread"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            sys.stdout.write(r.stdout)
            raise RuntimeError("link failed: " + " ".join(cmd))
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
