"""The per-rod shared-memory layout (ropephysics_b200/csrc/rp_layout.h), on
the CPU: every section of every layout the kernels carve must start on a
16-byte boundary and the total must be a multiple of 16 -- float4 rows,
the bulk copies that stage a rod, and the next rod's slice of a group all
rely on it, and a misaligned section faults on the GPU. The header is
compiled by g++ into a small program that sweeps rod sizes (odd and even
segment counts, ghost frames), primitive counts, self-collision, hash
tables, and every layout mode (full, lean, compensated, slots shared)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include "rp_layout.h"
int main() {
    long checked = 0;
    const int tables[] = {1, 63, 64, 100, 257, 1024, 4097};
    for (int nSt = 1; nSt <= 700; ++nSt)
        for (int ghosts = 0; ghosts <= 2; ++ghosts)
            for (int prims = 0; prims <= 5; prims += 1)
                for (int self = 0; self <= 1; ++self)
                    for (int table : tables)
                        for (int mode = 0; mode < 8; ++mode) {
                            const int nP = nSt + 1, nS = nSt + ghosts, nB = nSt - 1 + ghosts;
                            const int cap = nSt / 2 > 16 ? nSt / 2 : 16;
                            const int lean = mode & 1, comp = (mode >> 1) & 1, shared = (mode >> 2) & 1;
                            const rp::RodLayout L =
                                rp::rodLayout(nP, nS, nSt, nB, prims, self, table, cap, lean, comp, shared);
                            ++checked;
                            if (!rp::rodLayoutAligned(L)) {
                                std::printf("misaligned: nSt %d ghosts %d prims %d self %d table %d mode %d\n",
                                            nSt, ghosts, prims, self, table, mode);
                                return 1;
                            }
                        }
    std::printf("%ld layouts aligned\n", checked);
    return 0;
}
"""


def test_every_layout_section_is_16_byte_aligned(tmp_path):
    src = tmp_path / "layout_check.cpp"
    exe = tmp_path / "layout_check"
    src.write_text(PROGRAM)
    inc = os.path.join(ROOT, "ropephysics_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{inc}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    assert "layouts aligned" in out.stdout
