"""The multi-rank host logic of bench.py on CPU (gloo, world size 2).

Rods are independent, so N ranks each simulate their own shard of one seeded
batch of N x rods (sorted by length, every N-th rod) with no data-path
collective; the only cross-rank steps are the barrier around the timed region
and the max-over-ranks of the step time. This runs those steps as two gloo
ranks and checks that the shards are disjoint, cover the batch and are
balanced, that both ranks see the max of the two times, and that the
reference arm prints nothing on rank 1.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    class A:
        seed = 5

    w, r, _ = bench.dist_setup(A)
    assert (w, r) == (world, rank) and dist.get_backend() == "gloo"
    wl = bench.build_workload("uneven", 6, seed=A.seed, shard=(r, w))
    bench.barrier(w)
    t = bench.max_over_ranks(1.5 + r, w)
    shards = [None] * w
    dist.all_gather_object(shards, [int(s) for s in wl.segments])
    buf = io.StringIO()

    class R:
        workload, rods, seed, steps, warmup, cpu_rods, cpu_seconds = "uneven", 4, 0, 1, 0, 2, 0.1

    if r != 0:
        with redirect_stdout(buf):
            bench.run_reference(R)
    out[r] = (t, shards, buf.getvalue())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert set(res) == {0, 1}
    from ropephysics_b200 import synth
    whole = sorted(d.segments for d in synth.uneven(12, 5))
    for r in (0, 1):
        t, shards, printed = res[r]
        assert t == 2.5
        # the two shards of one seeded batch: disjoint, together the batch,
        # each the same spread of lengths (every other rod by length)
        assert sorted(shards[0] + shards[1]) == whole
        assert len(shards[0]) == len(shards[1]) == 6
        assert abs(sum(shards[0]) - sum(shards[1])) <= max(whole)
    assert res[1][2] == ""  # the reference arm runs on rank 0 alone
