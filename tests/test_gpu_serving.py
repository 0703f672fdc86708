"""The continuous-batching server (rp_server_*).

* A request's result is the same alone and in the mix: each request's final
  positions equal, bit for bit, a batch holding only that request's rods run
  for the same number of steps -- while other requests were admitted,
  stepped in the same launches and retired around it (tolerance: exact).
* Admission respects the HBM budget (peak resident bytes <= budget) and is
  continuous: requests queued behind the budget are admitted as earlier ones
  retire, and requests submitted while others run join them on the device.
* A request that can never fit is rejected with RP_ERR_BUDGET.
"""
import time

import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W

pytestmark = pytest.mark.gpu

PARAMS = rp.StepParams(dt=1.0 / 60, substeps=20, iterations=1)


def small_requests(seed, count):
    rng = np.random.default_rng(seed)
    return [W.served_request(rng, max_rods=24, min_seg=32, max_seg=160, min_steps=15, max_steps=60)
            for _ in range(count)]


def run_alone(req):
    b = rp.Batch.create_mixed(req.rods, req.worlds, [0] * len(req.rods), rp.Strategy.BATCHED)
    b.set_material_scales(req.youngs_scale, req.friction_scale)
    if req.drives is not None:
        b.set_drives(req.drives)
    b.step_many(PARAMS, req.steps)
    x = b.download_positions()
    b.close()
    return x


def submit(server, req):
    return server.submit(req.rods, req.steps, req.worlds, [0] * len(req.rods), req.drives,
                         req.youngs_scale, req.friction_scale)


def test_results_same_alone_and_in_the_mix():
    reqs = small_requests(3, 10)
    # every feature appears at least once among the requests
    for f in ("floor", "primitives", "driven", "self"):
        assert any(r.features[f] for r in reqs), f
    alone = [run_alone(r) for r in reqs]
    server = rp.Server(512 << 20, PARAMS)
    ids = []
    for i, r in enumerate(reqs):
        ids.append(submit(server, r))
        if i % 3 == 2:
            time.sleep(0.05)  # later requests arrive while earlier ones run
    for rid, x in zip(ids, alone):
        server.wait(rid, 300)
        assert np.array_equal(server.result(rid), x)
    st = server.stats()
    assert st["completed"] == len(reqs) and st["resident_bytes"] == 0
    infos = [server.info(i) for i in ids]
    # continuous batching: some request was admitted before another finished
    assert any(a["admit_s"] < b["done_s"] and a["submit_s"] > b["admit_s"]
               for a in infos for b in infos if a is not b)
    server.close()


def test_budget_admission_and_queueing():
    # requests of 48..53 rods x 128..138 segments: a few MiB resident each,
    # so a budget of 1.5x the largest holds one at a time
    reqs = []
    for k, r in enumerate(small_requests(5, 6)):
        n = 48 + k
        rod = rp.Rod.straight(128 + 2 * k, 1.0, W.GRID_MATERIAL, direction=(0.0, 0.0, -1.0))
        rod.pin_particle(0)
        drives = None if r.drives is None else [r.drives[0]] * n
        reqs.append(W.ServedRequest([rod] * n, r.steps, r.worlds, drives,
                                    np.resize(r.youngs_scale, n), np.resize(r.friction_scale, n), r.features))
    sizes = []
    probe = rp.Server(1 << 30, PARAMS)
    for r in reqs:
        rid = submit(probe, r)
        sizes.append(probe.info(rid)["resident_bytes"])
    probe.drain(300)
    probe.close()
    # the smallest budget, in steps of 1/8, whose arenas take every request
    # alone (the arenas split the budget in fixed proportions, so the request
    # that binds may be one with many contact slots rather than the largest):
    # the six cannot all be resident at once, so later ones wait for earlier
    # ones to retire
    budget = max(max(sizes), 1 << 20)
    for _ in range(64):
        fits = True
        for r in reqs:
            probe = rp.Server(budget, PARAMS)
            try:
                submit(probe, r)
            except rp.RopeError as e:
                assert e.status == 6
                fits = False
            probe.drain(300)
            probe.close()
            if not fits:
                break
        if fits:
            break
        budget = int(budget * 1.125)
    assert fits
    server = rp.Server(budget, PARAMS)
    ids = [submit(server, r) for r in reqs]
    server.drain(600)
    st = server.stats()
    assert st["completed"] == len(reqs)
    assert st["peak_resident_bytes"] <= budget
    assert st["peak_resident_bytes"] < sum(sizes)  # never all resident at once
    infos = [server.info(i) for i in ids]
    # FIFO: admissions in submission order, and some waited for an earlier retire
    admits = [i["admit_s"] for i in infos]
    assert admits == sorted(admits)
    assert any(infos[j]["admit_s"] >= min(i["done_s"] for i in infos[:j]) for j in range(1, len(infos)))
    for rid, r in zip(ids, reqs):
        assert np.array_equal(server.result(rid), run_alone(r))
    server.close()


def test_oversized_request_rejected():
    server = rp.Server(2 << 20, PARAMS)
    rod = rp.Rod.straight(512, 1.0, W.GRID_MATERIAL)
    with pytest.raises(rp.RopeError) as e:
        server.submit([rod] * 64, 10)
    assert e.value.status == 6
    server.close()


def test_concurrent_submitters():
    """Four host threads submit at once; every result still equals its request
    run alone (the submit path is thread-safe; ctypes releases the GIL)."""
    import threading
    reqs = small_requests(9, 12)
    alone = [run_alone(r) for r in reqs]
    server = rp.Server(512 << 20, PARAMS)
    ids = [None] * len(reqs)

    def worker(k):
        for i in range(k, len(reqs), 4):
            ids[i] = submit(server, reqs[i])

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert len(set(ids)) == len(reqs)
    for rid, x in zip(ids, alone):
        server.wait(rid, 300)
        assert np.array_equal(server.result(rid), x)
    server.close()
