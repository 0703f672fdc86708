"""Host side of the library on the CPU: the C ABI loads and exports what the
header declares; the descriptor builders, colouring and index gap equal the
oracle bit for bit; malformed input fails loudly; no GPU means a clear
RP_ERR_NO_DEVICE, never a silent CPU path."""
import ctypes as C
import math
import os

import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import _abi
from tests.helpers import REF_MAT, product_rod

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ropephysics_b200.h")
MAT = rp.Material(**REF_MAT)


def test_library_exports_every_header_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    declared = _abi.header_symbols(HEADER)
    assert len(declared) > 40
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python mirror declares exactly the header's functions
    assert sorted(_abi.SIGNATURES) == declared


def test_abi_version():
    assert rp.lib().rp_abi_version() == 1


def _same(prod, orod):
    n = orod.nP
    pairs = [("x", "x", n), ("inv_mass", "invMass", n), ("mass", "mass", n),
             ("q", "q", orod.nS), ("inertia", "inertia", orod.nS),
             ("inv_inertia", "invInertia", orod.nS), ("s_p0", "sP0", orod.nSt),
             ("s_p1", "sP1", orod.nSt), ("s_seg", "sSeg", orod.nSt), ("s_rest", "sRest", orod.nSt),
             ("s_compliance", "sComp", orod.nSt), ("b_a", "bA", orod.nB), ("b_b", "bB", orod.nB),
             ("b_rest", "bRest", orod.nB), ("b_compliance", "bComp", orod.nB),
             ("b_rest_darboux", "bRestD", orod.nB)]
    assert (prod.num_particles, prod.num_frames, prod.num_stretch, prod.num_bend) == \
        (orod.nP, orod.nS, orod.nSt, orod.nB)
    for a, b, k in pairs:
        assert np.array_equal(getattr(prod, a), getattr(orod, b)[:k]), a


@pytest.mark.parametrize("n", [2, 3, 16, 64, 513])
def test_straight_builder_bit_exact(oracle64, n):
    for tip in (False, True):
        for d in ((1, 0, 0), (0, 0, 1), (0, 0, -1), (0.3, -0.2, 0.9)):
            p = rp.Rod.straight(n, 1.3, MAT, origin=(0.1, -0.2, 0.3), direction=d)
            g = p.clamp_end(tip)
            o = oracle64.straight(n, 1.3, **REF_MAT, origin=(0.1, -0.2, 0.3), direction=d)
            assert g == oracle64.clamp(o, tip)
            _same(p, o)


def test_centerline_builder_bit_exact(oracle64):
    for n, twist, seed in ((10, 0.0, (0, 0, 1)), (121, 0.8, (0, 1, 0)), (300, -2.0, (1, 0, 0))):
        t = np.linspace(0, 4 * math.pi, n + 1)
        pts = np.stack([0.1 * np.cos(t), 0.1 * np.sin(t), 0.015 * t], 1)
        p = rp.Rod.centerline(pts, MAT, frame_seed=seed, twist_per_length=twist)
        o = oracle64.centerline(pts, **REF_MAT, frame_seed=seed, twist_per_length=twist)
        _same(p, o)
        p.x[:, 2] += 0.01 * np.sin(np.arange(n + 1))
        o.x[: n + 1, 2] += 0.01 * np.sin(np.arange(n + 1))
        p.set_rest_from_current()
        oracle64.set_rest_from_current(o)
        _same(p, o)


def test_from_arrays_roundtrip(oracle64):
    o = oracle64.straight(20, 1.0, **REF_MAT)
    oracle64.clamp(o, False)
    oracle64.clamp(o, True)
    _same(product_rod(o), o)


@pytest.mark.parametrize("n", [8, 32, 128, 512])
def test_coloring_matches_oracle_and_golden(oracle64, n):
    g = np.load(os.path.join(ROOT, "tests", "golden", "coloring.npz"))
    p = rp.Rod.straight(n, 1.0, MAT)
    p.clamp_end(False)
    for bend in (False, True):
        order, starts = p.coloring(bend)
        key = f"{'bend' if bend else 'stretch'}_{n}"
        assert np.array_equal(order, g[key + "_order"])
        assert np.array_equal(starts, g[key + "_start"])


def test_general_coloring_is_greedy_and_conflict_free(oracle64):
    rng = np.random.default_rng(3)
    count = 200
    res = [sorted(set(rng.integers(0, 60, size=rng.integers(1, 4)).tolist())) for _ in range(count)]
    start = np.cumsum([0] + [len(r) for r in res]).astype(np.int32)
    flat = np.array([x for r in res for x in r], np.int32)
    order = np.zeros(count, np.int32)
    cs = np.zeros(count + 1, np.int32)
    nc = C.c_int32()
    I = C.POINTER(C.c_int32)
    assert rp.lib().rp_color_constraints(count, start.ctypes.data_as(I), flat.ctypes.data_as(I),
                                         order.ctypes.data_as(I), cs.ctypes.data_as(I),
                                         C.byref(nc)) == 0
    # greedy reference: lowest colour no resource has taken (coloring.cpp:11-57)
    used = {}
    colour = []
    for r in res:
        c = 0
        while any(c in used.get(x, set()) for x in r):
            c += 1
        colour.append(c)
        for x in r:
            used.setdefault(x, set()).add(c)
    expect = sorted(range(count), key=lambda k: (colour[k], k))
    assert np.array_equal(order, expect)
    for c in range(nc.value):
        members = order[cs[c]:cs[c + 1]]
        seen = [x for k in members for x in res[k]]
        assert len(seen) == len(set(seen))


def test_self_collision_index_gap(oracle64):
    from oracle import World as OW
    for n, r in ((150, 5e-3), (16, 5e-3), (100, 4e-3), (30, 0.02)):
        p = rp.Rod.straight(n, 1.2, rp.Material(1e7, 0.35, 1000, r))
        o = oracle64.straight(n, 1.2, youngs=1e7, poisson=0.35, density=1000, radius=r)
        for skip in (2, 5):
            w = rp.World(self_collision=True, self_skip=skip)
            assert rp.self_collision_index_gap(p, w) == oracle64.self_gap(o, OW(self_skip=skip))


def test_invalid_descriptors_fail_loudly():
    with pytest.raises(rp.RopeError, match="segments"):
        rp.Rod.straight(1, 1.0, MAT)
    with pytest.raises(rp.RopeError):
        rp.Rod.straight(8, -1.0, MAT)
    with pytest.raises(rp.RopeError, match="coincident"):
        rp.Rod.centerline(np.zeros((5, 3)), MAT)
    good = rp.Rod.straight(8, 1.0, MAT)
    a = dict(x=good.x, v=good.v, inv_mass=good.inv_mass, q=good.q, inertia=good.inertia,
             inv_inertia=good.inv_inertia, s_p0=good.s_p0.copy(), s_p1=good.s_p1, s_seg=good.s_seg,
             s_rest=good.s_rest, s_compliance=good.s_compliance, b_a=good.b_a, b_b=good.b_b,
             b_rest=good.b_rest, b_compliance=good.b_compliance, b_rest_darboux=good.b_rest_darboux)
    a["s_p0"][3] = 99
    with pytest.raises(rp.RopeError, match="indexes outside"):
        rp.Rod.from_arrays(MAT, **a)
    a["s_p0"][3] = 3
    x = good.x.copy()
    x[2, 1] = np.nan
    with pytest.raises(rp.RopeError, match="non-finite"):
        rp.Rod.from_arrays(MAT, **dict(a, x=x))


def test_no_device_is_an_error_not_a_fallback():
    if rp.cuda_available():
        pytest.skip("a GPU is present")
    rod = rp.Rod.straight(8, 1.0, MAT)
    with pytest.raises(rp.RopeError) as e:
        rp.Batch.create(rod, 4, rp.Strategy.BATCHED)
    assert e.value.status == 2
    assert "no usable CUDA device" in rp.diagnostic()
    assert rp.max_fused_segments() == 0


def test_world_limits_rejected_before_any_device_work():
    """At most 64 primitives per world (the batched kernel culls them with a
    64-bit mask); self-collision needs a hash table of 1..2^20 buckets."""
    import ropephysics_b200 as rp
    rod = rp.Rod.straight(8, 0.2, rp.Material())
    many = [rp.Primitive.sphere((0, 0, -1.0 - k), 0.1, 0.5) for k in range(65)]
    with pytest.raises(rp.RopeError) as e:
        rp.Batch.create(rod, 1, rp.Strategy.BATCHED, rp.World(many))
    assert e.value.status == 1 and "64" in str(e.value)
    with pytest.raises(rp.RopeError) as e:
        rp.Batch.create(rod, 1, rp.Strategy.BATCHED, rp.World([], self_collision=True, hash_table_size=0))
    assert e.value.status == 1
