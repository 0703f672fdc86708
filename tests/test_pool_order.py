"""The self-contact pool built from touching pairs has the reference's order.

The batched kernel builds the pool of a substep with few touching pairs
without the spatial hash (`poolFromPairs`, csrc/rp_batched.cu): each
touching pair (j, k) gets one entry per cell t of the 27 around cell(j)
whose hash is k's bucket, and the entries are ranked by (j, t, k). The
reference's query (src/gpu/gpu_solver.cu:262-309, collision.cpp:119-151)
walks, for each segment j in order, the 27 cells in z/y/x order and in
each the bucket of that cell's hash in segment order (a stable counting
sort), appending every touching later segment; entries past the pool's
capacity are dropped. These host tests replay both on seeded layouts --
clustered segments, small hash tables so buckets collide, several touching
pairs per segment, capacities that cut the pool -- and require the same
entry sequence, using the kernel's ranking arithmetic (entries of pairs of
earlier segments, then cells below t, then smaller k in cell t).
"""
import numpy as np
import pytest

P1, P2, P3 = 73856093, 19349663, 83492791


def hash_cell(ix, iy, iz, table):
    h = ((ix * P1) & 0xFFFFFFFF) ^ ((iy * P2) & 0xFFFFFFFF) ^ ((iz * P3) & 0xFFFFFFFF)
    return h & (table - 1) if table & (table - 1) == 0 else h % table


def cells_around(cell):
    cx, cy, cz = cell
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                yield cx + dx, cy + dy, cz + dz


def reference_pool(cells, touching, table, capacity):
    """The reference's query order: buckets by a stable counting sort, then
    for each j the 27 cells, each bucket in segment order."""
    n = len(cells)
    buckets = [[] for _ in range(table)]
    for k in range(n):  # stable: segments in ascending order
        buckets[hash_cell(*cells[k], table)].append(k)
    pool = []
    for j in range(n):
        for c in cells_around(cells[j]):
            for k in buckets[hash_cell(*c, table)]:
                if (j, k) in touching:
                    pool.append((j, k))
    return pool[:capacity], len(pool)


def pool_from_pairs(cells, pairs, table, capacity):
    """The kernel's ranking: every pair's cell mask, then each entry's rank
    from the masks of the pairs that order before it."""
    masks = []
    for j, k in pairs:
        hk = hash_cell(*cells[k], table)
        m = 0
        for t, c in enumerate(cells_around(cells[j])):
            if hash_cell(*c, table) == hk:
                m |= 1 << t
        masks.append(m)
    total = sum(bin(m).count("1") for m in masks)
    pool = [None] * min(total, capacity)
    for (j, k), m in zip(pairs, masks):
        before = sum(bin(mq).count("1") for (jq, _), mq in zip(pairs, masks) if jq < j)
        for t in range(27):
            if not (m >> t) & 1:
                continue
            below = (1 << t) - 1
            rank = before
            for (jq, kq), mq in zip(pairs, masks):
                if jq != j:
                    continue
                rank += bin(mq & below).count("1") + (1 if (mq >> t) & 1 and kq < k else 0)
            if rank < capacity:
                assert pool[rank] is None, "two entries ranked alike"
                pool[rank] = (j, k)
    assert all(e is not None for e in pool), "a rank left empty"
    return pool, total


@pytest.mark.parametrize("table", [4, 8, 64, 7])
@pytest.mark.parametrize("seed", range(6))
def test_pool_from_pairs_equals_the_reference_query_order(table, seed):
    rng = np.random.default_rng(seed * 31 + table)
    n = int(rng.integers(8, 120))
    # segments clustered in a few cells, so buckets hold many segments and
    # touching pairs sit in neighbouring cells (as the cell size guarantees)
    cells = [tuple(int(v) for v in rng.integers(-2, 3, 3)) for _ in range(n)]
    touching = set()
    for _ in range(int(rng.integers(1, 40))):
        j = int(rng.integers(0, n - 1))
        k = int(rng.integers(j + 1, n))
        if max(abs(a - b) for a, b in zip(cells[j], cells[k])) <= 1:
            touching.add((j, k))
    if not touching:
        touching.add((0, n - 1))
        cells[n - 1] = cells[0]
    # the count appends pairs in no particular order
    pairs = sorted(touching, key=lambda p: rng.random())
    for capacity in (1, 3, 16, 1000):
        want, want_total = reference_pool(cells, touching, table, capacity)
        got, got_total = pool_from_pairs(cells, pairs, table, capacity)
        assert got_total == want_total
        assert got == want


def test_bucket_collisions_repeat_a_pair():
    # a one-bucket table: every cell of the 27 hashes to k's bucket, so each
    # touching pair appears 27 times, all before the next segment's entries
    cells = [(0, 0, 0), (0, 0, 1), (1, 0, 0), (5, 5, 5)]
    touching = {(0, 1), (0, 2), (1, 2)}
    want, total = reference_pool(cells, touching, 1, 1000)
    got, total2 = pool_from_pairs(cells, [(1, 2), (0, 2), (0, 1)], 1, 1000)
    assert total == total2 == 81 and got == want
    assert got[:2] == [(0, 1), (0, 2)] and got[54:] == [(1, 2)] * 27
