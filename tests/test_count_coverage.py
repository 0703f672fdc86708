"""The batched self-contact count reaches every pair the sphere test keeps.

The batched kernel's count (`countSelfByBlocks`, csrc/rp_batched.cu) does not
walk the reference's hash: it tests chain blocks of 8 segments. Block J's
pairs with itself run over a gap-ordered triangle (the 28 in-block pairs
ordered by b - a descending, so the pairs with b - a >= gap are a prefix),
its pairs with block J + 1 run unconditionally, and blocks K >= J + 2 are
first culled by box distance with a bound no tighter than the per-pair sphere
test's (FP32, with the kernel's margins). These host tests replay that
enumeration in float32 on seeded rods -- straight, coiled, folded, with
ragged last blocks and gaps from 1 to 12 -- and require that the pairs
passing the per-pair sphere test are exactly the ones the reference's
all-pairs walk (k - j >= gap) keeps.
"""
import numpy as np
import pytest

f32 = np.float32


def l1(c):
    return f32(f32(f32(f32(1.0) + abs(c[0])) + abs(c[1])) + abs(c[2]))


def blocks(c, h, n):
    out = []
    for J in range((n + 7) // 8):
        idx = range(8 * J, min(8 * J + 8, n))
        lo = np.array([min(c[j][d] for j in idx) for d in range(3)], f32)
        hi = np.array([max(c[j][d] for j in idx) for d in range(3)], f32)
        out.append((lo, max(h[j] for j in idx), hi, max(l1(c[j]) for j in idx)))
    return out


def sphere_keeps(c, h, j, k, two_r):
    d = c[k] - c[j]
    plim = f32(f32(f32(f32(h[j] + h[k]) + two_r) * f32(1.001)) + f32(f32(1e-6) * l1(c[j])))
    return not (f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) > f32(plim * plim))


def box_hit(bj, bk, two_r):
    jlo, jw, jhi, jl1 = bj
    klo, kw, khi, _ = bk
    g = [max(f32(0), max(f32(klo[d] - jhi[d]), f32(jlo[d] - khi[d]))) for d in range(3)]
    lim = f32(f32(f32(f32(jw + kw) + two_r) * f32(1.001)) + f32(f32(1e-6) * jl1))
    return not (f32(f32(g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]) > f32(f32(lim * lim) * f32(1.0001)))


def triangle(gap):
    """Lane -> (a, b) of the kernel's in-block round."""
    out = []
    for wl in range(32):
        e, pair = wl, None
        for d in range(7, 0, -1):
            if e < 8 - d:
                pair = (e, e + d)
                break
            e -= 8 - d
        if pair and pair[1] - pair[0] >= gap:
            out.append(pair)
    return out


def kernel_candidates(c, h, n, gap, two_r):
    B = blocks(c, h, n)
    nb = len(B)
    out = set()
    for J in range(nb):
        jmin = 8 * J
        if J + 1 < nb:  # J against J + 1, no box test
            for a in range(8):
                for b in range(8):
                    j, k = jmin + a, 8 * (J + 1) + b
                    if j < n and k < n and k - j >= gap:
                        out.add((j, k))
        for a, b in triangle(gap):  # J against itself
            if jmin + b < n:
                out.add((jmin + a, jmin + b))
        for K in range(J + 2, nb):  # far blocks, by box distance
            if min(8 * K + 7, n - 1) - jmin < gap or not box_hit(B[J], B[K], two_r):
                continue
            for a in range(8):
                for b in range(8):
                    j, k = jmin + a, 8 * K + b
                    if j < n and k < n and k - j >= gap:
                        out.add((j, k))
    return out


def rod(rng, n, kind):
    if kind == "straight":
        dirs = np.tile([1.0, 0.0, 0.0], (n, 1))
    elif kind == "coil":
        t = np.arange(n) * 0.35
        dirs = np.stack([-np.sin(t), np.cos(t), np.full(n, 0.08)], axis=1)
    else:  # folded: a random walk with sharp turns
        dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    seg = rng.uniform(0.8, 1.2, n)[:, None] * rng.uniform(0.003, 0.02)
    x = np.concatenate([[rng.uniform(-2, 2, 3)], np.cumsum(dirs * seg, axis=0)])
    x[1:] += x[0]
    x = x.astype(f32)
    c = ((x[:-1] + x[1:]) * f32(0.5)).astype(f32)
    h = (f32(0.5) * np.linalg.norm(x[1:] - x[:-1], axis=1)).astype(f32)
    return c, h


def test_triangle_is_every_in_block_pair_beyond_the_gap():
    for gap in range(1, 10):
        assert sorted(triangle(gap)) == [(a, b) for a in range(8) for b in range(8) if b - a >= gap]


@pytest.mark.parametrize("kind", ["straight", "coil", "folded"])
@pytest.mark.parametrize("seed", range(4))
def test_count_keeps_every_sphere_pair(kind, seed):
    rng = np.random.default_rng(seed * 7 + len(kind))
    n = int(rng.integers(3, 70))
    c, h = rod(rng, n, kind)
    seg = float(np.mean(2 * h))
    for radius_factor in (0.2, 0.8, 2.5):
        two_r = f32(2 * radius_factor * seg)
        gap = max(1, int(np.floor(float(two_r) / float(np.min(2 * h)))) + 2)
        gap = min(gap, 12)
        want = {(j, k) for j in range(n) for k in range(j + gap, n) if sphere_keeps(c, h, j, k, two_r)}
        got = {p for p in kernel_candidates(c, h, n, gap, two_r) if sphere_keeps(c, h, *p, two_r)}
        assert got == want, (kind, n, gap, sorted(want - got)[:5])
