"""Structural tests of the oracle's LBVH build and traversal.

Restates Partia.jl/test/neighbor_search_tests.jl: binary radix tree invariants for
n = 1..20 and offsets 0..4 on the deterministic prime-hash coordinates (:49-61) with the
Karras split rule recomputed independently here (:186-241), the identical-code case
(:245-256), AABB containment on a lattice (:260-296), node hmax against a recursive
reference (:300-314), LBVH_query! against brute force (:318-342), scatter and symmetric
pruning against brute force (:346-371), hmax pruning tightening the traversal (:375-422)
and line traversal against brute force (:424-466).
"""
import numpy as np
import pytest

import oracle

PRIMES = (37, 61, 97, 131, 197, 263)


def prime_coords(n, off, dim=3):
    return [np.array([((PRIMES[d] * i + PRIMES[d + dim] * off) % 1021) / 1021 for i in range(1, n + 1)])
            for d in range(dim)]


def lcp(c, i, j):   # 1-based indices, codes c is 0-based array
    a, b = int(c[i - 1]), int(c[j - 1])
    x = (i ^ j) if a == b else (a ^ b)
    return 64 - x.bit_length()


def find_range(c, i):
    n = len(c)
    dl = lcp(c, i, i - 1) if i > 1 else -1
    dr = lcp(c, i, i + 1) if i < n else -1
    d = 1 if dr - dl >= 0 else -1
    dmin = lcp(c, i, i - d) if 1 <= i - d <= n else -1
    lmax = 2
    while 1 <= i + lmax * d <= n and lcp(c, i, i + lmax * d) > dmin:
        lmax *= 2
    l, t = 0, lmax >> 1
    while t > 0:
        j = i + (l + t) * d
        if 1 <= j <= n and lcp(c, i, j) > dmin:
            l += t
        t >>= 1
    j = i + l * d
    return min(i, j), max(i, j)


def split_position(c, first, last):
    if c[first - 1] == c[last - 1]:
        return min(max((first + last) >> 1, first), last - 1)
    p = lcp(c, first, last)
    split, step = first, last - first
    while step > 1:
        step = (step + 1) >> 1
        if split + step < last and lcp(c, first, split + step) > p:
            split += step
    return split


@pytest.mark.parametrize("off", range(5))
def test_binary_radix_tree_invariants(off):
    for n in range(1, 21):
        x, y, z = prime_coords(n, off)
        t = oracle.OracleLBVH(x, y, z, np.full(n, 0.1))
        nt = 2 * n - 1
        assert len(t.left) == nt and len(t.parent) == nt
        assert t.root == (1 if n >= 2 else 0)
        if t.root:
            assert t.parent[t.root - 1] == 0
        assert ((t.parent >= 0) & (t.parent < nt + 1)).all()
        assert ((t.escape >= 0) & (t.escape <= nt)).all()
        assert (np.diff(t.codes.astype(object)) > 0).all() if n > 1 else True
        off_ = n - 1
        for i in range(1, n):
            lo, hi = find_range(t.codes, i)
            s = split_position(t.codes, lo, hi)
            l, r = t.left[i - 1], t.right[i - 1]
            assert l == (off_ + lo if s == lo else s)
            assert r == (off_ + hi if s + 1 == hi else s + 1)


@pytest.mark.parametrize("n", [1, 2, 8, 16])
def test_identical_codes(n):
    t = oracle.OracleLBVH(np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5))
    assert t.root == (1 if n >= 2 else 0)
    if n >= 2:
        assert t.parent[0] == 0
    assert np.count_nonzero(t.parent == 0) == 1
    # the duplicate bump makes the codes strictly increasing
    assert all(int(t.codes[i + 1]) == int(t.codes[i]) + 1 for i in range(n - 1))


def _child_box(t, c, d):
    n, nin = t.n, t.n - 1
    leaf = (t.x, t.y, t.z)
    if c >= n:
        v = leaf[d][c - n]
        return v, v
    return t.bmin[d * nin + c - 1], t.bmax[d * nin + c - 1]


@pytest.mark.parametrize("n", [2, 8, 32])
def test_aabb_containment(n):
    g = np.linspace(0.0, 1.0, n)
    t = oracle.OracleLBVH(g, g, g, np.full(n, 0.1))
    nin = n - 1
    for i in range(1, n):
        for d in range(3):
            lmn, lmx = _child_box(t, t.left[i - 1], d)
            rmn, rmx = _child_box(t, t.right[i - 1], d)
            assert t.bmin[d * nin + i - 1] == min(lmn, rmn)
            assert t.bmax[d * nin + i - 1] == max(lmx, rmx)


def test_node_hmax_recursive():
    g = np.random.default_rng(0xBEEF)
    n = 64
    x, y, z = g.random((3, n))
    t = oracle.OracleLBVH(x, y, z, g.random(n))

    def visit(node):
        if node >= n:
            return t.h[node - n]
        v = max(visit(t.left[node - 1]), visit(t.right[node - 1]))
        assert t.hmax[node - 1] == v
        return v

    visit(1)


def test_query_matches_brute_force():
    x = np.array([0.0, 1.0, 0.0, 1.0])
    y = np.array([0.0, 0.0, 1.0, 1.0])
    z = np.zeros(4)
    t = oracle.OracleLBVH(x, y, z, np.full(4, 0.1))
    for p, r in (((0.1, 0.1, 0.0), 0.25), ((0.9, 0.9, 0.0), 0.25), ((0.5, 0.5, 0.0), 0.75)):
        got, _ = t.query(p, r)
        d2 = (t.x - p[0]) ** 2 + (t.y - p[1]) ** 2 + (t.z - p[2]) ** 2
        assert np.array_equal(np.sort(got), np.nonzero(d2 <= r * r + 16 * np.finfo(float).eps)[0])
    g = np.random.default_rng(5)
    n = 3000
    x, y, z = g.random((3, n))
    t = oracle.OracleLBVH(x, y, z, np.full(n, 0.05))
    for _ in range(100):
        p, r = g.random(3), g.random() * 0.2
        got, near = t.query(p, r)
        d2 = (t.x - p[0]) ** 2 + (t.y - p[1]) ** 2 + (t.z - p[2]) ** 2
        exp = np.nonzero(d2 <= r * r)[0]
        assert np.array_equal(got, exp)          # DFS order == ascending leaf index
        if len(exp):
            assert near == exp[np.argmin(d2[exp])]


@pytest.mark.parametrize("strategy", ["itpScatter", "itpSymmetric", "itpGather"])
def test_pruned_traversal_accepts_brute_force_set(strategy):
    g = np.random.default_rng(0xCAFE)
    n = 500
    x, y, z = g.random((3, n))
    h = g.random(n) * 0.2 + 0.05
    t = oracle.OracleLBVH(x, y, z, h).attach(np.ones(n), np.ones(n), [np.ones(n)])
    cat = {"scalar_cols": [0], "scalar_shepard": [1]}
    q = g.random((3, 40))
    _, st = t.interp_points(cat, *q, strategy=strategy, stats=True)
    for i in range(q.shape[1]):
        p = q[:, i]
        d2 = (t.x - p[0]) ** 2 + (t.y - p[1]) ** 2 + (t.z - p[2]) ** 2
        hb = t.h
        if strategy == "itpScatter":
            r2 = (2.0 * hb) ** 2
        else:
            ha, _ = t.find_nearest_h(p)
            r2a = (2.0 * ha) ** 2
            r2 = np.full(n, r2a) if strategy == "itpGather" else np.maximum(r2a, (2.0 * hb) ** 2)
        assert st[i, 4] == np.count_nonzero(d2 <= r2)


def test_hmax_pruning_tightens_traversal():
    g = np.random.default_rng(0x1234)
    n = 256
    x, y, z = g.random((3, n))
    h = g.random(n) * 0.3 + 0.01
    t = oracle.OracleLBVH(x, y, z, h)
    p = (0.1, 0.2, 0.3)
    nin = n - 1

    def visits(hnode):
        cnt, node = 0, t.root
        while node != 0:
            if node >= n:
                node = t.escape[node - 1]
                continue
            cnt += 1
            d2 = 0.0
            for d, pd in enumerate(p):
                a, b = t.bmin[d * nin + node - 1], t.bmax[d * nin + node - 1]
                tt = a - pd if pd < a else (pd - b if pd > b else 0.0)
                d2 += tt * tt
            node = t.left[node - 1] if d2 <= hnode(node) ** 2 else t.escape[node - 1]
        return cnt

    assert visits(lambda i: t.hmax[i - 1]) <= visits(lambda i: h.max())


def test_line_traversal_matches_brute_force():
    g = np.random.default_rng(7)
    n = 400
    x, y, z = g.random((3, n))
    h = g.random(n) * 0.1 + 0.02
    t = oracle.OracleLBVH(x, y, z, h).attach(np.ones(n), np.ones(n), [np.ones(n)])
    cat = {"scalar_cols": [0], "scalar_shepard": [1]}
    m = g.normal(size=(3, 30))
    m /= np.linalg.norm(m, axis=0)
    o = g.random((3, 30))
    _, st = t.interp_lines(cat, tuple(o), tuple(m), stats=True)
    for i in range(30):
        P = np.stack([t.x, t.y, t.z]) - o[:, i:i + 1]
        d2 = (P ** 2).sum(0) - ((P * m[:, i:i + 1]).sum(0)) ** 2
        assert st[i, 2] == np.count_nonzero(d2 <= (2.0 * t.h) ** 2)
