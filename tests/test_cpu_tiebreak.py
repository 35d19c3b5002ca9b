"""The ATRBVH kernel replaces the reference's two shuffle-down reductions by
warp reductions over keys.  These tests check, on the CPU, that the keys pick
the same lane as the reference's trees on tie-heavy inputs:

* formTreelet's argmax (BVHRT-Core/src/Treelet.cuh:23-39): lane i takes lane
  i + floor(c/2) when that area is strictly larger, c = m, ceil(c/2), ... -- equal
  to "largest value, then lowest rank" with a per-m rank that the kernel
  builds by replaying the tree on tie patterns (argmax_priority in atrbvh.cu);
* findMinimumDistance (BVHRT-Core/src/AgglomerativeTreelet.cu:65-99): stride-32
  lane scans with strict <, then shuffle-down offsets 16..1 -- equal to the
  minimum of (distance, bit-reversed j mod 32, j).
"""
from __future__ import annotations

import itertools
import random

FLT_MAX = 3.4028234663852886e38


def _argmax_tree(vals):
    m = len(vals)
    v = list(vals) + [float("-inf")] * 32
    ix = list(range(m)) + [-1] * 32
    c, sh = m, m // 2
    while c > 1:
        for i in range(c - sh):  # all lanes read before any writes: i + sh > i
            if v[i + sh] > v[i]:
                v[i], ix[i] = v[i + sh], ix[i + sh]
        c = (c + 1) // 2
        sh = c // 2
    return ix[0]


def _ranks(m):
    """The kernel's rank table: remove tree winners of the all-tied pattern."""
    rem = set(range(m))
    rank = [0] * m
    k = 0
    while rem:
        w = _argmax_tree([1.0 if i in rem else 0.0 for i in range(m)])
        rank[w] = k
        k += 1
        rem.remove(w)
    return rank


def _argmin_reference(dist):
    bv = [FLT_MAX] * 32
    bi = [0] * 32
    for ln in range(32):
        for j in range(ln, len(dist), 32):
            if dist[j] < bv[ln]:
                bv[ln], bi[ln] = dist[j], j
    c, sh = 32, 16
    while c > 1:
        for i in range(c - sh):
            if bv[i + sh] < bv[i]:
                bv[i], bi[i] = bv[i + sh], bi[i + sh]
        c = (c + 1) // 2
        sh = c // 2
    return bi[0]


def _brev5(x):
    return int(format(x & 31, "05b")[::-1], 2)


def _argmin_key(dist):
    best = None
    for j, d in enumerate(dist):
        if d < FLT_MAX:
            k = (d, _brev5(j), j)
            if best is None or k < best:
                best = k
    return 0 if best is None else best[2]


def test_argmax_rank_order_exhaustive_small():
    for m in range(2, 11):
        rank = _ranks(m)
        for vals in itertools.product([0.0, 1.0, 2.0], repeat=m):
            top = max(vals)
            want = min((rank[i], i) for i in range(m) if vals[i] == top)[1]
            assert _argmax_tree(list(vals)) == want, (m, vals)


def test_argmax_rank_order_random_up_to_20():
    rng = random.Random(0)
    for m in range(2, 21):
        rank = _ranks(m)
        for _ in range(3000):
            vals = [rng.choice([0.0, 1.0, 2.0, 3.0, -FLT_MAX]) for _ in range(m)]
            top = max(vals)
            want = min((rank[i], i) for i in range(m) if vals[i] == top)[1]
            assert _argmax_tree(vals) == want, (m, vals)


def test_argmin_bit_reversed_key():
    rng = random.Random(1)
    for _ in range(20000):
        n = rng.randint(1, 190)
        dist = [rng.choice([1.0, 2.0, 3.0, FLT_MAX]) for _ in range(n)]
        assert _argmin_reference(dist) == _argmin_key(dist), dist
