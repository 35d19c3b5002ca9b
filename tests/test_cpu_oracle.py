"""CPU tests: the oracle against its invariants and the golden fixtures, the
product's build algorithm restated in Python, and the C ABI's exports."""
from __future__ import annotations

import json
import re
from pathlib import Path

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import CASES, check_tree, collapsed_digests, scene_case, tree_digests

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"

SMALL = ["u2", "u3", "u5", "u17", "u100", "u1000", "u4097", "clu4096", "dupes3000", "flat2000", "same64"]


@pytest.mark.parametrize("case", SMALL)
def test_oracle_lbvh_invariants(case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    t, sk, si = O.build_lbvh(v, mn, mx)
    check_tree(t, len(v))
    assert np.all(np.diff(sk.astype(np.int64)) >= 0)
    assert sorted(si.tolist()) == list(range(len(v)))


@pytest.mark.parametrize("case", ["u100", "u1000", "clu4096", "dupes3000", "flat2000", "same64"])
@pytest.mark.parametrize("treelet,iters", [(5, 1), (7, 2), (9, 2), (12, 1), (20, 1)])
def test_oracle_atrbvh_invariants(case, treelet, iters):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx)
    a = O.atrbvh(t, treelet, iters)
    check_tree(a, len(v))
    assert O.sah(a) <= O.sah(t) * (1 + 1e-6)


@pytest.mark.parametrize("case", ["u100", "u1000", "clu4096", "dupes3000"])
def test_oracle_trbvh_invariants(case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx)
    a = O.trbvh(t, 7, 3)
    check_tree(a, len(v))


def test_oracle_parallel_equals_serial():
    v = scene_case("clu65536")
    mn, mx = O.scene_aabb(v)
    t1, _, _ = O.build_lbvh(v, mn, mx, threads=1)
    t8, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    for f in ("parent", "left", "right", "data", "bbox_min", "bbox_max", "area"):
        assert np.array_equal(getattr(t1, f), getattr(t8, f)), f
    for fn in (lambda t, th: O.atrbvh(t, 9, 2, threads=th), lambda t, th: O.trbvh(t, 7, 2, threads=th)):
        a1, a8 = fn(t1, 1), fn(t1, 8)
        for f in ("parent", "left", "right", "data", "bbox_min", "bbox_max", "area"):
            assert np.array_equal(getattr(a1, f), getattr(a8, f)), f


def _clz(x: int, bits: int) -> int:
    return bits - x.bit_length()


def bottom_up_build(keys: np.ndarray, idx: np.ndarray, order: np.ndarray, bits: int = 32):
    """Python restatement of the product's fused build (atrbvh_b200/csrc/lbvh.cu
    k_build): leaves climb in `order`; the second sibling to arrive builds the
    parent.  Returns parent/left/right/data arrays."""
    n = len(keys)
    last = n - 1
    keys = [int(k) for k in keys]

    def delta(k):
        if keys[k] == keys[k + 1]:
            return bits + _clz(k ^ (k + 1), 32)
        return _clz(keys[k] ^ keys[k + 1], bits)

    nn = 2 * n - 1
    parent = np.zeros(nn, np.int32)
    left = np.zeros(nn, np.int32)
    right = np.zeros(nn, np.int32)
    data = np.zeros(nn, np.int32)
    slot = [-1] * max(n - 1, 1)
    for i in order:
        i = int(i)
        leaf = i + last
        left[leaf] = right[leaf] = -1
        data[leaf] = idx[i]
        l = r = i
        dl = delta(l - 1) if l > 0 else -1
        dr = delta(r) if r < last else -1
        while True:
            is_left = dr > dl
            split = r if is_left else l - 1
            other = slot[split]
            slot[split] = l if is_left else r
            if other < 0:
                break
            pl, pr = (l, other) if is_left else (other, r)
            lc = split + last if split == pl else split
            rc = split + 1 + last if split + 1 == pr else split + 1
            root = pl == 0 and pr == last
            p = 0
            if not root:
                dl = delta(pl - 1) if pl > 0 else -1
                dr = delta(pr) if pr < last else -1
                p = pr if dr > dl else pl
            left[p], right[p], data[p] = lc, rc, -1
            parent[lc] = parent[rc] = p
            if root:
                parent[0] = -1
                break
            l, r = pl, pr
    return parent, left, right, data


@pytest.mark.parametrize("case", ["u2", "u3", "u5", "u17", "u100", "u1000", "dupes3000", "flat2000", "same64"])
def test_bottom_up_build_matches_karras(case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    t, sk, si = O.build_lbvh(v, mn, mx)
    rng = np.random.default_rng(1)
    for order in (np.arange(len(v)), rng.permutation(len(v))):
        p, l, r, d = bottom_up_build(sk, si, order)
        assert np.array_equal(p, t.parent) and np.array_equal(l[: len(v) - 1], t.left[: len(v) - 1])
        assert np.array_equal(r[: len(v) - 1], t.right[: len(v) - 1]) and np.array_equal(d, t.data)


def test_bottom_up_build_matches_karras_63bit():
    v = scene_case("dupes3000")
    mn, mx = O.scene_aabb(v)
    t, sk, si = O.build_lbvh(v, mn, mx, bits=63)
    p, l, r, d = bottom_up_build(sk, si, np.random.default_rng(2).permutation(len(v)), bits=64)
    assert np.array_equal(p, t.parent) and np.array_equal(d, t.data)


def test_triangular_index_formula():
    """The kernel's row/column recovery (float sqrt + integer fix-up) over every
    flat index of a 20-leaf treelet, against TriangularMatrix.cuh's layout."""
    for k in range(190):
        r = int(np.float32(np.float32(1.0) + np.sqrt(np.float32(8 * k + 1))) * np.float32(0.5))
        if r * (r - 1) // 2 > k:
            r -= 1
        if (r + 1) * r // 2 <= k:
            r += 1
        c = k - r * (r - 1) // 2
        assert 0 <= c < r and r * (r - 1) // 2 + c == k


@pytest.mark.parametrize("treelet", range(3, 21))
def test_atrbvh_schedule_covers_all_pairs(treelet):
    """AgglomerativeScheduler::GenerateScheduleLower restated: every (i, j),
    j < i, appears once; the kernel computes the same pair set directly."""
    s = O.atrbvh_schedule(treelet)
    pairs = []
    for e in s.tolist():
        for sh in (16, 0):
            a, b = (e >> (sh + 8)) & 0xFF, (e >> sh) & 0xFF
            if a or b:
                pairs.append((a, b))
    assert sorted(pairs) == sorted((i, j) for i in range(treelet) for j in range(i))


def test_collapse_and_trace_oracle_consistent():
    v = scene_case("u1000")
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx)
    a = O.atrbvh(t, 9, 2)
    c = O.collapse(a)
    ll = O.leaf_lists(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v))
    assert sorted(x for l in ll.values() for x in l) == list(range(len(v)))
    cap = O.collapse(a, max_leaf=2)
    assert max(len(l) for l in O.leaf_lists(cap.left, cap.right, cap.data, cap.triangle_count,
                                              cap.triangle_indices, len(v)).values()) <= 2
    cp = O.flatten(c, v)
    rays = ab.gen_rays_random(512, mn, mx, seed=3)
    res = O.trace(cp, rays)
    assert (res[:, 0] >= -1).all() and (res[:, 0] < len(v)).all()


def test_workload_is_deterministic():
    a = ab.gen_scene(ab.SCENE_CLUSTERED, 5000, 9)
    b = ab.gen_scene(ab.SCENE_CLUSTERED, 5000, 9)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, ab.gen_scene(ab.SCENE_CLUSTERED, 5000, 10))
    sizes = ab.gen_batch_sizes(4096, 256, 262144, 0)
    assert sizes.min() >= 256 and sizes.max() <= 262144


def test_golden_workload_digests():
    """Generated scenes are pinned: the golden fixtures were made from them."""
    path = GOLDEN / "workload_digests.json"
    want = json.loads(path.read_text())
    from tests._util import digest
    for name, d in want.items():
        assert digest(scene_case(name)) == d, name


def _oracle_tree(rec):
    v = scene_case(rec["case"])
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx, bits=rec.get("bits", 30))
    if rec["optimizer"] == "atrbvh":
        t = O.atrbvh(t, rec["treelet"], rec["iterations"], threads=8)
    elif rec["optimizer"] == "trbvh":
        t = O.trbvh(t, rec["treelet"], rec["iterations"], threads=8)
    return v, t


def test_oracle_matches_reference_golden():
    """The oracle reproduces the SAH the reference's own CUDA build printed on
    single-block inputs (one run on a B200, transcribed into
    tests/golden/ref_golden.json with its log lines and provenance)."""
    gold = json.loads((GOLDEN / "ref_golden.json").read_text())
    for rec in gold["cases"]:
        v, t = _oracle_tree(rec)
        assert np.float32(O.sah(t)) == np.float32(rec["sah"]), rec["name"]
        if "tree" in rec:
            got = tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area)
            assert got == rec["tree"], f"{rec['name']}: tree differs from the reference"
        if "collapsed" in rec:
            c = O.collapse(t)
            assert collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v)) == \
                rec["collapsed"], rec["name"]
    # Cases the reference ran across several SMs are recorded with the oracle's
    # own value beside the reference's; the oracle must stay on it (a change
    # would be a regression, not parity).
    for rec in gold["multi_block_records"]:
        _, t = _oracle_tree(rec)
        assert np.float32(O.sah(t)) == np.float32(rec["oracle_sah"]), rec["name"]


def test_library_exports_header_symbols():
    """libatrbvh.so loads without a GPU and exports every function that
    include/atrbvh.h declares; the Python mirror binds each of them."""
    header = (ROOT / "include" / "atrbvh.h").read_text()
    declared = set(re.findall(r"\b(atr_[a-z0-9_]+)\s*\(", header))
    lib = ab.lib()
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert declared <= set(ab.EXPORTED), sorted(declared - set(ab.EXPORTED))


def test_library_reports_errors_without_device():
    """Entry points return a status (no exit) when called without a GPU or with
    bad arguments."""
    import ctypes as C
    h = C.c_void_p()
    st = ab.lib().atr_ctx_create(0, None, C.byref(h))
    if st == 0:
        ab.lib().atr_ctx_destroy(h)
        pytest.skip("a GPU is present")
    assert st in (2, 6)
    assert ab.lib().atr_last_error()
    assert ab.lib().atr_build_lbvh(None, None, 30, C.byref(h)) == 1


def test_oracle_workload_generators_match_product_and_digests():
    """The checker's own scene and ray generators (used by the host-core
    baseline and the reference arm of bench.py, which load nothing from the
    product library) produce the same bits as the product's generators and
    as the committed workload digests."""
    from tests._util import CASES, digest
    want = json.loads((GOLDEN / "workload_digests.json").read_text())
    kinds = {"uniform": O.SCENE_UNIFORM, "clustered": O.SCENE_CLUSTERED}
    for name, (kind, n, seed) in CASES.items():
        if kind in kinds:
            v = O.gen_scene(kinds[kind], n, seed)
            assert digest(v) == want[name], name
    for kind, n, seed in [(O.SCENE_CLUSTERED, 1 << 16, 0), (O.SCENE_UNIFORM, 3000, 4)]:
        a, b = O.gen_scene(kind, n, seed), ab.gen_scene(kind, n, seed)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (kind, n)
    a, b = O.gen_rays_pinhole(320, 200), ab.gen_rays_pinhole(320, 200)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    a, b = O.gen_rays_random(5000, [0, 0, 0], [1, 2, 3], 5), ab.gen_rays_random(5000, [0, 0, 0], [1, 2, 3], 5)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    sa, sb = O.gen_batch_sizes(4096, 256, 262144, 0), ab.gen_batch_sizes(4096, 256, 262144, 0)
    assert np.array_equal(sa, sb)
    assert np.array_equal(O.gen_batch_scene(sa[:40]).view(np.uint32), ab.gen_batch_scene(sb[:40]).view(np.uint32))


def test_cpu_golden_fullsize():
    """The committed full-size digests (tests/golden/fullsize_oracle.json,
    which the full-size GPU tests and bench.py's SAH check read) are the
    oracle's own outputs: the clustered 4,194,304-triangle pipeline end to
    end, and the 16,777,216-triangle LBVH and ATRBVH(9,2) trees."""
    from tests._util import collapsed_digests, digest, tree_digests
    gold = json.loads((GOLDEN / "fullsize_oracle.json").read_text())
    g = gold["c2"]
    v = O.gen_scene(O.SCENE_CLUSTERED, 4194304, 0)
    assert digest(v) == g["scene"]
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    t = O.atrbvh(base, 9, 2, threads=0)

    def tdig(x):
        return tree_digests(x.parent, x.left, x.right, x.data, x.bbox_min, x.bbox_max, x.area)

    assert tdig(base) == g["lbvh_tree"] and tdig(t) == g["tree"]
    assert np.float32(O.sah(t)) == np.float32(g["tree_sah"])
    c = O.collapse(t)
    assert np.float32(c.sah) == np.float32(g["collapsed_sah"])
    assert collapsed_digests(c.left, c.right, c.data, c.triangle_count, c.triangle_indices, len(v)) == g["collapsed"]
    cp = O.flatten(c, v)
    assert digest(cp.nodes) == g["compact2"]["nodes"] and digest(cp.tri_index) == g["compact2"]["tri_index"]
    assert digest(cp.woop) == g["compact2"]["woop"]
    rays = O.gen_rays_pinhole(1920, 1080)
    res = O.trace(cp, rays)
    assert digest(res[:, 0].copy()) == g["primary_hits"]["ids"] and digest(res[:, 1].copy()) == g["primary_hits"]["t"]
    g3 = gold["c3"]
    v = O.gen_scene(O.SCENE_UNIFORM, 16777216, 0)
    assert digest(v) == g3["scene"]
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    assert tdig(base) == g3["variants"]["lbvh"]["tree"]
    t = O.atrbvh(base, 9, 2, threads=0)
    assert tdig(t) == g3["variants"]["atrbvh_9_2"]["tree"]
