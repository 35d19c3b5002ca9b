"""Launch tuning and the autotuner: every tuning knob leaves the results
bit-exact (10-bit sort digits, ATRBVH block sizes, lane-group threshold), and
an autotuned batch equals the oracle built with each mesh's tuned parameters."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, scene_case

pytestmark = pytest.mark.gpu


@pytest.fixture()
def tuned_ctx():
    c = ab.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("case", ["u2", "u17", "u4097", "c1", "clu65536", "dupes3000", "same64"])
def test_ten_bit_sort_digits_bit_exact(tuned_ctx, case, bits):
    tuned_ctx.set_tuning(ab.TUNE_SORT_BITS, 10)
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    want, sk, si = O.build_lbvh(v, mn, mx, bits=bits, threads=8)
    scene = ab.SceneWrapper(tuned_ctx, v, mn, mx)
    tree = ab.LBVHBuilder(bits == 63).BuildTree(scene)
    keys, idx = tree.sorted_keys()
    assert np.array_equal(keys, sk) and np.array_equal(idx, si)
    assert_trees_equal(ab.BVHTreeInstanceManager().DeviceToHostTree(tree), want, f"{case}/{bits} 10-bit digits")


@pytest.mark.parametrize("warps,gmin,levels,qmin,wmax", [(2, 2, 16, 0, 0), (8, 2, 16, 0, 0), (4, 3, 0, 0, 0),
                                                         (4, 33, 0, -1, 0), (4, 2, 1, 0, 0), (4, 2, 4, -1, 0),
                                                         (2, 2, 64, 0, 0), (4, 2, 16, 0, 0), (4, 2, 16, -1, 0),
                                                         (8, 2, 64, 1000, 0), (8, 2, 12, -1, 1 << 30),
                                                         (2, 2, 16, 1000, 500), (8, 2, 12, 50000, 8192), (8, 2, 12, 20000, 4096)])
@pytest.mark.parametrize("treelet,iters", [(3, 1), (5, 2), (9, 2), (10, 3), (11, 2), (12, 1), (20, 1)])
def test_atrbvh_launch_tuning_bit_exact(tuned_ctx, warps, gmin, levels, qmin, wmax, treelet, iters):
    tuned_ctx.set_tuning(ab.TUNE_ATR_WARPS, warps)
    tuned_ctx.set_tuning(ab.TUNE_ATR_GROUP_MIN, gmin)
    tuned_ctx.set_tuning(ab.TUNE_ATR_LEVELS, levels)
    tuned_ctx.set_tuning(ab.TUNE_QUAD_MIN, qmin)
    tuned_ctx.set_tuning(ab.TUNE_WARP_MAX, wmax)
    v = scene_case("clu65536")
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    want = O.atrbvh(base, treelet, iters, threads=8)
    scene = ab.SceneWrapper(tuned_ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(treelet, iters).Optimize(tree)
    assert_trees_equal(ab.BVHTreeInstanceManager().DeviceToHostTree(tree), want,
                       f"ATRBVH({treelet},{iters}) warps {warps} group_min {gmin} levels {levels} quads {qmin} "
                       f"whole-warp {wmax}")


def test_tuning_rejects_bad_values(tuned_ctx):
    for knob, bad in [(ab.TUNE_ATR_WARPS, 3), (ab.TUNE_ATR_GROUP_MIN, 1), (ab.TUNE_SORT_BITS, 9),
                      (ab.TUNE_ATR_LEVELS, 65), (ab.TUNE_ATR_LEVELS, -1), (ab.TUNE_QUAD_MIN, -2), (ab.TUNE_WARP_MAX, -1), (7, 1)]:
        with pytest.raises(ab.AtrError):
            tuned_ctx.set_tuning(knob, bad)


def test_autotune_table_and_tuned_batch(tuned_ctx):
    warps0, bits0 = tuned_ctx.get_tuning(ab.TUNE_ATR_WARPS), tuned_ctx.get_tuning(ab.TUNE_SORT_BITS)
    table = ab.autotune(tuned_ctx, min_class=8, max_class=11, sample_triangles=1 << 15, reps=1)
    cls = table.classes()
    assert sorted(cls) == [8, 9, 10, 11]
    for c, e in cls.items():
        assert 5 <= e["treelet"] <= 9 and 1 <= e["iterations"] <= 3, e
        assert e["atr_warps"] in (2, 4, 8) and e["sort_bits"] in (8, 10), e
        assert e["sah_ratio"] <= 1.0 + 1e-6, e
        assert 0.0 < e["build_ms"] <= e["reference_ms"], e
        assert e["sample_meshes"] >= 2
    # The tuning context's own knobs are restored.
    assert tuned_ctx.get_tuning(ab.TUNE_ATR_WARPS) == warps0 and tuned_ctx.get_tuning(ab.TUNE_SORT_BITS) == bits0
    ts, it = table.class_arrays()
    assert ts[8] == cls[8]["treelet"] and ts[20] == cls[11]["treelet"] and ts[3] == cls[8]["treelet"]

    sizes = ab.gen_batch_sizes(24, 200, 5000, 4)
    v = ab.gen_batch_scene(sizes, 4)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    b = ab.Batch(tuned_ctx, v, off)
    b.apply_tuning(table)
    b.build(1, 9, 2, graph=True)
    b.build(1, 9, 2, graph=True)
    for m in range(len(sizes)):
        n = int(sizes[m])
        c = min(max(n.bit_length() - 1, 8), 11)
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        mn, mx = O.scene_aabb(vm)
        base, _, _ = O.build_lbvh(vm, mn, mx, threads=8)
        want = O.atrbvh(base, cls[c]["treelet"], cls[c]["iterations"], threads=8)
        assert_trees_equal(b.mesh(m), want, f"mesh {m} ({n} tris, class {c})")
    b.close()


def test_batch_autotune_never_slower_than_defaults(tuned_ctx):
    """atr_batch_autotune keeps its table only when the batch itself builds
    faster with it; either way the batch is left with parameters whose build
    equals the oracle's at those parameters, and the table's entries match
    what the batch uses."""
    sizes = ab.gen_batch_sizes(48, 256, 20000, 6)
    v = ab.gen_batch_scene(sizes, 6)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    b = ab.Batch(tuned_ctx, v, off)
    warps0, bits0 = tuned_ctx.get_tuning(ab.TUNE_ATR_WARPS), tuned_ctx.get_tuning(ab.TUNE_SORT_BITS)
    table, out = ab.batch_autotune(tuned_ctx, b, sample_triangles=1 << 15, reps=2)
    assert out["default_ms"] > 0 and out["tuned_ms"] > 0
    if out["kept"]:
        assert out["tuned_ms"] < out["default_ms"]
        assert out["tuned_sah"] <= out["default_sah"] * (1 + 1e-12)
    else:
        for e in table.classes().values():
            assert (e["treelet"], e["iterations"], e["atr_warps"], e["sort_bits"]) == (9, 2, warps0, bits0), e
        assert tuned_ctx.get_tuning(ab.TUNE_ATR_WARPS) == warps0
    present = {int(n).bit_length() - 1 for n in sizes}
    assert set(table.classes()) == present
    b.build(1, 9, 2, graph=True)
    for m in range(0, len(sizes), 5):
        e = table.classes()[int(sizes[m]).bit_length() - 1]
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        mn, mx = O.scene_aabb(vm)
        base, _, _ = O.build_lbvh(vm, mn, mx, threads=8)
        want = O.atrbvh(base, e["treelet"], e["iterations"], threads=8)
        assert_trees_equal(b.mesh(m), want, f"mesh {m}")
    b.close()
    tuned_ctx.set_tuning(ab.TUNE_ATR_WARPS, warps0)
    tuned_ctx.set_tuning(ab.TUNE_SORT_BITS, bits0)
