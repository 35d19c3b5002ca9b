"""GPU parity: Morton codes, sort, LBVH, refit and ATRBVH through the C ABI
against the oracle, bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, check_tree, scene_case

pytestmark = pytest.mark.gpu

CASES_LBVH = ["u2", "u3", "u5", "u17", "u100", "u1000", "u4097", "c1", "clu4096", "clu65536", "dupes3000",
              "flat2000", "same64"]


def _gpu_tree(ctx, v, bits=30, bounds=True):
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn if bounds else None, mx if bounds else None)
    tree = ab.LBVHBuilder(bits == 63).BuildTree(scene)
    return scene, tree


@pytest.mark.parametrize("case", ["u100", "c1", "clu65536", "dupes3000", "flat2000", "same64"])
def test_scene_bounds_on_device(ctx, case):
    v = scene_case(case)
    scene = ab.SceneWrapper(ctx, v)
    mn, mx = scene.bounds()
    omn, omx = O.scene_aabb(v)
    assert np.array_equal(mn, omn) and np.array_equal(mx, omx)


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("case", CASES_LBVH)
def test_lbvh_bit_exact(ctx, case, bits):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    want, sk, si = O.build_lbvh(v, mn, mx, bits=bits, threads=8)
    scene, tree = _gpu_tree(ctx, v, bits)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    keys, idx = tree.sorted_keys()
    assert np.array_equal(keys, sk), "sorted Morton keys"
    assert np.array_equal(idx, si), "sorted triangle order"
    assert_trees_equal(got, want, f"{case}/{bits}")
    check_tree(got, len(v))
    assert np.float32(got.SAH()) == np.float32(O.sah(want))
    assert np.float32(tree.sah()) == np.float32(O.sah(want))


def test_lbvh_device_bounds_equal_host_bounds(ctx):
    v = scene_case("clu65536")
    _, t1 = _gpu_tree(ctx, v, bounds=True)
    _, t2 = _gpu_tree(ctx, v, bounds=False)
    m = ab.BVHTreeInstanceManager()
    assert_trees_equal(m.DeviceToHostTree(t1), m.DeviceToHostTree(t2), "device vs host bounds")


def test_lbvh_full_size_c2(ctx):
    """4,194,304-triangle clustered scene: bit-exact against the oracle."""
    v = ab.gen_scene(ab.SCENE_CLUSTERED, 4194304, 0)
    mn, mx = O.scene_aabb(v)
    want, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    _, tree = _gpu_tree(ctx, v)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, "C2 LBVH")


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n", [1, 7, 4096, 4097, 100003, 3000000])
def test_device_sort_pairs_stable(ctx, n, bits):
    import torch
    rng = np.random.default_rng(n + bits)
    if bits == 32:
        keys = rng.integers(0, 1 << 12, n, dtype=np.uint32) * np.uint32(1 << 18) + rng.integers(0, 3, n, dtype=np.uint32)
    else:
        keys = rng.integers(0, 1 << 62, n, dtype=np.uint64) & np.uint64(0x7F000000000000FF)
    vals = np.arange(n, dtype=np.uint32)[::-1].copy()
    kd = torch.from_numpy(keys.view(np.int32 if bits == 32 else np.int64).copy()).cuda()
    vd = torch.from_numpy(vals.view(np.int32)).cuda()
    ab.check(ab.lib().atr_device_sort_pairs(ctx.handle, kd.data_ptr(), vd.data_ptr(), n, bits))
    ctx.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(kd.cpu().numpy().view(keys.dtype), keys[order])
    assert np.array_equal(vd.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("bits", [30, 63])
def test_device_morton(ctx, bits):
    import torch
    v = scene_case("c1")
    mn, mx = O.scene_aabb(v)
    vd = torch.from_numpy(v.reshape(-1)).cuda()
    kd = torch.empty(len(v), dtype=torch.int32 if bits == 30 else torch.int64, device="cuda")
    ab.check(ab.lib().atr_device_morton(ctx.handle, vd.data_ptr(), len(v), ab._f3(mn), ab._f3(mx), bits,
                                        kd.data_ptr()))
    got = kd.cpu().numpy().view(np.uint32 if bits == 30 else np.uint64)
    assert np.array_equal(got, O.morton(v, mn, mx, bits))


@pytest.mark.parametrize("case", ["u100", "c1", "clu65536", "dupes3000"])
def test_refit_bit_exact(ctx, case):
    """Refit of a resident optimised tree after vertex jitter equals the oracle's
    refit of the same topology."""
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene, tree = _gpu_tree(ctx, v)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    rng = np.random.default_rng(4)
    v2 = (v + rng.normal(0, 0.001, v.shape).astype(np.float32)).astype(np.float32)
    v2[:, :, 3] = 0
    scene.set_vertices(v2)
    ab.Refit(tree, scene)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    want = O.Tree(got.parent.copy(), got.left.copy(), got.right.copy(), got.data.copy(),
                  np.zeros_like(got.bbox_min), np.zeros_like(got.bbox_max), np.zeros_like(got.area))
    O.lib().orc_refit(O._ptr(v2), len(v2), *want.ptrs(), 1)
    assert_trees_equal(got, want, "refit")


ATR_CASES = ["u17", "u100", "u1000", "u4097", "clu4096", "dupes3000", "flat2000", "same64"]


@pytest.mark.parametrize("treelet,iters", [(3, 1), (5, 1), (7, 2), (9, 2), (9, 3), (10, 1), (11, 2), (12, 2), (16, 1), (20, 1)])
@pytest.mark.parametrize("case", ATR_CASES)
def test_atrbvh_bit_exact(ctx, case, treelet, iters):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    want = O.atrbvh(base, treelet, iters, threads=8)
    _, tree = _gpu_tree(ctx, v)
    ab.AgglomerativeTreeletOptimizer(treelet, iters).Optimize(tree)
    ctx.synchronize()
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, f"{case} ATRBVH({treelet},{iters})")
    assert np.float32(got.SAH()) == np.float32(O.sah(want))


@pytest.mark.parametrize("case", ["c1", "clu65536"])
def test_atrbvh_c1_bit_exact(ctx, case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    want = O.atrbvh(base, 9, 2, threads=0)
    _, tree = _gpu_tree(ctx, v)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, f"{case} ATRBVH(9,2)")
    check_tree(got, len(v))


def test_atrbvh_full_size_c2(ctx):
    """4,194,304 triangles, ATRBVH(9,2): bit-exact against the oracle."""
    v = ab.gen_scene(ab.SCENE_CLUSTERED, 4194304, 0)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    want = O.atrbvh(base, 9, 2, threads=0)
    _, tree = _gpu_tree(ctx, v)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, "C2 ATRBVH(9,2)")


def test_invalid_arguments_rejected(ctx):
    v = scene_case("u100")
    _, tree = _gpu_tree(ctx, v)
    with pytest.raises(ab.AtrError):
        ab.AgglomerativeTreeletOptimizer(21, 1).Optimize(tree)
    with pytest.raises(ab.AtrError):
        ab.AgglomerativeTreeletOptimizer(2, 1).Optimize(tree)
    with pytest.raises(ab.AtrError):
        ab.SceneWrapper(ctx, v[:1])
