"""GPU parity: TRBVH, collapse, Compact2 flatten and traversal through the C ABI
against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, check_tree, scene_case

pytestmark = pytest.mark.gpu


def _build(ctx, v, opt=None):
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    want = base
    if opt == "atrbvh":
        ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
        want = O.atrbvh(base, 9, 2, threads=8)
    elif opt == "trbvh":
        ab.TRBVHOptimizer(7, 3).Optimize(tree)
        want = O.trbvh(base, 7, 3, threads=8)
    return scene, tree, want


@pytest.mark.parametrize("iters", [1, 2, 3])
@pytest.mark.parametrize("case", ["u17", "u100", "u1000", "u4097", "clu4096", "dupes3000", "flat2000", "same64", "c1"])
def test_trbvh_bit_exact(ctx, case, iters):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    want = O.trbvh(base, 7, iters, threads=8)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.TRBVHOptimizer(7, iters).Optimize(tree)
    ctx.synchronize()
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, f"{case} TRBVH(7,{iters})")
    check_tree(got, len(v))


def test_trbvh_rejects_other_sizes(ctx):
    v = scene_case("u100")
    _, tree, _ = _build(ctx, v)
    with pytest.raises(ab.AtrError):
        ab.TRBVHOptimizer(6, 1).Optimize(tree)


def _collapsed_matches(got: ab.HostCollapsedTree, want: O.Collapsed, n: int) -> None:
    for f in ("parent", "left", "right", "triangle_count"):
        assert np.array_equal(getattr(got, f), getattr(want, f)), f
    for f in ("bbox_min", "bbox_max"):
        assert np.array_equal(getattr(got, f)[:, :3], getattr(want, f)[:, :3]), f
    # data: equal except list offsets of emitted leaves; compare lists instead.
    emitted = (want.triangle_count > 1) & (want.data >= 0)
    assert np.array_equal(got.data[~emitted], want.data[~emitted])
    assert np.array_equal(got.data >= 0, want.data >= 0)
    gl = O.leaf_lists(got.left, got.right, got.data, got.triangle_count, got.triangle_indices, n)
    wl = O.leaf_lists(want.left, want.right, want.data, want.triangle_count, want.triangle_indices, n)
    assert gl == wl


@pytest.mark.parametrize("max_leaf", [0, 4])
@pytest.mark.parametrize("case", ["u100", "u1000", "clu4096", "dupes3000", "flat2000", "same64", "c1", "clu65536"])
def test_collapse_matches_oracle(ctx, case, max_leaf):
    v = scene_case(case)
    _, tree, want_tree = _build(ctx, v, "atrbvh")
    col, sah = ab.BVHTreeCollapser().Collapse(tree, max_leaf=max_leaf)
    want = O.collapse(want_tree, max_leaf=max_leaf)
    assert np.float32(sah) == np.float32(want.sah)
    got = ab.BVHTreeInstanceManager().DeviceToHostCollapsedTree(col)
    _collapsed_matches(got, want, len(v))
    if max_leaf:
        ll = O.leaf_lists(got.left, got.right, got.data, got.triangle_count, got.triangle_indices, len(v))
        assert max(len(x) for x in ll.values()) <= max_leaf


def compact_arrays(bvh: ab.CudaBVH):
    nodes, woop, tri = bvh.download()
    return nodes, woop, tri, bvh.view().max_depth


@pytest.mark.parametrize("case", ["u100", "u1000", "clu4096", "dupes3000", "same64", "c1", "clu65536"])
def test_flatten_byte_identical(ctx, case):
    """The device-built Compact2 arrays equal the reference's host DFS layout
    (restated by the oracle) byte for byte."""
    v = scene_case(case)
    scene, tree, want_tree = _build(ctx, v, "atrbvh")
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    bvh = ab.CudaBVH(col, scene)
    nodes, woop, tri, depth = compact_arrays(bvh)
    want = O.flatten(O.collapse(want_tree), v)
    assert nodes.shape == want.nodes.shape and woop.shape == want.woop.shape
    assert np.array_equal(nodes, want.nodes)
    assert np.array_equal(woop.view(np.int32), want.woop.view(np.int32))
    assert np.array_equal(tri, want.tri_index)
    assert depth >= 1


def _trace_gpu(ctx, bvh, rays, any_hit=False):
    import torch
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rd.data_ptr(), len(rays), res.data_ptr(), any_hit=any_hit)
    ctx.synchronize()
    return res.cpu().numpy().reshape(-1, 4)


@pytest.mark.parametrize("any_hit", [False, True])
@pytest.mark.parametrize("case,opt", [("u1000", "atrbvh"), ("c1", "atrbvh"), ("c1", "trbvh"), ("c1", None),
                                      ("clu65536", "atrbvh"), ("dupes3000", "atrbvh"), ("same64", "atrbvh")])
def test_trace_bit_exact(ctx, case, opt, any_hit):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene, tree, want_tree = _build(ctx, v, opt)
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    bvh = ab.CudaBVH(col, scene)
    cp = O.flatten(O.collapse(want_tree), v)
    rays = np.concatenate([ab.gen_rays_random(60000, mn, mx, seed=7),
                           ab.gen_rays_pinhole(160, 120, eye=(0.5, 0.5, -1.5), fov_deg=60.0)])
    got = _trace_gpu(ctx, bvh, rays, any_hit)
    want = O.trace(cp, rays, any_hit=any_hit)
    assert (got[:, 0] >= 0).sum() > 0
    assert np.array_equal(got[:, 0], want[:, 0]), f"hit ids differ on {(got[:, 0] != want[:, 0]).sum()} rays"
    assert np.array_equal(got[:, 1], want[:, 1]), "hit t differs"


def test_trace_full_size_c3_rays(ctx):
    """16,777,216 uniform triangles, 8,388,608 random rays: hit ids and t
    equal the oracle's on a 65,536-ray sample and the hit fraction is sane."""
    v = ab.gen_scene(ab.SCENE_UNIFORM, 16777216, 0)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    bvh = ab.CudaBVH(col, scene)
    rays = ab.gen_rays_random(1 << 23, mn, mx, seed=3)
    got = _trace_gpu(ctx, bvh, rays)
    # Oracle on a sample, over the GPU tree's own collapsed arrays.
    m = ab.BVHTreeInstanceManager()
    hc = m.DeviceToHostCollapsedTree(col)
    oc = O.Collapsed(hc.parent, hc.left, hc.right, hc.data, hc.triangle_count, hc.bbox_min, hc.bbox_max,
                     hc.triangle_indices, np.zeros(0, np.float32), 0.0)
    cp = O.flatten(oc, v)
    idx = np.random.default_rng(0).choice(len(rays), 65536, replace=False)
    want = O.trace(cp, rays[idx])
    assert np.array_equal(got[idx, 0], want[:, 0])
    assert np.array_equal(got[idx, 1], want[:, 1])
    assert 0.2 < (got[:, 0] >= 0).mean() <= 1.0


def test_bounce_rays_trace(ctx):
    """Primary pinhole rays then one diffuse bounce per hit (the clustered
    scene's workload); bounce rays traced on the device match the oracle."""
    import torch
    v = scene_case("clu65536")
    mn, mx = O.scene_aabb(v)
    scene, tree, want_tree = _build(ctx, v, "atrbvh")
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    bvh = ab.CudaBVH(col, scene)
    prim = ab.gen_rays_pinhole(320, 240)
    pd = torch.from_numpy(prim.reshape(-1)).cuda()
    res = torch.zeros(len(prim) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(pd.data_ptr(), len(prim), res.data_ptr())
    bounce = torch.zeros_like(pd)
    ab.check(ab.lib().atr_gen_bounce_rays(ctx.handle, scene.handle, pd.data_ptr(), res.data_ptr(), len(prim), 5,
                                          bounce.data_ptr()))
    res2 = torch.zeros_like(res)
    bvh.trace(bounce.data_ptr(), len(prim), res2.data_ptr())
    ctx.synchronize()
    cp = O.flatten(O.collapse(want_tree), v)
    b = bounce.cpu().numpy().reshape(-1, 2, 4)
    want = O.trace(cp, b)
    got = res2.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(got[:, :2], want[:, :2])
    assert (res.cpu().numpy().reshape(-1, 4)[:, 0] >= 0).any()
