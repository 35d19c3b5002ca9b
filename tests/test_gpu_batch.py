"""Segmented batch builds: every mesh of a batch equals the build of that mesh
alone (and the oracle), with uniform and per-mesh parameters, eager and
graph-replayed."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, check_tree

pytestmark = pytest.mark.gpu


def _meshes(count: int, lo: int, hi: int, seed: int):
    sizes = ab.gen_batch_sizes(count, lo, hi, seed)
    v = ab.gen_batch_scene(sizes, seed)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    return v, off


def _oracle_mesh(v, off, m, opt, treelet, iters):
    vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
    mn, mx = O.scene_aabb(vm)
    t, _, _ = O.build_lbvh(vm, mn, mx, threads=8)
    if opt == 1:
        t = O.atrbvh(t, treelet, iters, threads=8)
    elif opt == 2:
        t = O.trbvh(t, 7, iters, threads=8)
    return t


@pytest.mark.parametrize("opt,treelet,iters", [(0, 9, 0), (1, 9, 2), (1, 5, 1), (2, 7, 2)])
def test_batch_meshes_equal_oracle(ctx, opt, treelet, iters):
    v, off = _meshes(40, 2, 20000, 1)
    # Include tiny meshes and a tile-boundary size.
    b = ab.Batch(ctx, v, off)
    b.build(opt, treelet, iters)
    rng = np.random.default_rng(0)
    for m in sorted(set(rng.choice(len(off) - 1, 12, replace=False).tolist()) | {0, len(off) - 2}):
        got = b.mesh(m)
        want = _oracle_mesh(v, off, m, opt, treelet, iters)
        assert_trees_equal(got, want, f"mesh {m} ({off[m + 1] - off[m]} tris)")
        check_tree(got, int(off[m + 1] - off[m]))


def test_batch_equals_plain_builds(ctx):
    """Every mesh of a 256-mesh batch equals atr_build_lbvh + ATRBVH of that
    mesh alone (plain per-mesh launches), and so do the per-mesh SAH values."""
    v, off = _meshes(256, 256, 65536, 3)
    b = ab.Batch(ctx, v, off)
    b.build(1, 9, 2, graph=True)
    b.build(1, 9, 2, graph=True)  # replay
    sah = b.sah()
    mgr = ab.BVHTreeInstanceManager()
    for m in range(0, 256, 17):
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        scene = ab.SceneWrapper(ctx, vm)
        tree = ab.LBVHBuilder().BuildTree(scene)
        ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
        plain = mgr.DeviceToHostTree(tree)
        assert_trees_equal(b.mesh(m), plain, f"mesh {m}")
        assert np.float32(sah[m]) == np.float32(plain.SAH())


def test_batch_per_mesh_params(ctx):
    v, off = _meshes(24, 100, 30000, 5)
    count = len(off) - 1
    rng = np.random.default_rng(1)
    ts = rng.choice([5, 7, 9], count).astype(np.uint8)
    it = rng.integers(0, 4, count).astype(np.uint8)
    b = ab.Batch(ctx, v, off)
    b.set_params(ts, it)
    b.build(1, 9, 2, graph=True)
    for m in range(count):
        want = _oracle_mesh(v, off, m, 1, int(ts[m]), int(it[m]))
        assert_trees_equal(b.mesh(m), want, f"mesh {m} ATRBVH({ts[m]},{it[m]})")


def test_batch_rejects_bad_offsets(ctx):
    v, off = _meshes(4, 10, 100, 2)
    bad = off.copy()
    bad[2] = bad[1] + 1  # a one-triangle mesh
    with pytest.raises(ab.AtrError):
        ab.Batch(ctx, v, bad)


def _single(ctx, vm, treelet=9, iters=2, max_leaf=0):
    scene = ab.SceneWrapper(ctx, vm)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(treelet, iters).Optimize(tree)
    col, sah = ab.BVHTreeCollapser().Collapse(tree, max_leaf=max_leaf)
    return scene, tree, col, sah, ab.CudaBVH(col, scene)


def _assert_compact_equal(got, want, what):
    gn, gw, gt = got
    wn, ww, wt = want
    assert gn.shape == wn.shape and gw.shape == ww.shape, what
    assert np.array_equal(gn, wn), what
    assert np.array_equal(gw.view(np.int32), ww.view(np.int32)), what
    assert np.array_equal(gt, wt), what


@pytest.mark.parametrize("max_leaf", [0, 4])
def test_batch_collapse_flatten_equal_single(ctx, max_leaf):
    """Per-mesh collapse SAH and Compact2 arrays of a batch equal
    atr_collapse + atr_flatten_compact2 of each mesh alone."""
    v, off = _meshes(30, 2, 20000, 7)
    b = ab.Batch(ctx, v, off)
    b.build(1, 9, 2)
    sah = b.collapse(max_leaf=max_leaf)
    b.flatten()
    count = len(off) - 1
    for m in sorted(set(range(0, count, 4)) | {count - 1}):
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        _, _, _, s, bvh = _single(ctx, vm, max_leaf=max_leaf)
        assert np.float32(sah[m]) == np.float32(s), f"mesh {m} sah"
        _assert_compact_equal(b.compact(m), bvh.download(), f"mesh {m}")
        assert b.compact_view(m).max_depth >= 1


def test_batch_merged_ray_queue_equals_single_traces(ctx):
    """One merged queue of ray groups (meshes repeated and out of order) gives
    the same closest hits as tracing each group against its mesh alone."""
    import torch
    v, off = _meshes(12, 500, 30000, 9)
    b = ab.Batch(ctx, v, off)
    b.build(1, 9, 2)
    b.collapse(want_sah=False)
    b.flatten()
    order = [3, 0, 11, 3, 7, 1, 5]
    groups, offsets, singles = [], [0], {}
    for g, m in enumerate(order):
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        mn = vm[:, :, :3].reshape(-1, 3).min(0)
        mx = vm[:, :, :3].reshape(-1, 3).max(0)
        r = ab.gen_rays_random(3000 + 517 * g, mn, mx, seed=g)
        groups.append(r)
        offsets.append(offsets[-1] + len(r))
        if m not in singles:
            singles[m] = _single(ctx, vm)
    rays = np.concatenate(groups)
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    b.trace(rd.data_ptr(), len(rays), offsets, order, res.data_ptr())
    ctx.synchronize()
    got = res.cpu().numpy().reshape(-1, 4)
    for g, m in enumerate(order):
        bvh = singles[m][4]
        r = groups[g]
        rg = torch.from_numpy(np.ascontiguousarray(r, np.float32).reshape(-1)).cuda()
        rs = torch.zeros(len(r) * 4, dtype=torch.int32, device="cuda")
        bvh.trace(rg.data_ptr(), len(r), rs.data_ptr())
        ctx.synchronize()
        want = rs.cpu().numpy().reshape(-1, 4)
        part = got[offsets[g]:offsets[g + 1]]
        assert (want[:, 0] >= 0).sum() > 0
        assert np.array_equal(part[:, :2], want[:, :2]), f"group {g} mesh {m}"


def test_batch_refit_mesh_equals_single_refit(ctx):
    """Refitting one resident mesh of a flattened batch equals refit +
    collapse + flatten of that mesh alone, and leaves the other meshes as
    they were."""
    v, off = _meshes(10, 1000, 20000, 4)
    b = ab.Batch(ctx, v, off)
    b.build(1, 9, 2)
    b.collapse(want_sah=False)
    b.flatten()
    count = len(off) - 1
    before = [b.compact(m) for m in range(count)]
    m = 6
    vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
    rng = np.random.default_rng(3)
    w = (vm + rng.normal(0, 0.002, vm.shape).astype(np.float32)).astype(np.float32)
    w[:, :, 3] = 0
    for _ in range(2):
        b.refit_mesh(m, w)
    scene, tree, _, _, _ = _single(ctx, vm)
    scene.set_vertices(w)
    ab.Refit(tree, scene)
    assert_trees_equal(b.mesh(m), ab.BVHTreeInstanceManager().DeviceToHostTree(tree), "refit tree")
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    _assert_compact_equal(b.compact(m), ab.CudaBVH(col, scene).download(), "refit compact")
    for k in range(count):
        if k != m:
            _assert_compact_equal(b.compact(k), before[k], f"untouched mesh {k}")
