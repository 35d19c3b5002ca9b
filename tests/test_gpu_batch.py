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
