"""GPU parity of atr_refit: boxes and areas of a resident topology after
vertex jitter equal the oracle's refit of the same topology, bit for bit --
the first refit of a topology (a climb over global memory) and the later ones
(the topology's refit plan, built by the second refit) -- on LBVH, ATRBVH and
TRBVH trees, on repeated refits that reuse the plan, after an optimiser
changed the topology (the plan is rebuilt), and at the clustered
4,194,304-triangle size."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, scene_case

pytestmark = pytest.mark.gpu


def _jitter(v, seed, sigma=0.001):
    rng = np.random.default_rng(seed)
    v2 = (v + rng.normal(0, sigma, v.shape)).astype(np.float32)
    v2[:, :, 3] = 0
    return v2


def _oracle_refit(got, v, threads=1):
    want = O.Tree(got.parent.copy(), got.left.copy(), got.right.copy(), got.data.copy(),
                  np.zeros_like(got.bbox_min), np.zeros_like(got.bbox_max), np.zeros_like(got.area))
    O.lib().orc_refit(O._ptr(v), len(v), *want.ptrs(), threads)
    return want


def _refit_and_check(scene, tree, v2, what, threads=1):
    scene.set_vertices(v2)
    ab.Refit(tree, scene)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, _oracle_refit(got, v2, threads), what)


@pytest.mark.parametrize("opt", ["lbvh", "atrbvh", "trbvh"])
@pytest.mark.parametrize("case", ["u2", "u3", "u5", "u17", "u1000", "u4097", "c1", "clu65536", "dupes3000",
                                  "flat2000", "same64"])
def test_planned_refit_matches_oracle(ctx, case, opt):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    if opt == "atrbvh":
        ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    elif opt == "trbvh":
        ab.TRBVHOptimizer(7, 1).Optimize(tree)
    _refit_and_check(scene, tree, _jitter(v, 4), f"{case}/{opt} first refit")
    _refit_and_check(scene, tree, _jitter(v, 5), f"{case}/{opt} planned refit")
    _refit_and_check(scene, tree, _jitter(v, 6), f"{case}/{opt} planned refit again")


def test_planned_refit_reuse_and_topology_change(ctx):
    """Three refits of one topology share a plan; an optimiser pass changes the
    topology and the next refit builds a new plan -- every result equals the
    oracle's refit of the tree as it stands."""
    v = scene_case("clu65536")
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    for k in range(3):
        _refit_and_check(scene, tree, _jitter(v, 10 + k), f"lbvh refit {k}")
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    for k in range(2):
        _refit_and_check(scene, tree, _jitter(v, 20 + k), f"atrbvh refit {k}")
    tree2 = ab.LBVHBuilder().BuildTree(scene)  # a new tree of the same scene: its own plan
    _refit_and_check(scene, tree2, _jitter(v, 30), "second tree")
    _refit_and_check(scene, tree, _jitter(v, 31), "first tree again")


@pytest.mark.parametrize("opt", ["lbvh", "atrbvh"])
def test_planned_refit_full_size_clustered(ctx, opt):
    """The clustered 4,194,304-triangle scene: LBVH or LBVH + ATRBVH(9,2), then
    two refits after jitter, each equal to the oracle's."""
    v = ab.gen_scene(ab.SCENE_CLUSTERED, 4194304, 0)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    if opt == "atrbvh":
        ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    threads = O.max_threads()
    for k in range(2):
        _refit_and_check(scene, tree, _jitter(v, 40 + k), f"4.2M {opt} refit {k}", threads)
