"""Build plans (atr_plan_*): the single-mesh build replayed from a CUDA graph
gives the same tree, collapsed tree, SAH and Compact2 bytes as the eager
calls and the oracle, across replays, vertex updates and launch-tuning
changes."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, scene_case

pytestmark = pytest.mark.gpu


def _oracle(v, opt, ts, it, bounds=None):
    mn, mx = O.scene_aabb(v) if bounds is None else bounds
    t, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    if opt == 1:
        t = O.atrbvh(t, ts, it, threads=0)
    elif opt == 2:
        t = O.trbvh(t, ts, it, threads=0)
    c = O.collapse(t)
    return t, c, O.flatten(c, v)


def _check(plan, v, opt, ts, it, what, bounds=None):
    t, c, cp = _oracle(v, opt, ts, it, bounds)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(plan.tree())
    assert_trees_equal(got, t, what)
    assert np.float32(plan.sah()) == np.float32(c.sah), what
    nodes, woop, tri = plan.compact().download()
    assert np.array_equal(nodes, cp.nodes) and np.array_equal(tri, cp.tri_index), what
    assert np.array_equal(woop.view(np.int32), cp.woop.view(np.int32)), what


@pytest.mark.parametrize("case,opt,ts,it", [("clu4096", 1, 9, 2), ("c1", 1, 9, 2), ("u4097", 1, 5, 3),
                                            ("dupes3000", 2, 7, 2), ("u1000", 0, 0, 0), ("clu65536", 1, 16, 1)])
def test_plan_graph_replays_match_oracle(ctx, case, opt, ts, it):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    plan = ab.BuildPlan(scene, optimizer=opt, treelet=ts, iterations=it)
    plan.run(graph=False)
    _check(plan, v, opt, ts, it, f"{case} eager")
    for k in range(3):
        plan.run(graph=True)
        _check(plan, v, opt, ts, it, f"{case} replay {k}")
    build_ms, flatten_ms = plan.times()
    assert build_ms > 0 and flatten_ms > 0
    plan.close()
    scene.close()


def test_plan_follows_vertex_updates_and_tuning(ctx):
    """A captured plan rebuilds whatever the scene holds when it runs; a
    change of launch tuning captures the graph again, with equal results."""
    v = scene_case("c1")
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    plan = ab.BuildPlan(scene)
    plan.run(graph=True)
    _check(plan, v, 1, 9, 2, "first")
    rng = np.random.default_rng(3)
    w = (v + rng.normal(0, 0.002, v.shape).astype(np.float32)).astype(np.float32)
    w[:, :, 3] = 0
    scene.set_vertices(w)  # the scene keeps the box it was created with
    plan.run(graph=True)
    _check(plan, w, 1, 9, 2, "after set_vertices", (mn, mx))
    ctx.set_tuning(ab.TUNE_ATR_WARPS, 4)
    try:
        plan.run(graph=True)
        _check(plan, w, 1, 9, 2, "after retuning", (mn, mx))
    finally:
        ctx.set_tuning(ab.TUNE_ATR_WARPS, 8)
    plan.close()
    scene.close()


def test_plan_rejects_bad_parameters(ctx):
    v = scene_case("u100")
    scene = ab.SceneWrapper(ctx, v)
    for kw in (dict(treelet=2), dict(optimizer=2, treelet=9), dict(morton_bits=31), dict(iterations=-1)):
        with pytest.raises(ab.AtrError):
            ab.BuildPlan(scene, **kw)
    scene.close()
