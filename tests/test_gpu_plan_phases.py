"""Phase marks recorded inside a build plan's graph when the context times
phases: one device time per phase of the last replay, positive, and summing to
about the build time measured around the same phases; none without."""
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import scene_case

pytestmark = pytest.mark.gpu


def test_plan_phase_times_after_replay(ctx):
    v = scene_case("c1")
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    plan = ab.BuildPlan(scene)
    with pytest.raises(ab.AtrError):
        plan.phase_times()  # no replay yet
    plan.run(graph=True)
    assert plan.phase_times() == []  # captured without phase timing: no marks
    ctx.set_timing(True)  # the next replay captures the graph again, with marks
    try:
        for _ in range(3):
            plan.run(graph=True)
        ph = dict(plan.phase_times())
    finally:
        ctx.set_timing(False)
    assert set(ph) == {"morton", "sort", "build", "atrbvh", "collapse", "flatten"}, ph
    assert all(t > 0 for t in ph.values())
    build_ms, flatten_ms = plan.times()
    inner = sum(ph[k] for k in ("morton", "sort", "build", "atrbvh", "collapse"))
    assert inner <= build_ms * 1.02 + 0.01
    assert ph["flatten"] <= flatten_ms * 1.02 + 0.01
    plan.close()
    scene.close()
