"""GPU parity of the triangle-splitting path: the splitting step
(atr_split_triangles) and the primitive-box LBVH (atr_build_lbvh_split, the
reference's LBVH.cu:99-161, 320-428, 572-669) against the oracle, bit for bit;
the whole pipeline (split -> primitive-box LBVH -> ATRBVH -> collapse ->
Compact2 -> traversal) against the oracle's, and its hits against the
unsplit pipeline's."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, scene_case

pytestmark = pytest.mark.gpu

CASES = ["u17", "u1000", "u4097", "c1", "dupes3000", "flat2000", "same64", "sliver20000", "sliver262144"]


@pytest.mark.parametrize("ratio", [0.0, 0.3, 1.0])
@pytest.mark.parametrize("case", CASES)
def test_split_fragments_match_oracle(ctx, case, ratio):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    bmin, bmax, data = ab.split_triangles(scene, ratio)
    wmin, wmax, wdata = O.split_triangles(v, ratio)
    assert len(data) == len(wdata)
    assert np.array_equal(data.cpu().numpy().astype(np.uint32), wdata)
    assert np.array_equal(bmin.cpu().numpy()[:, :3], wmin[:, :3])
    assert np.array_equal(bmax.cpu().numpy()[:, :3], wmax[:, :3])


@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("case", CASES)
def test_split_lbvh_matches_oracle(ctx, case, bits):
    """The primitive-box LBVH over the oracle's fragments equals the oracle's
    restatement of the reference's primitive-box kernels (which the CPU
    tests pin to the reference's own kernels)."""
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    wmin, wmax, wdata = O.split_triangles(v, 0.3)
    want = O.build_lbvh_split(wmin, wmax, wdata, mn, mx, bits, threads=8)
    tree = ab.build_lbvh_split(ctx, torch.from_numpy(wmin).cuda(), torch.from_numpy(wmax).cuda(),
                               torch.from_numpy(wdata.astype(np.int32)).cuda(), mn, mx, bits)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, f"{case} split {bits}-bit")


def _trace_gpu(ctx, bvh, rays):
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rd.data_ptr(), len(rays), res.data_ptr())
    ctx.synchronize()
    return res.cpu().numpy().reshape(-1, 4)


@pytest.mark.parametrize("case", ["u1000", "sliver20000", "sliver262144"])
def test_split_pipeline_matches_oracle(ctx, case):
    """Split on the device, primitive-box LBVH, ATRBVH(9,2), collapse, Compact2
    and closest-hit traversal: every stage equals the oracle's; the hits equal
    the unsplit pipeline's (splitting changes the tree, not what a ray hits);
    on the sliver scenes the split tree's SAH is lower."""
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    bmin, bmax, data = ab.split_triangles(scene, 0.3)
    tree = ab.build_lbvh_split(ctx, bmin, bmax, data, mn, mx)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    wmin, wmax, wdata = O.split_triangles(v, 0.3)
    want = O.atrbvh(O.build_lbvh_split(wmin, wmax, wdata, mn, mx, 30, threads=8), 9, 2, threads=8)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert_trees_equal(got, want, f"{case} split + ATRBVH")
    col, sah = ab.BVHTreeCollapser().Collapse(tree)
    wc = O.collapse(want)
    assert np.float32(sah) == np.float32(wc.sah)
    bvh = ab.CudaBVH(col, scene)
    nodes, woop, tri = bvh.download()
    wcp = O.flatten(wc, v)
    assert np.array_equal(nodes, wcp.nodes) and np.array_equal(tri, wcp.tri_index)
    assert np.array_equal(woop.view(np.int32), wcp.woop.view(np.int32))
    rays = ab.gen_rays_random(60000, mn, mx, seed=7)
    hits = _trace_gpu(ctx, bvh, rays)
    assert np.array_equal(hits[:, :2], O.trace(wcp, rays)[:, :2])
    base, _, _ = O.build_lbvh(v, mn, mx, threads=8)
    plain = O.atrbvh(base, 9, 2, threads=8)
    plain_hits = O.trace(O.flatten(O.collapse(plain), v), rays)
    assert (hits[:, 0] >= 0).sum() > 0
    assert np.array_equal(hits[:, :2], plain_hits[:, :2])
    if case.startswith("sliver"):
        assert O.sah(want) < 0.75 * O.sah(plain)


def test_split_tree_rejects_refit(ctx):
    v = scene_case("u1000")
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    bmin, bmax, data = ab.split_triangles(scene, 0.3)
    tree = ab.build_lbvh_split(ctx, bmin, bmax, data, mn, mx)
    with pytest.raises(ab.AtrError):
        ab.Refit(tree, scene)


def test_split_room_and_arguments(ctx):
    """Room for fewer primitives than triangles, or a negative ratio, is an
    argument error; room smaller than the budget caps the splits."""
    v = scene_case("sliver20000")
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    with pytest.raises(ab.AtrError):
        ab.split_triangles(scene, 0.3, max_primitives=len(v) - 1)
    with pytest.raises(ab.AtrError):
        ab.split_triangles(scene, -0.5)
    _, _, data = ab.split_triangles(scene, 1.0, max_primitives=len(v) + 100)
    assert len(v) <= len(data) <= len(v) + 100
