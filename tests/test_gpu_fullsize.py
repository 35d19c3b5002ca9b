"""GPU parity at the benchmark configurations' full sizes, against the oracle
(directly, and through the oracle's committed full-size digests in
tests/golden/fullsize_oracle.json, which test_cpu_golden_fullsize pins to the
oracle on the host).

  clustered 4,194,304 triangles (the timed bench step): LBVH + ATRBVH(9,2)
      tree, collapsed tree and SAH, Compact2 bytes, primary and diffuse-bounce
      closest-hit results;
  unit-cube 16,777,216 triangles: LBVH, TRBVH(7,3), ATRBVH(5/7/9 x 1-3);
  4096-mesh batch (151.5M triangles): a seeded sample of 64 meshes (the
      smallest and the largest among them) against the oracle on each mesh;
  serving: a 2M-triangle build and refit with 1M rays against the oracle."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import assert_trees_equal, collapsed_digests, digest, tree_digests

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "fullsize_oracle.json").read_text())


def _tdig(t):
    return tree_digests(t.parent, t.left, t.right, t.data, t.bbox_min, t.bbox_max, t.area)


def _trace_gpu(ctx, bvh, rays):
    import torch
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rd.data_ptr(), len(rays), res.data_ptr())
    ctx.synchronize()
    return rd, res


def test_clustered_4m_pipeline_matches_oracle(ctx):
    """The bench step at its full size: every stage's output equals the
    oracle's (tree bit-exact, collapsed leaves and SAH, Compact2 bytes, hit
    ids and t of the primary rays and of the device-made bounce rays)."""
    g = GOLD["c2"]
    v = ab.gen_scene(ab.SCENE_CLUSTERED, 4194304, 0)
    assert digest(v) == g["scene"]
    scene = ab.SceneWrapper(ctx, v)
    tree = ab.LBVHBuilder().BuildTree(scene)
    lb = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert _tdig(lb) == g["lbvh_tree"]
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert _tdig(got) == g["tree"]
    assert np.float32(tree.sah()) == np.float32(g["tree_sah"])
    col, csah = ab.BVHTreeCollapser().Collapse(tree)
    assert np.float32(csah) == np.float32(g["collapsed_sah"])
    hc = ab.BVHTreeInstanceManager().DeviceToHostCollapsedTree(col)
    assert collapsed_digests(hc.left, hc.right, hc.data, hc.triangle_count, hc.triangle_indices, len(v)) == \
        g["collapsed"]
    bvh = ab.CudaBVH(col, scene)
    nodes, woop, tri = bvh.download()
    assert digest(nodes) == g["compact2"]["nodes"]
    assert digest(woop) == g["compact2"]["woop"]
    assert digest(tri) == g["compact2"]["tri_index"]
    prim = ab.gen_rays_pinhole(1920, 1080)
    assert digest(prim) == g["primary_rays"]
    rd, res = _trace_gpu(ctx, bvh, prim)
    r = res.cpu().numpy().reshape(-1, 4)
    assert digest(r[:, 0].copy()) == g["primary_hits"]["ids"]
    assert digest(r[:, 1].copy()) == g["primary_hits"]["t"]
    # Bounce rays from the device generator, traced on the device and by the
    # oracle over the oracle's own Compact2 arrays.
    import torch
    bounce = torch.zeros_like(rd)
    ab.check(ab.lib().atr_gen_bounce_rays(ctx.handle, scene.handle, rd.data_ptr(), res.data_ptr(), len(prim), 1,
                                          bounce.data_ptr()))
    res2 = torch.zeros_like(res)
    bvh.trace(bounce.data_ptr(), len(prim), res2.data_ptr())
    ctx.synchronize()
    mn, mx = O.scene_aabb(v)
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    cp = O.flatten(O.collapse(O.atrbvh(base, 9, 2, threads=0)), v)
    b = bounce.cpu().numpy().reshape(-1, 2, 4)
    want = O.trace(cp, b)
    got2 = res2.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(got2[:, :2], want[:, :2])
    assert (got2[:, 0] >= 0).sum() > 100000


C3 = list(GOLD["c3"]["variants"])


@pytest.fixture(scope="module")
def c3_scene(ctx):
    v = ab.gen_scene(ab.SCENE_UNIFORM, 16777216, 0)
    assert digest(v) == GOLD["c3"]["scene"]
    scene = ab.SceneWrapper(ctx, v)
    yield scene
    scene.close()


@pytest.mark.parametrize("variant", C3)
def test_sweep_16m_matches_oracle(ctx, c3_scene, variant):
    """16,777,216 triangles: each optimiser's tree is bit-exact against the
    oracle's, with the same SAH and collapsed SAH."""
    want = GOLD["c3"]["variants"][variant]
    tree = ab.LBVHBuilder().BuildTree(c3_scene)
    if variant.startswith("atrbvh"):
        _, ts, it = variant.split("_")
        ab.AgglomerativeTreeletOptimizer(int(ts), int(it)).Optimize(tree)
    elif variant.startswith("trbvh"):
        _, ts, it = variant.split("_")
        ab.TRBVHOptimizer(int(ts), int(it)).Optimize(tree)
    got = ab.BVHTreeInstanceManager().DeviceToHostTree(tree)
    assert _tdig(got) == want["tree"], variant
    assert np.float32(tree.sah()) == np.float32(want["sah"])
    col, csah = ab.BVHTreeCollapser().Collapse(tree)
    assert np.float32(csah) == np.float32(want["collapsed_sah"])
    col.close()
    tree.close()


def test_batch_4096_meshes_sample_matches_oracle(ctx):
    """The whole 4096-mesh workload built as one segmented batch (graph
    replay); 64 meshes drawn with a fixed seed, plus the smallest and the
    largest, each equal to the oracle's LBVH + ATRBVH(9,2) of that mesh alone."""
    sizes = ab.gen_batch_sizes(4096, 256, 262144, 0)
    v = ab.gen_batch_scene(sizes, 0)
    off = np.concatenate([[0], np.cumsum(sizes, dtype=np.uint64)]).astype(np.uint32)
    batch = ab.Batch(ctx, v, off)
    batch.build(1, 9, 2, graph=True)
    batch.build(1, 9, 2, graph=True)  # replay
    sah = batch.sah()
    rng = np.random.default_rng(1234)
    pick = set(rng.choice(len(sizes), 64, replace=False).tolist())
    pick |= {int(np.argmin(sizes)), int(np.argmax(sizes))}
    for m in sorted(pick):
        vm = np.ascontiguousarray(v[off[m]:off[m + 1]])
        mn, mx = O.scene_aabb(vm)
        base, _, _ = O.build_lbvh(vm, mn, mx, threads=0)
        want = O.atrbvh(base, 9, 2, threads=0)
        assert_trees_equal(batch.mesh(m), want, f"mesh {m} ({sizes[m]} triangles)")
        assert np.float32(sah[m]) == np.float32(O.sah(want)), m
    batch.close()


def test_server_2m_build_and_refit_1m_rays_match_oracle():
    """A serving request at the configuration's largest sizes (2,000,000
    triangles, 1,048,576 rays): build + trace, then a refit of the resident
    mesh after vertex jitter + trace, each equal to the oracle."""
    n, nr = 2_000_000, 1 << 20
    v = ab.gen_scene(ab.SCENE_UNIFORM, n, 4242)
    mn, mx = O.scene_aabb(v)
    rays = ab.gen_rays_random(nr, mn, mx, seed=99)
    rng = np.random.default_rng(5)
    w = (v + rng.normal(0, 0.001, v.shape).astype(np.float32)).astype(np.float32)
    w[:, :, 3] = 0
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    t = O.atrbvh(base, 9, 2, threads=0)
    want_build = O.trace(O.flatten(O.collapse(t), v), rays)
    want_refit = O.trace(O.flatten(O.collapse(O.refit(t, w)), w), rays)
    srv = ab.Server(device=0, hbm_budget=120 << 30, lanes=2)
    out1 = np.full((nr, 4), -7, np.int32)
    r1 = srv.wait(srv.submit(ab.REQ_BUILD, 1, v, rays, out1, keep_resident=True))
    assert r1["status"] == 0, r1
    out2 = np.full((nr, 4), -7, np.int32)
    r2 = srv.wait(srv.submit(ab.REQ_REFIT, 1, w, rays, out2))
    assert r2["status"] == 0, r2
    srv.close()
    assert np.array_equal(out1[:, :2], want_build[:, :2])
    assert np.array_equal(out2[:, :2], want_refit[:, :2])
    assert (out1[:, 0] >= 0).mean() > 0.2
