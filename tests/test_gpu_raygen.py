"""Secondary-ray workloads against the oracle: ambient-occlusion rays
(gpu-ray-traversal/src/rt/ray/RayGenKernels.cu:114-223) generated in the
reference's batches, their traversal, and the Morton ray sort
(gpu-ray-traversal/src/rt/ray/RayBuffer.cpp:103-160)."""
from __future__ import annotations

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import scene_case

pytestmark = pytest.mark.gpu


def _dev(a, dtype=np.float32):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype).reshape(-1)).cuda()


def _scene_bvh(ctx, case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    return v, mn, mx, scene, ab.CudaBVH(col, scene), (tree, col)


def _trace(ctx, bvh, rays_t, n, any_hit=False):
    import torch
    res = torch.zeros(n * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rays_t.data_ptr(), n, res.data_ptr(), any_hit=any_hit)
    ctx.synchronize()
    return res


@pytest.mark.parametrize("case,samples", [("clu65536", 1), ("c1", 4), ("u4097", 16)])
def test_ao_rays_match_oracle_in_reference_batches(ctx, case, samples):
    import torch
    v, mn, mx, scene, bvh, keep = _scene_bvh(ctx, case)
    prim = ab.gen_rays_pinhole(160, 120, eye=(0.5, 0.5, -1.5))
    pd = _dev(prim)
    res = _trace(ctx, bvh, pd, len(prim))
    res_h = res.cpu().numpy().reshape(-1, 4)
    assert (res_h[:, 0] >= 0).any() and (res_h[:, 0] < 0).any()
    batches = list(ab.ray_batches(len(prim), samples, max_batch=1 << 12))
    assert len(batches) > 1
    for lo, hi in batches:
        out = torch.zeros((hi - lo) * samples * 8, dtype=torch.float32, device="cuda")
        ab.gen_ao_rays(scene, pd.data_ptr(), res.data_ptr(), lo, hi - lo, samples, 0.25, 1234, out.data_ptr())
        ctx.synchronize()
        got = out.cpu().numpy().reshape(-1, 2, 4)
        want = O.gen_ao_rays(v, prim, res_h, samples, 0.25, 1234, first=lo, count=hi - lo)
        assert np.array_equal(got.view(np.int32), want.view(np.int32)), (lo, hi)
        miss = np.repeat(res_h[lo:hi, 0] < 0, samples)
        assert np.all(got[miss, 1, 3] == -1.0) and np.all(got[~miss, 1, 3] == 0.25)
        # AO traversal (any hit, as the reference traces AO rays) equals the oracle's.
        cp = O.flatten(O.collapse(O.atrbvh(O.build_lbvh(v, mn, mx, threads=0)[0], 9, 2, threads=0)), v)
        for any_hit in (True, False):
            r2 = _trace(ctx, bvh, out, len(got), any_hit=any_hit).cpu().numpy().reshape(-1, 4)
            w2 = O.trace(cp, got, any_hit=any_hit)
            assert np.array_equal(r2[:, :2], w2[:, :2]), (lo, any_hit)
        break_after_two = lo >= batches[1][0]
        if break_after_two:
            break


@pytest.mark.parametrize("kind", ["random", "pinhole", "ao"])
def test_ray_sort_matches_oracle(ctx, kind):
    import torch
    v, mn, mx, scene, bvh, keep = _scene_bvh(ctx, "c1")
    if kind == "random":
        rays = ab.gen_rays_random(300000, mn, mx, seed=5)
    elif kind == "pinhole":
        rays = ab.gen_rays_pinhole(640, 480, eye=(0.5, 0.5, -1.5))
    else:
        prim = ab.gen_rays_pinhole(320, 240, eye=(0.5, 0.5, -1.5))
        pd = _dev(prim)
        res = _trace(ctx, bvh, pd, len(prim))
        out = torch.zeros(len(prim) * 4 * 8, dtype=torch.float32, device="cuda")
        ab.gen_ao_rays(scene, pd.data_ptr(), res.data_ptr(), 0, len(prim), 4, 0.5, 99, out.data_ptr())
        ctx.synchronize()
        rays = out.cpu().numpy().reshape(-1, 2, 4)
    n = len(rays)
    rd = _dev(rays)
    ids = np.random.default_rng(1).permutation(n).astype(np.int32)  # an arbitrary slot-to-id map
    idd = _dev(ids, np.int32)
    out_r = torch.zeros_like(rd)
    s2i = torch.zeros(n, dtype=torch.int32, device="cuda")
    i2s = torch.zeros(n, dtype=torch.int32, device="cuda")
    ab.sort_rays(ctx, rd.data_ptr(), n, out_r.data_ptr(), idd.data_ptr(), s2i.data_ptr(), i2s.data_ptr())
    ctx.synchronize()
    perm, _ = O.sort_rays(rays)
    got = out_r.cpu().numpy().reshape(-1, 2, 4)
    assert np.array_equal(got.view(np.int32), rays[perm].view(np.int32))
    s2i_h = s2i.cpu().numpy()
    assert np.array_equal(s2i_h, ids[perm])
    i2s_h = i2s.cpu().numpy()
    assert np.array_equal(i2s_h[s2i_h], np.arange(n))
    # Tracing the sorted batch gives each ray the same result.
    a = _trace(ctx, bvh, rd, n).cpu().numpy().reshape(-1, 4)
    b = _trace(ctx, bvh, out_r, n).cpu().numpy().reshape(-1, 4)
    assert np.array_equal(b[:, :2], a[perm, :2])


def test_ray_workloads_reject_bad_arguments(ctx):
    import torch
    v, mn, mx, scene, bvh, keep = _scene_bvh(ctx, "u100")
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    with pytest.raises(ab.AtrError):
        ab.gen_ao_rays(scene, buf.data_ptr(), buf.data_ptr(), 0, 4, 0, 1.0, 0, buf.data_ptr())
    with pytest.raises(ab.AtrError):
        ab.sort_rays(ctx, buf.data_ptr(), 4, buf.data_ptr())
