"""Serving loop: requests submitted together (continuous batching over two
lanes) give the same results as the same requests run one at a time, builds
equal the plain single-mesh pipeline, and admission by memory evicts idle
resident meshes."""
from __future__ import annotations

import time

import numpy as np
import pytest

import atrbvh_b200 as ab

pytestmark = pytest.mark.gpu


def _mesh(n: int, seed: int) -> np.ndarray:
    return ab.gen_scene(ab.SCENE_UNIFORM, n, seed)


def _rays(v: np.ndarray, count: int, seed: int) -> np.ndarray:
    p = v[:, :, :3].reshape(-1, 3)
    return ab.gen_rays_random(count, p.min(0), p.max(0), seed=seed)


def _jitter(v: np.ndarray, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = (v + rng.normal(0, 0.001, v.shape).astype(np.float32)).astype(np.float32)
    w[:, :, 3] = 0
    return w


def _workload(seed: int = 0):
    """Builds of log-uniform sizes and refits of some of them, with rays."""
    rng = np.random.default_rng(seed)
    reqs = []
    built = []
    for i in range(18):
        if built and rng.random() < 0.35:
            mid, base = built[int(rng.integers(len(built)))]
            w = _jitter(base, 1000 + i)
            reqs.append((ab.REQ_REFIT, mid, w, _rays(w, int(rng.integers(2000, 9000)), 50 + i)))
        else:
            n = int(np.exp(rng.uniform(np.log(1000), np.log(120000))))
            v = _mesh(n, 100 + i)
            reqs.append((ab.REQ_BUILD, i, v, _rays(v, int(rng.integers(2000, 9000)), 10 + i)))
            built.append((i, v))
    return reqs


def _run(server: ab.Server, reqs, together: bool, gap_s: float = 0.0):
    outs = [np.full((len(r[3]), 4), -7, np.int32) for r in reqs]
    results = [None] * len(reqs)
    if together:
        tickets = []
        for (kind, mid, v, rays), out in zip(reqs, outs):
            tickets.append(server.submit(kind, mid, v, rays, out))
            if gap_s:
                time.sleep(gap_s)
        for k, t in enumerate(tickets):
            results[k] = server.wait(t)
    else:
        for k, ((kind, mid, v, rays), out) in enumerate(zip(reqs, outs)):
            results[k] = server.wait(server.submit(kind, mid, v, rays, out))
    return outs, results


def test_server_mix_equals_alone():
    reqs = _workload(0)
    mix = ab.Server(lanes=2, max_batch_requests=8)
    outs_mix, res_mix = _run(mix, reqs, together=True, gap_s=0.002)
    st = mix.stats()
    mix.close()
    alone = ab.Server(lanes=1, max_batch_requests=1)
    outs_alone, res_alone = _run(alone, reqs, together=False)
    alone.close()
    assert all(r["status"] == 0 for r in res_mix), [r["error"] for r in res_mix if r["status"]]
    assert all(r["status"] == 0 for r in res_alone)
    assert max(r["batch_requests"] for r in res_mix) > 1, "no request shared a lane batch"
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for k in range(len(reqs)):
        assert np.array_equal(outs_mix[k], outs_alone[k]), f"request {k} kind {reqs[k][0]}"
        assert np.float32(res_mix[k]["sah"]) == np.float32(res_alone[k]["sah"]), k
        assert (outs_mix[k][:, 0] >= 0).any()


def test_server_build_equals_plain_pipeline(ctx):
    v = _mesh(30000, 7)
    rays = _rays(v, 20000, 3)
    srv = ab.Server(lanes=2)
    out = np.zeros((len(rays), 4), np.int32)
    r = srv.wait(srv.submit(ab.REQ_BUILD, 1, v, rays, out))
    srv.close()
    assert r["status"] == 0
    import torch
    scene = ab.SceneWrapper(ctx, v)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    col, sah = ab.BVHTreeCollapser().Collapse(tree)
    bvh = ab.CudaBVH(col, scene)
    rd = torch.from_numpy(rays.reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rd.data_ptr(), len(rays), res.data_ptr())
    ctx.synchronize()
    want = res.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(out[:, :2], want[:, :2])
    assert np.float32(r["sah"]) == np.float32(sah)


def test_server_budget_evicts_idle_meshes():
    n = 50000
    # Room for about two resident meshes of this size beside one in flight.
    srv = ab.Server(lanes=1, hbm_budget=int(n * 404 * 2.5 + n * 460), max_batch_requests=1)
    meshes = [_mesh(n, 40 + i) for i in range(5)]
    for i, v in enumerate(meshes):
        assert srv.wait(srv.submit(ab.REQ_BUILD, i, v))["status"] == 0
    st = srv.stats()
    assert st["evictions"] >= 2 and st["resident_meshes"] <= 3
    # The oldest mesh was evicted; the newest is resident.
    w = _jitter(meshes[0], 1)
    assert srv.wait(srv.submit(ab.REQ_REFIT, 0, w))["status"] == ab.ERR_NOT_RESIDENT
    w = _jitter(meshes[4], 2)
    rays = _rays(w, 5000, 9)
    out = np.zeros((len(rays), 4), np.int32)
    assert srv.wait(srv.submit(ab.REQ_REFIT, 4, w, rays, out))["status"] == 0
    assert (out[:, 0] >= 0).any()
    srv.release(4)
    with pytest.raises(ab.AtrError):
        srv.release(4)
    srv.close()


def test_server_rejects_bad_requests():
    srv = ab.Server(lanes=1, max_batch_triangles=1000)
    v = _mesh(2000, 1)
    with pytest.raises(ab.AtrError):
        srv.submit(ab.REQ_BUILD, 0, v)  # above the batch cap
    with pytest.raises(ab.AtrError):
        srv.submit(5, 0, v[:10])
    r = srv.wait(srv.submit(ab.REQ_REFIT, 123, v[:10]))
    assert r["status"] == ab.ERR_NOT_RESIDENT
    srv.close()


def test_server_pinned_request_buffers_equal_pageable():
    """Requests whose vertex, ray and result buffers are page-locked (copied to
    and from the device directly, no staging copy), mixed in one lane batch
    with pageable ones, give the same results as pageable requests alone."""
    reqs = _workload(1)
    pinned = []
    for k, (kind, mid, v, rays) in enumerate(reqs):
        if k % 2 == 0:
            v, rays = ab.pinned_like(v), ab.pinned_like(rays)
        pinned.append((kind, mid, v, rays))
    mix = ab.Server(lanes=2, max_batch_requests=8)
    outs = [np.full((len(r[3]), 4), -7, np.int32) for r in pinned]
    outs = [ab.pinned_like(o) if k % 3 == 0 else o for k, o in enumerate(outs)]
    tickets = [mix.submit(kind, mid, v, rays, out) for (kind, mid, v, rays), out in zip(pinned, outs)]
    res_mix = [mix.wait(t) for t in tickets]
    st = mix.stats()
    mix.close()
    alone = ab.Server(lanes=1, max_batch_requests=1)
    outs_alone, res_alone = _run(alone, reqs, together=False)
    alone.close()
    assert all(r["status"] == 0 for r in res_mix), [r["error"] for r in res_mix if r["status"]]
    assert st["host_copy_ms"] >= 0 and st["lane_batch_ms"] > 0
    for k in range(len(reqs)):
        assert np.array_equal(outs[k], outs_alone[k]), f"request {k}"
        assert np.float32(res_mix[k]["sah"]) == np.float32(res_alone[k]["sah"]), k
