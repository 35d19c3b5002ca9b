"""atr_refit_noalloc (the refit whose counters live in a fixed __device__ array
instead of freshly allocated memory) against atr_refit, through the C ABI.

The array keeps the previous call's contents, so every check runs two calls
in a row on different vertex sets: a call that skipped clearing the counters
would stop climbing at every internal node on its second run."""
import ctypes as C

import numpy as np
import pytest

import atrbvh_b200 as ab
from tests._util import scene_case

MAX_TRIANGLES = 1 << 20


def _tree(ctx, v):
    scene = ab.SceneWrapper(ctx, v)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    return scene, tree


def _jitter(v, seed):
    rng = np.random.default_rng(seed)
    w = (v + rng.normal(0, 0.001, v.shape).astype(np.float32)).astype(np.float32)
    w[:, :, 3] = 0
    return w


def _noalloc(ctx, scene, tree):
    tv = tree.view()
    ab.check(ab.lib().atr_refit_noalloc(C.c_void_p(ctx.stream), tv.num_triangles,
                                        C.c_void_p(scene.device_vertices()), tv.parent, tv.left, tv.right,
                                        tv.data, tv.bbox_min, tv.bbox_max, tv.area))
    ctx.synchronize()


def _host(tree):
    return ab.BVHTreeInstanceManager().DeviceToHostTree(tree)


def _assert_same(got, want, what):
    for f in ("parent", "left", "right", "data", "bbox_min", "bbox_max", "area"):
        a, b = getattr(got, f), getattr(want, f)
        assert a.shape == b.shape, (what, f)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (what, f)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["u17", "u4097", "c1", "clu65536"])
def test_noalloc_refit_matches_refit_twice(ctx, case):
    v = scene_case(case)
    scene_a, tree_a = _tree(ctx, v)          # refit by atr_refit
    scene_b, tree_b = _tree(ctx, v)          # refit by atr_refit_noalloc
    _assert_same(_host(tree_b), _host(tree_a), "identical builds")
    for call, seed in enumerate((11, 12)):
        w = _jitter(v, seed)
        scene_a.set_vertices(w)
        ab.Refit(tree_a, scene_a)
        scene_b.set_vertices(w)
        _noalloc(ctx, scene_b, tree_b)
        _assert_same(_host(tree_b), _host(tree_a), f"{case} call {call + 1}")


@pytest.mark.gpu
def test_noalloc_refit_alternating_meshes_and_max_size(ctx):
    """Calls on meshes of different sizes in a row, the largest at the fixed
    maximum, each equal to atr_refit on the same tree and vertices."""
    big = ab.gen_scene(ab.SCENE_UNIFORM, MAX_TRIANGLES, 5)
    small = scene_case("u4097")
    pairs = [(_tree(ctx, big), _tree(ctx, big)), (_tree(ctx, small), _tree(ctx, small))]
    for step, idx in enumerate((0, 1, 0, 1)):
        (sa, ta), (sb, tb) = pairs[idx]
        base = big if idx == 0 else small
        w = _jitter(base, 100 + step)
        sa.set_vertices(w)
        ab.Refit(ta, sa)
        sb.set_vertices(w)
        _noalloc(ctx, sb, tb)
        _assert_same(_host(tb), _host(ta), f"step {step} mesh {idx}")


@pytest.mark.gpu
def test_noalloc_refit_rejects_oversize_and_null(ctx):
    dummy = C.c_void_p(256)
    args = [dummy] * 8  # vertices, parent, left, right, data, bbox_min, bbox_max, area
    assert ab.lib().atr_refit_noalloc(None, MAX_TRIANGLES + 1, *args) == 1
    assert b"fixed maximum" in ab.lib().atr_last_error()
    assert ab.lib().atr_refit_noalloc(None, 1, *args) == 1
    assert ab.lib().atr_refit_noalloc(None, 100, None, *args[1:]) == 1


def _pool_used(device: int = 0) -> int:
    """Bytes in use in the device's default stream-ordered pool (where any
    cudaMallocAsync without an explicit pool would draw from)."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    assert err == rt.cudaError_t.cudaSuccess
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    return int(used)


@pytest.mark.gpu
def test_noalloc_refit_allocates_nothing(ctx):
    """After the first call on the device (which may load the library's module
    and with it the fixed array), further calls change neither the device's
    free memory, the stream-ordered pool's usage nor torch's allocator."""
    import torch
    scene, tree = _tree(ctx, scene_case("c1"))
    _noalloc(ctx, scene, tree)
    for seed in range(5):
        scene.set_vertices(_jitter(scene_case("c1"), 200 + seed))
        torch.cuda.synchronize()
        before = (torch.cuda.mem_get_info(0)[0], _pool_used(0), torch.cuda.memory_allocated(0))
        _noalloc(ctx, scene, tree)
        _noalloc(ctx, scene, tree)
        torch.cuda.synchronize()
        after = (torch.cuda.mem_get_info(0)[0], _pool_used(0), torch.cuda.memory_allocated(0))
        assert after == before, (seed, before, after)


@pytest.mark.gpu
def test_noalloc_refit_allocates_nothing(ctx):
    """The entry point's promise itself: once a first call has run (it loads
    the kernel and looks up the array's address), further calls leave the
    device's free memory exactly as it was."""
    import torch

    v = scene_case("clu65536")
    scene, tree = _tree(ctx, v)
    _noalloc(ctx, scene, tree)
    torch.cuda.mem_get_info()  # the query's own first-use set-up, if any, happens here
    free0, _ = torch.cuda.mem_get_info()
    for seed in range(5):
        scene.set_vertices(_jitter(v, 20 + seed))
        _noalloc(ctx, scene, tree)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
