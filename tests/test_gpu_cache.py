"""On-disk cache of the traversal layout (atr_compact_serialize /
atr_compact_deserialize / atr_cache_key) against the reference's CudaBVH
stream format (gpu-ray-traversal/src/rt/cuda/CudaBVH.cpp:108-123,
framework/gpu/Buffer.cpp:331-362) and the oracle's Compact2 arrays."""
from __future__ import annotations

import struct

import numpy as np
import pytest

import atrbvh_b200 as ab
import oracle as O
from tests._util import scene_case

pytestmark = pytest.mark.gpu


def _pipeline(ctx, v):
    mn, mx = O.scene_aabb(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    col, _ = ab.BVHTreeCollapser().Collapse(tree)
    return scene, tree, col, ab.CudaBVH(col, scene)


def _reference_image(cp: O.Compact) -> bytes:
    """The stream CudaBVH::serialize writes: S32 layout, then each buffer as
    S64 size and bytes (little-endian)."""
    out = struct.pack("<i", 5)
    for a in (cp.nodes, cp.woop, cp.tri_index):
        b = np.ascontiguousarray(a).tobytes()
        out += struct.pack("<q", len(b)) + b
    return out


def _trace(ctx, bvh, rays):
    import torch
    rd = torch.from_numpy(np.ascontiguousarray(rays, np.float32).reshape(-1)).cuda()
    res = torch.zeros(len(rays) * 4, dtype=torch.int32, device="cuda")
    bvh.trace(rd.data_ptr(), len(rays), res.data_ptr())
    ctx.synchronize()
    return res.cpu().numpy().reshape(-1, 4)


@pytest.mark.parametrize("case", ["u100", "clu4096", "dupes3000", "c1", "clu65536"])
def test_cache_image_is_reference_stream_and_round_trips(ctx, case):
    v = scene_case(case)
    mn, mx = O.scene_aabb(v)
    _, _, _, bvh = _pipeline(ctx, v)
    image = bvh.serialize()
    base, _, _ = O.build_lbvh(v, mn, mx, threads=0)
    want = _reference_image(O.flatten(O.collapse(O.atrbvh(base, 9, 2, threads=0)), v))
    assert image == want
    loaded = ab.CudaBVH.from_image(ctx, image)
    assert loaded.view().max_depth == bvh.view().max_depth
    assert loaded.view().num_nodes == bvh.view().num_nodes
    assert loaded.serialize() == image
    rays = np.concatenate([ab.gen_rays_random(20000, mn, mx, seed=4), ab.gen_rays_pinhole(64, 48)])
    assert np.array_equal(_trace(ctx, loaded, rays), _trace(ctx, bvh, rays))


def test_cache_directory_by_key(ctx, tmp_path):
    v = scene_case("clu4096")
    cache = ab.BVHCache(tmp_path)
    key = ab.cache_key(v)
    assert cache.load(ctx, key) is None
    _, _, _, bvh = _pipeline(ctx, v)
    cache.store(key, bvh)
    assert cache.path(key).name == f"{key:016x}.dat"
    loaded = cache.load(ctx, key)
    assert loaded is not None and loaded.serialize() == bvh.serialize()
    assert ab.cache_key(v, treelet=7) != key


def test_cache_rejects_damaged_images(ctx):
    v = scene_case("u1000")
    _, _, _, bvh = _pipeline(ctx, v)
    good = bytearray(bvh.serialize())
    nodes_bytes = struct.unpack_from("<q", good, 4)[0]
    bad = [bytes(good[:-1]),                       # truncated
           bytes(good + b"\0"),                    # trailing bytes
           struct.pack("<i", 4) + bytes(good[4:]),  # another layout
           bytes(good[:20])]
    cut = bytearray(good)                          # inner reference pointing backwards
    struct.pack_into("<i", cut, 12 + 64 * 1 + 48, 0)
    bad.append(bytes(cut))
    leaf = bytearray(good)                         # leaf reference past the Woop buffer
    struct.pack_into("<i", leaf, 12 + 48, ~(10 ** 8))
    bad.append(bytes(leaf))
    odd = bytearray(good)                          # node buffer not a whole number of nodes
    struct.pack_into("<q", odd, 4, nodes_bytes - 16)
    bad.append(bytes(odd))
    for k, image in enumerate(bad):
        with pytest.raises(ab.AtrError):
            ab.CudaBVH.from_image(ctx, image)
