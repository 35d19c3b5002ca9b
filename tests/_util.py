"""Shared helpers for the parity tests: seeded cases, array digests, tree checks."""
from __future__ import annotations

import hashlib

import numpy as np

import atrbvh_b200 as ab


def scene_case(name: str) -> np.ndarray:
    """Seeded triangle soups (n, 3, 4) used across tests and golden fixtures."""
    kind, n, seed = CASES[name]
    if kind == "uniform":
        return ab.gen_scene(ab.SCENE_UNIFORM, n, seed)
    if kind == "clustered":
        return ab.gen_scene(ab.SCENE_CLUSTERED, n, seed)
    if kind == "dupes":
        # Many identical triangles: equal Morton keys exercise the index tie-break.
        base = ab.gen_scene(ab.SCENE_UNIFORM, max(n // 16, 1), seed)
        return np.ascontiguousarray(np.repeat(base, 16, axis=0)[:n])
    if kind == "flat":
        # All centroids in one plane: a zero-extent scene axis.
        v = ab.gen_scene(ab.SCENE_UNIFORM, n, seed).copy()
        v[:, :, 1] = 0.25
        return v
    if kind == "same":
        v = ab.gen_scene(ab.SCENE_UNIFORM, 1, seed)
        return np.ascontiguousarray(np.repeat(v, n, axis=0))
    if kind == "sliver":
        # Long thin triangles along random directions (the case triangle
        # splitting is for): 90% small triangles of the uniform scene, 10%
        # slivers of length 0.2-0.6 and width 0.002.
        v = ab.gen_scene(ab.SCENE_UNIFORM, n, seed).copy()
        rng = np.random.default_rng(seed)
        k = n // 10
        idx = rng.choice(n, size=k, replace=False)
        p0 = rng.uniform(0.0, 1.0, (k, 3)).astype(np.float32)
        d = rng.normal(size=(k, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        w = np.cross(d, rng.normal(size=(k, 3)))
        w /= np.linalg.norm(w, axis=1, keepdims=True)
        length = rng.uniform(0.2, 0.6, (k, 1))
        v[idx, 0, :3] = p0
        v[idx, 1, :3] = (p0 + length * d).astype(np.float32)
        v[idx, 2, :3] = (p0 + 0.002 * w).astype(np.float32)
        v[:, :, 3] = 0
        return np.ascontiguousarray(v)
    raise KeyError(name)


CASES = {
    "u2": ("uniform", 2, 11),
    "u3": ("uniform", 3, 12),
    "u5": ("uniform", 5, 13),
    "u17": ("uniform", 17, 14),
    "u100": ("uniform", 100, 15),
    "u1000": ("uniform", 1000, 16),
    "u4097": ("uniform", 4097, 17),
    "c1": ("uniform", 65536, 0),
    "clu4096": ("clustered", 4096, 2),
    "clu65536": ("clustered", 65536, 0),
    "dupes3000": ("dupes", 3000, 5),
    "flat2000": ("flat", 2000, 6),
    "same64": ("same", 64, 7),
    "sliver20000": ("sliver", 20000, 8),
    "sliver262144": ("sliver", 262144, 9),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:32]


def tree_digests(parent, left, right, data, bmin, bmax, area) -> dict:
    """Digests of the reference SoA arrays; box .w lanes are excluded (the
    reference leaves them uninitialised)."""
    return {
        "parent": digest(np.asarray(parent, np.int32)),
        "left": digest(np.asarray(left, np.int32)),
        "right": digest(np.asarray(right, np.int32)),
        "data": digest(np.asarray(data, np.int32)),
        "bbox_min": digest(np.asarray(bmin, np.float32)[:, :3]),
        "bbox_max": digest(np.asarray(bmax, np.float32)[:, :3]),
        "area": digest(np.asarray(area, np.float32)),
    }


def reachable_leaves(left, right, data, count, tri_indices):
    """Leaves reachable from the root of a collapsed tree, ascending by node,
    with their triangle counts and their triangle lists end to end (level by
    level over numpy arrays, so it stays quick at millions of nodes)."""
    left, right, data, count = (np.asarray(a) for a in (left, right, data, count))
    tri_indices = np.asarray(tri_indices)
    leaves = []
    frontier = np.zeros(1, np.int64)
    while frontier.size:
        ch = np.concatenate([left[frontier], right[frontier]]).astype(np.int64)
        is_leaf = data[ch] >= 0
        leaves.append(ch[is_leaf])
        frontier = ch[~is_leaf]
    nodes = np.sort(np.concatenate(leaves)) if leaves else np.zeros(0, np.int64)
    cnt = np.maximum(count[nodes].astype(np.int64), 1)
    start = np.where(count[nodes] > 1, data[nodes], -1).astype(np.int64)
    # Flat list: leaf k contributes tri_indices[start_k : start_k + cnt_k], or
    # its own data index when it holds one triangle.
    first = np.repeat(np.cumsum(cnt) - cnt, cnt)
    within = np.arange(int(cnt.sum()), dtype=np.int64) - first
    owner = np.repeat(np.arange(len(nodes)), cnt)
    multi = start[owner] >= 0
    flat = np.where(multi, tri_indices[np.where(multi, start[owner] + within, 0)], data[nodes][owner])
    return nodes, cnt, flat.astype(np.int64)


def collapsed_digests(left, right, data, count, tri_indices, n) -> dict:
    """Order-independent digest of a collapsed tree: reachable leaves with
    their triangle lists (the reference assigns list offsets by atomicAdd)."""
    nodes, cnt, flat = reachable_leaves(left, right, data, count, tri_indices)
    return {"leaf_nodes": digest(nodes), "leaf_counts": digest(cnt), "leaf_lists": digest(flat),
            "num_leaves": int(len(nodes))}


def check_tree(t, n: int) -> None:
    """Structural invariants of a BVH in the reference layout."""
    parent, left, right, data = (np.asarray(x) for x in (t.parent, t.left, t.right, t.data))
    bmin, bmax = np.asarray(t.bbox_min), np.asarray(t.bbox_max)
    assert parent[0] == -1
    nn = 2 * n - 1
    seen = np.zeros(nn, bool)
    st = [0]
    while st:
        x = st.pop()
        assert not seen[x]
        seen[x] = True
        if x < n - 1:
            l, r = int(left[x]), int(right[x])
            assert parent[l] == x and parent[r] == x
            assert np.array_equal(bmin[x, :3], np.minimum(bmin[l, :3], bmin[r, :3]))
            assert np.array_equal(bmax[x, :3], np.maximum(bmax[l, :3], bmax[r, :3]))
            assert data[x] == -1
            st += [l, r]
        else:
            assert left[x] == -1 and right[x] == -1 and data[x] >= 0
    assert seen.all()
    assert sorted(data[n - 1:].tolist()) == list(range(n))


def assert_trees_equal(a, b, what: str = "") -> None:
    for f in ("parent", "left", "right", "data", "area"):
        x, y = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        if not np.array_equal(x, y):
            bad = np.nonzero(x != y)[0]
            raise AssertionError(f"{what}: {f} differs at {len(bad)} nodes, first {bad[:8].tolist()}: "
                                 f"{x[bad[:4]].tolist()} vs {y[bad[:4]].tolist()}")
    for f in ("bbox_min", "bbox_max"):
        x, y = np.asarray(getattr(a, f))[:, :3], np.asarray(getattr(b, f))[:, :3]
        if not np.array_equal(x.view(np.int32), y.view(np.int32)):
            bad = np.nonzero((x.view(np.int32) != y.view(np.int32)).any(1))[0]
            raise AssertionError(f"{what}: {f} differs at {len(bad)} nodes, first {bad[:8].tolist()}")
