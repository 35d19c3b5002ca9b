"""Mesh sharding across ranks for batched builds on several GPUs.

Meshes are independent units (no exchange step), so a batch is split by
mesh: longest-processing-time greedy over the triangle counts, ties broken
by mesh index and then by rank, so every rank computes the same assignment
without communication.  Each rank then builds its own meshes as one
segmented batch.
"""
from __future__ import annotations

import heapq

import numpy as np


def assign_meshes(sizes, world: int) -> list[np.ndarray]:
    """Mesh indices (ascending) of each of `world` ranks; every mesh goes to
    exactly one rank, largest first to the least-loaded rank."""
    if world < 1:
        raise ValueError(f"world size {world}")
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.lexsort((np.arange(len(sizes)), -sizes))  # size descending, index ascending
    heap = [(0, r) for r in range(world)]
    owned: list[list[int]] = [[] for _ in range(world)]
    for m in order:
        load, r = heapq.heappop(heap)
        owned[r].append(int(m))
        heapq.heappush(heap, (load + int(sizes[m]), r))
    return [np.array(sorted(o), dtype=np.int64) for o in owned]


def rank_meshes(sizes, world: int, rank: int) -> np.ndarray:
    """The meshes of one rank."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return assign_meshes(sizes, world)[rank]


def rank_loads(sizes, world: int) -> np.ndarray:
    """Triangles per rank under assign_meshes."""
    sizes = np.asarray(sizes, dtype=np.int64)
    return np.array([int(sizes[o].sum()) for o in assign_meshes(sizes, world)], dtype=np.int64)
