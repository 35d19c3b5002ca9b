"""Mesh sharding for multi-GPU batches, checked over world-size-2 gloo ranks
on the CPU: the ranks agree on a partition of the meshes without exchanging
it, and the triangle loads are balanced."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from atrbvh_b200.shard import assign_meshes, rank_loads, rank_meshes


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, sizes: np.ndarray, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = rank_meshes(sizes, world, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine.tolist())
        out[rank] = gathered
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_a_partition_gloo():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(256), np.log(262144), 4096)).astype(np.int64)
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), sizes, out), nprocs=world, join=True,
                           start_method="spawn")
        views = [out[r] for r in range(world)]
    assert views[0] == views[1], "ranks computed different assignments"
    parts = [np.array(p) for p in views[0]]
    allm = np.concatenate(parts)
    assert len(allm) == len(sizes) and np.array_equal(np.sort(allm), np.arange(len(sizes)))
    loads = [int(sizes[p].sum()) for p in parts]
    assert max(loads) - min(loads) <= int(sizes.max())


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_assignment_properties(world):
    rng = np.random.default_rng(world)
    sizes = rng.integers(2, 100000, 500)
    parts = assign_meshes(sizes, world)
    assert len(parts) == world
    allm = np.concatenate(parts)
    assert np.array_equal(np.sort(allm), np.arange(len(sizes)))
    loads = rank_loads(sizes, world)
    assert loads.sum() == sizes.sum()
    assert loads.max() - loads.min() <= sizes.max()
    for p in parts:
        assert np.all(np.diff(p) > 0)


def test_more_ranks_than_meshes_and_bad_args():
    parts = assign_meshes([5, 3], 4)
    assert sum(len(p) for p in parts) == 2 and sum(len(p) == 0 for p in parts) == 2
    with pytest.raises(ValueError):
        assign_meshes([1], 0)
    with pytest.raises(ValueError):
        rank_meshes([1, 2], 2, 2)
