"""Multi-process host logic of the data-parallel paths, on CPU: mesh sharding by tet count and the
max-over-ranks / sum-over-ranks combination, run as world_size 2 over gloo."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from vbd_tetmesh_b200 import meshgen
from vbd_tetmesh_b200.sharding import combine_over_ranks, shard_meshes


def test_shard_meshes_partition_and_balance():
    rng = np.random.default_rng(0)
    counts = rng.integers(100, 50000, 97)
    for world in (1, 2, 3, 8):
        shards = shard_meshes(counts, world)
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(len(counts)))
        loads = [int(counts[s].sum()) if s else 0 for s in shards]
        # greedy largest-first: no rank exceeds the mean by more than the largest mesh
        assert max(loads) <= counts.sum() / world + counts.max()
        assert shard_meshes(counts, world) == shards  # deterministic


def test_shard_meshes_of_the_batched_configuration():
    meshes = meshgen.batched_blocks(num_meshes=64, seed=2024)
    counts = [m.num_tets for m in meshes]
    shards = shard_meshes(counts, 2)
    loads = [sum(counts[k] for k in s) for s in shards]
    assert abs(loads[0] - loads[1]) <= max(counts)


def test_single_process_combine_is_identity():
    assert combine_over_ranks([1.5, 2.0], [3.0]) == ([1.5, 2.0], [3.0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        counts = [m.num_tets for m in meshgen.batched_blocks(num_meshes=24, lo=2, hi=8, seed=5)]
        mine = shard_meshes(counts, world)[rank]
        times = [10.0 + rank, 5.0 - rank]           # per-rank device times (ms)
        units = [float(sum(counts[k] for k in mine)), 1.0]
        (t0, t1), (tets, ranks) = combine_over_ranks(times, units, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([t0, t1, tets, ranks, float(sum(counts)), float(len(set(sum(gathered, []))))]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_ranks_over_gloo(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for rank in range(world):
        t0, t1, tets, ranks, total, covered = np.load(tmp_path / f"rank{rank}.npy")
        assert t0 == 11.0 and t1 == 5.0      # max over ranks
        assert tets == total and ranks == 2  # sums over ranks: every tet counted once
        assert covered == 24                 # the two shards partition the meshes
