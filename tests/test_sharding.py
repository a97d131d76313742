"""Multi-process host logic of the data-parallel paths, on CPU: mesh sharding by tet count and the
max-over-ranks / sum-over-ranks combination, run as world_size 2 over gloo; and a sharded batch
whose per-rank shards are stepped (by the oracle, standing in for each rank's batched GPU solver)
and gathered, checked against the whole batch stepped in one process."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import pyoracle as po
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


# A small batch of the batched configuration's kind, stepped as VBDsolver::step with Chebyshev.
SHARD_BATCH = dict(num_meshes=10, lo=2, hi=5, seed=5)
SHARD_STEPS, SHARD_ITERS, SHARD_DT, SHARD_RHO = 3, 10, 1.0 / 60.0, 0.9


def _union(meshes):
    """The meshes as one mesh (global vertex ids), the form a rank's batched solver steps."""
    b = meshgen.concat(meshes)
    tets = np.concatenate([m.tets + b.vert_offsets[k] for k, m in enumerate(meshes)]).astype(np.int32)
    return SimpleNamespace(rest=b.rest, x=b.x, v=b.v, tets=tets, fixed=b.fixed, mu=b.mu, lam=b.lam,
                           density=meshes[0].density), b


def _step_batch(meshes):
    """Per-mesh positions after stepping the meshes together as one batch (FP32 oracle)."""
    u, b = _union(meshes)
    r = po.simulate(u, SHARD_STEPS, SHARD_DT, SHARD_ITERS, (0.0, -9.8, 0.0), True, SHARD_RHO, precision=32,
                    mode=po.CLOSED)
    return b.split(r["x"])


def _shard_worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        meshes = meshgen.batched_blocks(**SHARD_BATCH)
        mine = shard_meshes([m.num_tets for m in meshes], world)[rank]
        xs = _step_batch([meshes[k] for k in mine])
        results = {k: x for k, x in zip(mine, xs)}
        # vertex-iterations of this rank's shard, summed over ranks as bench.py combines them
        units = float(sum(meshes[k].num_verts for k in mine) * SHARD_ITERS * SHARD_STEPS)
        _, (total_units,) = combine_over_ranks([], [units], dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, results)
        if rank == 0:
            merged = {}
            for part in gathered:
                assert not set(part) & set(merged)  # no mesh stepped by two ranks
                merged.update(part)
            np.savez(os.path.join(out_dir, "gathered.npz"), units=total_units,
                     **{f"m{k}": merged[k] for k in sorted(merged)})
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_sharded_batch_equals_single_process_batch(tmp_path):
    """Whole meshes sharded over two gloo ranks, each rank stepping its shard as one batch: the
    gathered per-mesh positions equal, bit for bit, those of the whole batch stepped in one process
    (meshes are independent, so a mesh's arithmetic does not depend on its batch-mates)."""
    world = 2
    mp.spawn(_shard_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    g = np.load(tmp_path / "gathered.npz")
    meshes = meshgen.batched_blocks(**SHARD_BATCH)
    whole = _step_batch(meshes)
    assert sorted(k for k in g.files if k.startswith("m")) == sorted(f"m{k}" for k in range(len(meshes)))
    for k, x in enumerate(whole):
        np.testing.assert_array_equal(g[f"m{k}"], x)
    assert float(g["units"]) == sum(m.num_verts for m in meshes) * SHARD_ITERS * SHARD_STEPS
