"""Multi-GPU host logic of the data-parallel paths: one process per GPU, no collective on the data
path.

* A single mesh does not shard (a halo exchange after every colour would be latency-bound), so
  ``bench.py --gpus N`` runs one replica per rank.
* Batches of independent meshes shard by whole meshes: :func:`shard_meshes` balances ranks by tet
  count (greedy, largest first).  Each rank then runs one batched solver over its own meshes.
* Timings are combined after the timed region: :func:`combine_over_ranks` takes the max of the
  per-rank times and the sum of the per-rank counts (a ``torch.distributed`` all-reduce, NCCL on
  GPUs or gloo on the host).
"""
from __future__ import annotations


def shard_meshes(tet_counts, world: int) -> list[list[int]]:
    """Mesh indices per rank (each list ascending): meshes are taken largest first (ties by index)
    and each goes to the rank with the least load so far (ties to the lowest rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(tet_counts)), key=lambda k: (-int(tet_counts[k]), k)):
        r = min(range(world), key=lambda r: (load[r], r))
        load[r] += int(tet_counts[k])
        shards[r].append(k)
    return [sorted(s) for s in shards]


def combine_over_ranks(times, counts, dist=None, device="cpu"):
    """(max of each time over ranks, sum of each count over ranks) as Python floats.  With
    ``dist`` None (one process) the inputs come back unchanged.  Every rank must call it, with the
    same number of values."""
    times = [float(t) for t in times]
    counts = [float(c) for c in counts]
    if dist is None:
        return times, counts
    import torch

    t = torch.tensor(times, dtype=torch.float64, device=device)
    c = torch.tensor(counts, dtype=torch.float64, device=device)
    if len(times):
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if len(counts):
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()], [float(v) for v in c.cpu()]
