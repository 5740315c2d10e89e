"""Multi-process plumbing of the benchmark and of sharded work (one process
per GPU, torch.distributed).  The TD path itself has no exchange step: pairs
are independent, so assembly shards by element columns with no collective,
many independent cracks shard by crack (each rank solves its own), and the
dense LU of one system runs per replica (it would need a panel broadcast to
shard).  The only collectives are the timing barrier and the max over ranks
of a step time."""
from __future__ import annotations


def column_block(n, rank, world):
    """Contiguous block [j0, j1) of n element columns owned by `rank` of
    `world` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n), int(world))
    j0 = rank * base + min(rank, extra)
    return j0, j0 + base + (1 if rank < extra else 0)


def crack_shard(sizes, rank, world):
    """Indices of the cracks (sizes = triangles per crack) that `rank` of
    `world` solves: largest first, each to the rank with the least work so
    far (work ~ (3N)^3, the dense factorisation's), ties to the lower rank.
    Every rank computes the same assignment; the shards are disjoint and
    cover every crack.  Returned in increasing index order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    load = [0.0] * world
    mine = []
    for i in sorted(range(len(sizes)), key=lambda c: (-int(sizes[c]), c)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += float(sizes[i]) ** 3
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(value, device=None):
    """The largest `value` over all ranks (the step time a multi-GPU run
    reports); `value` itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, ms_max, world):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, timed as the slowest rank's `ms_max`."""
    return world * float(units_per_rank) / (ms_max * 1e-3)
