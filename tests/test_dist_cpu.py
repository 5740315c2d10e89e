"""The multi-rank host logic of the benchmark on CPU with the gloo backend
(world size 2): column blocks tile the element range, crack shards are
disjoint and cover the batch, the step time is the maximum over ranks, the
whole-job throughput counts every replica."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from cutanddisplacejulia_b200 import dist as cd
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        j0, j1 = cd.column_block(1001, rank, world)
        sizes = [(37 * c) % 1800 + 200 for c in range(61)]
        mine = cd.crack_shard(sizes, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        ms = 10.0 + 5.0 * rank                       # rank 1 is the slow one
        dist.barrier()
        mx = cd.max_over_ranks(ms)
        out[rank] = (j0, j1, mx, cd.replica_throughput(1000, mx, world), got)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    blocks = sorted((out[r][0], out[r][1]) for r in range(world))
    assert blocks[0][0] == 0 and blocks[-1][1] == 1001 and blocks[0][1] == blocks[1][0]
    for r in range(world):
        assert out[r][2] == 15.0
        assert out[r][3] == pytest.approx(2 * 1000 / 15e-3)
        # every rank saw the same shards: disjoint, covering all 61 cracks
        shards = out[r][4]
        assert shards == out[0][4]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(61))


@pytest.mark.parametrize("count,world", [(0, 2), (5, 8), (512, 2), (512, 8), (61, 3)])
def test_crack_shard_balance(count, world):
    import numpy as np

    from cutanddisplacejulia_b200 import dist as cd
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(200), np.log(2000), count))]
    shards = [cd.crack_shard(sizes, r, world) for r in range(world)]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(count))
    work = [sum(float(sizes[i]) ** 3 for i in s) for s in shards]
    if count >= 8 * world:
        # greedy largest-first: no rank above the mean by more than one largest crack
        assert max(work) <= sum(work) / world + max(sizes) ** 3
    with pytest.raises(ValueError):
        cd.crack_shard(sizes, world, world)


@pytest.mark.parametrize("n,world", [(0, 3), (7, 3), (1001, 8), (5, 8)])
def test_column_block_partition(n, world):
    from cutanddisplacejulia_b200 import dist as cd
    spans = [cd.column_block(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1
