"""Multi-rank host logic on CPU: network placement and the max-over-ranks
timing reduction, with world-size-2 gloo process groups on 127.0.0.1."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from demystification_dfn_b200.sharding import reduce_timing, shard_by_work


def test_shard_by_work_partitions_and_balances():
    sizes = [2000 + 37 * ((i * 7919) % 101) for i in range(64)]
    for world in (1, 2, 3, 8):
        parts = [shard_by_work(sizes, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(sizes[i] ** 2 for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(s ** 2 for s in sizes)
    with pytest.raises(ValueError):
        shard_by_work(sizes, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [1000 + 10 * i for i in range(10)]
        mine = shard_by_work(sizes, world, rank)
        ms, work = reduce_timing(10.0 + 5.0 * rank, float(len(mine)), dist=dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out[rank] = (ms, work, sorted(i for g in gathered for i in g))
    finally:
        dist.destroy_process_group()


def test_reduce_timing_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            ms, work, allidx = out[r]
            assert ms == 15.0 and work == 10.0 and allidx == list(range(10))


def test_reduce_timing_without_group_is_local():
    assert reduce_timing(3.0, 7.0) == (3.0, 7.0)
