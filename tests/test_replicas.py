"""The N>1 path (independent replicas): root sharding and max/sum over ranks,
run as two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cggraph_b200.replicas import shard


def test_shard_partitions_roots():
    roots = list(range(10))
    parts = [shard(roots, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == roots
    assert parts[0] == [0, 3, 6, 9]
    with pytest.raises(ValueError):
        shard(roots, 3, 3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from cggraph_b200.replicas import max_over_ranks, shard, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard(list(range(10)), rank, world)
        t = max_over_ranks(1.0 + rank)
        s = sum_over_ranks(len(mine))
        dist.barrier()
        q.put((rank, mine, t, s))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    assert res[0][1] == [0, 2, 4, 6, 8] and res[1][1] == [1, 3, 5, 7, 9]
    assert res[0][2] == res[1][2] == 2.0
    assert res[0][3] == res[1][3] == 10.0
