"""The multi-GPU host logic on CPU: two gloo ranks shard the batched
specimens with no overlap and no gap, and the timing and count reductions
combine them as bench.py does (max of times, sum of counts)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from icflow_b200.shard import dist_env, reduce_max, reduce_sum, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    ws, r, lr = dist_env()
    mine = shard(64, r, ws)
    t = reduce_max([1.0 + r, 5.0 - r])
    n = reduce_sum([len(mine)])
    q.put((r, mine, t, n))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    items = sorted(i for _, mine, _, _ in out for i in mine)
    assert items == list(range(64))
    assert set(out[0][1]).isdisjoint(out[1][1])
    for _, _, t, n in out:
        assert t == [2.0, 5.0] and n == [64.0]


def test_shard_arguments():
    assert shard(5, 0, 1) == [0, 1, 2, 3, 4]
    assert shard(5, 1, 2) == [1, 3]
    with pytest.raises(ValueError):
        shard(5, 2, 2)
