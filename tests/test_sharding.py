"""Multi-rank host logic on CPU: two gloo ranks shard the units and reduce
the timings as bench.py does on NVLink-connected GPUs."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from csdecomp_b200.shard import shard, shard_range


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 2), (10, 3), (257, 8)])
def test_shard_range_covers_exactly_once(n, world):
    seen = []
    for r in range(world):
        b, e = shard_range(n, r, world)
        seen.extend(range(b, e))
        assert e - b in (n // world, n // world + 1)
    assert seen == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from csdecomp_b200.shard import reduce_timing
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    items = list(range(11))
    mine = shard(items, rank, world)
    dev_s, wall_s, units = reduce_timing(dist, torch.device("cpu"), 1.0 + rank, 2.0 * (rank + 1), float(len(mine)))
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    out[rank] = (dev_s, wall_s, units, sorted(x for g in gathered for x in g))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            dev_s, wall_s, units, allitems = out[r]
            assert dev_s == 2.0 and wall_s == 4.0  # max over ranks
            assert units == 11.0  # sum over ranks
            assert allitems == list(range(11))
