"""Multi-rank host logic on CPU: gloo ranks shard the units as bench.py does
on NVLink-connected GPUs (contiguous ranges of equal predicted cost), run
their inflations independently, and reduce the timings; no data crosses
ranks on the data path."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from csdecomp_b200.shard import cost_balanced_ranges, shard, shard_range


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 2), (10, 3), (257, 8)])
def test_shard_range_covers_exactly_once(n, world):
    seen = []
    for r in range(world):
        b, e = shard_range(n, r, world)
        seen.extend(range(b, e))
        assert e - b in (n // world, n // world + 1)
    assert seen == list(range(n))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_cost_balanced_ranges_cover_and_balance(world):
    rng = np.random.default_rng(world)
    costs = rng.uniform(1, 10, 512) * np.where(np.arange(512) % 2, 4.0, 1.0)  # two plant families
    r = cost_balanced_ranges(costs, world)
    assert r[0][0] == 0 and r[-1][1] == len(costs)
    assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
    sums = np.array([costs[b:e].sum() for b, e in r])
    # every cut is within one unit of its ideal position
    assert sums.max() - sums.min() <= 2 * costs.max()
    assert all(e > b for b, e in r)


def test_cost_balanced_ranges_edge_cases():
    assert cost_balanced_ranges([], 3) == [(0, 0)] * 3
    assert cost_balanced_ranges([5.0], 2) in ([(0, 1), (1, 1)], [(0, 0), (0, 1)])
    r = cost_balanced_ranges([1.0, 100.0, 1.0, 1.0], 2)
    assert r == [(0, 1), (1, 4)] or r == [(0, 2), (2, 4)]
    with pytest.raises(ValueError):
        cost_balanced_ranges([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        cost_balanced_ranges([1.0], 0)


def test_scene_cost_reads_the_seed_only():
    from csdecomp_b200 import scenes
    seeds = scenes.batch_scene_seeds(6)
    for i, s in enumerate(seeds):
        c = scenes.batch_scene_cost(i, s)
        sc = scenes.batch_scene(i, s)
        n = int(sc.description.split(",")[1].split()[0])
        assert c == sc.dim ** 2 * n


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _small_inflations():
    """Eight small 7-DOF inflations with uneven obstacle counts (the units)."""
    from csdecomp_b200 import scenes
    from oracle import oracle as O
    out = []
    for i in range(8):
        sc = scenes.arm_scene(500 + i, num_spheres=12, num_world_boxes=4 + 3 * i, num_world_spheres=4 + 3 * i,
                              keepout=0.8)
        e = scenes.seed_edges(sc, 1, 600 + i, lambda q, sc=sc: O.check_points(sc.plant, q, O.RULE_GPU, nthreads=1),
                              lambda a, b, sc=sc: O.check_edges(sc.plant, a, b, nthreads=1)[0], length=(0.1, 0.4))
        assert e, i
        out.append((sc, e[0], float(sc.dim ** 2 * (8 + 6 * i))))
    return out


def _inflate(sc, edge):
    from csdecomp_b200.api import EizoOptions
    from oracle import oracle as O
    d = sc.dim
    A0 = np.zeros((2 * d, d), np.float32)
    for k in range(d):
        A0[2 * k, k], A0[2 * k + 1, k] = -1, 1
    b0 = np.concatenate([[-sc.lower()[k], sc.upper()[k]] for k in range(d)]).astype(np.float32)
    opt = EizoOptions(num_particles=100, mixing_steps=10, bisection_steps=5, max_iterations=3)
    A, b, _ = O.eizo(sc.plant, edge[0], edge[1], A0, b0, opt, sc.inspector.robot_geometry_ids, capacity=200,
                     nthreads=1)
    return A, b


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from csdecomp_b200.shard import reduce_timing
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    units = _small_inflations()
    b, e = cost_balanced_ranges([c for _, _, c in units], world)[rank]
    mine = [(i, _inflate(sc, edge)) for i, (sc, edge, _) in enumerate(units[b:e], start=b)]
    dev_s, wall_s, n = reduce_timing(dist, torch.device("cpu"), 1.0 + rank, 2.0 * (rank + 1), float(len(mine)))
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    out[rank] = (dev_s, wall_s, n, sorted((i, A.tolist(), bb.tolist()) for g in gathered for i, (A, bb) in g))
    dist.destroy_process_group()


def test_two_gloo_ranks_inflate_their_shards():
    """Each rank inflates its cost-balanced range of eight inflations (oracle
    EI-ZO); the gathered regions equal a one-rank run unit for unit, and the
    timing reduction takes the max over ranks and the sum of the units."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        ref = [(i, *(_x.tolist() for _x in _inflate(sc, edge))) for i, (sc, edge, _) in enumerate(_small_inflations())]
        for r in range(2):
            dev_s, wall_s, n, regions = out[r]
            assert dev_s == 2.0 and wall_s == 4.0  # max over ranks
            assert n == 8.0  # sum over ranks
            assert [x[0] for x in regions] == list(range(8))
            for (i, A, b), (j, A1, b1) in zip(regions, ref):
                assert i == j and A == A1 and b == b1, i
        assert any(len(A) > 14 for _, A, _ in ref)  # the inflations placed faces
