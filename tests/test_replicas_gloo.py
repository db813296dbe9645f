"""The multi-rank plumbing of bench.py and the sharding module on CPU with gloo (world size 2 and 3).

A single pour does not shard, so N GPUs run N independent replicas; the only cross-rank steps are
the barrier and the max/sum reductions of the timing, exercised here with two CPU ranks. The
ensemble and the Poisson batch shard by pour and by snapshot, partitioned by estimated cost: every
pour and every snapshot lands on exactly one rank, every rank computes the same partition, the
loads are balanced, and the per-pour stats gathered from all ranks cover every pour once.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    bench.barrier(world)
    mx = bench.allmax(10.0 + rank, world, device="cpu")
    sm = bench.allsum(1.5 * (rank + 1), world, device="cpu")
    q.put((rank, mx, sm))
    dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, mx, sm in res:
        assert mx == 11.0
        assert sm == pytest.approx(4.5)


def _shard_rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from teapotfluidsimulation_b200 import engine as E
    from teapotfluidsimulation_b200 import sharding

    cfgs = E.ensemble_configs(2026, 11, 10.0, 20.0)
    pours = bench.shard_pours(cfgs, rank, world)
    snaps = bench.shard_snapshots(16, 4 * world, rank, world)
    # each rank reports stats for its own pours; the gather merges them on every rank
    stats = sharding.gather_stats({i: {"rank": rank, "cells": i * 10} for i in pours}, world)
    got = [None] * world
    dist.all_gather_object(got, (pours, snaps))
    q.put((rank, got, stats))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ensemble_and_poisson_shards_cover_everything_once(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    results = [q.get(timeout=10) for _ in range(world)]
    for rank, got, stats in results:
        pours = sorted(x for pr, _ in got for x in pr)
        snaps = sorted(x for _, sn in got for x in sn)
        assert pours == list(range(11))
        assert snaps == list(range(4 * world))
        assert sorted(stats) == list(range(11))
        assert all(stats[i]["rank"] == r for r, (pr, _) in enumerate(got) for i in pr)
    assert all(res[1] == results[0][1] for res in results)  # the same partition on every rank


def test_partition_by_cost_balances_uneven_units():
    from teapotfluidsimulation_b200 import sharding

    costs = [100, 1, 1, 1, 1, 50, 50, 3, 97, 2]
    parts = sharding.partition_by_cost(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    # the largest load stays within Graham's 4/3 of the lower bound max(mean load, largest unit)
    bound = max(sum(costs) / 3, max(costs))
    assert max(loads) <= 4 / 3 * bound
    assert sharding.partition_by_cost(costs, 3) == parts  # deterministic
    assert sharding.partition_by_cost([], 2) == [[], []]
    assert sharding.contiguous_runs([5, 1, 2, 3, 7, 8]) == [(1, 3), (5, 1), (7, 2)]
    with pytest.raises(ValueError):
        sharding.partition_by_cost([1.0, float("nan")], 2)


def test_pour_and_snapshot_costs_follow_the_sizes():
    from teapotfluidsimulation_b200 import engine as E
    from teapotfluidsimulation_b200 import sharding

    cfgs = E.ensemble_configs(2026, 6, 10.0, 20.0)
    costs = sharding.pour_costs(cfgs)
    sizes = [E.plan(c)["sizes"] for c in cfgs]
    work = [s.nx * s.ny * s.nz + s.n for s in sizes]
    assert all(c > 0 for c in costs)
    assert costs[work.index(max(work))] > costs[work.index(min(work))]
    sc = sharding.snapshot_costs(16, 0, 4)
    cell, _ = E.poisson_generate(16, 0, 4)
    assert sc == [float(v) for v in ((cell & 3) == 1).sum(axis=1)]
