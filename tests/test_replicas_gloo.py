"""The multi-rank plumbing of bench.py on CPU with gloo (world size 2).

A single pour does not shard, so N GPUs run N independent replicas; the only cross-rank steps are
the barrier and the max/sum reductions of the timing, exercised here with two CPU ranks. The
ensemble and the Poisson batch shard by pour and by snapshot: every pour and every snapshot lands on
exactly one rank.
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

    pours = bench.shard_pours(list(range(11)), rank, world)
    first = bench.poisson_first_snapshot(rank, 4)
    got = [None] * world
    dist.all_gather_object(got, (pours, list(range(first, first + 4))))
    q.put((rank, got))
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
        p.join(120)
        assert p.exitcode == 0
    for _ in range(world):
        rank, got = q.get(timeout=10)
        pours = sorted(x for pr, _ in got for x in pr)
        snaps = sorted(x for _, sn in got for x in sn)
        assert pours == list(range(11))
        assert snaps == list(range(4 * world))
