"""The multi-rank plumbing of bench.py on CPU with gloo (world size 2).

A single pour does not shard, so N GPUs run N independent replicas; the only cross-rank steps are
the barrier and the max/sum reductions of the timing, exercised here with two CPU ranks.
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
