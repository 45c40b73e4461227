"""Multi-rank host logic on CPU (gloo, world size 2): the partition of
independent problems over ranks and the max/sum reductions the benchmark
uses for its whole-job numbers."""
import os
import socket

import pytest

from felspa_b200.replicas import aggregate_rate, partition


def test_partition_covers_once():
    for n in (0, 1, 7, 256):
        for world in (1, 2, 3, 8):
            got = sorted(i for r in range(world) for i in partition(n, r, world))
            assert got == list(range(n))
            sizes = [len(partition(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(4, 2, 2)


def test_aggregate_rate():
    assert aggregate_rate(1e9, 500.0, 4) == 8e9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from felspa_b200.replicas import max_over_ranks, partition, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mine = partition(256, rank, world)
    import torch
    t = torch.zeros(256, dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    out.put((rank, int(t.min()), int(t.max()), max_over_ranks(10.0 + rank), sum_over_ranks(len(mine))))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmin, tmax, mx, sm in res:
        assert (tmin, tmax) == (1, 1)      # every problem owned exactly once
        assert mx == 11.0 and sm == 256
