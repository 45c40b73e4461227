"""Multi-GPU host logic.  The level-set path shards without a data-path
collective: independent problems (batch members, benchmark replicas) are
partitioned over ranks, one process per GPU, and only the timings and
diagnostics are reduced (max of device time, sum of work) at the end.
"""


def partition(n_items, rank, world):
    """Contiguous, balanced block of item indices owned by `rank`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return list(range(start, stop))


def _reduce(value, op):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM)


def aggregate_rate(work_per_rank, ms_per_rank_max, world):
    """Whole-job throughput: total work of all ranks over the slowest rank's time."""
    return work_per_rank * world / (ms_per_rank_max * 1e-3)
