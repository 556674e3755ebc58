"""Multi-rank plumbing of the benchmark: one process per GPU, every rank
advancing its own independent case (replicas of a channel, or its share of an
ensemble); no data-path collective, only a barrier and the max-over-ranks of
the timed interval.  The path itself does not need to shard to run on N GPUs:
a channel at these sizes fits one B200, so N GPUs run N cases (weak scaling).
"""
import os


def dist_env():
    """(world size, rank, local rank) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init(backend, timeout_s=120):
    """Initialises the process group when WORLD_SIZE > 1 (rendezvous on
    127.0.0.1 through the torchrun environment); returns the module or None."""
    ws, _, _ = dist_env()
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def replica_seed(base, rank):
    """Seed of rank `rank`'s replica: distinct per rank, base on rank 0."""
    return int(base) + int(rank)


def ensemble_share(n, ws, rank):
    """Indices of the ensemble members rank `rank` advances: a contiguous
    block, sizes differing by at most one."""
    lo = n * rank // ws
    hi = n * (rank + 1) // ws
    return list(range(lo, hi))


def max_over_ranks(value, dist, device=None):
    """The max of a float over all ranks (the timed interval of the job)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device=None):
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
