"""One process per GPU, each evaluating its own independent system (replicas).

The treecode needs no data exchange between GPUs when every rank owns whole systems, so
the only collectives are the ones measurement needs: a barrier before and after the
timed region and the maximum of the ranks' device times.  Rank, world size and local
rank come from the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK).
"""
import datetime
import os


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend="nccl", timeout_s=600):
    """Join the process group when there is more than one rank; returns the
    torch.distributed module, or None for a single process."""
    _, world, _ = rank_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(value, dist, device=None):
    """The largest value over all ranks (every rank gets it)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def system_seed(rank, base=1):
    """Each rank evaluates its own seeded system of the same size (weak scaling)."""
    return base + rank


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
