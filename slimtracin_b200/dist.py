"""Multi-GPU plumbing for the tracing path: replicas only.

Rays, pixels and requests are independent and scenes are read-only during a frame, so every rank
holds a full scene replica and works on its own share of views; nothing is exchanged on the data
path.  The only collectives are the barrier around timed regions and the max over ranks of device
times (torch.distributed; NCCL on GPUs, gloo in the CPU tests).
"""
import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def shard(items, rank, world):
    """The contiguous share of `items` that `rank` of `world` works on (sizes differ by at most 1)."""
    n = len(items)
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return items[begin:begin + base + (1 if rank < extra else 0)]


def max_over_ranks(value, device=None):
    """The largest `value` over all ranks (every rank gets it); the identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
