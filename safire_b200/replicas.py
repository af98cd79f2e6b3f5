"""Replica bookkeeping for several GPUs of one node (bench.py under torchrun).

The propagation does not shard: every rank runs its own walker population of the same system with
its own seed, and no collective touches the data path. The only cross-rank steps are the job's
timing, the maximum over ranks of each rank's device time, and the job's throughput, the
walker-steps of all ranks over that time.
"""
import datetime


def seed_for(rank, base=1000):
    """The walker-population seed of a rank: independent replicas."""
    return base + int(rank)


def init(world, backend="nccl", timeout_s=300):
    """The process group for world > 1 (None for one rank); a short timeout ends waits on a lost rank."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x, dist=None, device="cuda"):
    """The maximum of x over all ranks (x itself for one rank)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms_max):
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return float(units_per_rank) * int(world) / (float(ms_max) * 1e-3)
