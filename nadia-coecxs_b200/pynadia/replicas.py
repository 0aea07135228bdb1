"""Replicas across GPUs, one process per GPU.

Reconstructions are independent, so a job with several GPUs splits into whole
reconstructions (batch members, restart seeds, requests) assigned to ranks;
nothing crosses between GPUs while they iterate.  The only communication is
on the host side after the work: the job's time is the slowest rank's time
and its throughput is the units all ranks processed divided by that time.
The functions work with any torch.distributed backend (NCCL between GPUs,
gloo on the CPU); every rank must call them in the same order."""


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def shard(n_items, rank, world):
    """Indices of the items rank `rank` of `world` processes (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return list(range(rank, n_items, world))


def _reduce(value, op, device):
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    """The largest `value` over all ranks (the job's time)."""
    dist = _dist()
    return _reduce(value, dist.ReduceOp.MAX if dist else None, device)


def sum_over_ranks(value, device="cpu"):
    dist = _dist()
    return _reduce(value, dist.ReduceOp.SUM if dist else None, device)


def job_rate(units, seconds, device="cpu"):
    """Units processed by all ranks per second of the slowest rank."""
    total = sum_over_ranks(units, device)
    slowest = max_over_ranks(seconds, device)
    return total / slowest
