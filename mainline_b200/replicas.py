"""Independent DMC replicas, one process per GPU (the population does not
shard across GPUs; QWalk's MPI walkers become separate seeded replicas).

The only cross-rank operations are the start barrier and the max-over-ranks
of the timed durations; throughput is the units all replicas processed over
the slowest replica's time.
"""
from __future__ import annotations


def replica_seed(base: int, rank: int) -> int:
    """Seed of replica `rank`: distinct walks on every rank."""
    return base + 7919 * rank


def max_over_ranks(values, device: str = "cuda"):
    """Element-wise maximum of `values` (floats) over all ranks of the
    default process group (NCCL on GPUs, gloo on CPU); identity on one rank."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def aggregate_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return units_per_rank * world / (max_ms / 1e3)
