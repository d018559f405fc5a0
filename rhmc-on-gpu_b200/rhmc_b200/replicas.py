"""Replica parallelism across GPUs (one process per GPU).

The reference is a single-GPU program and its hot path has no data exchange at one-GPU
volumes, so several GPUs run independent replicas (independent Markov chains, or independent
pseudofermion sets): each rank gets its own seeds and its own fields, nothing crosses ranks in
the data path, and the only collectives are the timing reductions of the benchmark
(max over ranks of the elapsed time, sum of the work).
"""
import os


def world():
    """(rank, world_size, local_rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base, rank):
    """Seed of `rank`'s replica: distinct per rank, reproducible."""
    return int(base) + 7919 * int(rank)


def max_over_ranks(value, dist=None, device="cpu"):
    """Largest `value` over all ranks (the job time of a weak-scaling step)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device="cpu"):
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_this_rank, elapsed_this_rank, dist=None, device="cpu"):
    """Whole-job throughput: units processed by all ranks / max over ranks of the elapsed time."""
    total = sum_over_ranks(units_this_rank, dist, device)
    t = max_over_ranks(elapsed_this_rank, dist, device)
    return total / t if t > 0 else 0.0
