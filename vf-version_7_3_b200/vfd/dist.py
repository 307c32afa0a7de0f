"""Multi-GPU plumbing of the diffusion path: one process per GPU, independent
units per rank, no data-path collective.

The path shards naturally (the reference splits its chemicals over GPUs by
ic % N_GPU with no exchange, DiffusionHelper.cpp:386-392): worlds, fields or
requests are independent.  The only collective is the timing reduction
(max over ranks) used by the benchmark.
"""
import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_units, rank, world_size):
    """Units of this rank, round-robin (unit i -> rank i % world_size)."""
    return [i for i in range(n_units) if i % world_size == rank]


def max_over_ranks(value, device=None):
    """Max of a scalar over all ranks of the default process group (identity
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, elapsed_s, world_size):
    """Whole-job throughput when every rank processed `units_per_rank` units
    and the job took the max-over-ranks `elapsed_s` (weak scaling)."""
    return world_size * units_per_rank / elapsed_s
