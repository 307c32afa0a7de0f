"""Multi-GPU plumbing of the diffusion path: one process per GPU, independent
units per rank, no data-path collective.

The path shards naturally (the reference splits its chemicals over GPUs by
ic % N_GPU with no exchange, DiffusionHelper.cpp:386-392): worlds of an
ensemble, requests of a serving stream and fields of one world are
independent units.  Unit i goes to rank i % world_size.  The collectives
here are for timing and reporting only (max of the elapsed time, sum of the
work done, gathering results for a check), never on the data path.
"""
import os


def env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_units, rank, world_size):
    """Units of this rank, round-robin (unit i -> rank i % world_size), the
    reference's chemical-to-GPU rule generalised to any unit."""
    return [i for i in range(n_units) if i % world_size == rank]


def _group():
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier():
    """Barrier over the default process group (no-op without one)."""
    if _group():
        import torch.distributed as dist
        dist.barrier()


def _reduce(value, op, device):
    import torch
    import torch.distributed as dist
    if not _group():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device=None):
    """Max of a scalar over all ranks of the default process group (identity
    when no group is initialised)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX if dist.is_available() else None, device)


def sum_over_ranks(value, device=None):
    """Sum of a scalar over all ranks (identity without a group)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM if dist.is_available() else None, device)


def aggregate_rate(units_per_rank, elapsed_s, world_size):
    """Whole-job throughput when every rank processed `units_per_rank` units
    and the job took the max-over-ranks `elapsed_s` (weak scaling)."""
    return world_size * units_per_rank / elapsed_s


def gather_units(local, device=None):
    """{unit index: value} of every rank merged on every rank (all_gather of
    Python objects; a reporting/check step, not the data path)."""
    if not _group():
        return dict(local)
    import torch.distributed as dist
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, dict(local))
    merged = {}
    for d in out:
        merged.update(d)
    return merged
