"""Host-side helpers for one process per GPU (replicas / independent shards).

The solve does not exchange data between GPUs: N processes run N independent
problems, and only their timings meet, as the maximum over ranks. These
helpers work with any torch.distributed backend: NCCL needs the value on the
rank's CUDA device, gloo on the CPU (which is how they are tested without a
GPU)."""


def max_over_ranks(value, dist=None, device=None):
    """Maximum of a float over all ranks of the default process group
    (``value`` itself when ``dist`` is None)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=f"cuda:{device}" if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, seconds_max):
    """Whole-job throughput of ``world`` replicas that each processed
    ``units_per_rank`` units, timed as the slowest rank's seconds."""
    return world * units_per_rank / seconds_max
