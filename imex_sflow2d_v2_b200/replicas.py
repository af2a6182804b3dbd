"""Whole-job throughput of independent replicas (one per rank).

The time step does not shard: on N GPUs each rank advances its own grid, with
no data exchanged.  The job's rate is then all ranks' cell-updates divided by
the slowest rank's time.  The reduction is the only collective; with the
`gloo` backend it runs on the CPU (tests), with `nccl` on the GPUs (bench)."""


def job_rate(local_seconds, units_per_rank, dist=None, device="cpu"):
    """(units/s over all ranks, max seconds over ranks)."""
    if dist is None or not dist.is_initialized():
        return units_per_rank / local_seconds, local_seconds
    import torch
    t = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    slowest = float(t.item())
    return dist.get_world_size() * units_per_rank / slowest, slowest
