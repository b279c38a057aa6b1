"""Replica runs over torch.distributed (one process per GPU).

A solve is one heightmap whose state fits one GPU, so a multi-GPU run is N
independent replicas: no collective touches the data path.  The ranks meet
only at barriers around the timed region and in one max-reduction of their
device-timed durations, so the job's time is that of its slowest rank, and
rank 0 reports the whole job's throughput.
"""
from __future__ import annotations


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of `values` (floats) over the ranks of the
    default process group, or `values` unchanged without one."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_rate(world: int, steps: int, units_per_step: float, elapsed_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed in `steps` steps
    (each rank the same work), over the slowest rank's elapsed time."""
    if elapsed_ms <= 0:
        raise ValueError("elapsed time must be positive")
    return world * steps * units_per_step / (elapsed_ms * 1e-3)
