"""Replica parallelism for several GPUs of one node.

The sTDA path shards only across independent molecules: each rank (one
process per GPU) solves its own molecules with its own engine and there is no
exchange on the data path.  The only collectives are the barrier around the
timed region and the maximum of the timed region over ranks, from which the
whole-job rate is computed.
"""
from __future__ import annotations


def _tensor(value, device):
    import torch
    return torch.tensor([float(value)], dtype=torch.float64,
                        device=device if device is not None else "cpu")


def barrier(dist, device=None) -> None:
    """All ranks reach this point (an all-reduce of a zero, then a device sync)."""
    if dist is None:
        return
    import torch
    t = _tensor(0.0, device)
    dist.all_reduce(t)
    if device is not None and str(device).startswith("cuda"):
        torch.cuda.synchronize(device)


def max_over_ranks(dist, value: float, device=None) -> float:
    """The largest `value` over all ranks (the job's timed region is the slowest rank's)."""
    if dist is None:
        return float(value)
    t = _tensor(value, device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, max_seconds: float) -> float:
    """Units processed by all ranks divided by the slowest rank's time."""
    return world * units_per_rank / max_seconds
