"""Replica parallelism for several GPUs of one node.

The sTDA path shards only across independent molecules: each rank (one
process per GPU) solves its own molecules with its own engine and there is no
exchange on the data path.  The only collectives are the barrier around the
timed region and the maximum of the timed region over ranks, from which the
whole-job rate is computed.  A set of molecules is split over the ranks by
shard_by_cost (every rank computes the same split from the same costs, so no
message carries it).
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


def shard_by_cost(costs, world: int):
    """Split items of the given costs over `world` ranks (longest-processing-
    time bin-pack: items in decreasing cost, ties by index, each to the rank
    with the least load so far, ties to the lower rank).  Deterministic;
    returns one ascending index list per rank, every index exactly once.  The
    largest load exceeds the smallest by at most the largest single cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(x) for x in out]
