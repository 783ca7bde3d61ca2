"""Multi-GPU form of the solver: replicas only.

The hot path has no exchange step: impurity instances, sectors, c / c^+
excitation runs and served requests are independent units, so N GPUs run N
replicas of the single-GPU solver (one process per GPU) on disjoint shares of
the units, with no data-path collective.  The only communication is the
timing reduction (max over ranks) and, for the batched form, the gather of
small per-unit results (E0, G) to rank 0.  A sector larger than one GPU's HBM
(which no workload here reaches) would need a row-block split with a halo
exchange per H.v and is not implemented.

Units are assigned by longest-processing-time first on their cost (sum over
Lanczos runs of dim x steps), deterministically, so every rank computes the
same partition without communicating.
"""

from __future__ import annotations

from typing import Sequence


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Partition unit indices 0..len(costs)-1 over `world` ranks, LPT order:
    the costliest unit goes to the least loaded rank (ties: lower rank, lower
    index).  Returns the index list of every rank, each in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def my_units(costs: Sequence[float], rank: int, world: int) -> list[int]:
    """The units rank `rank` of `world` runs."""
    return shard(costs, world)[rank]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar (a timed region's length) over all ranks;
    the identity without a process group."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(obj, dist=None, world: int = 1):
    """Every rank's picklable result on rank 0 (list by rank); [obj] alone."""
    if dist is None or world == 1:
        return [obj]
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out
