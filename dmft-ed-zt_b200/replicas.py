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
    """Every rank's picklable result, on every rank (list by rank); [obj] alone."""
    if dist is None or world == 1:
        return [obj]
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def instance_cost(inst, maxnstep: int) -> float:
    """Cost of one impurity solve for the partition: the sum over its Lanczos
    runs of dimension x steps (ground-state scan and eigenvector pass of every
    sector, plus the c / c^+ runs of the ground-state sector's neighbours,
    bounded by the largest neighbouring dimension)."""
    from math import comb
    m = inst["model"]
    ns = m.nsite
    dims = [comb(ns, u) * comb(ns, d) for u, d in inst["sectors"]]
    nruns = 4 * m.norb if int(inst.get("nspin", 1)) == 2 else 2 * m.norb
    return float(maxnstep) * (2.0 * sum(dims) + nruns * max(dims))


def sharded_batch(solve_batch, instances, maxnstep: int, rank: int, world: int, dist=None):
    """The batched form over `world` ranks: rank `rank` solves its LPT share
    of the instances (by instance_cost) with solve_batch(list) -> dict of
    isector [n], e0 [n] and G_cl (list of n arrays); the shares are gathered
    to every rank and returned in instance order, with this rank's indices.
    No data-path collective: the only exchange is the final gather of the
    small results."""
    costs = [instance_cost(inst, maxnstep) for inst in instances]
    mine = my_units(costs, rank, world)
    part = solve_batch([instances[i] for i in mine]) if mine else {"isector": [], "e0": [], "G_cl": []}
    local = (mine, [int(v) for v in part["isector"]], [float(v) for v in part["e0"]], list(part["G_cl"]))
    shares = gather_to_root(local, dist, world)
    n = len(instances)
    isector, e0, G = [None] * n, [None] * n, [None] * n
    for idx, isec, ee, gg in shares:
        for j, i in enumerate(idx):
            isector[i], e0[i], G[i] = isec[j], ee[j], gg[j]
    return {"isector": isector, "e0": e0, "G_cl": G}, mine
