"""Multi-GPU host logic (replicas only), as world-size-2 gloo ranks on CPU.

The same functions run bench.py's N > 1 path over NCCL: a deterministic
cost-balanced partition of independent units (every rank computes it alone),
the max-over-ranks timing reduction and the gather of small results.
"""

import importlib
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_pkg


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        load_pkg()
        rp = importlib.import_module("dmft_ed_zt_b200.replicas")
        mine = rp.my_units(costs, rank, world)
        load = sum(costs[i] for i in mine)
        t_max = rp.max_over_ranks(load, dist)
        allp = rp.gather_to_root(mine, dist, world)
        if rank == 0:
            out_q.put((t_max, allp))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_is_a_balanced_partition(pkg):
    from random import Random
    rp = importlib.import_module("dmft_ed_zt_b200.replicas")
    rng = Random(3)
    costs = [rng.uniform(1, 100) for _ in range(37)]
    for world in (1, 2, 3, 8):
        parts = rp.shard(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9      # LPT bound
        assert parts == rp.shard(costs, world)                    # deterministic
    assert rp.shard([], 2) == [[], []]
    with pytest.raises(ValueError):
        rp.shard([1.0], 0)


def test_two_gloo_ranks_partition_and_reduce(pkg):
    costs = [5.0, 3.0, 8.0, 1.0, 7.0, 2.0, 6.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    t_max, parts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(parts[0] + parts[1]) == list(range(len(costs)))
    assert not set(parts[0]) & set(parts[1])
    loads = [sum(costs[i] for i in p) for p in parts]
    assert t_max == max(loads)


class _Inst:
    def __init__(self, ns):
        self.nsite, self.norb = ns, 1


def _batch_rank(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import numpy as np
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        load_pkg()
        rp = importlib.import_module("dmft_ed_zt_b200.replicas")
        insts = [dict(model=_Inst(ns), sectors=[(ns // 2, ns // 2)], nspin=1 + (i % 2), tag=i)
                 for i, ns in enumerate([8, 12, 9, 14, 10, 8, 13, 11])]
        solved = []

        def fake_solve_batch(lst):                  # stands in for Solver.solve_batch
            solved.extend(inst["tag"] for inst in lst)
            return {"isector": [inst["tag"] % 3 for inst in lst], "e0": [-1.0 * inst["tag"] for inst in lst],
                    "G_cl": [np.full((1, 1, 4), inst["tag"], dtype=complex) for inst in lst]}
        res, mine = rp.sharded_batch(fake_solve_batch, insts, 300, rank, world, dist)
        out_q.put((rank, sorted(solved), mine, res["isector"], res["e0"], [g[0, 0, 0].real for g in res["G_cl"]]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sharded_batch(pkg):
    """The batched form's multi-GPU driver on two gloo ranks: the instances
    are split by cost with no overlap, every rank solves only its share, and
    the gathered results come back in instance order on every rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    (r0, s0, m0, isec0, e00, g0), (r1, s1, m1, isec1, e01, g1) = got
    assert s0 == m0 and s1 == m1 and not set(m0) & set(m1) and sorted(m0 + m1) == list(range(8))
    assert m0 and m1                                            # both ranks get work
    assert isec0 == isec1 == [i % 3 for i in range(8)]
    assert e00 == e01 == [-1.0 * i for i in range(8)]
    assert g0 == g1 == [float(i) for i in range(8)]
