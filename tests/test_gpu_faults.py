"""Failure detection without a GPU fault (the reference only aborts).

Every failure here is made on the host or by a wait that is allowed to run
out: invalid or non-finite input, a request beyond the memory budget, a
cancelled request, a pass cap too small for the run, and a persistent launch
in which one CTA leaves without arriving at the grid barrier, so the others'
bounded wait expires and the kernel reports it through its status word.
After each, the same context still gives correct results.
"""

import ctypes as C
import time

import numpy as np
import pytest

from conftest import oracle_for, random_model


def test_footprint_query_without_gpu(pkg, configs):
    """edzt_instance_footprint needs no device: it grows with the sector sizes
    and rejects invalid requests."""
    pkg.build()
    L = pkg.load_library()
    keep = []
    sizes = []
    for ns in (8, 10, 12):
        m = pkg.Model(1, ns - 1, np.zeros((1, 2)), np.zeros((ns - 1, 2)), np.full((1, ns - 1, 2), 0.5), U=2.0)
        rec = pkg._instance(dict(model=m, sectors=configs.near_half_sectors(ns), nspin=2), keep)
        b = C.c_longlong()
        assert L.edzt_instance_footprint(C.byref(rec), C.byref(b)) == pkg.EDZT_OK
        sizes.append(b.value)
    assert sizes[0] < sizes[1] < sizes[2]
    assert sizes[2] >= 32 * 9 * 700000                    # the nsite-12 scan's pair buffers
    bad = pkg._instance(dict(model=m, sectors=[(30, 1)], nspin=1), keep)
    assert L.edzt_instance_footprint(C.byref(bad), C.byref(b)) == pkg.EDZT_ERR_ARG


@pytest.mark.gpu
def test_non_finite_model_rejected(pkg, solver):
    rng = np.random.default_rng(3)
    m = random_model(pkg, rng, 1, 5)
    for attr in ("U", "mu"):
        bad = random_model(pkg, np.random.default_rng(3), 1, 5)
        setattr(bad, attr, float("nan"))
        with pytest.raises(pkg.EDError) as e:
            solver.set_model(bad)
        assert e.value.code == pkg.EDZT_ERR_ARG
    bad = random_model(pkg, np.random.default_rng(3), 1, 5)
    bad.vmk[0, 2, 1] = np.inf
    with pytest.raises(pkg.EDError):
        solver.set_model(bad)
    solver.set_model(m)                                   # still usable
    assert solver.dim(3, 3) == 400


@pytest.mark.gpu
def test_server_rejects_over_budget_and_cancels(pkg, solver, configs):
    rng = np.random.default_rng(9)
    reqs = [dict(model=random_model(pkg, rng, 1, 7), sectors=configs.near_half_sectors(8), nspin=1, seed=i)
            for i in range(4)]
    omega = pkg.matsubara(32, 20.0)
    fp = solver.footprint(reqs[0])
    small = pkg.Server(solver, 60, omega, hbm_budget=fp // 2)
    try:
        with pytest.raises(pkg.EDError) as e:
            small.submit(reqs[0])
        assert e.value.code == pkg.EDZT_ERR_OOM
    finally:
        small.close()
    ref = []
    for r in reqs:
        solver.set_model(r["model"])
        ref.append(solver.solve(r["sectors"], 60, omega, nspin=1, seed=r["seed"]))
    sv = pkg.Server(solver, 60, omega, hbm_budget=int(2.5 * fp))                  # two run at a time
    try:
        sv.set_step_ms(0.01)                                                        # one launch per step
        ids = [sv.submit(r) for r in reqs]
        sv.step()                                                                   # 0, 1 running; 2, 3 queued
        sv.cancel(ids[1])                                                           # a running request
        sv.cancel(ids[3])                                                           # a queued one
        with pytest.raises(pkg.EDError):
            sv.cancel(12345)
        res = {}
        for _ in range(5000):
            if len(res) == 2:
                break
            sv.step()
            for i in (0, 2):
                if i not in res:
                    r = sv.result(ids[i])
                    if r is not None:
                        res[i] = r
        for i in (0, 2):
            assert res[i]["isector"] == ref[i]["isector"]
            assert abs(res[i]["e0"] - ref[i]["e0"]) <= 1e-10 * max(1.0, abs(ref[i]["e0"]))
            assert np.abs(res[i]["G_cl"] - ref[i]["G_cl"]).max() <= 1e-8
        with pytest.raises(pkg.EDError):
            sv.result(ids[1])                                                       # cancelled
        assert sv.step() == (0, 0, 0)
    finally:
        sv.close()


@pytest.mark.gpu
def test_pass_cap_and_stalled_barrier(pkg, solver, oracle_mod):
    rng = np.random.default_rng(21)
    m = random_model(pkg, rng, 1, 9)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    v0 = oracle_mod.start_vector(5, 0, o.dim(5, 5))
    try:
        solver.set_fault_test(pass_cap=3)                 # the run needs ~2 * 60 passes
        with pytest.raises(pkg.EDError) as e:
            solver.lanczos_iteration(5, 5, v0, 60)
        assert e.value.code == pkg.EDZT_ERR_NUMERIC
        solver.set_fault_test(wait_seconds=0.2, stall_cta=0)
        t0 = time.perf_counter()
        with pytest.raises(pkg.EDError) as e:
            solver.lanczos_iteration(5, 5, v0, 60)
        assert e.value.code == pkg.EDZT_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 5.0
    finally:
        solver.set_fault_test()
    n, a, b = solver.lanczos_iteration(5, 5, v0, 60)     # the context is still good
    n_ref, a_ref, b_ref = o.lanczos_iteration(5, 5, v0, 60)
    assert n == n_ref and np.abs(a[:40] - a_ref[:40]).max() <= 1e-8
