"""GPU parity of the served form (edzt_server_*): continuous batching.

Requests that arrive while others are on the GPU join the next persistent
launch; each request's result must be the same alone (edzt_solve on it) and
in the mix, within the solve tolerances (E0 1e-10 relative, G(i w) 1e-8),
whatever the arrival pattern or the memory budget.
"""

import numpy as np
import pytest

from conftest import random_model

pytestmark = pytest.mark.gpu
E_TOL = 1e-10
G_TOL = 1e-8


def _requests(pkg, configs, n=6, seed=31):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ns = int(rng.integers(6, 11))
        nspin = int(rng.integers(1, 3))
        m = random_model(pkg, rng, 1, ns - 1, spin_dep=(nspin == 2))
        out.append(dict(model=m, sectors=configs.near_half_sectors(ns), nspin=nspin, seed=int(rng.integers(1 << 40))))
    return out


def _alone(solver, reqs, omega, maxnstep):
    out = []
    for r in reqs:
        solver.set_model(r["model"])
        out.append(solver.solve(r["sectors"], maxnstep, omega, nspin=r["nspin"], seed=r["seed"]))
    return out


def _same(got, ref):
    assert got["isector"] == ref["isector"]
    assert abs(got["e0"] - ref["e0"]) <= E_TOL * max(1.0, abs(ref["e0"]))
    assert np.abs(got["G_cl"] - ref["G_cl"]).max() <= G_TOL


def test_server_mix_equals_alone(pkg, solver, configs):
    reqs = _requests(pkg, configs)
    omega = pkg.matsubara(128, 40.0)
    ref = _alone(solver, reqs, omega, 100)
    sv = pkg.Server(solver, 100, omega)
    try:
        ids = [sv.submit(r) for r in reqs[:3]]             # three at once
        sv.step()                                           # they are on the GPU (scan) ...
        ids += [sv.submit(r) for r in reqs[3:5]]            # ... when two more arrive
        sv.step()
        ids.append(sv.submit(reqs[5]))
        res = {}
        for _ in range(2000):
            na, nq, nf = sv.step()
            for i, rid in enumerate(ids):
                if i not in res:
                    r = sv.result(rid)
                    if r is not None:
                        res[i] = r
            if len(res) == len(reqs):
                break
        assert len(res) == len(reqs)
        for i in range(len(reqs)):
            _same(res[i], ref[i])
        assert sv.step() == (0, 0, 0)                       # idle
    finally:
        sv.close()


def test_server_budget_admits_one_at_a_time(pkg, solver, configs):
    rng = np.random.default_rng(32)
    reqs = [dict(model=random_model(pkg, rng, 1, 7), sectors=configs.near_half_sectors(8), nspin=1,
                 seed=int(rng.integers(1 << 40))) for _ in range(3)]                   # equal footprints
    omega = pkg.matsubara(64, 30.0)
    ref = _alone(solver, reqs, omega, 80)
    budget = int(1.5 * max(solver.footprint(r) for r in reqs))                      # one fits at a time
    sv = pkg.Server(solver, 80, omega, hbm_budget=budget)
    try:
        sv.set_step_ms(0.01)                                # one launch of two phases per step
        ids = [sv.submit(r) for r in reqs]
        na, nq, nf = sv.step()
        assert na == 1 and nq == 2                          # the budget holds the others back
        res = {}
        for _ in range(5000):
            if len(res) == len(reqs):
                break
            sv.step()
            for i, rid in enumerate(ids):
                if i not in res:
                    r = sv.result(rid)
                    if r is not None:
                        res[i] = r
        for i in range(len(reqs)):
            _same(res[i], ref[i])
    finally:
        sv.close()


def test_serve_loop_with_arrivals(pkg, solver, configs):
    reqs = _requests(pkg, configs, n=5, seed=33)
    omega = pkg.matsubara(64, 30.0)
    ref = _alone(solver, reqs, omega, 80)
    sv = pkg.Server(solver, 80, omega)
    try:
        arrivals = [0.0, 0.001, 0.02, 0.02, 0.05]
        done, lat, total = pkg.serve(sv, reqs, arrivals)
        for i in range(len(reqs)):
            _same(done[i], ref[i])
        assert np.all(lat > 0) and total >= max(arrivals)
    finally:
        sv.close()


def test_server_rejects_bad_requests(pkg, solver, configs):
    omega = pkg.matsubara(16, 10.0)
    sv = pkg.Server(solver, 20, omega)
    try:
        r = _requests(pkg, configs, n=1)[0]
        with pytest.raises(pkg.EDError):
            sv.submit(dict(r, nspin=3))
        with pytest.raises(pkg.EDError):
            sv.submit(dict(r, sectors=[(40, 1)]))
        assert sv.step() == (0, 0, 0)
    finally:
        sv.close()
