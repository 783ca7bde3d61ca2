"""GPU parity at the large sizes of the workloads, against the CPU oracle.

  * nsite 14, sector (7, 7), 11,778,624 states: the first 50 Lanczos a_n, b_n
    of lanczos_iteration and E0 of diag_lanczos (the reference's
    src/lanczos_solver.f90:20-173);
  * nsite 16, sector (8, 8), 165,636,900 states (beyond the reference's
    int32 states, src/ed_basis.f90:16-17,135): the first 30 a_n, b_n;
  * one instance of nsite 13 in a batched launch (edzt_solve_batch) and one
    request of nsite 12 in the served form (edzt_server_*), each against the
    oracle's ground_state + cluster_green_ftn.

Tolerances: a_n, b_n 1e-8; E0 1e-10 relative; G(i w_n) 1e-8.  The oracle
runs on all host threads; the step counts keep it within about a minute per
case on a 16-thread host.
"""

import numpy as np
import pytest

from conftest import ab_compare_len, oracle_for, random_model

pytestmark = pytest.mark.gpu
E_TOL = 1e-10
AB_TOL = 1e-8
G_TOL = 1e-8


def _single_orbital(pkg, nsite, seed):
    """Half-filled single-orbital impurity: eps ~ U(-2,2), V ~ U(0.1,1), U = 3."""
    rng = np.random.default_rng(seed)
    nb = nsite - 1
    ek = rng.uniform(-2.0, 2.0, nb)
    V = rng.uniform(0.1, 1.0, nb)
    return pkg.Model(1, nb, np.zeros((1, 2)), np.stack([ek, ek], 1), np.stack([V, V], 1).reshape(1, nb, 2),
                     U=3.0, mu=1.5)


def test_nsite14_lanczos_coefficients_and_e0(pkg, solver, oracle_mod):
    m = _single_orbital(pkg, 14, 1414)
    o = oracle_for(oracle_mod, m)
    n_states = o.dim(7, 7)
    assert n_states == 3432 ** 2
    seed, stream, steps = 21, 3, 120
    v0 = oracle_mod.start_vector(seed, stream, n_states)
    n_ref, a_ref, b_ref = o.lanczos_iteration(7, 7, v0, steps)
    solver.set_model(m)
    n, a, b = solver.lanczos_iteration(7, 7, v0, steps)
    assert n == n_ref == steps
    k = ab_compare_len(b_ref, n)
    assert k == 50
    assert np.abs(a[:k] - a_ref[:k]).max() <= AB_TOL
    assert np.abs(b[:k] - b_ref[:k]).max() <= AB_TOL
    e_ref, _ = oracle_mod.tridiag_lowest(a_ref, b_ref, n_ref)
    r = solver.diag_lanczos(7, 7, steps, seed=seed, stream=stream)      # same start vector by (seed, stream)
    assert abs(r["e0"] - e_ref) <= E_TOL * max(1.0, abs(e_ref))
    assert r["residual"] < 1e-8


def test_nsite16_lanczos_coefficients(pkg, solver, oracle_mod):
    m = _single_orbital(pkg, 16, 1616)
    o = oracle_for(oracle_mod, m)
    n_states = o.dim(8, 8)
    assert n_states == 12870 ** 2
    steps = 30
    v0 = oracle_mod.start_vector(5, 0, n_states)
    n_ref, a_ref, b_ref = o.lanczos_iteration(8, 8, v0, steps)
    solver.set_model(m)
    n, a, b = solver.lanczos_iteration(8, 8, v0, steps)
    del v0
    assert n == n_ref == steps
    assert np.abs(a - a_ref).max() <= AB_TOL
    assert np.abs(b - b_ref).max() <= AB_TOL


def _oracle_solve(oracle_mod, inst, maxnstep, omega):
    o = oracle_for(oracle_mod, inst["model"])
    gs = o.ground_state(inst["sectors"], maxnstep, seed=inst["seed"])
    cg = o.cluster_green_ftn(inst["nspin"], *gs["sector"], gs["vec"], gs["e0"], maxnstep, omega)
    return gs, cg


def test_batched_nsite13_instance_against_oracle(pkg, solver, configs, oracle_mod):
    """One nsite-13 instance solved in a batched launch together with two
    smaller ones, against the oracle."""
    rng = np.random.default_rng(1313)
    insts = []
    for ns in (13, 8, 10):
        m = random_model(pkg, rng, 1, ns - 1)
        insts.append(dict(model=m, sectors=configs.near_half_sectors(ns), nspin=1, seed=int(rng.integers(1 << 40))))
    maxnstep = 100
    omega = pkg.matsubara(256, 100.0)
    res = solver.solve_batch(insts, maxnstep, omega)
    gs, cg = _oracle_solve(oracle_mod, insts[0], maxnstep, omega)
    assert res["isector"][0] == gs["isector"]
    assert abs(res["e0"][0] - gs["e0"]) <= E_TOL * max(1.0, abs(gs["e0"]))
    assert np.abs(res["G_cl"][0] - cg["G_cl"]).max() <= G_TOL


def test_served_nsite12_request_against_oracle(pkg, solver, configs, oracle_mod):
    """One nsite-12 request served together with a smaller one that arrives
    while it runs, against the oracle."""
    rng = np.random.default_rng(1212)
    reqs = []
    for ns in (12, 9):
        m = random_model(pkg, rng, 1, ns - 1)
        reqs.append(dict(model=m, sectors=configs.near_half_sectors(ns), nspin=1, seed=int(rng.integers(1 << 40))))
    maxnstep = 100
    omega = pkg.matsubara(256, 100.0)
    sv = pkg.Server(solver, maxnstep, omega)
    try:
        big = sv.submit(reqs[0])
        sv.step()
        small = sv.submit(reqs[1])
        got = {}
        for _ in range(200):
            sv.step()
            for rid in (big, small):
                if rid not in got:
                    r = sv.result(rid)
                    if r is not None:
                        got[rid] = r
            if len(got) == 2:
                break
    finally:
        sv.close()
    assert len(got) == 2
    gs, cg = _oracle_solve(oracle_mod, reqs[0], maxnstep, omega)
    r = got[big]
    assert r["isector"] == gs["isector"]
    assert abs(r["e0"] - gs["e0"]) <= E_TOL * max(1.0, abs(gs["e0"]))
    assert np.abs(r["G_cl"] - cg["G_cl"]).max() <= G_TOL
