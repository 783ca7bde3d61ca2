"""GPU parity of the batched form (edzt_solve_batch): every instance's result
is the same alone (edzt_solve on that instance) and in the mix, and matches
the oracle.  Tolerances as the single-solve tests: E0 1e-10 relative, G(i w)
1e-8.
"""

import numpy as np
import pytest

from conftest import oracle_for, random_model

pytestmark = pytest.mark.gpu
E_TOL = 1e-10
G_TOL = 1e-8


def _instances(pkg, configs):
    rng = np.random.default_rng(2718)
    out = []
    for ns, nspin in [(6, 1), (8, 2), (7, 1), (10, 2), (9, 1), (6, 2)]:
        m = random_model(pkg, rng, 1, ns - 1, spin_dep=(nspin == 2))
        out.append(dict(model=m, sectors=configs.near_half_sectors(ns), nspin=nspin, seed=int(rng.integers(1 << 40))))
    k = configs.kanamori_n10()
    out.append(dict(model=k["model"], sectors=k["sectors"][1:4], nspin=1, seed=5))
    return out


def _check_against_alone(solver, insts, res, omega, maxnstep):
    for i, inst in enumerate(insts):
        solver.set_model(inst["model"])
        one = solver.solve(inst["sectors"], maxnstep, omega, nspin=inst["nspin"], seed=inst["seed"])
        assert res["isector"][i] == one["isector"], i
        assert abs(res["e0"][i] - one["e0"]) <= E_TOL * max(1.0, abs(one["e0"])), i
        assert np.abs(res["G_cl"][i] - one["G_cl"]).max() <= G_TOL, i


def test_batch_matches_single_solves(pkg, solver, configs):
    insts = _instances(pkg, configs)
    omega = pkg.matsubara(256, 50.0)
    res = solver.solve_batch(insts, 120, omega)
    _check_against_alone(solver, insts, res, omega, 120)


def test_batch_in_waves_and_against_oracle(pkg, solver, configs, oracle_mod):
    insts = _instances(pkg, configs)[:4]
    omega = pkg.matsubara(128, 40.0)
    one_wave = solver.solve_batch(insts, 100, omega)
    waves = solver.solve_batch(insts, 100, omega, hbm_budget=1)     # one instance per wave
    assert np.array_equal(one_wave["isector"], waves["isector"])
    assert np.abs(one_wave["e0"] - waves["e0"]).max() <= E_TOL * max(1.0, np.abs(one_wave["e0"]).max())
    for g1, g2 in zip(one_wave["G_cl"], waves["G_cl"]):
        assert np.abs(g1 - g2).max() <= G_TOL
    inst = insts[1]                                                  # nsite 8, nspin 2
    o = oracle_for(oracle_mod, inst["model"])
    gs = o.ground_state(inst["sectors"], 100, seed=inst["seed"])
    cg = o.cluster_green_ftn(2, *gs["sector"], gs["vec"], gs["e0"], 100, omega)
    assert one_wave["isector"][1] == gs["isector"]
    assert abs(one_wave["e0"][1] - gs["e0"]) <= E_TOL * max(1.0, abs(gs["e0"]))
    assert np.abs(one_wave["G_cl"][1] - cg["G_cl"]).max() <= G_TOL


def test_batch_arguments(pkg, solver, configs):
    insts = _instances(pkg, configs)[:1]
    omega = pkg.matsubara(16, 10.0)
    bad = dict(insts[0], nspin=3)
    with pytest.raises(pkg.EDError) as e:
        solver.solve_batch([bad], 50, omega)
    assert e.value.code == pkg.EDZT_ERR_ARG
    bad = dict(insts[0], sectors=[(99, 1)])
    with pytest.raises(pkg.EDError):
        solver.solve_batch([bad], 50, omega)
    empty = solver.solve_batch([], 50, omega)
    assert len(empty["e0"]) == 0
