"""GPU parity of the ARPACK path (diag_arpack, src/arpack_solver.f90:19-124,
and ground_state with diag_solver = 2) against ARPACK itself: the oracle runs
scipy's eigsh (ARPACK dsaupd/dseupd) with the reference's settings on the
oracle's hx.  Both converge to machine precision, so the bounds are the
solve tolerances: E0 and the three Ritz values 1e-10 relative, the
eigenvector to 1e-10 in |<x_gpu|x_arpack>| (its sign is arbitrary in both),
G(i w) from the ARPACK ground state 1e-8."""

import numpy as np
import pytest

from conftest import oracle_for, random_model

pytestmark = pytest.mark.gpu
E_TOL = 1e-10
G_TOL = 1e-8


@pytest.fixture
def arpack_solver(solver, pkg):
    solver.set_diag_solver(pkg.DIAG_ARPACK)
    yield solver
    solver.set_diag_solver(pkg.DIAG_LANCZOS)


@pytest.mark.parametrize("norb,nbath,sec,seed", [(1, 7, (4, 4), 11), (1, 9, (5, 4), 12), (2, 6, (4, 4), 13),
                                                 (1, 5, (1, 2), 14)])
def test_diag_arpack_matches_arpack(pkg, solver, oracle_mod, norb, nbath, sec, seed):
    rng = np.random.default_rng(seed)
    m = random_model(pkg, rng, norb, nbath, J=0.3 if norb == 2 else 0.0)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    ref = o.diag_arpack(*sec, seed=7, stream=2)
    got = solver.diag_arpack(*sec, seed=7, stream=2)
    scale = max(1.0, abs(ref["e0"]))
    assert abs(got["e0"] - ref["e0"]) <= E_TOL * scale
    assert np.abs(got["ritz"] - ref["ritz"]).max() <= E_TOL * scale
    assert abs(abs(got["vec"] @ ref["vec"]) - 1.0) <= 1e-10
    assert abs(np.linalg.norm(got["vec"]) - 1.0) <= 1e-12
    assert got["resid"].max() <= 1e-10 * scale and got["nmult"] > 0


def test_ground_state_arpack_and_green(pkg, arpack_solver, configs, oracle_mod):
    rng = np.random.default_rng(21)
    m = random_model(pkg, rng, 1, 7)
    arpack_solver.set_model(m)
    sectors = [(u, d) for u in (3, 4, 5) for d in (3, 4, 5)]
    o = oracle_for(oracle_mod, m)
    ref = o.ground_state_arpack(sectors, seed=3)
    got = arpack_solver.ground_state(sectors, 100, seed=3)
    assert got["isector"] == ref["isector"]
    assert abs(got["e0"] - ref["e0"]) <= E_TOL * max(1.0, abs(ref["e0"]))
    assert np.nanmax(np.abs(got["e_sector"] - ref["e_sector"])) <= E_TOL * max(1.0, abs(ref["e0"]))
    assert abs(abs(got["vec"] @ ref["vec"]) - 1.0) <= 1e-10
    omega = pkg.matsubara(256, 50.0)
    g = arpack_solver.cluster_green_ftn(1, 150, omega)
    cg = o.cluster_green_ftn(1, *ref["sector"], ref["vec"], ref["e0"], 150, omega)
    assert np.abs(g["G_cl"] - cg["G_cl"]).max() <= G_TOL
    lz = o.ground_state(sectors, 150, seed=3)                  # the Lanczos path finds the same state
    assert lz["isector"] == got["isector"] and abs(lz["e0"] - got["e0"]) <= E_TOL * max(1.0, abs(lz["e0"]))


def test_solve_with_arpack(pkg, arpack_solver, oracle_mod):
    rng = np.random.default_rng(22)
    m = random_model(pkg, rng, 1, 6)
    arpack_solver.set_model(m)
    sectors = [(3, 4), (4, 3), (4, 4), (3, 3)]
    omega = pkg.matsubara(128, 40.0)
    got = arpack_solver.solve(sectors, 120, omega, nspin=1, seed=9)
    o = oracle_for(oracle_mod, m)
    ref = o.ground_state_arpack(sectors, seed=9)
    cg = o.cluster_green_ftn(1, *ref["sector"], ref["vec"], ref["e0"], 120, omega)
    assert got["isector"] == ref["isector"]
    assert abs(got["e0"] - ref["e0"]) <= E_TOL * max(1.0, abs(ref["e0"]))
    assert np.abs(got["G_cl"] - cg["G_cl"]).max() <= G_TOL


def test_arpack_arguments(pkg, solver, oracle_mod):
    rng = np.random.default_rng(23)
    m = random_model(pkg, rng, 1, 5)                              # nsite 6
    solver.set_model(m)
    with pytest.raises(pkg.EDError) as e:
        solver.set_diag_solver(3)                                 # "invalid diag solver"
    assert e.value.code == pkg.EDZT_ERR_ARG
    assert solver.dim(6, 1) == 6 and solver.dim(6, 0) == 1
    with pytest.raises(pkg.EDError) as e:
        solver.diag_arpack(6, 0)                                  # dimension 1 < ncv = 6
    assert e.value.code == pkg.EDZT_ERR_ARG
    r = solver.diag_arpack(6, 1)                                  # dimension 6 = ncv: the space is exhausted
    H = oracle_for(oracle_mod, m).dense_h(6, 1)
    assert abs(r["e0"] - np.linalg.eigvalsh(H)[0]) <= E_TOL * max(1.0, abs(r["e0"]))
    solver.set_diag_solver(pkg.DIAG_ARPACK)
    try:                                                          # diag_lanczos stays Lanczos
        got = solver.diag_lanczos(3, 3, 80, seed=4)
        ref = oracle_for(oracle_mod, m).diag_lanczos(3, 3, 80, seed=4)
        assert abs(got["e0"] - ref["e0"]) <= E_TOL * max(1.0, abs(ref["e0"]))
        assert np.abs(got["vec"] - ref["vec"]).max() <= 1e-8
    finally:
        solver.set_diag_solver(pkg.DIAG_LANCZOS)
