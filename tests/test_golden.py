"""Golden vectors (tests/golden/edzt_golden.npz, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces every golden vector (it is the checker of
all other parity tests, so it must not drift).  GPU: the library reproduces
them through the C ABI within the parity tolerances: basis bit-exact, H.v
and apply_c to 1e-13 of the vector scale, energies 1e-10 relative, the first
12 Lanczos and 10 continued-fraction coefficients 1e-8, G(i w) 1e-8.
"""

import os

import numpy as np
import pytest

from conftest import ROOT, oracle_for

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "edzt_golden.npz"))


def kanamori_small(pkg):
    p = GOLD["kan6_params"]
    norb, nbath = 2, 4
    em = p[:4].reshape(norb, 2)
    ek = p[4:12].reshape(nbath, 2)
    vmk = p[12:28].reshape(norb, nbath, 2)
    U, Up, J, Jp, mu = p[28:33]
    return pkg.Model(norb, nbath, em, ek, vmk, U=U, Up=Up, Jex=J, Jp=Jp, mu=mu)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(1.0, np.abs(b).max())


def test_golden_file_is_complete():
    for k in ["basis_n6_3", "basis_n12_6", "kan6_hx_33", "kan6_applyc_111", "kan6_applyc_222", "tri_e0",
              "bethe_e_sector", "bethe_G64", "bethe_coeffs10", "kan10_e0"]:
        assert k in GOLD.files, k


def test_oracle_reproduces_golden(pkg, configs, oracle_mod):
    for ns, n in [(6, 3), (10, 4), (12, 6)]:
        s, _ = oracle_mod.spin_basis(ns, n)
        assert np.array_equal(s, GOLD[f"basis_n{ns}_{n}"])
    o = oracle_for(oracle_mod, kanamori_small(pkg))
    x = GOLD["kan6_x_33"]
    assert np.array_equal(o.hx(3, 3, x), GOLD["kan6_hx_33"])
    for pm in (1, 2):
        for ispin in (1, 2):
            for iorb in (1, 2):
                assert np.array_equal(o.apply_c(3, 3, x, pm, iorb, ispin), GOLD[f"kan6_applyc_{pm}{iorb}{ispin}"])
    e0, _ = oracle_mod.tridiag_lowest(GOLD["tri_a"], GOLD["tri_b"], 60)
    assert abs(e0 - GOLD["tri_e0"][0]) < 1e-12
    cfg = configs.bethe_n6()
    o = oracle_for(oracle_mod, cfg["model"])
    gs = o.ground_state(cfg["sectors"], cfg["maxnstep"], seed=7)
    assert gs["isector"] == GOLD["bethe_isector"][0]
    assert np.abs(gs["e_sector"] - GOLD["bethe_e_sector"]).max() < 1e-12
    omega = oracle_mod.matsubara(cfg["nw"], cfg["beta"])
    cg = o.cluster_green_ftn(1, *gs["sector"], gs["vec"], gs["e0"], cfg["maxnstep"], omega)
    assert np.abs(cg["G_cl"][0, 0, :64] - GOLD["bethe_G64"]).max() < 1e-12
    assert np.abs(cg["coeffs"][0, 0, :, :10] - GOLD["bethe_coeffs10"]).max() < 1e-12


@pytest.mark.gpu
def test_gpu_reproduces_golden(pkg, solver, configs, oracle_mod):
    for ns, n in [(6, 3), (10, 4), (12, 6)]:
        nb = ns - 1
        m = pkg.Model(1, nb, np.zeros((1, 2)), np.zeros((nb, 2)), np.full((1, nb, 2), 0.5), U=1.0)
        solver.set_model(m)
        up, dn = solver.generate_basis(n, n)
        assert np.array_equal(np.asarray(up, dtype=np.int64), GOLD[f"basis_n{ns}_{n}"])
    solver.set_model(kanamori_small(pkg))
    x = GOLD["kan6_x_33"]
    y = solver.hx(3, 3, x)
    assert _rel(y, GOLD["kan6_hx_33"]) <= 1e-13
    for pm in (1, 2):
        for ispin in (1, 2):
            for iorb in (1, 2):
                out = solver.apply_c(3, 3, x, pm, iorb, ispin)
                assert np.array_equal(out, GOLD[f"kan6_applyc_{pm}{iorb}{ispin}"])
    cfg = configs.bethe_n6()
    solver.set_model(cfg["model"])
    gs = solver.ground_state(cfg["sectors"], cfg["maxnstep"], seed=7)
    assert gs["isector"] == GOLD["bethe_isector"][0]
    ref = GOLD["bethe_e_sector"]
    assert np.all(np.abs(gs["e_sector"] - ref) <= 1e-10 * np.maximum(1.0, np.abs(ref)))
    nu, nd = gs["sector"]
    v0 = oracle_mod.start_vector(7, gs["isector"], solver.dim(nu, nd))     # the input only
    n, a, b = solver.lanczos_iteration(nu, nd, v0, cfg["maxnstep"])
    assert np.abs(a[:12] - GOLD["bethe_gs_a20"][:12]).max() <= 1e-8
    assert np.abs(b[:12] - GOLD["bethe_gs_b20"][:12]).max() <= 1e-8
    omega = pkg.matsubara(cfg["nw"], cfg["beta"])
    cg = solver.cluster_green_ftn(1, cfg["maxnstep"], omega)
    assert np.abs(cg["G_cl"][0, 0, :64] - GOLD["bethe_G64"]).max() <= 1e-8
    assert np.abs(cg["coeffs"][0, 0, :, :10] - GOLD["bethe_coeffs10"]).max() <= 1e-8
    cfg = configs.kanamori_n10()
    solver.set_model(cfg["model"])
    gs = solver.ground_state(cfg["sectors"], cfg["maxnstep"], seed=1)
    assert gs["isector"] == GOLD["kan10_isector"][0]
    assert abs(gs["e0"] - GOLD["kan10_e0"][0]) <= 1e-10 * max(1.0, abs(GOLD["kan10_e0"][0]))

