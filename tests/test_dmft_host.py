"""The host DMFT loop (dmft.py) on CPU: the Bethe local Green's function, the
bath-fit cost gradient, the conjugate-gradient minimiser and a short loop on
the oracle solver."""

import importlib

import numpy as np
import pytest


def _dmft(pkg):
    return importlib.import_module("dmft_ed_zt_b200.dmft")


def oracle_solver(oracle_mod, m, sectors, maxnstep, omega, nspin=1, seed=0):
    def solve(em, ek, vmk):
        o = oracle_mod.Oracle(m.norb, m.nbath, em, ek, vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)
        gs = o.ground_state(sectors, maxnstep, seed=seed)
        return o.cluster_green_ftn(nspin, *gs["sector"], gs["vec"], gs["e0"], maxnstep, omega)["G_cl"]
    return solve


def test_local_green_semicircle(pkg, oracle_mod):
    """With i w + mu - Sigma = i w the quadrature gives the semicircle's
    Hilbert transform -2i (sqrt(w^2 + 1) - w)."""
    d = _dmft(pkg)
    w = oracle_mod.matsubara(64, 20.0)
    G_cl = (1.0 / (1j * w))[None, None, :]
    G = d.local_green(np.zeros((1, 2)), np.zeros_like(G_cl), G_cl)
    exact = -2j * (np.sqrt(w * w + 1.0) - w)
    assert np.abs(G[0, 0] - exact).max() < 2e-4


def test_bath_fit_gradient_and_minimiser(pkg, oracle_mod):
    d = _dmft(pkg)
    rng = np.random.default_rng(4)
    w = oracle_mod.matsubara(128, 50.0)
    em, ek, V = rng.uniform(-.5, .5, (1, 2)), rng.uniform(-1, 1, (4, 2)), rng.uniform(.2, .8, (1, 4, 2))
    D = d.hybridization(ek, V, w, 1)
    G_cl = 1.0 / (1j * w - 0.3 - D[0, 0] + 0.2 / (1j * w))[None, None, :]
    G_loc = 0.9 * G_cl
    bf = d.BathFit(em, D, G_cl, G_loc, w, 0)
    x = np.concatenate([em[:, 0], ek[:, 0], V[:, :, 0].T.ravel()]) + rng.normal(0, .05, 9)
    g = bf.df(x)
    h = 1e-6
    num = np.array([(bf.f(x + h * e) - bf.f(x - h * e)) / (2 * h) for e in np.eye(9)])
    assert np.abs(g - num).max() <= 1e-6 * max(1.0, np.abs(num).max())
    xm, it, fret = d.conjugate_gradient(bf.f, bf.df, x)
    assert fret <= bf.f(x) and np.abs(bf.df(xm)).max() < 1e-3
    rosen = lambda p: (1 - p[0]) ** 2 + 100 * (p[1] - p[0] ** 2) ** 2
    drosen = lambda p: np.array([-2 * (1 - p[0]) - 400 * p[0] * (p[1] - p[0] ** 2), 200 * (p[1] - p[0] ** 2)])
    p, it, f = d.conjugate_gradient(rosen, drosen, np.array([-1.2, 1.0]), ftol=1e-12)
    assert np.abs(p - 1.0).max() < 1e-3


def test_short_loop_on_the_oracle(pkg, configs, oracle_mod, tmp_path):
    d = _dmft(pkg)
    cfg = configs.bethe_n6()
    m = cfg["model"]
    w = oracle_mod.matsubara(128, cfg["beta"])
    solve = oracle_solver(oracle_mod, m, cfg["sectors"], 40, w)
    res = d.dmft_loop(solve, m.em, m.ek, m.vmk, w, m.nbath, nspin=1, nloop=3, scf_tol=0.0, mixing=0.5,
                      writer=lambda it, em, ek, vmk, D, Gc, Gl: d.write_green(str(tmp_path), w, D, Gc, Gl))
    assert res.iterations == 3 and len(res.history) == 3 and np.all(np.isfinite(res.history))
    assert np.allclose(res.ek[:, 0], res.ek[:, 1]) and np.allclose(res.vmk[..., 0], res.vmk[..., 1])
    rows = open(tmp_path / "green.dat.1.1").read().split("\n")
    assert rows[0].split() == ["128", "1", "1"] and len(rows[1]) == 7 * 12
    d.write_h_imp(str(tmp_path / "h_imp.dat"), res.em, res.ek, res.vmk, 1)
    vals = open(tmp_path / "h_imp.dat").read().split()
    assert vals[:3] == ["1", "5", "1"] and len(vals) == 3 + 1 + 5 + 5
    S = d.self_energy(res.em, res.D_cl, res.G_cl, w, m.mu)
    Z = d.quasiparticle_weight(S, w)
    assert np.all(S[0, 0].imag < 0) and 0.0 < Z[0, 0] < 1.0        # U = 2: a correlated metal
    d.write_sigma(str(tmp_path), w, S)
    assert open(tmp_path / "sigma.dat.1.1").read().split("\n")[0].split() == ["128", "1", "1"]


def test_self_energy_vanishes_without_interaction(pkg, oracle_mod):
    d = _dmft(pkg)
    rng = np.random.default_rng(6)
    w = oracle_mod.matsubara(64, 30.0)
    em, ek, V = rng.uniform(-.5, .5, (2, 2)), rng.uniform(-1, 1, (3, 2)), rng.uniform(.2, .8, (2, 3, 2))
    mu = 0.7
    D = d.hybridization(ek, V, w, 2)
    G0 = np.array([[1.0 / (1j * w + mu - em[a, s] - D[s, a]) for a in range(2)] for s in range(2)])
    S = d.self_energy(em, D, G0, w, mu)
    assert np.abs(S).max() < 1e-12
    assert np.allclose(d.quasiparticle_weight(S, w), 1.0)
    G0[0, 0] *= 0.5
    S = d.self_energy(em, D, G0, w, mu)
    assert np.allclose(d.quasiparticle_weight(S, w, literal=True), 1.0)        # only (iorb 2, ispin 2) is kept
    assert d.quasiparticle_weight(S, w)[0, 0] != 1.0


def test_library_host_loop_pieces_match_restatement(pkg, oracle_mod):
    """The library's C++ DMFT pieces (hybridization, Bethe G_loc, bath fit;
    no device needed) against this module's Python restatement of them."""
    d = _dmft(pkg)
    pkg.build()
    rng = np.random.default_rng(8)
    w = oracle_mod.matsubara(256, 40.0)
    for norb, nbath, nspin in [(1, 5, 1), (2, 3, 2)]:
        em = rng.uniform(-.5, .5, (norb, 2))
        ek = rng.uniform(-1, 1, (nbath, 2))
        V = rng.uniform(.2, .8, (norb, nbath, 2))
        if nspin == 1:
            em[:, 1], ek[:, 1], V[..., 1] = em[:, 0], ek[:, 0], V[..., 0]
        D = d.hybridization(ek, V, w, nspin)
        assert np.abs(pkg.hybridization(ek, V, w, nspin) - D).max() <= 1e-14
        G_cl = 1.0 / (1j * w[None, None, :] - 0.2 - D + 0.3 / (1j * w[None, None, :] + 0.4))
        G_loc = d.local_green(em, D, G_cl, 0.05)
        assert np.abs(pkg.local_green_bethe(em, D, G_cl, 0.05) - G_loc).max() <= 1e-12
        # a fit whose minimum is flat (couplings go to zero): the same cost
        em0, ek0, V0 = em + 0.03, ek * 1.05, V * 0.95
        emp, ekp, Vp, info = d.fit_bath(em0, ek0, V0, D, G_cl, G_loc, w, nspin, ftol=1e-13)
        emc, ekc, Vc, cost = pkg.fit_bath(em0, ek0, V0, D, G_cl, G_loc, w, nspin, ftol=1e-13)
        for s in range(nspin):
            assert abs(cost[s] - info[s][1]) <= 1e-10 * info[s][1] + 1e-16
        # with G_loc = G_cl the target is em0 + D(ek, V), which a bath of this
        # size represents exactly: both fits return em0 and a bath giving D
        # (the cost goes to zero, where the relative stop needs a looser ftol)
        emc, ekc, Vc, cost = pkg.fit_bath(em0, ek0, V0, D, G_cl, G_cl, w, nspin, ftol=1e-9)
        emp, ekp, Vp, info = d.fit_bath(em0, ek0, V0, D, G_cl, G_cl, w, nspin, ftol=1e-9)
        assert cost.max() < 1e-12
        for got in ((emc, ekc, Vc), (emp, ekp, Vp)):
            assert np.abs(got[0] - em0).max() <= 1e-6
            assert np.abs(d.hybridization(got[1], got[2], w, nspin) - D).max() <= 1e-5
    with pytest.raises(pkg.EDError):
        pkg.fit_bath(em, ek, V, D, G_cl, G_loc, w, nspin, ftol=0.0)


def _dmft_golden():
    import importlib.util
    import os
    from conftest import ROOT
    path = os.path.join(ROOT, "tests", "golden", "make_dmft_golden.py")
    spec = importlib.util.spec_from_file_location("make_dmft_golden", path)
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    return gen, np.load(gen.OUT)


def test_dmft_loop_reproduces_golden(pkg):
    """The Python DMFT loop on the oracle reproduces the committed record of
    a short run (tests/golden/make_dmft_golden.py) within the DMFT bound."""
    gen, gold = _dmft_golden()
    _, r = gen.run_oracle_loop()
    for key in ("D_cl", "G_cl", "G_loc", "em", "ek"):
        assert np.abs(getattr(r, key) - gold[key]).max() <= 1e-6, key
    assert np.allclose(r.history, gold["history"], rtol=1e-4, atol=0)


def test_bath_sign_alignment(pkg):
    """Before mixing, each fitted bath site keeps the overall sign of its
    previous couplings: the fit's cost is blind to it (only V_a V_b of a site
    enter), and mixing columns of opposite sign would shrink the bath."""
    d = _dmft(pkg)
    old = np.array([[[0.5, 0.5], [0.3, 0.3], [-0.2, -0.2]],
                    [[0.1, 0.1], [-0.4, -0.4], [0.6, 0.6]]])          # (norb 2, nbath 3, spin 2)
    new = old * np.array([-1.0, 1.0, -1.0])[None, :, None] * 1.1
    got = d.align_bath_signs(new, old)
    assert np.allclose(got, old * 1.1)
    assert np.array_equal(d.align_bath_signs(old, old), old)
