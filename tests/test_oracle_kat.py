"""Independent known-answer tests that pin the CPU oracle (no GPU).

The reference has no tests and cannot be run here, so the restatement is
pinned to mathematics instead: dense diagonalisation, the U = 0 free-fermion
limit, the atomic limit, sum rules, particle-hole and spin symmetry,
Hermiticity, an ARPACK cross-check and LAPACK's tridiagonal solver.
Tolerances: energies 1e-10 relative, Green's functions 1e-8 absolute.
"""

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse.linalg as spla

from conftest import oracle_for, random_model

E_TOL = 1e-10
G_TOL = 1e-8


def test_dense_h_symmetric_and_lanczos_e0(pkg, oracle_mod):
    rng = np.random.default_rng(11)
    for norb, nbath, J in [(1, 5, 0.0), (2, 4, 0.625), (3, 3, 0.3)]:
        m = random_model(pkg, rng, norb, nbath, J=J, spin_dep=True)
        o = oracle_for(oracle_mod, m)
        ns = norb + nbath
        for nu, nd in [(ns // 2, ns // 2), (ns // 2 + 1, ns // 2 - 1), (1, 2)]:
            H = o.dense_h(nu, nd)
            assert np.abs(H - H.T).max() <= 1e-14 * max(1.0, np.abs(H).max())
            ev = np.linalg.eigvalsh(H)
            r = o.diag_lanczos(nu, nd, 200, seed=3)
            assert abs(r["e0"] - ev[0]) <= E_TOL * max(1.0, abs(ev[0]))
            assert r["residual"] < 1e-12
            w, V = np.linalg.eigh(H)
            if w[1] - w[0] > 1e-6:
                assert abs(abs(V[:, 0] @ r["vec"]) - 1.0) < 1e-9


def test_hermiticity(pkg, oracle_mod):
    rng = np.random.default_rng(5)
    m = random_model(pkg, rng, 2, 6, J=0.5, spin_dep=True, zero_frac=0.3)
    o = oracle_for(oracle_mod, m)
    for nu, nd in [(4, 4), (3, 5)]:
        n = o.dim(nu, nd)
        u, v = rng.standard_normal(n), rng.standard_normal(n)
        lhs, rhs = u @ o.hx(nu, nd, v), o.hx(nu, nd, u) @ v
        assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + 1.0)


def _one_body(m, sigma):
    ns = m.norb + m.nbath
    h = np.zeros((ns, ns))
    for a in range(m.norb):
        h[a, a] = m.em[a, sigma] - m.mu
    for l in range(m.nbath):
        h[m.norb + l, m.norb + l] = m.ek[l, sigma]
        for a in range(m.norb):
            h[a, m.norb + l] = h[m.norb + l, a] = m.vmk[a, l, sigma]
    return h


def test_free_fermion_limit(pkg, oracle_mod):
    """U = J = 0: E0(n_up, n_dn) = sum of the lowest one-body levels; G = [(iw - h)^-1]_00."""
    rng = np.random.default_rng(8)
    nb = 6
    em = rng.uniform(-0.3, 0.3, (1, 2))
    ek = rng.uniform(-2, 2, (nb, 2))
    V = rng.uniform(0.2, 1.0, (1, nb, 2))
    m = pkg.Model(1, nb, em, ek, V, U=0.0, Up=0.0, Jex=0.0, Jp=0.0, mu=0.1)
    o = oracle_for(oracle_mod, m)
    e_up = np.linalg.eigvalsh(_one_body(m, 0))
    e_dn = np.linalg.eigvalsh(_one_body(m, 1))
    for nu, nd in [(3, 4), (4, 4), (2, 5), (0, 3)]:
        exact = e_up[:nu].sum() + e_dn[:nd].sum()
        r = oracle_mod.Oracle.diag_lanczos(o, nu, nd, 200, seed=1, want_vec=False)
        assert abs(r["e0"] - exact) <= E_TOL * max(1.0, abs(exact))
    # Green's function of the ground-state sector vs the one-body resolvent
    sectors = [(u, d) for u in range(nb + 2) for d in range(nb + 2)]
    gs = o.ground_state(sectors, 200, seed=2)
    nu, nd = gs["sector"]
    assert abs(gs["e0"] - min(e_up[:u].sum() + e_dn[:d].sum() for u, d in sectors)) < 1e-9
    omega = oracle_mod.matsubara(32, 50.0)
    for ispin, e_s in ((1, e_up), (2, e_dn)):
        h = _one_body(m, ispin - 1)
        g = o.green_diag(nu, nd, gs["vec"], gs["e0"], 1, ispin, 200, omega)["g"]
        # non-degenerate Fermi sea: exact resolvent
        nocc = nu if ispin == 1 else nd
        if 0 < nocc < h.shape[0] and e_s[nocc] - e_s[nocc - 1] > 1e-3:
            exact = np.array([np.linalg.inv(1j * w * np.eye(h.shape[0]) - h)[0, 0] for w in omega])
            assert np.abs(g - exact).max() < G_TOL


def test_atomic_limit(pkg, oracle_mod):
    """nsite = 1 (no bath) at half filling: G = 1/2 [1/(iw+U/2) + 1/(iw-U/2)]."""
    U = 2.0
    m = pkg.Model(1, 0, np.zeros((1, 2)), np.zeros((0, 2)), np.zeros((1, 0, 2)), U=U, Up=U, Jex=0.0, Jp=0.0,
                  mu=U / 2)
    o = oracle_for(oracle_mod, m)
    sectors = [(0, 0), (1, 0), (0, 1), (1, 1)]
    gs = o.ground_state(sectors, 50, seed=0)
    assert gs["sector"] == (1, 0) and abs(gs["e0"] + U / 2) < 1e-15
    omega = oracle_mod.matsubara(16, 10.0)
    nu, nd = gs["sector"]
    res = o.cluster_green_ftn(1, nu, nd, gs["vec"], gs["e0"], 50, omega)
    exact = 0.5 * (1 / (1j * omega + U / 2) + 1 / (1j * omega - U / 2))
    assert np.abs(res["G_cl"][0, 0] - exact).max() < 1e-14


def test_sum_rules_and_occupation(configs, oracle_mod):
    cfg = configs.bethe_n6()
    m = cfg["model"]
    o = oracle_for(oracle_mod, m)
    gs = o.ground_state(cfg["sectors"], 100, seed=4)
    nu, nd = gs["sector"]
    up, dn = o.basis(nu, nd)
    vec = gs["vec"].reshape(len(dn), len(up))
    n_up = float(((up & 1)[None, :] * vec ** 2).sum())
    n_dn = float(((dn & 1)[:, None] * vec ** 2).sum())
    omega = oracle_mod.matsubara(8, 100.0)
    for ispin, n_s in ((1, n_up), (2, n_dn)):
        r = o.green_diag(nu, nd, gs["vec"], gs["e0"], 1, ispin, 100, omega)
        bp1, bm1 = r["bp"][0], r["bm"][0]
        assert abs(bp1 ** 2 + bm1 ** 2 - 1.0) < 1e-12
        assert abs(bp1 ** 2 - (1 - n_s)) < 1e-12 and abs(bm1 ** 2 - n_s) < 1e-12


def test_particle_hole_and_spin_symmetry(pkg, oracle_mod):
    nb = 5
    ek = np.array([-1.3, -0.4, 0.0, 0.4, 1.3])
    V = np.array([0.6, 0.3, 0.5, 0.3, 0.6])
    U = 2.0
    m = pkg.Model(1, nb, np.zeros((1, 2)), np.stack([ek, ek], 1), np.stack([V, V], 1).reshape(1, nb, 2),
                  U=U, Up=U, Jex=0.0, Jp=0.0, mu=U / 2)
    o = oracle_for(oracle_mod, m)
    ns = nb + 1
    E = {}
    for u in range(ns + 1):
        for d in range(ns + 1):
            E[(u, d)] = o.diag_lanczos(u, d, 150, seed=1, want_vec=False)["e0"]
    for (u, d), e in E.items():
        assert abs(e - E[(d, u)]) < 1e-10 * max(1, abs(e))                 # spin
        assert abs(e - E[(ns - u, ns - d)]) < 1e-10 * max(1, abs(e))       # particle-hole
    gs = o.ground_state([(3, 3)], 150, seed=1)
    omega = oracle_mod.matsubara(32, 100.0)
    g = o.green_diag(3, 3, gs["vec"], gs["e0"], 1, 1, 150, omega)["g"]
    assert np.abs(g.real).max() < 1e-9


def test_arpack_cross_check(pkg, oracle_mod):
    """DiagSolver = 2 semantics: eigsh(which='SA') on the same H.v."""
    rng = np.random.default_rng(21)
    m = random_model(pkg, rng, 1, 9, spin_dep=False)
    o = oracle_for(oracle_mod, m)
    nu = nd = 5
    n = o.dim(nu, nd)
    op = spla.LinearOperator((n, n), matvec=lambda x: o.hx(nu, nd, np.ascontiguousarray(x.ravel())),
                             dtype=np.float64)
    w = spla.eigsh(op, k=1, which="SA", tol=1e-13, v0=np.ones(n))[0]
    r = o.diag_lanczos(nu, nd, 200, seed=9, want_vec=False)
    assert abs(r["e0"] - w[0]) <= E_TOL * abs(w[0])


def test_tridiag_vs_lapack(oracle_mod):
    rng = np.random.default_rng(2)
    for n in (1, 2, 3, 17, 120, 300):
        a = rng.uniform(-3, 3, n)
        b = np.concatenate([[0.0], rng.uniform(0.1, 2, n - 1)])
        e0, z = oracle_mod.tridiag_lowest(a, b, n)
        w, V = sla.eigh_tridiagonal(a, b[1:]) if n > 1 else (a.copy(), np.ones((1, 1)))
        assert abs(e0 - w[0]) <= 4e-15 * max(1.0, np.abs(w).max())
        if n > 1 and w[1] - w[0] > 1e-8:
            assert abs(abs(V[:, 0] @ z) - 1.0) < 1e-12


def test_continued_fraction_matches_resolvent(pkg, oracle_mod):
    rng = np.random.default_rng(4)
    m = random_model(pkg, rng, 1, 5, spin_dep=True)
    o = oracle_for(oracle_mod, m)
    gs = o.ground_state([(3, 3), (3, 2), (2, 3)], 120, seed=6)
    nu, nd = gs["sector"]
    omega = oracle_mod.matsubara(16, 20.0)
    r = o.green_diag(nu, nd, gs["vec"], gs["e0"], 1, 1, 120, omega)
    Hp, Hm = o.dense_h(nu + 1, nd), o.dense_h(nu - 1, nd)
    vp = o.apply_c(nu, nd, gs["vec"], 1, 1, 1)
    vm = o.apply_c(nu, nd, gs["vec"], 2, 1, 1)
    E0 = gs["e0"]
    exact = []
    for w in omega:
        gp = vp @ np.linalg.solve((1j * w + E0) * np.eye(len(vp)) - Hp, vp)
        gm = vm @ np.linalg.solve((1j * w - E0) * np.eye(len(vm)) + Hm, vm)
        exact.append(gp + gm)
    assert np.abs(r["g"] - np.array(exact)).max() < G_TOL


def test_edge_cases(pkg, oracle_mod):
    rng = np.random.default_rng(0)
    m = random_model(pkg, rng, 1, 3)
    o = oracle_for(oracle_mod, m)
    ns = 4
    # vacuum (dim 1): breakdown at the second step, E = 0
    r = o.diag_lanczos(0, 0, 10, seed=0)
    assert r["nstep"] == 1 and r["e0"] == 0.0
    # full sector (dim 1)
    r = o.diag_lanczos(ns, ns, 10, seed=0)
    assert r["nstep"] == 1
    # excitation into an empty sector contributes nothing; zero vector too
    gs = o.ground_state([(ns, ns)], 10)
    g = o.green_diag(ns, ns, gs["vec"], gs["e0"], 1, 1, 10, oracle_mod.matsubara(4, 10.0))
    assert g["nstep"][0] == 0 and np.all(np.isfinite(g["g"]))
    # start vector: U[0,1), reproducible, distinct streams
    v1 = oracle_mod.start_vector(5, 0, 1000)
    assert np.all((v1 >= 0) & (v1 < 1)) and np.array_equal(v1, oracle_mod.start_vector(5, 0, 1000))
    assert not np.array_equal(v1, oracle_mod.start_vector(5, 1, 1000))


def test_arpack_oracle_matches_dense(pkg, oracle_mod):
    """The oracle's ARPACK path (scipy's eigsh = ARPACK dsaupd/dseupd) against
    dense diagonalisation: lowest three eigenvalues and the ground state."""
    m = random_model(pkg, np.random.default_rng(31), 2, 3, J=0.4)
    o = oracle_for(oracle_mod, m)
    r = o.diag_arpack(2, 3, seed=1, stream=0)
    w, v = np.linalg.eigh(o.dense_h(2, 3))
    assert np.abs(r["ritz"] - w[:3]).max() <= 1e-12 * max(1.0, abs(w[0]))
    assert abs(abs(r["vec"] @ v[:, 0]) - 1.0) <= 1e-12
    assert r["resid"].max() <= 1e-12
    gs = o.ground_state_arpack([(2, 3), (3, 3), (3, 2)], seed=1)
    es = [np.linalg.eigvalsh(o.dense_h(u, d))[0] for u, d in [(2, 3), (3, 3), (3, 2)]]
    assert np.abs(gs["e_sector"] - es).max() <= 1e-12 * max(1.0, abs(min(es)))
    assert abs(gs["e0"] - min(es)) <= 1e-12 * max(1.0, abs(min(es)))
