"""Generate tests/golden/edzt_golden.npz: golden vectors for the hot path.

The reference has no tests, fixtures or known-answer vectors, and cannot be
built in this environment (Fortran + MPI + MKL + PARPACK), so these vectors
come from the CPU oracle (oracle/edzt_oracle.c).  Before anything is written
the generator cross-checks the oracle against the two independent pins that
exist:
  - oracle/ref_literal.py, a literal transliteration of the reference's basis,
    hx and apply_c that keeps its integer state representation, 1-based loops
    and evaluation order: basis, H.v and apply_c must agree bit for bit;
  - LAPACK (scipy.linalg.eigh_tridiagonal) for the tridiagonal ground state,
    dense eigh for sector ground energies of the small model.
Run from the repository root:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O          # noqa: E402
from oracle import ref_literal as R     # noqa: E402

OUT = os.path.join(HERE, "edzt_golden.npz")


def load_configs():
    pkg_dir = os.path.join(ROOT, "dmft-ed-zt_b200")
    spec = importlib.util.spec_from_file_location("dmft_ed_zt_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dmft_ed_zt_b200"] = mod
    spec.loader.exec_module(mod)
    import dmft_ed_zt_b200.configs as cfgs
    return mod, cfgs


def oracle_of(m):
    return O.Oracle(m.norb, m.nbath, m.em, m.ek, m.vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)


def kanamori_small(pkg):
    """Two-orbital Hubbard-Kanamori impurity, 2 bath sites per orbital (nsite 6), seed 606."""
    rng = np.random.default_rng(606)
    norb, nbath = 2, 4
    em = rng.uniform(-0.5, 0.5, (norb, 2))
    ek = rng.uniform(-2.0, 2.0, (nbath, 2))
    V = rng.uniform(0.1, 1.0, (norb, nbath, 2))
    U, J = 2.5, 0.625
    return pkg.Model(norb, nbath, em, ek, V, U=U, Up=U - 2 * J, Jex=J, Jp=J, mu=2.1875)


def main():
    pkg, cfgs = load_configs()
    g = {}

    # ---- basis (ed_basis.f90:42-114), bit exact against the literal restatement
    for ns, n in [(6, 3), (10, 4), (12, 6)]:
        s, idx = O.spin_basis(ns, n)
        lit = R.Basis(ns, n, 0).up
        assert s.tolist() == lit, (ns, n)
        g[f"basis_n{ns}_{n}"] = s.astype(np.int64)

    # ---- H.v and apply_c on a two-orbital model with spin-flip and pair-hopping
    km = kanamori_small(pkg)
    o = oracle_of(km)
    md = o.model_dict()
    rng = np.random.default_rng(607)
    B = R.Basis(6, 3, 3)
    x = rng.standard_normal(B.ntot)
    y = o.hx(3, 3, x)
    assert np.array_equal(np.array(R.hx(md, B, list(x))), y)
    g["kan6_params"] = np.concatenate([km.em.ravel(), km.ek.ravel(), km.vmk.ravel(),
                                       [km.U, km.Up, km.Jex, km.Jp, km.mu]])
    g["kan6_x_33"] = x
    g["kan6_hx_33"] = y
    for pm in (1, 2):
        for ispin in (1, 2):
            for iorb in (1, 2):
                d = 1 if pm == 1 else -1
                nu, nd = 3 + (d if ispin == 1 else 0), 3 + (d if ispin == 2 else 0)
                out = o.apply_c(3, 3, x, pm, iorb, ispin)
                lit = np.array(R.apply_c(6, B, list(x), pm, iorb, ispin, R.Basis(6, nu, nd)))
                assert np.array_equal(out, lit)
                g[f"kan6_applyc_{pm}{iorb}{ispin}"] = out
    # sector ground energies against dense diagonalisation
    es = []
    for nu in range(7):
        H = o.dense_h(nu, 6 - nu)
        es.append(np.linalg.eigvalsh(H)[0])
    g["kan6_dense_e_n6"] = np.array(es)

    # ---- tridiagonal lowest eigenpair (dstevx replacement) against LAPACK
    from scipy.linalg import eigh_tridiagonal
    rng = np.random.default_rng(608)
    a = rng.uniform(-2, 2, 60)
    b = np.concatenate([[0.0], rng.uniform(0.1, 1.0, 59)])
    e0, z = O.tridiag_lowest(a, b, 60)
    w, v = eigh_tridiagonal(a, b[1:], select="i", select_range=(0, 0))
    assert abs(e0 - w[0]) < 1e-12 and abs(abs(z @ v[:, 0]) - 1) < 1e-10
    g["tri_a"], g["tri_b"], g["tri_e0"] = a, b, np.array([w[0]])

    # ---- the CPU-runnable workload: ground state and Green's function
    cfg = cfgs.bethe_n6()
    m = cfg["model"]
    o = oracle_of(m)
    gs = o.ground_state(cfg["sectors"], cfg["maxnstep"], seed=7)
    for i, (nu, nd) in enumerate(cfg["sectors"]):
        if o.dim(nu, nd) <= 400:
            ed = np.linalg.eigvalsh(o.dense_h(nu, nd))[0]
            assert abs(ed - gs["e_sector"][i]) < 1e-9 * max(1, abs(ed)), (nu, nd)
    omega = O.matsubara(cfg["nw"], cfg["beta"])
    nu, nd = gs["sector"]
    cg = o.cluster_green_ftn(1, nu, nd, gs["vec"], gs["e0"], cfg["maxnstep"], omega)
    v0 = O.start_vector(7, gs["isector"], o.dim(nu, nd))
    n, aa, bb = o.lanczos_iteration(nu, nd, v0, cfg["maxnstep"])
    g["bethe_e_sector"] = np.asarray(gs["e_sector"])
    g["bethe_e0"] = np.array([gs["e0"]])
    g["bethe_isector"] = np.array([gs["isector"]])
    g["bethe_gs_a20"] = aa[:20]
    g["bethe_gs_b20"] = bb[:20]
    g["bethe_G64"] = np.asarray(cg["G_cl"])[0, 0, :64]
    g["bethe_coeffs10"] = np.asarray(cg["coeffs"])[0, 0, :, :10]

    # ---- the two-orbital workload's ground state
    cfg = cfgs.kanamori_n10()
    o = oracle_of(cfg["model"])
    gs = o.ground_state(cfg["sectors"], cfg["maxnstep"], seed=1)
    g["kan10_e_sector"] = np.asarray(gs["e_sector"])
    g["kan10_e0"] = np.array([gs["e0"]])
    g["kan10_isector"] = np.array([gs["isector"]])

    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes,", len(g), "arrays")


if __name__ == "__main__":
    main()
