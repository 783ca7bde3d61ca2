"""The oracle against golden vectors computed by the reference's own Fortran
source (tests/golden/make_ref_golden.py runs the reference's procedures
through oracle/f90run.py; the fixture records the SHA-256 of every reference
file it read).  This pins the oracle, and through it every GPU parity test,
to the reference:

  basis strings, H.v (both py forms), apply_c    bit-exact
  Lanczos a_n, b_n (first 40-50)                 1e-12 (dot products summed in
                                                 another order than the
                                                 reference's sum(A*B))
  ground-state sector, E0, eigenvector           same sector, 1e-12, |overlap| 1 - 1e-12
  G(i w_n) with z = dcmplx(E0, w_n)              1e-12
The reference itself builds z = cmplx(E0, w_n) without a kind, i.e. in single
precision (src/dmft_green.f90:223,253); its literal G differs from the
double-precision one by about 1e-7, which the last test records."""

import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "ref_golden.npz"))


def _model(O, p):
    norb, nbath = int(p[0]), int(p[1])
    U, Up, Jex, Jp, mu = p[2:7]
    k = 7
    em = p[k:k + 2 * norb].reshape((norb, 2), order="F")
    k += 2 * norb
    ek = p[k:k + 2 * nbath].reshape((nbath, 2), order="F")
    k += 2 * nbath
    vmk = p[k:k + 2 * norb * nbath].reshape((norb, nbath, 2), order="F")
    return O.Oracle(norb, nbath, em, ek, vmk, U, Up, Jex, Jp, mu)


CASES = sorted(k[len("model_"):] for k in GOLD.files if k.startswith("model_"))
LZ = sorted(k[len("lzmodel_"):] for k in GOLD.files if k.startswith("lzmodel_"))


def test_fixture_provenance():
    assert len(GOLD["src_files"]) == len(GOLD["src_sha256"]) >= 10
    assert "impurity_hamiltonian.f90" in list(GOLD["src_files"])
    assert all(len(h) == 64 for h in GOLD["src_sha256"])
    assert len(CASES) >= 5 and len(LZ) >= 2


def test_basis_strings_match_reference(oracle_mod):
    n = 0
    for key in GOLD.files:
        if not key.startswith("basis_"):
            continue
        _, ns, ne = key.split("_")
        got, _ = oracle_mod.spin_basis(int(ns), int(ne))
        assert np.array_equal(np.asarray(got, dtype=np.int64), GOLD[key]), key
        n += 1
    assert n >= 20


@pytest.mark.parametrize("case", CASES)
def test_hx_and_apply_c_match_reference_bit_for_bit(oracle_mod, case):
    o = _model(oracle_mod, GOLD[f"model_{case}"])
    nu, nd = (int(v) for v in GOLD[f"sector_{case}"])
    x = GOLD[f"hx_{case}_x"]
    assert np.array_equal(o.hx(nu, nd, x), GOLD[f"hx_{case}_y"])
    y = GOLD[f"hx_{case}_y0"].copy()
    assert np.array_equal(o.hx(nu, nd, x, y, py=True), GOLD[f"hx_{case}_yacc"])
    for key in GOLD.files:
        if key.startswith(f"applyc_{case}_"):
            pm, iorb, ispin = (int(c) for c in key.rsplit("_", 1)[1])
            assert np.array_equal(o.apply_c(nu, nd, x, pm, iorb, ispin), GOLD[key]), key


@pytest.mark.parametrize("case", LZ)
def test_lanczos_coefficients_match_reference(oracle_mod, case):
    o = _model(oracle_mod, GOLD[f"lzmodel_{case}"])
    nu, nd = (int(v) for v in GOLD[f"lz_{case}_sector"])
    a_ref, b_ref = GOLD[f"lz_{case}_a"], GOLD[f"lz_{case}_b"]
    n_ref = int(GOLD[f"lz_{case}_nstep"][0])
    n, a, b = o.lanczos_iteration(nu, nd, GOLD[f"lz_{case}_v"], len(a_ref))
    assert n == n_ref
    k = min(n, 50)
    assert np.abs(a[:k] - a_ref[:k]).max() <= 1e-12
    assert np.abs(b[:k] - b_ref[:k]).max() <= 1e-12


def test_ground_state_and_green_match_reference(oracle_mod):
    em, ek, V = np.zeros((1, 2)), np.stack([np.linspace(-1.0, 1.0, 5)] * 2, 1), np.full((1, 5, 2), 0.5)
    o = oracle_mod.Oracle(1, 5, em, ek, V, 2.0, 2.0, 0.0, 0.0, 1.0)
    sectors = [tuple(int(v) for v in s) for s in GOLD["gs_sectors"]]
    gs = o.ground_state(sectors, 60, seed=0)
    assert gs["isector"] + 1 == int(GOLD["gs_isector"][0])          # the reference counts from 1
    assert abs(gs["e0"] - GOLD["gs_e0"][0]) <= 1e-12 * max(1.0, abs(gs["e0"]))
    assert abs(abs(gs["vec"] @ GOLD["gs_vec"]) - 1.0) <= 1e-12
    cg = o.cluster_green_ftn(1, *gs["sector"], gs["vec"], gs["e0"], 60, GOLD["G_omega"])
    assert np.abs(cg["G_cl"][0, 0] - GOLD["G_double"]).max() <= 1e-12


def test_reference_single_precision_frequency_argument():
    """The reference's own G(i w_n) carries the single-precision rounding of
    z = cmplx(E0, w_n): about 1e-7 from the double-precision value."""
    d = np.abs(GOLD["G_literal"] - GOLD["G_double"]).max()
    assert 1e-9 < d < 1e-6
