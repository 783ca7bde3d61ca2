"""GPU parity against golden vectors computed by the reference's own Fortran
source (tests/golden/make_ref_golden.py; see tests/test_ref_golden.py for how
the oracle matches them bit for bit).  Through the C ABI:

  apply_c                                   bit-exact
  H.v, y = H x and y = y0 + H x             1e-13 of the vector scale
  first Lanczos a_n, b_n (up to 50)         1e-8
  ground-state sector, E0                   same sector, 1e-10 relative
  G(i w_n) (z = dcmplx(E0, w_n))            1e-8
"""

import os

import numpy as np
import pytest

from conftest import ROOT, ab_compare_len

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "ref_golden.npz"))
CASES = sorted(k[len("model_"):] for k in GOLD.files if k.startswith("model_"))
LZ = sorted(k[len("lzmodel_"):] for k in GOLD.files if k.startswith("lzmodel_"))


def _model(pkg, p):
    norb, nbath = int(p[0]), int(p[1])
    U, Up, Jex, Jp, mu = (float(v) for v in p[2:7])
    k = 7
    em = p[k:k + 2 * norb].reshape((norb, 2), order="F")
    k += 2 * norb
    ek = p[k:k + 2 * nbath].reshape((nbath, 2), order="F")
    k += 2 * nbath
    vmk = p[k:k + 2 * norb * nbath].reshape((norb, nbath, 2), order="F")
    return pkg.Model(norb, nbath, em, ek, vmk, U=U, Up=Up, Jex=Jex, Jp=Jp, mu=mu)


@pytest.mark.parametrize("case", CASES)
def test_hx_and_apply_c_against_reference(pkg, solver, case):
    solver.set_model(_model(pkg, GOLD[f"model_{case}"]))
    nu, nd = (int(v) for v in GOLD[f"sector_{case}"])
    x = GOLD[f"hx_{case}_x"]
    y = solver.hx(nu, nd, x)
    ref = GOLD[f"hx_{case}_y"]
    assert np.abs(y - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    yacc = solver.hx(nu, nd, x, GOLD[f"hx_{case}_y0"].copy(), py=True)
    ref = GOLD[f"hx_{case}_yacc"]
    assert np.abs(yacc - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    for key in GOLD.files:
        if key.startswith(f"applyc_{case}_"):
            pm, iorb, ispin = (int(c) for c in key.rsplit("_", 1)[1])
            assert np.array_equal(solver.apply_c(nu, nd, x, pm, iorb, ispin), GOLD[key]), key


@pytest.mark.parametrize("case", LZ)
def test_lanczos_coefficients_against_reference(pkg, solver, case):
    solver.set_model(_model(pkg, GOLD[f"lzmodel_{case}"]))
    nu, nd = (int(v) for v in GOLD[f"lz_{case}_sector"])
    a_ref, b_ref = GOLD[f"lz_{case}_a"], GOLD[f"lz_{case}_b"]
    n_ref = int(GOLD[f"lz_{case}_nstep"][0])
    n, a, b = solver.lanczos_iteration(nu, nd, GOLD[f"lz_{case}_v"], len(a_ref))
    assert n == n_ref
    k = ab_compare_len(b_ref, n)
    assert k >= 20
    assert np.abs(a[:k] - a_ref[:k]).max() <= 1e-8
    assert np.abs(b[:k] - b_ref[:k]).max() <= 1e-8


def test_ground_state_and_green_against_reference(pkg, solver):
    em, ek, V = np.zeros((1, 2)), np.stack([np.linspace(-1.0, 1.0, 5)] * 2, 1), np.full((1, 5, 2), 0.5)
    solver.set_model(pkg.Model(1, 5, em, ek, V, U=2.0, mu=1.0))
    sectors = [tuple(int(v) for v in s) for s in GOLD["gs_sectors"]]
    omega = GOLD["G_omega"]
    gs = solver.ground_state(sectors, 60, seed=0)
    assert gs["isector"] + 1 == int(GOLD["gs_isector"][0])
    e_ref = float(GOLD["gs_e0"][0])
    assert abs(gs["e0"] - e_ref) <= 1e-10 * max(1.0, abs(e_ref))
    assert abs(abs(gs["vec"] @ GOLD["gs_vec"]) - 1.0) <= 1e-8
    G = solver.cluster_green_ftn(1, 60, omega)["G_cl"][0, 0]
    assert np.abs(G - GOLD["G_double"]).max() <= 1e-8
