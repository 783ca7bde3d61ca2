"""The C oracle against the literal transliteration of the reference (CPU).

oracle/ref_literal.py keeps the reference's own state representation and
evaluation order, so basis strings, H.v and apply_c must agree bit for bit.
"""

import numpy as np
import pytest

from conftest import oracle_for, random_model
from oracle import ref_literal as R


@pytest.mark.parametrize("norb,nbath,J", [(1, 5, 0.0), (2, 4, 0.6), (3, 3, 0.4)])
def test_hx_bit_exact(pkg, oracle_mod, norb, nbath, J):
    rng = np.random.default_rng(7 + norb)
    m = random_model(pkg, rng, norb, nbath, J=J, spin_dep=True, zero_frac=0.2)
    o = oracle_for(oracle_mod, m)
    md = o.model_dict()
    ns = norb + nbath
    for nu, nd in [(ns // 2, ns // 2), (ns // 2 - 1, ns // 2 + 1), (0, 1), (ns, ns - 1), (1, 0)]:
        B = R.Basis(ns, nu, nd)
        x = rng.standard_normal(B.ntot)
        y0 = rng.standard_normal(B.ntot)
        assert np.array_equal(np.array(R.hx(md, B, list(x))), o.hx(nu, nd, x))
        assert np.array_equal(np.array(R.hx(md, B, list(x), py=True, y=list(y0))), o.hx(nu, nd, x, y0, py=True))


@pytest.mark.parametrize("ns", [1, 4, 7, 10])
def test_spin_basis_bit_exact(oracle_mod, ns):
    for n in range(ns + 1):
        strings, idx = oracle_mod.spin_basis(ns, n)
        B = R.Basis(ns, n, 0)
        assert strings.tolist() == B.up
        for rank, s in enumerate(B.up, start=1):
            assert idx[s] == rank
        assert int((idx > 0).sum()) == len(B.up)


def test_apply_c_bit_exact(pkg, oracle_mod):
    rng = np.random.default_rng(3)
    m = random_model(pkg, rng, 2, 4, J=0.5)
    o = oracle_for(oracle_mod, m)
    ns = 6
    for nu, nd in [(3, 3), (2, 4), (6, 0), (0, 6)]:
        B = R.Basis(ns, nu, nd)
        x = rng.standard_normal(B.ntot)
        for pm in (1, 2):
            for ispin in (1, 2):
                for iorb in (1, 2):
                    d = 1 if pm == 1 else -1
                    ou, od = nu + (d if ispin == 1 else 0), nd + (d if ispin == 2 else 0)
                    if not (0 <= ou <= ns and 0 <= od <= ns):
                        continue
                    Bo = R.Basis(ns, ou, od)
                    ref = np.array(R.apply_c(ns, B, list(x), pm, iorb, ispin, Bo))
                    assert np.array_equal(ref, o.apply_c(nu, nd, x, pm, iorb, ispin))


def test_random_models_bit_exact(pkg, oracle_mod):
    """A seeded sweep over 40 random models (1-3 orbitals, up to 7 sites,
    random J, spin dependence and switched-off hops) and random sectors:
    hx (both forms) and apply_c agree with the literal transliteration bit
    for bit."""
    rng = np.random.default_rng(2024)
    for case in range(40):
        norb = int(rng.integers(1, 4))
        nbath = int(rng.integers(0, 8 - norb))
        ns = norb + nbath
        J = float(rng.uniform(0.0, 0.8)) if norb > 1 else 0.0
        m = random_model(pkg, rng, norb, nbath, J=J, spin_dep=bool(rng.integers(0, 2)),
                         zero_frac=float(rng.choice([0.0, 0.3])))
        o = oracle_for(oracle_mod, m)
        md = o.model_dict()
        sectors = {(int(rng.integers(0, ns + 1)), int(rng.integers(0, ns + 1))), (ns // 2, (ns + 1) // 2)}
        for nu, nd in sorted(sectors):
            B = R.Basis(ns, nu, nd)
            x = rng.standard_normal(B.ntot)
            y0 = rng.standard_normal(B.ntot)
            assert np.array_equal(np.array(R.hx(md, B, list(x))), o.hx(nu, nd, x)), (case, nu, nd)
            assert np.array_equal(np.array(R.hx(md, B, list(x), py=True, y=list(y0))),
                                  o.hx(nu, nd, x, y0, py=True)), (case, nu, nd)
            pm, ispin, iorb = int(rng.integers(1, 3)), int(rng.integers(1, 3)), int(rng.integers(1, norb + 1))
            d = 1 if pm == 1 else -1
            ou, od = nu + (d if ispin == 1 else 0), nd + (d if ispin == 2 else 0)
            if 0 <= ou <= ns and 0 <= od <= ns:
                Bo = R.Basis(ns, ou, od)
                ref = np.array(R.apply_c(ns, B, list(x), pm, iorb, ispin, Bo))
                assert np.array_equal(ref, o.apply_c(nu, nd, x, pm, iorb, ispin)), (case, nu, nd, pm, iorb, ispin)
