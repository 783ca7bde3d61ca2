"""GPU parity: kernel (a) basis tables (bit-exact) and kernel (b) H.v (FP64).

H.v tolerance: the GPU sums each row in a different order than the
reference's row loop, so entries may differ by a few ulps of the row's
terms: |y_gpu - y_oracle| <= 1e-13 * (max|y| + 1).
"""

import numpy as np
import pytest

from conftest import oracle_for, random_model

pytestmark = pytest.mark.gpu
HX_TOL = 1e-13


def _tol(y):
    return HX_TOL * (np.abs(y).max() + 1.0)


@pytest.mark.parametrize("nsite", list(range(1, 13)) + [14, 16])
def test_basis_bit_exact(pkg, solver, oracle_mod, nsite):
    nb = nsite - 1
    m = pkg.Model(1, nb, np.zeros((1, 2)), np.zeros((nb, 2)), np.zeros((1, nb, 2)), U=1.0, mu=0.5)
    solver.set_model(m)
    ns_list = range(nsite + 1) if nsite <= 12 else [0, 1, nsite // 2 - 1, nsite // 2, nsite]
    for n in ns_list:
        ref_str, ref_idx = oracle_mod.spin_basis(nsite, n)
        up, dn = solver.generate_basis(n, n)
        assert np.array_equal(up.astype(np.int64), ref_str.astype(np.int64))
        assert np.array_equal(dn, up)
        rank = solver.basis_rank(n)
        assert np.array_equal(rank, ref_idx - 1)   # 0-based, -1 outside the sector


CASES = [
    # norb, nbath, J, spin-dependent, fraction of switched-off hops
    (1, 5, 0.0, False, 0.0),
    (1, 7, 0.0, True, 0.3),
    (2, 4, 0.625, False, 0.0),
    (2, 6, 0.5, True, 0.25),
    (3, 3, 0.4, True, 0.0),
    (1, 0, 0.0, False, 0.0),
]


@pytest.mark.parametrize("case", CASES)
def test_hx_parity(pkg, solver, oracle_mod, case):
    norb, nbath, J, sd, zf = case
    rng = np.random.default_rng(100 + norb * 10 + nbath)
    m = random_model(pkg, rng, norb, nbath, J=J, spin_dep=sd, zero_frac=zf)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    ns = norb + nbath
    sectors = {(ns // 2, ns // 2), (ns // 2, (ns + 1) // 2), (0, 0), (ns, ns), (1, ns - 1), (ns - 1, 1)}
    for nu, nd in sorted(sectors):
        n = o.dim(nu, nd)
        x = rng.standard_normal(n)
        y0 = rng.standard_normal(n)
        y_ref = o.hx(nu, nd, x)
        y = solver.hx(nu, nd, x)
        assert np.abs(y - y_ref).max() <= _tol(y_ref), (nu, nd)
        ya_ref = o.hx(nu, nd, x, y0, py=True)
        ya = solver.hx(nu, nd, x, y0, py=True)
        assert np.abs(ya - ya_ref).max() <= _tol(ya_ref), (nu, nd)


def test_hx_cfg_aim_n12_full(solver, configs, oracle_mod):
    cfg = configs.aim_n12()
    m = cfg["model"]
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    rng = np.random.default_rng(12)
    for nu, nd in [(6, 6), (5, 7)]:
        x = rng.standard_normal(o.dim(nu, nd))
        y_ref = o.hx(nu, nd, x)
        assert np.abs(solver.hx(nu, nd, x) - y_ref).max() <= _tol(y_ref)


def test_hx_kanamori_full(solver, configs, oracle_mod):
    cfg = configs.kanamori_n10()
    m = cfg["model"]
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    x = np.random.default_rng(3).standard_normal(o.dim(5, 5))
    y_ref = o.hx(5, 5, x)
    assert np.abs(solver.hx(5, 5, x) - y_ref).max() <= _tol(y_ref)


@pytest.mark.parametrize("nsite", [14, 15, 16])
def test_hx_large_rows_and_hermiticity(pkg, solver, oracle_mod, nsite):
    """Full-size sectors: oracle rows at three offsets, <u,Hv> = <Hu,v> on the
    device, for y = H x and y += H x.  They run k_hx with 512 (nsite 14)
    and 1024 threads per CTA (nsite 15 and 16)."""
    import torch
    rng = np.random.default_rng(nsite)
    m = random_model(pkg, rng, 1, nsite - 1)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    nu = nd = nsite // 2
    n = o.dim(nu, nd)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(nsite)
    x = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    u = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    y = torch.empty_like(x)
    hu = torch.empty_like(x)
    solver.hx(nu, nd, x, y)
    solver.hx(nu, nd, u, hu)
    torch.cuda.synchronize()
    lhs = float(torch.dot(u, y))
    rhs = float(torch.dot(hu, x))
    scale = float(torch.linalg.norm(u) * torch.linalg.norm(y))
    assert abs(lhs - rhs) <= 1e-11 * scale
    z = u.clone()                                           # the accumulating form: z = u + H x
    solver.hx(nu, nd, x, z, py=True)
    torch.cuda.synchronize()
    assert float((z - u - y).abs().max()) <= 1e-13 * (float(y.abs().max()) + float(u.abs().max()) + 1.0)
    xh = x.cpu().numpy()
    yh = y.cpu().numpy()
    for r0 in (0, n // 2 - 20000, n - 40000):
        r1 = r0 + 40000
        ref = o.hx_rows(nu, nd, xh, r0, r1)
        assert np.abs(yh[r0:r1] - ref).max() <= _tol(ref)


def _random_element_cases(n=6, seed=77, max_dim=600):
    """Seeded random (norb, nbath, J, sector) with sector dimension <= max_dim."""
    from math import comb
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        norb = int(rng.integers(1, 4))
        nbath = int(rng.integers(1, 8 - norb))
        ns = norb + nbath
        nu, nd = int(rng.integers(0, ns + 1)), int(rng.integers(0, ns + 1))
        if 2 <= comb(ns, nu) * comb(ns, nd) <= max_dim:
            out.append((norb, nbath, float(rng.uniform(0.0, 0.8)) if norb > 1 else 0.0, (nu, nd)))
    return out


@pytest.mark.parametrize("norb,nbath,J,sector", [(1, 5, 0.0, (3, 3)), (1, 5, 0.0, (2, 4)), (2, 4, 0.6, (3, 3)),
                                                 (3, 3, 0.4, (3, 2))] + _random_element_cases())
def test_hx_matrix_elements_bit_exact(pkg, solver, oracle_mod, norb, nbath, J, sector):
    """Every (ket index, sign) of the GPU's hop tables, bit for bit: column j
    of H is H e_j, and each off-diagonal element is one product (+-V or
    +-Jp) times 1.0, so the GPU's and the oracle's dense H must agree exactly
    off the diagonal.  The diagonal sums several terms (ulp-level bound)."""
    import torch
    rng = np.random.default_rng(40 + norb)
    m = random_model(pkg, rng, norb, nbath, J=J, spin_dep=True)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    nu, nd = sector
    H_ref = o.dense_h(nu, nd)
    n = H_ref.shape[0]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    H = np.zeros((n, n))
    for j in range(n):
        x.zero_()
        x[j] = 1.0
        solver.hx(nu, nd, x, y)
        H[:, j] = y.cpu().numpy()
    off = ~np.eye(n, dtype=bool)
    assert np.array_equal(H[off], H_ref[off])
    assert np.count_nonzero(H_ref[off]) > 0
    assert np.abs(np.diag(H) - np.diag(H_ref)).max() <= 1e-14 * np.abs(np.diag(H_ref)).max()


def test_hx_device_pointers_accumulate(pkg, solver, oracle_mod):
    import torch
    rng = np.random.default_rng(9)
    m = random_model(pkg, rng, 2, 5, J=0.3)
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    n = o.dim(3, 4)
    x = rng.standard_normal(n)
    y0 = rng.standard_normal(n)
    xd = torch.tensor(x, device="cuda")
    yd = torch.tensor(y0, device="cuda")
    solver.hx(3, 4, xd, yd, py=True)
    ref = o.hx(3, 4, x, y0, py=True)
    assert np.abs(yd.cpu().numpy() - ref).max() <= _tol(ref)


def test_apply_c_bit_exact(pkg, solver, oracle_mod):
    rng = np.random.default_rng(31)
    for norb, nbath in [(1, 7), (2, 6)]:
        m = random_model(pkg, rng, norb, nbath, J=0.4)
        solver.set_model(m)
        o = oracle_for(oracle_mod, m)
        ns = norb + nbath
        for nu, nd in [(ns // 2, ns // 2), (ns // 2 + 1, ns // 2 - 1), (0, ns), (ns, 0)]:
            x = rng.standard_normal(o.dim(nu, nd))
            for pm in (1, 2):
                for ispin in (1, 2):
                    for iorb in range(1, norb + 1):
                        d = 1 if pm == 1 else -1
                        ou, od = nu + (d if ispin == 1 else 0), nd + (d if ispin == 2 else 0)
                        if not (0 <= ou <= ns and 0 <= od <= ns):
                            with pytest.raises(pkg.EDError):
                                solver.apply_c(nu, nd, x, pm, iorb, ispin)
                            continue
                        ref = o.apply_c(nu, nd, x, pm, iorb, ispin)
                        assert np.array_equal(solver.apply_c(nu, nd, x, pm, iorb, ispin), ref)


def test_argument_errors(pkg, solver):
    m = pkg.Model(1, 3, np.zeros((1, 2)), np.zeros((3, 2)), np.full((1, 3, 2), 0.5), U=1.0, mu=0.5)
    solver.set_model(m)
    with pytest.raises(pkg.EDError) as e:
        solver.hx(5, 1, np.zeros(4))
    assert e.value.code == pkg.EDZT_ERR_ARG
    with pytest.raises(pkg.EDError):
        solver.apply_c(2, 2, np.zeros(36), 3, 1, 1)
