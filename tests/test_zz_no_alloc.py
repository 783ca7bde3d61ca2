"""edzt_lanczos_iteration_noalloc (the variant that allocates no device
memory) against edzt_lanczos_iteration, through the C ABI.

Collected last on purpose: it must pass both in a fresh process and after
every other test has used (and grown) the library's allocations.  Tolerance:
the first 50 Lanczos coefficients within 1e-8, as the Lanczos parity tests.
"""

import ctypes as C

import numpy as np
import pytest

from conftest import ab_compare_len, random_model

pytestmark = pytest.mark.gpu
AB_TOL = 1e-8


def _compare(ref, got):
    n_ref, a_ref, b_ref = ref
    n, a, b = got
    assert n == n_ref
    k = ab_compare_len(b_ref, n_ref)
    assert np.abs(a[:k] - a_ref[:k]).max() <= AB_TOL
    assert np.abs(b[:k] - b_ref[:k]).max() <= AB_TOL
    assert b[0] == 0.0


def test_noalloc_matches_lanczos_iteration(pkg, solver):
    rng = np.random.default_rng(2024)
    m = random_model(pkg, rng, 1, 9, spin_dep=True)
    solver.set_model(m)
    for nu, nd in [(5, 5), (4, 6), (2, 1)]:               # dims 63504, 52920, 450
        v0 = np.random.default_rng(nu * 10 + nd).random(solver.dim(nu, nd))
        ref = solver.lanczos_iteration(nu, nd, v0, 120)   # allocating call: builds the tables
        first = solver.lanczos_iteration_noalloc(nu, nd, v0, 120)
        second = solver.lanczos_iteration_noalloc(nu, nd, v0, 120)
        _compare(ref, first)
        _compare(ref, second)


def test_noalloc_device_start_vector(pkg, solver):
    import torch
    rng = np.random.default_rng(7)
    m = random_model(pkg, rng, 1, 7)
    solver.set_model(m)
    nu, nd = 4, 4
    v0 = np.random.default_rng(3).random(solver.dim(nu, nd))
    ref = solver.lanczos_iteration(nu, nd, v0, 80)
    dv = torch.from_numpy(v0).to("cuda:0")
    for _ in range(2):
        a = np.zeros(80)
        b = np.zeros(80)
        n = C.c_int()
        rc = solver._L.edzt_lanczos_iteration_noalloc(solver._h, nu, nd, C.c_void_p(dv.data_ptr()), 80,
                                                      C.byref(n), a.ctypes.data, b.ctypes.data)
        assert rc == pkg.EDZT_OK, solver._L.edzt_last_error(solver._h)
        _compare(ref, (n.value, a, b))


def test_noalloc_limits_and_state(pkg, solver):
    rng = np.random.default_rng(11)
    m = random_model(pkg, rng, 1, 11)                     # nsite 12: (6,6) has 853776 states
    solver.set_model(m)
    v0 = np.zeros(1)
    with pytest.raises(pkg.EDError) as e:
        solver.lanczos_iteration_noalloc(6, 6, v0, 10)
    assert e.value.code == pkg.EDZT_ERR_ARG and "no-allocation limit" in str(e.value)
    with pytest.raises(pkg.EDError) as e:                 # tables of (1,1) not built yet
        solver.lanczos_iteration_noalloc(1, 1, np.ones(144), 10)
    assert e.value.code == pkg.EDZT_ERR_STATE
    solver.lanczos_iteration(1, 1, np.ones(144), 10)
    with pytest.raises(pkg.EDError) as e:
        solver.lanczos_iteration_noalloc(1, 1, np.ones(144), pkg.NOALLOC_MAX_STEPS + 1)
    assert e.value.code == pkg.EDZT_ERR_ARG
    n, a, b = solver.lanczos_iteration_noalloc(1, 1, np.ones(144), 10)
    n_ref, a_ref, b_ref = solver.lanczos_iteration(1, 1, np.ones(144), 10)
    _compare((n_ref, a_ref, b_ref), (n, a, b))
