"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = "dmft_ed_zt_b200"
PKG_DIR = os.path.join(ROOT, "dmft-ed-zt_b200")


def load_pkg():
    """Import the package directory dmft-ed-zt_b200/ as module dmft_ed_zt_b200."""
    if PKG_NAME in sys.modules:
        return sys.modules[PKG_NAME]
    spec = importlib.util.spec_from_file_location(PKG_NAME, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[PKG_NAME] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def configs(pkg):
    import importlib
    return importlib.import_module(PKG_NAME + ".configs")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def solver(pkg):
    """One CUDA context for the whole GPU session (fails loudly without libedzt.so / a GPU)."""
    pkg.build()
    s = pkg.Solver(0)
    yield s
    s.close()


@pytest.fixture(autouse=True)
def _device_checks(request):
    """With a bounds-checked library build, fail a GPU test whose kernels recorded a bad index."""
    yield
    if "gpu" not in request.keywords:
        return
    L = sys.modules.get(PKG_NAME)
    lib = getattr(L, "_lib", None) if L else None
    if lib is None or not hasattr(lib, "edzt_debug_bad"):
        return
    import ctypes as C
    bad = (C.c_longlong * 4)()
    lib.edzt_debug_bad(bad)
    assert bad[0] == 0, f"device bounds check {list(bad)}"


def oracle_for(O, m):
    """CPU oracle of a package Model."""
    return O.Oracle(m.norb, m.nbath, m.em, m.ek, m.vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)


def random_model(pkg, rng, norb, nbath, J=0.0, spin_dep=False, zero_frac=0.0):
    """Generic impurity model with optional spin dependence and switched-off hops."""
    em = rng.uniform(-0.5, 0.5, (norb, 2))
    ek = rng.uniform(-2.0, 2.0, (nbath, 2))
    V = rng.uniform(0.1, 1.0, (norb, nbath, 2))
    if not spin_dep:
        em[:, 1] = em[:, 0]
        ek[:, 1] = ek[:, 0]
        V[:, :, 1] = V[:, :, 0]
    if zero_frac > 0:
        V[rng.random(V.shape) < zero_frac] = 0.0
    U = float(rng.uniform(1.0, 4.0))
    return pkg.Model(norb, nbath, em, ek, V, U=U, Jex=J, mu=U / 2)


def ab_compare_len(b_ref, nstep, first=50):
    """Number of leading Lanczos coefficients that are comparable between two
    FP64 implementations: at most `first`, and none past the first tiny b
    (an exhausted Krylov space, after which the recurrence runs on rounding noise)."""
    k = min(first, nstep)
    b = np.abs(np.asarray(b_ref[:nstep]))
    if nstep > 1:
        tiny = np.nonzero(b[1:] < 1e-8 * b.max())[0]
        if tiny.size:
            k = min(k, int(tiny[0]) + 1)
    return k


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
