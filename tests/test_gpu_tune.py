"""The tile-shape autotuner (edzt_tune_sector): it picks a shape that fits,
records it on the context, and runs with the tuned shape give the oracle's
Lanczos coefficients (first 50 within 1e-8) and the same E0 (1e-10)."""

import numpy as np
import pytest

from conftest import oracle_for, random_model

pytestmark = pytest.mark.gpu


def test_tuned_shape_keeps_results(pkg, solver, oracle_mod):
    rng = np.random.default_rng(404)
    m = random_model(pkg, rng, 1, 11)                     # nsite 12
    solver.set_model(m)
    o = oracle_for(oracle_mod, m)
    v0 = oracle_mod.start_vector(8, 2, o.dim(6, 6))
    n_ref, a_ref, b_ref = o.lanczos_iteration(6, 6, v0, 80)
    try:
        t = solver.tune_sector(6, 6, steps=8)
        assert t["cols_per_slab"] in (2, 4, 8, 16) and t["rows_per_tile"] in (1, 2, 4, 8)
        assert t["block"] in (256, 512) and 0.0 < t["ms_per_step"] < 1000.0
        n, a, b = solver.lanczos_iteration(6, 6, v0, 80)
        assert n == n_ref
        assert np.abs(a[:50] - a_ref[:50]).max() <= 1e-8 and np.abs(b[:50] - b_ref[:50]).max() <= 1e-8
        e_tuned = solver.diag_lanczos(6, 6, 80, seed=3, stream=1)["e0"]
    finally:
        solver.clear_tuning()
    e_rule = solver.diag_lanczos(6, 6, 80, seed=3, stream=1)["e0"]
    assert abs(e_tuned - e_rule) <= 1e-10 * max(1.0, abs(e_rule))
    with pytest.raises(pkg.EDError):
        solver.tune_sector(6, 6, steps=1)
