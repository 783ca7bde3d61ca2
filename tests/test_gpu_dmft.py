"""The CPU-runnable workload end to end: nsite-6 Bethe-lattice DMFT, 20
iterations with linear mixing 0.5, 200 Lanczos steps, 2048 Matsubara points
at beta 100, run by the same host loop on the GPU library and on the oracle.
The converged hybridization D_cl(i w) must agree to 1e-6; G_cl, G_loc and the
quasiparticle weight are held to the same bound.

Both loops fit the bath to a relative tolerance of 1e-13.  With the
reference's 1e-6 the fit stops on a flat stretch of the cost before the
parameters settle, and the loop is not reproducible to 1e-6 even against
itself: a 1e-11 relative change of G_cl, well inside the solver's parity,
moves the 20th iteration's D_cl by about 1e-4 on the oracle alone."""

import importlib

import numpy as np
import pytest

from test_dmft_host import oracle_solver

pytestmark = pytest.mark.gpu


def test_bethe_dmft_gpu_matches_oracle(pkg, solver, configs, oracle_mod):
    d = importlib.import_module("dmft_ed_zt_b200.dmft")
    cfg = configs.bethe_n6()
    m = cfg["model"]
    w = pkg.matsubara(cfg["nw"], cfg["beta"])
    gpu = d.gpu_solver(pkg, solver, m.norb, m.nbath, m.U, m.Up, m.Jex, m.Jp, m.mu, cfg["sectors"], cfg["maxnstep"], w)
    cpu = oracle_solver(oracle_mod, m, cfg["sectors"], cfg["maxnstep"], w)
    kw = dict(nloop=20, scf_tol=0.0, mixing=0.5, fit_ftol=1e-13)
    r_gpu = d.dmft_loop(gpu, m.em, m.ek, m.vmk, w, m.nbath, **kw)
    r_cpu = d.dmft_loop(cpu, m.em, m.ek, m.vmk, w, m.nbath, **kw)
    assert r_gpu.iterations == r_cpu.iterations == 20
    assert np.abs(r_gpu.D_cl - r_cpu.D_cl).max() <= 1e-6
    assert np.abs(r_gpu.G_cl - r_cpu.G_cl).max() <= 1e-6
    assert np.abs(r_gpu.G_loc - r_cpu.G_loc).max() <= 1e-6
    z_gpu = d.quasiparticle_weight(d.self_energy(r_gpu.em, r_gpu.D_cl, r_gpu.G_cl, w, m.mu), w)
    z_cpu = d.quasiparticle_weight(d.self_energy(r_cpu.em, r_cpu.D_cl, r_cpu.G_cl, w, m.mu), w)
    assert np.abs(z_gpu - z_cpu).max() <= 1e-6
    assert r_gpu.history[-1] < 1e-3 * r_gpu.history[0]     # the loop converges
