"""Generate tests/golden/dmft_golden.npz: a short DMFT run as a golden record.

The nsite-6 Bethe-lattice workload (1 impurity + 5 bath sites, U = 2,
half filling, all 49 sectors) cut down so the oracle finishes in seconds:
the first 128 Matsubara points at beta 100, 60 Lanczos steps, 4 iterations
with linear mixing 0.5 and the bath fit to a relative tolerance of 1e-13
(looser fits leave the bath on a flat stretch of the cost, where rounding
differences between implementations grow from iteration to iteration).
The loop is dmft_ed_zt_b200/dmft.py on the CPU oracle solver.  The record
holds the last iteration's bath, D_cl, G_cl, G_loc and the convergence
measure of every iteration.
Run from the repository root:  python tests/golden/make_dmft_golden.py
"""

from __future__ import annotations

import importlib
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O          # noqa: E402

OUT = os.path.join(HERE, "dmft_golden.npz")
NW, BETA, MAXNSTEP, NLOOP, MIXING, FIT_FTOL = 128, 100.0, 60, 4, 0.5, 1e-13


def load_pkg():
    pkg_dir = os.path.join(ROOT, "dmft-ed-zt_b200")
    if "dmft_ed_zt_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("dmft_ed_zt_b200", os.path.join(pkg_dir, "__init__.py"),
                                                      submodule_search_locations=[pkg_dir])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["dmft_ed_zt_b200"] = mod
        spec.loader.exec_module(mod)
    return (sys.modules["dmft_ed_zt_b200"], importlib.import_module("dmft_ed_zt_b200.configs"),
            importlib.import_module("dmft_ed_zt_b200.dmft"))


def run_oracle_loop():
    """The recorded run: returns (config, result of dmft_loop)."""
    pkg, cfgs, d = load_pkg()
    O.build()
    cfg = cfgs.bethe_n6()
    m = cfg["model"]
    w = O.matsubara(NW, BETA)

    def solve(em, ek, vmk):
        o = O.Oracle(m.norb, m.nbath, em, ek, vmk, m.U, m.Up, m.Jex, m.Jp, m.mu)
        gs = o.ground_state(cfg["sectors"], MAXNSTEP, seed=0)
        return o.cluster_green_ftn(1, *gs["sector"], gs["vec"], gs["e0"], MAXNSTEP, w)["G_cl"]

    res = d.dmft_loop(solve, m.em, m.ek, m.vmk, w, m.nbath, nspin=1, nloop=NLOOP, scf_tol=0.0, mixing=MIXING,
                      fit_ftol=FIT_FTOL)
    return cfg, res


def main():
    cfg, r = run_oracle_loop()
    assert r.iterations == NLOOP and r.history[-1] < r.history[0]
    np.savez_compressed(OUT, em=r.em, ek=r.ek, vmk=r.vmk, D_cl=r.D_cl, G_cl=r.G_cl, G_loc=r.G_loc,
                        history=np.array(r.history),
                        settings=np.array([NW, BETA, MAXNSTEP, NLOOP, MIXING, FIT_FTOL]))
    print("wrote", OUT, "history", r.history)


if __name__ == "__main__":
    main()
