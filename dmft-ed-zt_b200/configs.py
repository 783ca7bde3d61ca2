"""Seeded synthetic impurity models for the workloads the solver is measured on.

The reference quotes no data set; every input here is synthetic, drawn with
numpy's PCG64 generator from a recorded seed:

  bethe_n6      single-orbital Anderson impurity, 5 bath sites (nsite 6),
                U = 2, mu = U/2, bath levels linspace(-1, 1), V = 0.5; all
                49 (n_up, n_dn) sectors; 200 Lanczos steps
  aim_n12       single-orbital impurity, 11 bath sites (nsite 12), U = 3,
                half filling (mu = U/2), eps ~ U(-2,2), V ~ U(0.1,1) (seed 12);
                sectors n_up, n_dn in {5,6,7}; 300 Lanczos steps
  kanamori_n10  two-orbital Hubbard-Kanamori impurity, U = 2.5, J = U/4,
                U' = U - 2J, Jp = J, 4 bath sites per orbital (nsite 10),
                particle-hole symmetric mu, eps ~ U(-2,2), V ~ U(0.1,1)
                (seed 10); half-filled sectors; 200 Lanczos steps
  batch(n)      single-orbital instances, nsite ~ U{8..14}, U ~ U(1,4),
                mu = U/2, eps ~ U(-2,2), V ~ U(0.1,1) (seed 4); sectors within
                one electron of half filling in each spin; nspin = 2 so the
                Green's function takes c and c^+ runs for both spins
"""

from __future__ import annotations

import numpy as np

from . import Model


def _single_orbital(nbath, ek, V, U, mu):
    em = np.zeros((1, 2))
    ekk = np.stack([ek, ek], axis=1)
    vmk = np.stack([V, V], axis=1).reshape(1, nbath, 2)
    return Model(1, nbath, em, ekk, vmk, U=U, Up=U, Jex=0.0, Jp=0.0, mu=mu)


def bethe_n6():
    nbath = 5
    U = 2.0
    m = _single_orbital(nbath, np.linspace(-1.0, 1.0, nbath), np.full(nbath, 0.5), U, U / 2)
    sectors = [(u, d) for u in range(7) for d in range(7)]
    return dict(name="bethe_n6", model=m, sectors=sectors, maxnstep=200, beta=100.0, nw=2048, nspin=1)


def aim_n12(seed: int = 12):
    rng = np.random.default_rng(seed)
    nbath = 11
    U = 3.0
    ek = rng.uniform(-2.0, 2.0, nbath)
    V = rng.uniform(0.1, 1.0, nbath)
    m = _single_orbital(nbath, ek, V, U, U / 2)
    sectors = [(u, d) for u in (5, 6, 7) for d in (5, 6, 7)]
    return dict(name="aim_n12", model=m, sectors=sectors, maxnstep=300, beta=100.0, nw=2048, nspin=1)


def kanamori_n10(seed: int = 10):
    rng = np.random.default_rng(seed)
    norb, nb = 2, 4
    nbath = norb * nb
    U = 2.5
    J = U / 4
    Up = U - 2 * J
    mu = U / 2 + (norb - 1) * (2 * Up - J) / 2
    ek1 = rng.uniform(-2.0, 2.0, nbath)
    V = rng.uniform(0.1, 1.0, nbath)
    vmk = np.zeros((norb, nbath, 2))
    for a in range(norb):
        for l in range(a * nb, (a + 1) * nb):
            vmk[a, l, :] = V[l]
    m = Model(norb, nbath, np.zeros((norb, 2)), np.stack([ek1, ek1], 1), vmk, U=U, Up=Up, Jex=J, Jp=J, mu=mu)
    ns = norb + nbath
    sectors = [(u, ns - u) for u in range(ns // 2 - 2, ns // 2 + 3)]
    return dict(name="kanamori_n10", model=m, sectors=sectors, maxnstep=200, beta=100.0, nw=2048, nspin=1)


def near_half_sectors(nsite: int):
    lo, hi = (nsite - 1) // 2, (nsite + 2) // 2
    if nsite % 2 == 0:
        ns = [nsite // 2 - 1, nsite // 2, nsite // 2 + 1]
    else:
        ns = [lo, hi]
    return [(u, d) for u in ns for d in ns]


def batch(n: int = 256, seed: int = 4, nsite_range=(8, 14)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ns = int(rng.integers(nsite_range[0], nsite_range[1] + 1))
        U = float(rng.uniform(1.0, 4.0))
        nbath = ns - 1
        ek = rng.uniform(-2.0, 2.0, nbath)
        V = rng.uniform(0.1, 1.0, nbath)
        m = _single_orbital(nbath, ek, V, U, U / 2)
        # nspin = 2: c and c^+ for both spins, the 4 excitation runs per instance
        out.append(dict(name=f"batch{i}", model=m, sectors=near_half_sectors(ns), maxnstep=300, beta=100.0,
                        nw=2048, nspin=2))
    return out
