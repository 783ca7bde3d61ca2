"""Host DMFT self-consistency loop around the impurity solver, Bethe lattice.

Restates the reference's host loop (src/dmft.f90:38-137) for the
semicircular density of states of half-bandwidth 1 (TBHamiltonian 2,
src/dmft_lattice.f90:75-103), so that the CPU-runnable workload (nsite 6,
20 iterations) runs end to end on either impurity solver:

  iteration 1:   the initial bath (em, ek, vmk)
  iteration > 1: fit (em, ek, vmk) to the previous iteration's
                 G_0^-1 corrected by G_loc^-1 - G_cl^-1
                 (src/ed_projection.f90:23-553), optionally mixed linearly
                 with the previous parameters (the workload's mixing 0.5,
                 which the reference does not have; 1.0 reproduces it)
  then           D_cl  = sum_l V_l^2 / (i w - e_l)        (dmft_green.f90:24-45)
                 G_cl  = the impurity solve (ground_state + cluster_green_ftn)
                 G_loc = int dos(x) / (em + D_cl + 1/G_cl - x) dx  (:128-170)
                 stop when sum |G_cl - G_loc|^2 / (norb nbath nw) < scf_tol

The fit minimises the reference's cost (ed_projection.f90:154-250) by a
nonlinear conjugate gradient with Polak-Ribiere directions, as the reference
does, with a line search of this module's own design that uses the cost's
analytic gradient (line_minimum: fourfold step growth to a bracket, then
safeguarded Hermite-cubic steps).  ftol is the reference's relative stopping
tolerance (1e-6 by default).
The impurity solver is a callback: the GPU library (gpu_solver) or the CPU
oracle (used by the tests) give the same loop.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Green's functions on the Matsubara grid
# ---------------------------------------------------------------------------
def hybridization(ek, vmk, omega, nspin):
    """D_cl[ispin, iorb, iw] = sum_l vmk(iorb,l,ispin)^2 / (i w - ek(l,ispin))."""
    ek = np.asarray(ek, dtype=float)
    vmk = np.asarray(vmk, dtype=float)
    iw = 1j * np.asarray(omega, dtype=float)
    norb = vmk.shape[0]
    D = np.zeros((nspin, norb, len(iw)), dtype=complex)
    for s in range(nspin):
        for a in range(norb):
            D[s, a] = (vmk[a, :, s][:, None] ** 2 / (iw[None, :] - ek[:, s][:, None])).sum(axis=0)
    return D


def local_green(em, D, G_cl, hfield=0.0, ne=10000):
    """G_loc of the Bethe lattice by the reference's quadrature: ne equally
    spaced points on [-1, 1], weights 2/pi sqrt(1 - x^2), sum times 2/(ne-1)."""
    em = np.asarray(em, dtype=float)
    nspin, norb, nw = G_cl.shape
    x = -1.0 + np.arange(ne) * 2.0 / (ne - 1)
    w = 2.0 / math.pi * np.sqrt(np.maximum(1.0 - x * x, 0.0))
    hs = (hfield, -hfield)
    G = np.zeros_like(G_cl)
    for s in range(nspin):
        for a in range(norb):
            zeta = em[a, s] + hs[s] + D[s, a] + 1.0 / G_cl[s, a]          # i w + mu - Sigma
            G[s, a] = (w[:, None] / (zeta[None, :] - x[:, None])).sum(axis=0) * 2.0 / (ne - 1)
    return G


def scf_diff(G_cl, G_loc, nbath, nw):
    """The convergence measure of dmft.f90:105-134."""
    norb = G_cl.shape[1]
    return float((np.abs(G_cl - G_loc) ** 2).sum() / (norb * nbath * nw))


# ---------------------------------------------------------------------------
# bath fit (ed_projection.f90)
# ---------------------------------------------------------------------------
class BathFit:
    """Cost and gradient of the fit of spin `s` (ed_projection.f90:154-250):
    f(x) = sum_{a,w} |em - em_old + D(x) - D_old + 1/G_loc - 1/G_cl|^2 / w
    / (norb nw), x = (em(1..norb), ek(1..nbath), vmk(iorb fast, ibath))."""

    def __init__(self, em_old, D_old, G_cl, G_loc, omega, s):
        self.norb = D_old.shape[1]
        self.s = s
        self.omega = np.asarray(omega, dtype=float)
        self.wgt = 1.0 / self.omega
        self.em_old = np.asarray(em_old, dtype=float)[:, s].copy()
        # constant part of the difference: - em_old - D_old + 1/G_loc - 1/G_cl
        self.c = -self.em_old[:, None] - D_old[s] + 1.0 / G_loc[s] - 1.0 / G_cl[s]
        self.nw = len(self.omega)

    def split(self, x):
        norb = self.norb
        nbath = (len(x) - norb) // (1 + norb)
        em = x[:norb]
        ek = x[norb:norb + nbath]
        V = x[norb + nbath:].reshape(nbath, norb).T              # V[iorb, ibath]
        return em, ek, V

    def diff(self, x):
        em, ek, V = self.split(x)
        iw = 1j * self.omega
        den = iw[None, :] - ek[:, None]                          # [l, w]
        D = (V[:, :, None] ** 2 / den[None, :, :]).sum(axis=1)   # [a, w]
        return em[:, None] + D + self.c, den, V

    def f(self, x):
        d, _, _ = self.diff(x)
        return float(((np.abs(d) ** 2) * self.wgt[None, :]).sum() / (self.norb * self.nw))

    def df(self, x):
        d, den, V = self.diff(x)
        norb = self.norb
        nbath = V.shape[1]
        g = np.zeros_like(x)
        scale = 1.0 / (norb * self.nw)
        g[:norb] = (2.0 * d.real * self.wgt[None, :]).sum(axis=1) * scale
        cden = np.conj(den)                                      # -i w - e_l
        for l in range(nbath):
            fac = V[:, l][:, None] ** 2 / cden[l][None, :] ** 2                  # dD/de_l, conjugated
            g[norb + l] = (2.0 * (d * fac).real * self.wgt[None, :]).sum() * scale
            fac = 2.0 * V[:, l][:, None] / cden[l][None, :]                      # dD/dV_al, conjugated
            g[norb + nbath + l * norb:norb + nbath + (l + 1) * norb] = \
                (2.0 * (d * fac).real * self.wgt[None, :]).sum(axis=1) * scale
        return g


def _cubic_step(lo, flo, slo, hi, fhi, shi):
    """Minimiser of the cubic that matches value and slope at both ends of
    [lo, hi] (Hermite interpolation); None when that cubic has no interior
    minimum."""
    h = hi - lo
    d1 = slo + shi - 3.0 * (fhi - flo) / h
    disc = d1 * d1 - slo * shi
    if not disc >= 0.0:
        return None
    d2 = math.copysign(math.sqrt(disc), h)
    den = shi - slo + 2.0 * d2
    if den == 0.0:
        return None
    t = hi - h * (shi + d2 - d1) / den
    return t if math.isfinite(t) else None


def line_minimum(phi, f0, s0, t0, rtol=1.0e-10, maxeval=200):
    """Minimum of phi(t) = f(p + t d) over t > 0 for a descent direction
    (slope s0 < 0 at t = 0), from values and slopes: phi(t) -> (f, slope).

    Search: steps grow fourfold from t0 until the slope turns non-negative or
    the value rises above that of the last descending point `lo`, which
    brackets a minimum between `lo` and that point `hi`.  The bracket then shrinks
    around the Hermite-cubic minimiser of its two ends, held to the middle 80%
    of the bracket (else its midpoint), keeping a descending point as `lo`.
    Stops when the slope has fallen below rtol |s0| or the bracket below
    rtol (|t| + rtol).  Returns (t, f, slope) of the lowest point evaluated."""
    lo, flo, slo = 0.0, f0, s0
    best = (0.0, f0, s0)
    t = t0
    hi = None
    n = 0
    while hi is None:
        ft, st = phi(t)
        n += 1
        if not (math.isfinite(ft) and math.isfinite(st)):
            hi, fhi, shi = t, math.inf, math.inf
            break
        if ft < best[1]:
            best = (t, ft, st)
        if st >= 0.0 or ft > flo:
            hi, fhi, shi = t, ft, st
            break
        lo, flo, slo = t, ft, st
        if abs(st) <= rtol * abs(s0):
            return best
        if n >= maxeval:
            raise RuntimeError("line search found no bracket")
        t = 4.0 * t
    while n < maxeval:
        w = hi - lo
        if w <= rtol * (abs(lo) + rtol):
            break
        t = _cubic_step(lo, flo, slo, hi, fhi, shi) if math.isfinite(fhi) else None
        if t is None or not (lo + 0.1 * w <= t <= hi - 0.1 * w):
            t = lo + 0.5 * w
        ft, st = phi(t)
        n += 1
        if ft < best[1]:
            best = (t, ft, st)
        if st < 0.0 and ft <= flo:
            lo, flo, slo = t, ft, st
        else:
            hi, fhi, shi = t, ft, st
        if abs(st) <= rtol * abs(s0) and ft <= best[1]:
            break
    return best


def conjugate_gradient(f, df, p, ftol=1.0e-6, itmax=20000):
    """Nonlinear conjugate gradient with Polak-Ribiere directions, restarted
    along the steepest descent whenever the update coefficient is negative or
    the direction does not descend, and line minimisation by line_minimum.
    Stops when an iteration lowers f by no more than ftol relative to f,
    2 (f_old - f_new) <= ftol (|f_old| + |f_new| + 1e-10 |f_start|), where
    the last term keeps a cost that falls towards zero from needing ever
    smaller steps, or when the gradient vanishes.  Returns (p, iterations,
    f(p))."""
    p = np.array(p, dtype=float)
    fp = float(f(p))
    floor = 1.0e-10 * abs(fp)
    g = np.asarray(df(p), dtype=float)
    d = -g
    step = 1.0
    for it in range(1, itmax + 1):
        s0 = float(g @ d)
        if not s0 < 0.0:                           # not a descent direction: restart
            d = -g
            s0 = float(g @ d)
            if not s0 < 0.0:
                return p, it, fp

        def phi(t):
            q = p + t * d
            return float(f(q)), float(np.asarray(df(q), dtype=float) @ d)

        t, fn, _ = line_minimum(phi, fp, s0, step)
        p = p + t * d
        gn = np.asarray(df(p), dtype=float)
        if 2.0 * (fp - fn) <= ftol * (abs(fp) + abs(fn) + floor):
            return p, it, fn
        beta = max(0.0, float(gn @ (gn - g)) / float(g @ g))
        d = -gn + beta * d
        step = t if t > 0.0 else 1.0
        g, fp = gn, fn
    raise RuntimeError("conjugate gradient did not converge")


def fit_bath(em, ek, vmk, D, G_cl, G_loc, omega, nspin, ftol=1.0e-6):
    """New (em, ek, vmk) (ed_projection.f90:23-101): one fit per spin; with
    nspin 1 spin down copies spin up.  ftol is the conjugate gradient's
    relative stopping tolerance (the reference's 1e-6 by default)."""
    em, ek, vmk = (np.array(a, dtype=float) for a in (em, ek, vmk))
    norb, nbath = vmk.shape[0], vmk.shape[1]
    info = []
    for s in range(nspin):
        bf = BathFit(em, D, G_cl, G_loc, omega, s)
        x0 = np.concatenate([em[:, s], ek[:, s], vmk[:, :, s].T.reshape(-1)])
        x, it, fret = conjugate_gradient(bf.f, bf.df, x0, ftol=ftol)
        em[:, s] = x[:norb]
        ek[:, s] = x[norb:norb + nbath]
        vmk[:, :, s] = x[norb + nbath:].reshape(nbath, norb).T
        info.append((it, fret))
    if nspin == 1:
        em[:, 1], ek[:, 1], vmk[:, :, 1] = em[:, 0], ek[:, 0], vmk[:, :, 0]
    return em, ek, vmk, info


# ---------------------------------------------------------------------------
# the loop
# ---------------------------------------------------------------------------
@dataclass
class DMFTResult:
    em: np.ndarray
    ek: np.ndarray
    vmk: np.ndarray
    D_cl: np.ndarray
    G_cl: np.ndarray
    G_loc: np.ndarray
    iterations: int
    converged: bool
    history: list = field(default_factory=list)


def align_bath_signs(vmk_new, vmk_old):
    """vmk_new with each bath site's couplings (the column vmk[:, l, s]) given
    the sign that best matches vmk_old.  The fit's cost depends on the
    couplings only through products V_a V_b of one site, so a site's overall
    sign is free and the conjugate gradient may return either; linear mixing
    of vmk is only meaningful between columns of the same sign."""
    v = np.array(vmk_new, dtype=float, copy=True)
    old = np.asarray(vmk_old, dtype=float)
    for s in range(v.shape[2]):
        for l in range(v.shape[1]):
            if float(v[:, l, s] @ old[:, l, s]) < 0.0:
                v[:, l, s] = -v[:, l, s]
    return v


def dmft_loop(solve, em, ek, vmk, omega, nbath, nspin=1, nloop=20, scf_tol=1.0e-6, mixing=1.0, hfield=0.0,
              writer=None, fit_ftol=1.0e-6):
    """The DMFT iterations of dmft.f90:55-98 with `solve(em, ek, vmk)` ->
    G_cl[ispin, iorb, iw] as the impurity solver.  mixing mixes the fitted
    parameters with the previous ones (1: the reference's loop); before a
    mixing below 1 the fitted bath sites take the signs of the previous ones
    (align_bath_signs).

    fit_ftol is the bath fit's stopping tolerance.  At the reference's 1e-6
    the fit stops where the cost is flat but the parameters are not settled,
    so after 20 iterations a 1e-11 relative change of G_cl moves D_cl by
    about 1e-4; at 1e-13 the same change moves it by about 1e-7."""
    em, ek, vmk = (np.array(a, dtype=float) for a in (em, ek, vmk))
    omega = np.asarray(omega, dtype=float)
    nw = len(omega)
    hist = []
    D = G_cl = G_loc = None
    converged = False
    it = 0
    for it in range(1, nloop + 1):
        if it > 1:
            em_f, ek_f, vmk_f, info = fit_bath(em, ek, vmk, D, G_cl, G_loc, omega, nspin, fit_ftol)
            if mixing < 1.0:
                vmk_f = align_bath_signs(vmk_f, vmk)
            em = mixing * em_f + (1.0 - mixing) * em
            ek = mixing * ek_f + (1.0 - mixing) * ek
            vmk = mixing * vmk_f + (1.0 - mixing) * vmk
        D = hybridization(ek, vmk, omega, nspin)
        G_cl = solve(em, ek, vmk)
        G_loc = local_green(em, D, G_cl, hfield)
        diff = scf_diff(G_cl, G_loc, nbath, nw)
        hist.append(diff)
        if writer is not None:
            writer(it, em, ek, vmk, D, G_cl, G_loc)
        if diff < scf_tol:
            converged = True
            break
    return DMFTResult(em, ek, vmk, D, G_cl, G_loc, it, converged, hist)


def gpu_solver(pkg, solver, norb, nbath, U, Up, Jex, Jp, mu, sectors, maxnstep, omega, nspin=1, seed=0):
    """Impurity solve on the GPU library for dmft_loop: edzt_set_model +
    edzt_solve with the fixed interaction and sector list."""
    def solve(em, ek, vmk):
        m = pkg.Model(norb, nbath, em, ek, vmk, U=U, Up=Up, Jex=Jex, Jp=Jp, mu=mu)
        solver.set_model(m)
        return solver.solve(sectors, maxnstep, omega, nspin=nspin, seed=seed)["G_cl"]
    return solve


# ---------------------------------------------------------------------------
# self-energy and quasiparticle weight (post_process.f90:39-57, :121-185)
# ---------------------------------------------------------------------------
def self_energy(em, D, G_cl, omega, mu):
    """Sigma[ispin, iorb, iw] = i w + mu - em - D_cl - 1/G_cl."""
    em = np.asarray(em, dtype=float)
    nspin, norb, nw = G_cl.shape
    iw = 1j * np.asarray(omega, dtype=float)
    S = np.zeros_like(G_cl)
    for s in range(nspin):
        for a in range(norb):
            S[s, a] = iw + mu - em[a, s] - D[s, a] - 1.0 / G_cl[s, a]
    return S


def quasiparticle_weight(Sigma, omega, literal=False):
    """Z[iorb, ispin] = 1 / (1 - Im Sigma(i w_1) / w_1).  The reference zeroes
    the whole Sigma array before each (iorb, ispin) of dump_sigma, so the Z it
    prints is 1 for every pair but the last; literal=True reproduces that."""
    nspin, norb, _ = Sigma.shape
    Z = np.ones((norb, nspin))
    for s in range(nspin):
        for a in range(norb):
            if literal and (a, s) != (norb - 1, nspin - 1):
                continue
            Z[a, s] = 1.0 / (1.0 - Sigma[s, a, 0].imag / omega[0])
    return Z


def write_sigma(directory, omega, Sigma):
    """sigma.dat.<iorb>.<ispin>: 'nw iorb ispin', then rows of w, Re/Im Sigma."""
    nspin, norb, nw = Sigma.shape
    for s in range(nspin):
        for a in range(norb):
            with open(os.path.join(directory, f"sigma.dat.{a + 1}.{s + 1}"), "w") as f:
                f.write(f" {nw:11d} {a + 1:11d} {s + 1:11d}\n")
                for i in range(nw):
                    f.write("".join(f"{v:12.8f}" for v in (omega[i], Sigma[s, a, i].real, Sigma[s, a, i].imag)) + "\n")


# ---------------------------------------------------------------------------
# the reference's output files (dump_data.f90:29-83)
# ---------------------------------------------------------------------------
def write_h_imp(path, em, ek, vmk, nspin):
    """h_imp.dat: 'norb nbath nspin', then per spin em, ek and vmk (iorb
    fastest), one value per line."""
    norb, nbath = vmk.shape[0], vmk.shape[1]
    with open(path, "w") as f:
        f.write(f" {norb:11d} {nbath:11d} {nspin:11d}\n")
        for s in range(nspin):
            for a in range(norb):
                f.write(f" {em[a, s]:25.16E}\n")
            for l in range(nbath):
                f.write(f" {ek[l, s]:25.16E}\n")
            for l in range(nbath):
                for a in range(norb):
                    f.write(f" {vmk[a, l, s]:25.16E}\n")


def write_green(directory, omega, D, G_cl, G_loc):
    """green.dat.<iorb>.<ispin>: 'nw iorb ispin', then rows of w, Re/Im D_cl,
    Re/Im G_cl, Re/Im G_loc in 7F12.8."""
    nspin, norb, nw = G_cl.shape
    for s in range(nspin):
        for a in range(norb):
            with open(os.path.join(directory, f"green.dat.{a + 1}.{s + 1}"), "w") as f:
                f.write(f" {nw:11d} {a + 1:11d} {s + 1:11d}\n")
                for i in range(nw):
                    row = (omega[i], D[s, a, i].real, D[s, a, i].imag, G_cl[s, a, i].real, G_cl[s, a, i].imag,
                           G_loc[s, a, i].real, G_loc[s, a, i].imag)
                    f.write("".join(f"{v:12.8f}" for v in row) + "\n")
