"""Literal pure-Python transliteration of the reference's basis, hx and apply_c.

TEST INFRASTRUCTURE ONLY (a second, independent restatement used to check the
C oracle in oracle/edzt_oracle.c on small sectors; never imported by the
product).  It keeps the reference's own representation: one integer Fock
state ``up + 2**nsite * down`` (src/ed_basis.f90:135), BTEST/IBSET/IBCLR on
that integer, 1-based loops, and the same floating-point evaluation order, so
its H.v must agree with the C oracle bit for bit.  Python integers do not
overflow, so this also covers nsite = 16.  Pure-Python loops: keep sectors to
a few thousand states.
"""

from __future__ import annotations

import math


def btest(i: int, k: int) -> bool:
    return (i >> k) & 1 == 1


def ibset(i: int, k: int) -> int:
    return i | (1 << k)


def ibclr(i: int, k: int) -> int:
    return i & ~(1 << k)


def icom(n: int, m: int) -> int:
    """numeric_utils.f90:207-222 (binomial)."""
    return math.comb(n, m)


class Basis:
    """basis_t (ed_basis.f90:19-37) for one rank (nloc = ntot)."""

    def __init__(self, nsite: int, ne_up: int, ne_down: int):
        # generate_basis, ed_basis.f90:42-114
        self.nsite = nsite
        self.ne_up = ne_up
        self.ne_down = ne_down
        self.nup = icom(nsite, ne_up)
        self.ndown = icom(nsite, ne_down)
        self.ntot = self.nup * self.ndown
        self.up: list[int] = []
        self.down: list[int] = []
        self.idx_up: dict[int, int] = {}
        self.idx_down: dict[int, int] = {}
        for ispin, n in ((1, ne_up), (2, ne_down)):
            minrange = sum(2 ** (i - 1) for i in range(1, n + 1))        # :81-84
            maxrange = sum(2 ** (nsite - i) for i in range(1, n + 1))
            counts = 0
            for i in range(minrange, maxrange + 1):                      # :94-112
                nbit = sum(1 for j in range(nsite) if btest(i, j))
                if nbit == n:
                    counts += 1
                    if ispin == 1:
                        self.up.append(i)
                        self.idx_up[i] = counts
                    else:
                        self.down.append(i)
                        self.idx_down[i] = counts

    def get(self, idx: int) -> int:
        """ed_basis_get, ed_basis.f90:122-136 (1-based idx)."""
        iup = (idx - 1) % self.nup + 1
        idown = (idx - 1) // self.nup + 1
        return self.up[iup - 1] + 2 ** self.nsite * self.down[idown - 1]

    def idx(self, state: int) -> int:
        """ed_basis_idx, ed_basis.f90:139-151 (1-based result)."""
        u = state % (2 ** self.nsite)
        d = state // (2 ** self.nsite)
        return (self.idx_down[d] - 1) * self.nup + self.idx_up[u]


def _sgn(state: int, i: int, j: int) -> int:
    """impurity_hamiltonian.f90:249-260."""
    s = 1
    for k in range(i, j):
        if btest(state, k - 1):
            s = -s
    return s


def _sgn2(state: int, i: int, j: int, nsite: int) -> int:
    """impurity_hamiltonian.f90:262-276."""
    s = 1
    for k in range(i, j):
        if btest(state, k - 1):
            s = -s
        if btest(state, nsite + k - 1):
            s = -s
    return s


def hx(model: dict, basis: Basis, x, py: bool = False, y=None):
    """hx, impurity_hamiltonian.f90:77-247.

    model: norb, nbath, em[norb][2], ek[nbath][2], vmk[norb][nbath][2],
    U, Up, Jex, Jp, mu (0-based nested lists, values as in the Fortran).
    """
    norb, nbath = model["norb"], model["nbath"]
    nsite = norb + nbath
    em, ek, vmk = model["em"], model["ek"], model["vmk"]
    U, Up, Jex, Jp, mu = model["U"], model["Up"], model["Jex"], model["Jp"], model["mu"]
    out = list(y) if (py and y is not None) else [0.0] * basis.ntot
    for b in range(1, basis.ntot + 1):                                   # :98
        bra = basis.get(b)
        rowsum = 0.0
        xb = x[b - 1]
        for iorb in range(1, norb + 1):
            ni = [1 if btest(bra, iorb - 1) else 0, 1 if btest(bra, nsite + iorb - 1) else 0]
            rowsum = rowsum + ((em[iorb - 1][0] - mu) * ni[0]
                               + (em[iorb - 1][1] - mu) * ni[1]
                               + U * ni[0] * ni[1]) * xb                  # :119-121
            for jorb in range(iorb + 1, norb + 1):                       # :126-141
                nj = [1 if btest(bra, jorb - 1) else 0, 1 if btest(bra, nsite + jorb - 1) else 0]
                rowsum = rowsum + ((Up - Jex) * (ni[0] * nj[0] + ni[1] * nj[1])
                                   + Up * (ni[0] * nj[1] + ni[1] * nj[0])) * xb
            for ispin in (1, 2):                                         # :146-174
                for jbath in range(1, nbath + 1):
                    v = vmk[iorb - 1][jbath - 1][ispin - 1]
                    if abs(v) < 1.0e-16:
                        continue
                    isite = (ispin - 1) * nsite + iorb
                    jsite = (ispin - 1) * nsite + norb + jbath
                    jb = btest(bra, jsite - 1)
                    if ni[ispin - 1] == 0 and jb:
                        ket = ibset(ibclr(bra, jsite - 1), isite - 1)
                        a = basis.idx(ket)
                        rowsum = rowsum + float(_sgn(bra, isite, jsite)) * v * x[a - 1]
                    elif ni[ispin - 1] != 0 and not jb:
                        ket = ibset(ibclr(bra, isite - 1), jsite - 1)
                        a = basis.idx(ket)
                        rowsum = rowsum - float(_sgn(bra, isite, jsite)) * v * x[a - 1]
            for jorb in range(1, norb + 1):                              # :179-226
                if iorb == jorb:
                    continue
                nj = [1 if btest(bra, jorb - 1) else 0, 1 if btest(bra, nsite + jorb - 1) else 0]
                imin, imax = min(iorb, jorb), max(iorb, jorb)
                if ni[0] == 0 and nj[0] != 0 and nj[1] == 0 and ni[1] != 0:
                    ket = ibclr(bra, nsite + iorb - 1)
                    ket = ibset(ket, nsite + jorb - 1)
                    ket = ibclr(ket, jorb - 1)
                    ket = ibset(ket, iorb - 1)
                    a = basis.idx(ket)
                    rowsum = rowsum - float(_sgn2(bra, imin, imax, nsite)) * Jp * x[a - 1]
                if ni[0] == 0 and ni[1] == 0 and nj[0] != 0 and nj[1] != 0:
                    ket = ibclr(bra, nsite + jorb - 1)
                    ket = ibset(ket, nsite + iorb - 1)
                    ket = ibclr(ket, jorb - 1)
                    ket = ibset(ket, iorb - 1)
                    a = basis.idx(ket)
                    rowsum = rowsum + float(_sgn2(bra, imin, imax, nsite)) * Jp * x[a - 1]
        for jbath in range(1, nbath + 1):                                # :232-239
            if btest(bra, norb + jbath - 1):
                rowsum = rowsum + ek[jbath - 1][0] * xb
            if btest(bra, nsite + norb + jbath - 1):
                rowsum = rowsum + ek[jbath - 1][1] * xb
        if py:
            out[b - 1] = out[b - 1] + rowsum
        else:
            out[b - 1] = rowsum
    return out


def apply_c(nsite: int, basis: Basis, vec, pm: int, iorb: int, ispin: int, basis_out: Basis):
    """apply_c, ed_operator.f90:13-57."""
    out = [0.0] * basis_out.ntot
    for i in range(1, basis_out.ntot + 1):
        basis_i = basis_out.get(i)
        isite = (ispin - 1) * nsite + iorb
        ssum = sum(1 for k in range(1, isite) if btest(basis_i, k - 1))   # sgn(basis_i,1,isite-1)
        sgntot = -1 if ssum % 2 else 1
        if pm == 1:
            if not btest(basis_i, isite - 1):
                sgntot = 0
            basis_j = ibclr(basis_i, isite - 1)
        else:
            if btest(basis_i, isite - 1):
                sgntot = 0
            basis_j = ibset(basis_i, isite - 1)
        if sgntot == 0:
            continue
        j = basis.idx(basis_j)
        out[i - 1] = out[i - 1] + vec[j - 1] * sgntot
    return out
