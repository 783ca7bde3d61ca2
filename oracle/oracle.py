"""ctypes front end of the CPU oracle (oracle/edzt_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs as the checker; the product never imports it.
Parity status: pinned to the reference's own source through the golden
vectors of tests/golden/ref_golden.npz, which oracle/f90run.py computes by
running the reference's Fortran procedures; see the header of edzt_oracle.c.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None
_lock = threading.Lock()

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (seconds)."""
    src = os.path.join(HERE, "edzt_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "-B", "liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(LIB_PATH)
            L.or_create.restype = C.c_void_p
            L.or_create.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp] + [C.c_double] * 5
            L.or_destroy.argtypes = [C.c_void_p]
            L.or_sector_dim.restype = C.c_longlong
            L.or_sector_dim.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.or_basis.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip]
            L.or_generate_spin_basis.argtypes = [C.c_int, C.c_int, _ip, _ip]
            L.or_icom.argtypes = [C.c_int, C.c_int]
            L.or_hx.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_int]
            L.or_hx_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_longlong, C.c_longlong]
            L.or_apply_c.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp]
            L.or_lanczos_iteration.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _ip, _dp, _dp]
            L.or_tridiag_lowest.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
            L.or_diag_lanczos.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                          _dp, _dp, _dp, _ip, _dp, _dp]
            L.or_ground_state.argtypes = [C.c_void_p, C.c_int, _ip, C.c_int, C.c_uint64, _ip, _dp, _dp,
                                          _dp, _dp]
            L.or_continued_fraction.argtypes = [C.c_double, C.c_double, C.c_int, _dp, _dp, C.c_int, _dp, _dp]
            L.or_green_diag.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_double, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _ip]
            L.or_cluster_green_ftn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, C.c_double,
                                               C.c_int, C.c_int, _dp, _dp, _dp]
            L.or_start_vector.argtypes = [C.c_uint64, C.c_uint64, C.c_longlong, _dp]
            L.or_dot.restype = C.c_double
            L.or_dot.argtypes = [_dp, _dp, C.c_longlong]
            L.or_num_threads.restype = C.c_int
            L.or_set_num_threads.argtypes = [C.c_int]
            _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def set_num_threads(n: int) -> None:
    lib().or_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().or_num_threads())


def spin_basis(nsite: int, n: int):
    """Ascending popcount-n strings and the dense 1-based rank table (ed_basis.f90:76-113)."""
    L = lib()
    cnt = L.or_icom(nsite, n) if 0 <= n <= nsite else 0
    strings = np.zeros(max(cnt, 1), dtype=np.int32)
    idx = np.zeros(1 << nsite, dtype=np.int32)
    got = L.or_generate_spin_basis(nsite, n, _i(strings), _i(idx))
    return strings[:got].copy(), idx


def start_vector(seed: int, stream: int, n: int) -> np.ndarray:
    v = np.empty(max(n, 1), dtype=np.float64)
    lib().or_start_vector(C.c_uint64(seed), C.c_uint64(stream), n, _d(v))
    return v[:n]


def dot(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return float(lib().or_dot(_d(a), _d(b), a.size))


def tridiag_lowest(a: np.ndarray, b: np.ndarray, n: int):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    e0 = C.c_double()
    z = np.zeros(max(n, 1), dtype=np.float64)
    rc = lib().or_tridiag_lowest(n, _d(a), _d(b), C.byref(e0), _d(z))
    if rc != 0:
        raise ValueError("tridiag_lowest failed")
    return e0.value, z[:n]


def continued_fraction(z: complex, n: int, a, b, sign: int) -> complex:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    fr, fi = C.c_double(), C.c_double()
    lib().or_continued_fraction(z.real, z.imag, n, _d(a), _d(b), sign, C.byref(fr), C.byref(fi))
    return complex(fr.value, fi.value)


def matsubara(nw: int, beta: float) -> np.ndarray:
    """omega(i) = (2(i-1)+1) pi / beta, dmft_grid.f90:42-52 (one rank)."""
    return np.array([(2.0 * float(i) + 1.0) * np.pi / beta for i in range(nw)], dtype=np.float64)


class Oracle:
    """One impurity model (em, ek, vmk, U, Up, J, Jp, mu) on the CPU.

    em: (norb, 2); ek: (nbath, 2); vmk: (norb, nbath, 2) — the reference's
    Fortran shapes; stored column-major as the reference lays them out.
    """

    def __init__(self, norb, nbath, em, ek, vmk, U, Up, Jex, Jp, mu):
        self.norb, self.nbath = int(norb), int(nbath)
        self.nsite = self.norb + self.nbath
        self.em = np.asfortranarray(np.asarray(em, dtype=np.float64).reshape(self.norb, 2))
        self.ek = np.asfortranarray(np.asarray(ek, dtype=np.float64).reshape(self.nbath, 2))
        self.vmk = np.asfortranarray(np.asarray(vmk, dtype=np.float64).reshape(self.norb, self.nbath, 2))
        self.U, self.Up, self.Jex, self.Jp, self.mu = map(float, (U, Up, Jex, Jp, mu))
        emf = np.ascontiguousarray(self.em.ravel(order="F"))
        ekf = np.ascontiguousarray(self.ek.ravel(order="F"))
        vmf = np.ascontiguousarray(self.vmk.ravel(order="F"))
        self._h = lib().or_create(self.norb, self.nbath, _d(emf), _d(ekf), _d(vmf),
                                  self.U, self.Up, self.Jex, self.Jp, self.mu)
        if not self._h:
            raise ValueError("or_create rejected the model")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.or_destroy(h)
            self._h = None

    def model_dict(self) -> dict:
        return dict(norb=self.norb, nbath=self.nbath, em=self.em.tolist(), ek=self.ek.tolist(),
                    vmk=self.vmk.tolist(), U=self.U, Up=self.Up, Jex=self.Jex, Jp=self.Jp, mu=self.mu)

    def dim(self, ne_up: int, ne_dn: int) -> int:
        return int(lib().or_sector_dim(self._h, ne_up, ne_dn))

    def basis(self, ne_up: int, ne_dn: int):
        nup = lib().or_icom(self.nsite, ne_up)
        ndn = lib().or_icom(self.nsite, ne_dn)
        up = np.zeros(max(nup, 1), dtype=np.int32)
        dn = np.zeros(max(ndn, 1), dtype=np.int32)
        if lib().or_basis(self._h, ne_up, ne_dn, _i(up), _i(dn)) != 0:
            raise ValueError("bad sector")
        return up[:nup].copy(), dn[:ndn].copy()

    def hx(self, ne_up: int, ne_dn: int, x: np.ndarray, y: np.ndarray | None = None, py: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.array(y, dtype=np.float64, copy=True) if (py and y is not None) else np.zeros_like(x)
        if lib().or_hx(self._h, ne_up, ne_dn, _d(x), _d(out), 1 if py else 0) != 0:
            raise ValueError("bad sector")
        return out

    def hx_rows(self, ne_up: int, ne_dn: int, x: np.ndarray, r0: int, r1: int) -> np.ndarray:
        """Rows [r0, r1) of H x (for spot checks of sectors too large for a full CPU H.v)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(x.size)
        if lib().or_hx_rows(self._h, ne_up, ne_dn, _d(x), _d(y), r0, r1) != 0:
            raise ValueError("bad sector")
        return y[r0:r1].copy()

    def apply_c(self, ne_up, ne_dn, vec, pm, iorb, ispin):
        vec = np.ascontiguousarray(vec, dtype=np.float64)
        d = 1 if pm == 1 else -1
        oup = ne_up + (d if ispin == 1 else 0)
        odn = ne_dn + (d if ispin == 2 else 0)
        n = self.dim(oup, odn)
        out = np.zeros(max(n, 1), dtype=np.float64)
        rc = lib().or_apply_c(self._h, ne_up, ne_dn, _d(vec), pm, iorb, ispin, _d(out))
        if rc < 0:
            raise ValueError("bad apply_c arguments")
        return out[:n]

    def lanczos_iteration(self, ne_up, ne_dn, v_init, maxnstep):
        v_init = np.ascontiguousarray(v_init, dtype=np.float64)
        a = np.zeros(maxnstep)
        b = np.zeros(maxnstep)
        nstep = C.c_int()
        if lib().or_lanczos_iteration(self._h, ne_up, ne_dn, _d(v_init), maxnstep, C.byref(nstep),
                                      _d(a), _d(b)) != 0:
            raise ValueError("bad sector")
        return nstep.value, a, b

    def diag_lanczos(self, ne_up, ne_dn, maxnstep, seed=0, stream=0, want_vec=True):
        n = self.dim(ne_up, ne_dn)
        ev = C.c_double()
        res = C.c_double()
        vec = np.zeros(n) if want_vec else None
        nstep = C.c_int()
        a = np.zeros(maxnstep)
        b = np.zeros(maxnstep)
        rc = lib().or_diag_lanczos(self._h, ne_up, ne_dn, maxnstep, C.c_uint64(seed), C.c_uint64(stream),
                                   C.byref(ev), _d(vec), C.byref(res), C.byref(nstep), _d(a), _d(b))
        if rc != 0:
            raise ValueError("diag_lanczos failed")
        return dict(e0=ev.value, vec=vec, residual=res.value, nstep=nstep.value, a=a, b=b)

    def ground_state(self, sectors, maxnstep, seed=0):
        sec = np.ascontiguousarray(np.asarray(sectors, dtype=np.int32).reshape(-1, 2))
        maxdim = max(self.dim(int(u), int(d)) for u, d in sec)
        vec = np.zeros(max(maxdim, 1))
        es = np.zeros(len(sec))
        isec = C.c_int()
        e0 = C.c_double()
        res = C.c_double()
        rc = lib().or_ground_state(self._h, len(sec), _i(sec), maxnstep, C.c_uint64(seed), C.byref(isec),
                                   C.byref(e0), _d(vec), _d(es), C.byref(res))
        if rc != 0:
            raise ValueError("ground_state failed")
        u, d = sec[isec.value]
        return dict(isector=isec.value, e0=e0.value, vec=vec[: self.dim(int(u), int(d))].copy(),
                    e_sector=es, residual=res.value, sector=(int(u), int(d)))

    def green_diag(self, ne_up, ne_dn, gsvec, e0, iorb, ispin, maxnstep, omega):
        gsvec = np.ascontiguousarray(gsvec, dtype=np.float64)
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        nw = omega.size
        ap, bp, am, bm = (np.zeros(maxnstep) for _ in range(4))
        g = np.zeros(2 * nw)
        ns = np.zeros(2, dtype=np.int32)
        rc = lib().or_green_diag(self._h, ne_up, ne_dn, _d(gsvec), e0, iorb, ispin, maxnstep, nw, _d(omega),
                                 _d(ap), _d(bp), _d(am), _d(bm), _d(g), _i(ns))
        if rc != 0:
            raise ValueError("green_diag failed")
        return dict(g=g[0::2] + 1j * g[1::2], ap=ap, bp=bp, am=am, bm=bm, nstep=(int(ns[0]), int(ns[1])))

    def cluster_green_ftn(self, nspin, ne_up, ne_dn, gsvec, e0, maxnstep, omega):
        gsvec = np.ascontiguousarray(gsvec, dtype=np.float64)
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        nw = omega.size
        G = np.zeros(2 * nw * self.norb * nspin)
        coeffs = np.zeros(self.norb * 2 * 4 * maxnstep)
        lib().or_cluster_green_ftn(self._h, nspin, ne_up, ne_dn, _d(gsvec), e0, maxnstep, nw, _d(omega),
                                   _d(G), _d(coeffs))
        Gc = (G[0::2] + 1j * G[1::2]).reshape(nspin, self.norb, nw)   # (ispin, iorb, iw)
        return dict(G_cl=Gc, coeffs=coeffs.reshape(self.norb, 2, 4, maxnstep))

    def occupancy(self, ne_up, ne_dn, gsvec, nspin):
        """occ[ispin][iorb] and docc[iorb] of a ground state
        (post_process.f90:62-112): |x_i|^2 summed over the states whose
        orbital bit is set (both spins for docc)."""
        up, dn = self.basis(ne_up, ne_dn)
        up = np.asarray(up, dtype=np.int64)
        dn = np.asarray(dn, dtype=np.int64)
        w = (np.asarray(gsvec, dtype=np.float64) ** 2).reshape(len(dn), len(up))
        occ = np.zeros((nspin, self.norb))
        docc = np.zeros(self.norb)
        for a in range(self.norb):
            bu = ((up >> a) & 1).astype(bool)
            bd = ((dn >> a) & 1).astype(bool)
            occ[0, a] = w[:, bu].sum()
            if nspin == 2:
                occ[1, a] = w[bd, :].sum()
            docc[a] = w[np.ix_(bd, bu)].sum()
        return occ, docc

    def green_run(self, v_init, nu, nd, pm, e0, maxnstep, omega):
        """One c^+ (pm=1) or c (pm=2) run of green_diag (dmft_green.f90:204-257)
        from an explicit start vector in sector (nu, nd): Lanczos, b(1) =
        |v_init|, continued fraction on E0 + i w (c^+) or -E0 + i w (c)."""
        n, a, b = self.lanczos_iteration(nu, nd, v_init, maxnstep)
        g = np.zeros(len(omega), dtype=complex)
        if n < 1:
            return g
        b = b.copy()
        b[0] = np.sqrt(dot(v_init, v_init))
        nl = 2 if (n == 1 and maxnstep >= 2) else n
        for i, w in enumerate(omega):
            if pm == 1:
                g[i] = continued_fraction(complex(e0, w), nl, a, b, -1)
            else:
                g[i] = continued_fraction(complex(-e0, w), nl, a, b, +1)
        return g

    def cluster_green_matrix(self, nspin, ne_up, ne_dn, gsvec, e0, maxnstep, omega):
        """The full G_ab(ispin, a, b, iw): the diagonal as cluster_green_ftn,
        G_ab = (G_(a+b) - G_aa - G_bb) / 2 with G_(a+b) from runs on
        (c_a + c_b)^(+)|gs> (an extension beyond the reference, which
        computes the diagonal only, dmft_green.f90:71-121)."""
        norb = self.norb
        even = not (nspin == 2 or ne_up != ne_dn)
        nsp = 1 if even else 2
        gm = np.zeros((nsp, norb, norb, len(omega)), dtype=complex)

        def exc(pm, ispin):
            d = 1 if pm == 1 else -1
            return ne_up + (d if ispin == 1 else 0), ne_dn + (d if ispin == 2 else 0)

        def start(pm, orbs, ispin):
            v = None
            for a in orbs:
                w = self.apply_c(ne_up, ne_dn, gsvec, pm, a, ispin)
                v = w if v is None else v + w
            return v

        for sp in range(nsp):
            for a in range(norb):
                for pm in (1, 2):
                    nu, nd = exc(pm, sp + 1)
                    if self.dim(nu, nd) > 0:
                        gm[sp, a, a] += self.green_run(start(pm, [a + 1], sp + 1), nu, nd, pm, e0, maxnstep, omega)
            for a in range(norb):
                for b in range(a + 1, norb):
                    gab = np.zeros(len(omega), dtype=complex)
                    for pm in (1, 2):
                        nu, nd = exc(pm, sp + 1)
                        if self.dim(nu, nd) > 0:
                            gab += self.green_run(start(pm, [a + 1, b + 1], sp + 1), nu, nd, pm, e0, maxnstep,
                                                  omega)
                    gm[sp, a, b] = gm[sp, b, a] = 0.5 * (gab - gm[sp, a, a] - gm[sp, b, b])
        if even:
            return np.repeat(gm, nspin, axis=0)
        if nspin == 1:
            return 0.5 * (gm[0:1] + gm[1:2])
        return gm

    def diag_arpack(self, ne_up, ne_dn, seed=0, stream=0):
        """diag_arpack (src/arpack_solver.f90:19-124) through ARPACK itself:
        scipy's eigsh wraps ARPACK's dsaupd/dseupd, the serial form of the
        reference's pdsaupd/pdseupd, here with the reference's settings
        (nev 3, ncv 6, which 'SA', tol 0, maxitr 20000) on this oracle's hx
        and the library's start vector (ARPACK would draw its own)."""
        from scipy.sparse.linalg import LinearOperator, eigsh
        n = self.dim(ne_up, ne_dn)
        op = LinearOperator((n, n), matvec=lambda x: self.hx(ne_up, ne_dn, np.ascontiguousarray(x, dtype=float)),
                            dtype=float)
        w, v = eigsh(op, k=3, ncv=6, which="SA", tol=0.0, maxiter=20000,
                     v0=start_vector(seed, stream, n))
        order = np.argsort(w)
        w, v = w[order], v[:, order]
        resid = np.array([np.linalg.norm(self.hx(ne_up, ne_dn, v[:, i].copy()) - w[i] * v[:, i]) for i in range(3)])
        return dict(e0=float(w[0]), vec=v[:, 0].copy(), ritz=w, resid=resid)

    def ground_state_arpack(self, sectors, seed=0):
        """ground_state with diag_solver = 2 (ground_state.f90:53-68): the
        lowest diag_arpack energy over the sectors, sector i on stream i."""
        best = None
        es = np.full(len(sectors), np.nan)
        for i, (u, d) in enumerate(sectors):
            if self.dim(u, d) <= 0:
                continue
            r = self.diag_arpack(u, d, seed, i)
            es[i] = r["e0"]
            if best is None or r["e0"] < best[1] - 1e-10 * max(1.0, abs(best[1])):
                best = (i, r["e0"], r["vec"])
        i, e0, vec = best
        return dict(isector=i, e0=e0, vec=vec, e_sector=es, sector=tuple(int(x) for x in sectors[i]))

    def dense_h(self, ne_up, ne_dn) -> np.ndarray:
        """H assembled column by column from hx (the idea of debug.f90:13-57)."""
        n = self.dim(ne_up, ne_dn)
        H = np.zeros((n, n))
        e = np.zeros(n)
        for j in range(n):
            e[:] = 0.0
            e[j] = 1.0
            H[:, j] = self.hx(ne_up, ne_dn, e)
        return H
