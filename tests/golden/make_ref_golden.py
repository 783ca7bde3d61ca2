"""Generate tests/golden/ref_golden.npz: golden vectors computed by the
reference's own Fortran source.

The reference (yw-choi/DMFT-ED-ZT) cannot be compiled here (no Fortran
compiler).  oracle/f90run.py translates its hot-path procedures statement by
statement into Python and runs them, so every value below comes from the
reference's source text:

  src/ed_basis.f90          generate_basis, ed_basis_get, ed_basis_idx
  src/numeric_utils.f90     icom, mpi_dot_product, mpi_norm, continued_fraction_p/m
  src/impurity_hamiltonian.f90  hx, sgn, sgn2
  src/ed_operator.f90       apply_c, sgn
  src/lanczos_solver.f90    diag_lanczos, lanczos_iteration, lanczos_diagonalize,
                            lanczos_ground_state
  src/ground_state.f90      ground_state
  src/dmft_green.f90        cluster_green_ftn, green_diag

with the external libraries supplied as oracle/f90run.py states (MPI with one
rank, Netlib daxpy, LAPACK's tridiagonal eigensolver for MKL's dstevx, and the
start vectors through the random_number hook: the hash stream the library and
the oracle use, since the reference's generator is unseeded).

Recorded cases (seeded inputs):
  basis_<nsite>_<n>            generate_basis strings (ascending)
  hx_<case>_{x,y,y0,yacc}      y = H x (py false) and y0 + H x (py true)
  applyc_<case>_<pm><iorb><ispin>   apply_c of x_<case>
  lz_<case>_{v,a,b,nstep}      lanczos_iteration from v
  gs_{isector,e0,vec}          ground_state over 9 sectors of the nsite-6 Bethe model
  G_{omega,double,literal}     cluster_green_ftn on 32 Matsubara points:
                               `double` with z = dcmplx(E0, w); `literal` with
                               the reference's cmplx(E0, w), which Fortran makes
                               single precision (dmft_green.f90:223,253)
  src_sha256                   SHA-256 of every reference file read
Run from the repository root (needs the reference tree at /root/reference):
    python tests/golden/make_ref_golden.py
"""

from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import f90run as F          # noqa: E402
from oracle import oracle as O          # noqa: E402

REF = os.environ.get("EDZT_REFERENCE_SRC", "/root/reference/src")
OUT = os.path.join(HERE, "ref_golden.npz")
FILES = ["mpi.f90", "dmft_params.f90", "constants.f90", "io_units.f90", "timer.f90", "dmft_grid.f90",
         "eigpair.f90", "numeric_utils.f90", "ed_basis.f90", "impurity_hamiltonian.f90", "ed_operator.f90",
         "lanczos_solver.f90", "ground_state.f90", "dmft_green.f90"]
ONLY = {"mpi": [], "dmft_params": [], "constants": [], "io_units": [], "timer": [], "dmft_grid": [], "eigpair": [],
        "numeric_utils": ["icom", "ip", "ifact", "mpi_dot_product", "mpi_norm", "continued_fraction_p",
                          "continued_fraction_m"],
        "ed_basis": ["generate_basis", "ed_basis_get", "ed_basis_idx", "get_bitidx", "dealloc_basis"],
        "impurity_hamiltonian": ["hx", "sgn", "sgn2"], "ed_operator": ["apply_c", "sgn"],
        "lanczos_solver": ["diag_lanczos", "lanczos_iteration", "lanczos_diagonalize", "lanczos_ground_state"],
        "dmft_green": ["cluster_green_ftn", "green_diag"], "": ["ground_state"]}


def farr(a, kind="real"):
    a = np.asarray(a)
    fa = F.FArray([(1, n) for n in a.shape], kind)
    conv = int if kind == "integer" else float
    fa.d = [conv(v) for v in a.flatten(order="F")]
    return fa


class Ref:
    """The reference's procedures for one impurity model (module globals of
    dmft_params set as its FDF input would)."""

    def __init__(self, norb, nbath, em, ek, vmk, U, Up, Jex, Jp, mu, maxnstep=60, double_z=False):
        self.P = P = F.Program()
        for f in FILES:
            P.load(os.path.join(REF, f), only=ONLY)
        if double_z:                       # z = cmplx(E0, w) kept in double precision
            P.intr.cmplx = staticmethod(F.Intrinsics.dcmplx)
        P.init_scopes()
        P.module_vars("mpi").update(nprocs=1, taskid=0, mpierr=0, comm=0, master=True)
        P.module_vars("dmft_params").update(norb=norb, nbath=nbath, nsite=norb + nbath, u=U, up=Up, jex=Jex, jp=Jp,
                                            mu=mu, maxnstep=maxnstep, nspin=1, diag_solver=1, hfield=0.0)
        self.norb, self.nbath = norb, nbath
        self.em, self.ek, self.vmk = farr(em), farr(ek), farr(vmk)

    def basis(self, nu, nd):
        b = self.P.new_type("basis_t")
        self.P.proc("generate_basis", "ed_basis")(nu, nd, b)
        return b

    def hx(self, nu, nd, x, y0=None):
        b = self.basis(nu, nd)
        y = farr(y0) if y0 is not None else F.FArray([(1, b.nloc)], "real")
        xall = F.FArray([(1, b.ntot)], "real")
        self.P.proc("hx", "impurity_hamiltonian")(self.em, self.ek, self.vmk, b, farr(x), y, xall, y0 is not None)
        return np.array(y.d)

    def apply_c(self, nu, nd, x, pm, iorb, ispin):
        b = self.basis(nu, nd)
        d = 1 if pm == 1 else -1
        bo = self.basis(nu + (d if ispin == 1 else 0), nd + (d if ispin == 2 else 0))
        out = F.FArray([(1, bo.nloc)], "real")
        self.P.proc("apply_c", "ed_operator")(b, farr(x), pm, iorb, ispin, bo, out)
        return np.array(out.d)

    def lanczos_iteration(self, nu, nd, v, maxnstep):
        self.P.module_vars("dmft_params")["maxnstep"] = maxnstep
        b = self.basis(nu, nd)
        a, bb = F.FArray([(1, maxnstep)], "real"), F.FArray([(1, maxnstep)], "real")
        r = self.P.proc("lanczos_iteration", "lanczos_solver")(self.em, self.ek, self.vmk, b, farr(v), 0, a, bb)
        return r[0], np.array(a.d), np.array(bb.d)

    def solve(self, sectors, maxnstep, omega, seed=0):
        """ground_state over `sectors` (start vector of sector i: the hash
        stream i of `seed`), then cluster_green_ftn with nspin 1."""
        P = self.P
        pv = P.module_vars("dmft_params")
        pv["maxnstep"] = maxnstep
        S = F.FArray([(1, len(sectors)), (1, 3)], "integer")
        for i, (u, d) in enumerate(sectors):
            S.d[S.off((i + 1, 1))], S.d[S.off((i + 1, 2))] = u, d
        pv.update(nsector=len(sectors), sectors=S)
        P.module_vars("dmft_grid").update(nwloc=len(omega), omega=farr(omega))
        st = {"sector": -1, "i": 0, "v": None}

        def hook(ev):
            if ev == "seed":                       # diag_lanczos calls random_seed once per sector
                st["sector"] += 1
                st["i"] = 0
                st["v"] = None
                return None
            if st["v"] is None:
                st["v"] = O.start_vector(seed, st["sector"], 1 << 20)
            v = float(st["v"][st["i"]])
            st["i"] += 1
            return v
        P.ext.random_hook = hook
        gs = P.new_type("eigpair_t")
        P.proc("ground_state")(self.em, self.ek, self.vmk, gs)
        G = F.FArray([(1, len(omega)), (1, self.norb), (1, 1)], "complex")
        P.proc("cluster_green_ftn", "dmft_green")(self.em, self.ek, self.vmk, gs, G)
        return gs.isector, gs.val, np.array(gs.vec.d), np.array(G.d).reshape(len(omega), self.norb, order="F")


def model(rng, norb, nbath, J=0.0, spin_dep=False):
    em = rng.uniform(-0.5, 0.5, (norb, 2))
    ek = rng.uniform(-2.0, 2.0, (nbath, 2))
    V = rng.uniform(0.1, 1.0, (norb, nbath, 2))
    if not spin_dep:
        em[:, 1], ek[:, 1], V[:, :, 1] = em[:, 0], ek[:, 0], V[:, :, 0]
    U = float(rng.uniform(1.0, 4.0))
    Up, Jp = U - 2.0 * J, J
    mu = U / 2 + (norb - 1) * (2 * Up - J) / 2
    return dict(norb=norb, nbath=nbath, em=em, ek=ek, vmk=V, U=U, Up=Up, Jex=J, Jp=Jp, mu=mu)


def params_array(m):
    return np.concatenate([[m["norb"], m["nbath"], m["U"], m["Up"], m["Jex"], m["Jp"], m["mu"]],
                           m["em"].ravel(order="F"), m["ek"].ravel(order="F"), m["vmk"].ravel(order="F")])


# (name, model seed, norb, nbath, J, spin-dependent, sector, apply_c operators)
HX_CASES = [
    ("o1n6", 11, 1, 5, 0.0, False, (3, 3), [(1, 1, 1), (2, 1, 2)]),
    ("o1n8s", 12, 1, 7, 0.0, True, (4, 3), [(1, 1, 2), (2, 1, 1)]),
    ("o2n6", 13, 2, 4, 0.5, True, (3, 3), [(1, 1, 1), (2, 2, 2), (1, 2, 1), (2, 1, 2)]),
    ("o3n6", 14, 3, 3, 0.4, False, (3, 3), [(1, 3, 2), (2, 2, 1)]),
    ("o2n8", 15, 2, 6, 0.3, False, (4, 4), [(1, 2, 2)]),
]
LZ_CASES = [("o1n8", 21, 1, 7, 0.0, False, (4, 4), 50), ("o2n6", 22, 2, 4, 0.5, True, (3, 3), 40)]


def main():
    t0 = time.time()
    out = {}
    # basis strings
    for ns in (4, 6, 8, 10):
        P = Ref(1, ns - 1, np.zeros((1, 2)), np.zeros((ns - 1, 2)), np.zeros((1, ns - 1, 2)), 1.0, 1.0, 0.0, 0.0, 0.5)
        for n in range(0, ns + 1):
            b = P.basis(n, n)
            out[f"basis_{ns}_{n}"] = np.array(b.up.d, dtype=np.int64)
    # H.v and apply_c
    for name, seed, norb, nbath, J, sd, (nu, nd), ops in HX_CASES:
        rng = np.random.default_rng(seed)
        m = model(rng, norb, nbath, J, sd)
        ref = Ref(**m)
        dim = O.Oracle(m["norb"], m["nbath"], m["em"], m["ek"], m["vmk"], m["U"], m["Up"], m["Jex"], m["Jp"],
                       m["mu"]).dim(nu, nd)
        x = rng.uniform(-1.0, 1.0, dim)
        y0 = rng.uniform(-1.0, 1.0, dim)
        out[f"model_{name}"] = params_array(m)
        out[f"sector_{name}"] = np.array([nu, nd])
        out[f"hx_{name}_x"] = x
        out[f"hx_{name}_y"] = ref.hx(nu, nd, x)
        out[f"hx_{name}_y0"] = y0
        out[f"hx_{name}_yacc"] = ref.hx(nu, nd, x, y0)
        for pm, iorb, ispin in ops:
            out[f"applyc_{name}_{pm}{iorb}{ispin}"] = ref.apply_c(nu, nd, x, pm, iorb, ispin)
        print(name, dim, f"{time.time() - t0:.1f}s", flush=True)
    # Lanczos coefficients
    for name, seed, norb, nbath, J, sd, (nu, nd), steps in LZ_CASES:
        rng = np.random.default_rng(seed)
        m = model(rng, norb, nbath, J, sd)
        ref = Ref(**m)
        dim = O.Oracle(m["norb"], m["nbath"], m["em"], m["ek"], m["vmk"], m["U"], m["Up"], m["Jex"], m["Jp"],
                       m["mu"]).dim(nu, nd)
        v = O.start_vector(seed, 0, dim)
        n, a, b = ref.lanczos_iteration(nu, nd, v, steps)
        out[f"lzmodel_{name}"] = params_array(m)
        out[f"lz_{name}_sector"] = np.array([nu, nd])
        out[f"lz_{name}_v"] = v
        out[f"lz_{name}_nstep"] = np.array([n])
        out[f"lz_{name}_a"] = a
        out[f"lz_{name}_b"] = b
        print("lanczos", name, dim, f"{time.time() - t0:.1f}s", flush=True)
    # ground state and Green's function of the nsite-6 Bethe model (60 steps, 9 sectors)
    em, ek, V = np.zeros((1, 2)), np.stack([np.linspace(-1.0, 1.0, 5)] * 2, 1), np.full((1, 5, 2), 0.5)
    sectors = [(u, d) for u in (2, 3, 4) for d in (2, 3, 4)]
    omega = O.matsubara(32, 100.0)
    for double_z, key in ((True, "double"), (False, "literal")):
        ref = Ref(1, 5, em, ek, V, 2.0, 2.0, 0.0, 0.0, 1.0, maxnstep=60, double_z=double_z)
        isec, e0, vec, G = ref.solve(sectors, 60, omega, seed=0)
        out[f"G_{key}"] = G[:, 0]
        if double_z:
            out["gs_isector"] = np.array([isec])
            out["gs_e0"] = np.array([e0])
            out["gs_vec"] = vec
        print("solve", key, f"{time.time() - t0:.1f}s", flush=True)
    out["gs_sectors"] = np.array(sectors)
    out["G_omega"] = omega
    out["src_files"] = np.array(FILES)
    out["src_sha256"] = np.array([hashlib.sha256(open(os.path.join(REF, f), "rb").read()).hexdigest() for f in FILES])
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, f"{time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
