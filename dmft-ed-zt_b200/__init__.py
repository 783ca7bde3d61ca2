"""B200 (sm_100a) zero-temperature ED impurity solver: Python host mirror.

A thin ctypes front end over the C ABI in include/edzt.h (libedzt.so, built
in this directory).  The classes and methods mirror the Fortran procedures
of the reference (yw-choi/DMFT-ED-ZT) that the library replaces:

  generate_basis      src/ed_basis.f90:42-114
  hx                  src/impurity_hamiltonian.f90:77-247
  apply_c             src/ed_operator.f90:13-57
  lanczos_iteration   src/lanczos_solver.f90:92-173
  diag_lanczos        src/lanczos_solver.f90:20-90
  diag_arpack         src/arpack_solver.f90:19-124
  ground_state        src/ground_state.f90:1-81
  green_diag          src/dmft_green.f90:177-260
  cluster_green_ftn   src/dmft_green.f90:47-126

Errors raise EDError carrying the library's status code (the reference
aborts through die()).  There is no CPU fallback: if libedzt.so or a CUDA
device is missing, constructing a Solver raises.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
# EDZT_LIBRARY selects another build of the same C ABI (e.g. one compiled with
# device-side bounds checks); the default is the in-tree libedzt.so.
LIB_PATH = os.environ.get("EDZT_LIBRARY") or os.path.join(PKG_DIR, "libedzt.so")
REPO_ROOT = os.path.dirname(PKG_DIR)

EDZT_OK = 0
EDZT_ERR_ARG = 1
EDZT_ERR_CUDA = 2
EDZT_ERR_OOM = 3
EDZT_ERR_STATE = 4
EDZT_ERR_TIMEOUT = 5
EDZT_ERR_NUMERIC = 6
ENGINE_FUSED = 0
ENGINE_PLAIN = 1

# Every symbol include/edzt.h declares.
EXPORTS = (
    "edzt_ctx_create", "edzt_ctx_destroy", "edzt_last_error", "edzt_version", "edzt_set_model",
    "edzt_set_engine", "edzt_basis", "edzt_basis_rank", "edzt_sector_dim", "edzt_hx", "edzt_apply_c",
    "edzt_lanczos_iteration", "edzt_diag_lanczos", "edzt_ground_state", "edzt_gs_dim",
    "edzt_green_diag", "edzt_cluster_green_ftn", "edzt_solve", "edzt_launch_count", "edzt_get_stream",
    "edzt_kernel_stats", "edzt_reset_stats", "edzt_kernel_launch_log", "edzt_lanczos_iteration_noalloc", "edzt_solve_batch",
    "edzt_cluster_green_matrix", "edzt_gs_occupancy", "edzt_green_real", "edzt_server_create", "edzt_server_submit", "edzt_server_step", "edzt_server_result", "edzt_server_destroy",
    "edzt_server_cancel", "edzt_server_set_step_ms", "edzt_tune_sector", "edzt_clear_tuning",
    "edzt_instance_footprint", "edzt_set_fault_test", "edzt_diag_arpack",
    "edzt_set_diag_solver", "edzt_set_keep_vectors", "edzt_hybridization", "edzt_local_green_bethe", "edzt_fit_bath", "edzt_dmft_bethe",
)
# ground_state's diag_solver values (src/ground_state.f90:53-60).
DIAG_LANCZOS = 1
DIAG_ARPACK = 2
# Limits of edzt_lanczos_iteration_noalloc (its static scratch array).
NOALLOC_MAX_DIM = 262144
NOALLOC_MAX_STEPS = 2048


class Instance(C.Structure):
    """edzt_instance of include/edzt.h: one impurity solve of a batch."""
    _fields_ = [("norb", C.c_int), ("nbath", C.c_int),
                ("em", C.c_void_p), ("ek", C.c_void_p), ("vmk", C.c_void_p),
                ("U", C.c_double), ("Up", C.c_double), ("Jex", C.c_double), ("Jp", C.c_double),
                ("mu", C.c_double), ("nsector", C.c_int), ("sectors", C.c_void_p), ("nspin", C.c_int),
                ("seed", C.c_uint64)]


def _instance(inst, keep):
    m = inst["model"]
    em, ek, vmk = m.fortran_arrays()
    sec = np.ascontiguousarray(np.asarray(inst["sectors"], dtype=np.int32).reshape(-1, 2))
    keep += [em, ek, vmk, sec]
    return Instance(m.norb, m.nbath, em.ctypes.data, ek.ctypes.data, vmk.ctypes.data, m.U, m.Up, m.Jex, m.Jp, m.mu,
                    len(sec), sec.ctypes.data, int(inst.get("nspin", 1)), int(inst.get("seed", 0)))


class DMFTParams(C.Structure):
    """edzt_dmft_params of include/edzt.h: settings of the DMFT loop."""
    _fields_ = [("norb", C.c_int), ("nbath", C.c_int), ("nspin", C.c_int),
                ("U", C.c_double), ("Up", C.c_double), ("Jex", C.c_double), ("Jp", C.c_double),
                ("mu", C.c_double), ("hfield", C.c_double), ("nsector", C.c_int), ("sectors", C.c_void_p),
                ("maxnstep", C.c_int), ("seed", C.c_uint64), ("nw", C.c_int), ("omega", C.c_void_p),
                ("nloop", C.c_int), ("scf_tol", C.c_double), ("mixing", C.c_double), ("fit_ftol", C.c_double),
                ("outdir", C.c_char_p)]


class EDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"edzt error {code}: {msg}")
        self.code = code


STAMP_PATH = LIB_PATH + ".stamp"


def source_hash() -> str:
    """SHA-256 over the library's sources: the Makefile, csrc/ and the C ABI
    header, in sorted path order."""
    import hashlib
    h = hashlib.sha256()
    files = [os.path.join(PKG_DIR, "Makefile"), os.path.join(REPO_ROOT, "include", "edzt.h")]
    csrc = os.path.join(PKG_DIR, "csrc")
    files += sorted(os.path.join(csrc, f) for f in os.listdir(csrc))
    for f in files:
        h.update(os.path.relpath(f, REPO_ROOT).encode() + b"\0")
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = True) -> str:
    """Compile libedzt.so for sm_100a with nvcc (cross-compiles without a GPU).

    The library is rebuilt from scratch whenever the hash of its sources
    differs from the stamp written beside it by the last build (or either is
    missing), so a shipped library is reused only if it was built from these
    exact sources.  Logs which of the two happened on stderr."""
    import sys
    if os.environ.get("EDZT_LIBRARY"):
        return LIB_PATH
    want = source_hash()
    try:
        with open(STAMP_PATH) as f:
            have = f.read().strip()
    except OSError:
        have = ""
    if not force and have == want and os.path.exists(LIB_PATH):
        if verbose:
            print(f"libedzt: reusing {os.path.basename(LIB_PATH)} built from sources {want[:16]}", file=sys.stderr)
        return LIB_PATH
    if os.path.exists(STAMP_PATH):
        os.remove(STAMP_PATH)
    subprocess.run(["make", "-s", "-C", PKG_DIR, "-j8", "-B", "libedzt.so"], check=True)
    with open(STAMP_PATH, "w") as f:
        f.write(want + "\n")
    if verbose:
        print(f"libedzt: rebuilt from sources {want[:16]} (stamp was {have[:16] or 'missing'})", file=sys.stderr)
    return LIB_PATH


_lib = None
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def load_library(path: str = LIB_PATH):
    """Load libedzt.so and declare argument types (no GPU needed to load)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise EDError(EDZT_ERR_STATE, f"{path} is missing: run build() (make -C {PKG_DIR})")
    L = C.CDLL(path)
    L.edzt_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    L.edzt_ctx_destroy.argtypes = [_vp]
    L.edzt_ctx_destroy.restype = None
    L.edzt_last_error.argtypes = [_vp]
    L.edzt_last_error.restype = C.c_char_p
    L.edzt_version.restype = C.c_char_p
    L.edzt_set_model.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp, _vp] + [C.c_double] * 5
    L.edzt_set_engine.argtypes = [_vp, C.c_int]
    L.edzt_basis.argtypes = [_vp, C.c_int, C.c_int, _ip, _ip, _vp, _vp]
    L.edzt_basis_rank.argtypes = [_vp, C.c_int, _vp]
    L.edzt_sector_dim.argtypes = [_vp, C.c_int, C.c_int]
    L.edzt_sector_dim.restype = C.c_longlong
    L.edzt_hx.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp, C.c_int]
    L.edzt_apply_c.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_int, _vp]
    L.edzt_lanczos_iteration.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int, _ip, _vp, _vp]
    L.edzt_lanczos_iteration_noalloc.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int, _ip, _vp, _vp]
    L.edzt_cluster_green_matrix.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp]
    L.edzt_gs_occupancy.argtypes = [_vp, C.c_int, _vp, _vp]
    L.edzt_green_real.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_double, _vp]
    L.edzt_solve_batch.argtypes = [_vp, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_size_t]
    L.edzt_server_create.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_size_t, C.POINTER(C.c_void_p)]
    L.edzt_server_submit.argtypes = [_vp, _vp, C.POINTER(C.c_longlong)]
    L.edzt_server_step.argtypes = [_vp, _ip, _ip, _ip]
    L.edzt_server_result.argtypes = [_vp, C.c_longlong, _ip, _ip, _dp, _vp]
    L.edzt_server_destroy.argtypes = [_vp]
    L.edzt_server_destroy.restype = None
    L.edzt_server_cancel.argtypes = [_vp, C.c_longlong]
    L.edzt_server_set_step_ms.argtypes = [_vp, C.c_double]
    L.edzt_tune_sector.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _dp]
    L.edzt_clear_tuning.argtypes = [_vp]
    L.edzt_instance_footprint.argtypes = [_vp, C.POINTER(C.c_longlong)]
    L.edzt_set_fault_test.argtypes = [_vp, C.c_int, C.c_double, C.c_int]
    L.edzt_diag_lanczos.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64, _dp, _vp, _dp]
    L.edzt_diag_arpack.argtypes = [_vp, C.c_int, C.c_int, C.c_uint64, C.c_uint64, _dp, _vp, _vp, _vp, _ip]
    L.edzt_set_diag_solver.argtypes = [_vp, C.c_int]
    L.edzt_set_keep_vectors.argtypes = [_vp, C.c_int]
    L.edzt_hybridization.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp]
    L.edzt_local_green_bethe.argtypes = [C.c_int, C.c_int, C.c_int, _vp, C.c_double, _vp, _vp, _vp]
    L.edzt_fit_bath.argtypes = [C.c_int] * 4 + [_vp] * 7 + [C.c_double, _vp]
    L.edzt_dmft_bethe.argtypes = [_vp, C.POINTER(DMFTParams)] + [_vp] * 7 + [_ip, _vp, _ip]
    L.edzt_ground_state.argtypes = [_vp, C.c_int, _vp, C.c_int, C.c_uint64, _ip, _dp, _vp, _vp]
    L.edzt_gs_dim.argtypes = [_vp]
    L.edzt_gs_dim.restype = C.c_longlong
    L.edzt_green_diag.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp]
    L.edzt_cluster_green_ftn.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]
    L.edzt_solve.argtypes = [_vp, C.c_int, _vp, C.c_int, C.c_uint64, C.c_int, C.c_int, _vp, _ip, _dp, _vp, _vp]
    L.edzt_launch_count.argtypes = [_vp]
    L.edzt_launch_count.restype = C.c_longlong
    L.edzt_get_stream.argtypes = [_vp, C.POINTER(C.c_void_p)]
    L.edzt_kernel_stats.argtypes = [_vp, C.POINTER(C.c_longlong), _dp, _dp]
    L.edzt_reset_stats.argtypes = [_vp]
    L.edzt_kernel_launch_log.argtypes = [_vp, C.c_int, _ip, _vp, _vp, _vp]
    _lib = L
    return L


def _ptr(a) -> int | None:
    """Address of a numpy array or a torch tensor (device pointers pass through)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return int(a.data_ptr())
    raise TypeError(f"unsupported buffer type {type(a)}")


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class Model:
    """Impurity model in the reference's shapes: em(norb,2), ek(nbath,2), vmk(norb,nbath,2)."""

    def __init__(self, norb, nbath, em, ek, vmk, U, Up=None, Jex=0.0, Jp=None, mu=0.0):
        self.norb, self.nbath = int(norb), int(nbath)
        self.nsite = self.norb + self.nbath
        self.em = np.asarray(em, dtype=np.float64).reshape(self.norb, 2)
        self.ek = np.asarray(ek, dtype=np.float64).reshape(self.nbath, 2)
        self.vmk = np.asarray(vmk, dtype=np.float64).reshape(self.norb, self.nbath, 2)
        self.U = float(U)
        self.Jex = float(Jex)
        # rotational-invariance defaults of src/dmft_params.f90:90-96
        self.Up = float(self.U - 2 * self.Jex) if (Up is None or Up < 0) else float(Up)
        self.Jp = float(self.Jex) if (Jp is None or Jp < 0) else float(Jp)
        self.mu = float(mu)

    def fortran_arrays(self):
        return (np.ascontiguousarray(self.em.ravel(order="F")),
                np.ascontiguousarray(self.ek.ravel(order="F")),
                np.ascontiguousarray(self.vmk.ravel(order="F")))


def _host_check(rc: int, what: str):
    if rc != EDZT_OK:
        raise EDError(rc, what)


def _cplx_f(G) -> np.ndarray:
    """Complex [nspin][norb][nw] as the interleaved Fortran array (nw, norb, nspin)."""
    return np.ascontiguousarray(np.asarray(G, dtype=np.complex128)).view(np.float64).ravel()


def hybridization(ek, vmk, omega, nspin) -> np.ndarray:
    """D_cl[ispin, iorb, iw] by the library (edzt_hybridization); no device needed."""
    ek, vmk, omega = (np.asarray(a, dtype=np.float64) for a in (ek, vmk, omega))
    norb, nbath = vmk.shape[0], vmk.shape[1]
    D = np.zeros((nspin, norb, omega.size), dtype=np.complex128)
    ekf, vmf, om = (np.ascontiguousarray(a.ravel(order="F")) for a in (ek, vmk, omega))
    _host_check(load_library().edzt_hybridization(norb, nbath, nspin, omega.size, _ptr(om), _ptr(ekf), _ptr(vmf),
                                                  D.ctypes.data), "edzt_hybridization")
    return D


def local_green_bethe(em, D, G_cl, hfield=0.0) -> np.ndarray:
    """G_loc[ispin, iorb, iw] of the Bethe lattice by the library (edzt_local_green_bethe)."""
    em = np.ascontiguousarray(np.asarray(em, dtype=np.float64).ravel(order="F"))
    nspin, norb, nw = np.shape(G_cl)
    G = np.zeros((nspin, norb, nw), dtype=np.complex128)
    Df, Gf = _cplx_f(D), _cplx_f(G_cl)
    _host_check(load_library().edzt_local_green_bethe(norb, nspin, nw, _ptr(em), float(hfield), _ptr(Df), _ptr(Gf),
                                                      G.ctypes.data), "edzt_local_green_bethe")
    return G


def fit_bath(em, ek, vmk, D, G_cl, G_loc, omega, nspin, ftol=1.0e-6):
    """New (em, ek, vmk) by the library's conjugate-gradient bath fit
    (edzt_fit_bath); returns them with the final cost per spin."""
    em = np.array(em, dtype=np.float64)
    ek = np.array(ek, dtype=np.float64)
    vmk = np.array(vmk, dtype=np.float64)
    norb, nbath = vmk.shape[0], vmk.shape[1]
    omega = _f64(omega)
    emf, ekf, vmf = (np.ascontiguousarray(a.ravel(order="F")) for a in (em, ek, vmk))
    cost = np.zeros(nspin)
    Df, Gc, Gl = _cplx_f(D), _cplx_f(G_cl), _cplx_f(G_loc)
    _host_check(load_library().edzt_fit_bath(norb, nbath, nspin, omega.size, _ptr(omega), _ptr(emf), _ptr(ekf),
                                             _ptr(vmf), _ptr(Df), _ptr(Gc), _ptr(Gl), float(ftol), _ptr(cost)),
                "edzt_fit_bath")
    return (emf.reshape(em.shape, order="F"), ekf.reshape(ek.shape, order="F"), vmf.reshape(vmk.shape, order="F"),
            cost)


def matsubara(nw: int, beta: float) -> np.ndarray:
    """omega_n = (2n+1) pi / beta, n = 0..nw-1 (src/dmft_grid.f90:42-52 on one rank)."""
    return (2.0 * np.arange(nw, dtype=np.float64) + 1.0) * np.pi / beta


class Solver:
    """One CUDA context of the ED solver (edzt_ctx)."""

    def __init__(self, device: int = 0, engine: int = ENGINE_FUSED):
        self._L = load_library()
        h = C.c_void_p()
        rc = self._L.edzt_ctx_create(int(device), C.byref(h))
        if rc != EDZT_OK:
            raise EDError(rc, "edzt_ctx_create failed (no CUDA device?)")
        self._h = h
        self.model: Model | None = None
        self.set_engine(engine)

    def close(self):
        if getattr(self, "_h", None):
            self._L.edzt_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != EDZT_OK:
            raise EDError(rc, self._L.edzt_last_error(self._h).decode())

    def set_engine(self, engine: int):
        self._check(self._L.edzt_set_engine(self._h, int(engine)))

    def launch_count(self) -> int:
        return int(self._L.edzt_launch_count(self._h))

    def stream_ptr(self) -> int:
        """cudaStream_t of this context (all its kernels run there)."""
        p = C.c_void_p()
        self._check(self._L.edzt_get_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def kernel_stats(self) -> dict:
        """Persistent Lanczos kernel: launches, device ms (CUDA events) and algorithmic bytes."""
        n, ms, by = C.c_longlong(), C.c_double(), C.c_double()
        self._check(self._L.edzt_kernel_stats(self._h, C.byref(n), C.byref(ms), C.byref(by)))
        return dict(launches=n.value, ms=ms.value, bytes=by.value)

    def reset_stats(self):
        self._check(self._L.edzt_reset_stats(self._h))

    def launch_log(self) -> list:
        """Per persistent launch since the last reset: dict(ms, bytes, states)."""
        ms, by, st = np.zeros(256), np.zeros(256), np.zeros(256)
        n = C.c_int()
        self._check(self._L.edzt_kernel_launch_log(self._h, 256, C.byref(n), _ptr(ms), _ptr(by), _ptr(st)))
        return [dict(ms=float(ms[i]), bytes=float(by[i]), states=float(st[i])) for i in range(n.value)]

    def set_model(self, m: Model):
        em, ek, vmk = m.fortran_arrays()
        self._check(self._L.edzt_set_model(self._h, m.norb, m.nbath, _ptr(em), _ptr(ek), _ptr(vmk),
                                           m.U, m.Up, m.Jex, m.Jp, m.mu))
        self.model = m
        self._keep = (em, ek, vmk)

    def dim(self, ne_up: int, ne_dn: int) -> int:
        return int(self._L.edzt_sector_dim(self._h, ne_up, ne_dn))

    # generate_basis
    def generate_basis(self, ne_up: int, ne_dn: int):
        nup, ndn = C.c_int(), C.c_int()
        self._check(self._L.edzt_basis(self._h, ne_up, ne_dn, C.byref(nup), C.byref(ndn), None, None))
        up = np.zeros(max(nup.value, 1), dtype=np.uint32)
        dn = np.zeros(max(ndn.value, 1), dtype=np.uint32)
        self._check(self._L.edzt_basis(self._h, ne_up, ne_dn, None, None, _ptr(up), _ptr(dn)))
        return up[: nup.value], dn[: ndn.value]

    def basis_rank(self, ne: int) -> np.ndarray:
        r = np.zeros(1 << self.model.nsite, dtype=np.int32)
        self._check(self._L.edzt_basis_rank(self._h, ne, _ptr(r)))
        return r

    def hx(self, ne_up, ne_dn, x, y=None, py: bool = False):
        """y = H x (py=False) or y += H x (py=True).  numpy in/out, or device tensors in place."""
        if isinstance(x, np.ndarray) or not hasattr(x, "data_ptr"):
            x = _f64(x)
            out = np.array(y, dtype=np.float64, copy=True) if (py and y is not None) else np.zeros_like(x)
            self._check(self._L.edzt_hx(self._h, ne_up, ne_dn, _ptr(x), _ptr(out), 1 if py else 0))
            return out
        self._check(self._L.edzt_hx(self._h, ne_up, ne_dn, _ptr(x), _ptr(y), 1 if py else 0))
        return y

    def apply_c(self, ne_up, ne_dn, vec, pm, iorb, ispin):
        vec = _f64(vec)
        d = 1 if pm == 1 else -1
        ou = ne_up + (d if ispin == 1 else 0)
        od = ne_dn + (d if ispin == 2 else 0)
        out = np.zeros(max(self.dim(ou, od), 1))
        self._check(self._L.edzt_apply_c(self._h, ne_up, ne_dn, _ptr(vec), pm, iorb, ispin, _ptr(out)))
        return out[: self.dim(ou, od)]

    def lanczos_iteration(self, ne_up, ne_dn, v_init, maxnstep):
        v_init = _f64(v_init)
        a = np.zeros(maxnstep)
        b = np.zeros(maxnstep)
        n = C.c_int()
        self._check(self._L.edzt_lanczos_iteration(self._h, ne_up, ne_dn, _ptr(v_init), maxnstep, C.byref(n),
                                                   _ptr(a), _ptr(b)))
        return n.value, a, b

    def lanczos_iteration_noalloc(self, ne_up, ne_dn, v_init, maxnstep):
        """lanczos_iteration from the library's static scratch array (no
        device allocation; sector dim <= NOALLOC_MAX_DIM, maxnstep <=
        NOALLOC_MAX_STEPS; the sector's tables must exist on the context)."""
        v_init = _f64(v_init)
        a = np.zeros(maxnstep)
        b = np.zeros(maxnstep)
        n = C.c_int()
        self._check(self._L.edzt_lanczos_iteration_noalloc(self._h, ne_up, ne_dn, _ptr(v_init), maxnstep,
                                                           C.byref(n), _ptr(a), _ptr(b)))
        return n.value, a, b

    def diag_lanczos(self, ne_up, ne_dn, maxnstep, seed=0, stream=0):
        ev, res = C.c_double(), C.c_double()
        vec = np.zeros(self.dim(ne_up, ne_dn))
        self._check(self._L.edzt_diag_lanczos(self._h, ne_up, ne_dn, maxnstep, C.c_uint64(seed),
                                              C.c_uint64(stream), C.byref(ev), _ptr(vec), C.byref(res)))
        return dict(e0=ev.value, vec=vec, residual=res.value)

    def diag_arpack(self, ne_up, ne_dn, seed=0, stream=0, want_resid=True):
        """diag_arpack (src/arpack_solver.f90:19-124): the lowest eigenpair by
        the restarted Lanczos with ARPACK's settings (nev 3, ncv 6, 'SA', tol 0)."""
        ev = C.c_double()
        nmult = C.c_int()
        vec = np.zeros(self.dim(ne_up, ne_dn))
        ritz = np.zeros(3)
        resid = np.zeros(3) if want_resid else None
        self._check(self._L.edzt_diag_arpack(self._h, ne_up, ne_dn, C.c_uint64(seed), C.c_uint64(stream),
                                             C.byref(ev), _ptr(vec), _ptr(ritz), _ptr(resid), C.byref(nmult)))
        return dict(e0=ev.value, vec=vec, ritz=ritz, resid=resid, nmult=nmult.value)

    def set_diag_solver(self, diag_solver: int):
        """ground_state's diag_solver: DIAG_LANCZOS (1) or DIAG_ARPACK (2)."""
        self._check(self._L.edzt_set_diag_solver(self._h, int(diag_solver)))

    def set_keep_vectors(self, keep: int):
        """edzt_set_keep_vectors: 1 (default) keep the scan's Lanczos vectors
        for the eigenvector when they fit, 0 rerun the recurrence."""
        self._check(self._L.edzt_set_keep_vectors(self._h, int(keep)))

    def ground_state(self, sectors, maxnstep, seed=0, want_vec=True):
        sec = np.ascontiguousarray(np.asarray(sectors, dtype=np.int32).reshape(-1, 2))
        isec, e0 = C.c_int(), C.c_double()
        es = np.zeros(len(sec))
        vec = None
        if want_vec:
            vec = np.zeros(max(max(self.dim(int(u), int(d)) for u, d in sec), 1))
        self._check(self._L.edzt_ground_state(self._h, len(sec), _ptr(sec), maxnstep, C.c_uint64(seed),
                                              C.byref(isec), C.byref(e0), _ptr(vec), _ptr(es)))
        out = dict(isector=isec.value, e0=e0.value, e_sector=es, sector=tuple(int(v) for v in sec[isec.value]))
        if want_vec:
            out["vec"] = vec[: int(self._L.edzt_gs_dim(self._h))].copy()
        return out

    def green_diag(self, iorb, ispin, maxnstep, omega):
        omega = _f64(omega)
        nw = omega.size
        ap, bp, am, bm = (np.zeros(maxnstep) for _ in range(4))
        g = np.zeros(2 * nw)
        self._check(self._L.edzt_green_diag(self._h, iorb, ispin, maxnstep, nw, _ptr(omega), _ptr(ap), _ptr(bp),
                                            _ptr(am), _ptr(bm), _ptr(g)))
        return dict(g=g[0::2] + 1j * g[1::2], ap=ap, bp=bp, am=am, bm=bm)

    def cluster_green_ftn(self, nspin, maxnstep, omega):
        omega = _f64(omega)
        nw = omega.size
        norb = self.model.norb
        G = np.zeros(2 * nw * norb * nspin)
        coeffs = np.zeros(norb * 2 * 4 * maxnstep)
        self._check(self._L.edzt_cluster_green_ftn(self._h, nspin, maxnstep, nw, _ptr(omega), _ptr(G),
                                                   _ptr(coeffs)))
        Gc = (G[0::2] + 1j * G[1::2]).reshape(nspin, norb, nw)
        return dict(G_cl=Gc, coeffs=coeffs.reshape(norb, 2, 4, maxnstep))

    def dmft_bethe(self, model, sectors, maxnstep, omega, nspin=1, nloop=20, scf_tol=1.0e-6, mixing=1.0,
                   fit_ftol=1.0e-6, hfield=0.0, seed=0, outdir=None):
        """The DMFT loop of src/dmft.f90:38-137 on the Bethe lattice, in the
        library (edzt_dmft_bethe): starts from model's bath, returns the last
        iteration's em[a,s], ek[l,s], vmk[a,l,s], D_cl/G_cl/G_loc[s,a,w],
        Z[a,s], the per-iteration convergence measure and the iteration count."""
        omega = _f64(omega)
        sec = np.ascontiguousarray(np.asarray(sectors, dtype=np.int32).reshape(-1, 2))
        em, ek, vmk = model.fortran_arrays()
        em, ek, vmk = em.copy(), ek.copy(), vmk.copy()
        norb, nbath, nw = model.norb, model.nbath, omega.size
        P = DMFTParams(norb, nbath, nspin, model.U, model.Up, model.Jex, model.Jp, model.mu, float(hfield), len(sec),
                       sec.ctypes.data, maxnstep, int(seed), nw, omega.ctypes.data, nloop, float(scf_tol),
                       float(mixing), float(fit_ftol), None if outdir is None else os.fsencode(outdir))
        D, Gc, Gl = (np.zeros((nspin, norb, nw), dtype=np.complex128) for _ in range(3))
        Z = np.zeros(norb * nspin)
        hist = np.zeros(nloop)
        it, conv = C.c_int(), C.c_int()
        self._check(self._L.edzt_dmft_bethe(self._h, C.byref(P), _ptr(em), _ptr(ek), _ptr(vmk), D.ctypes.data,
                                            Gc.ctypes.data, Gl.ctypes.data, _ptr(Z), C.byref(it), _ptr(hist),
                                            C.byref(conv)))
        return dict(em=em.reshape(norb, 2, order="F"), ek=ek.reshape(nbath, 2, order="F"),
                    vmk=vmk.reshape(norb, nbath, 2, order="F"), D_cl=D, G_cl=Gc, G_loc=Gl,
                    Z=Z.reshape(norb, nspin, order="F"), history=hist[: it.value], iterations=it.value,
                    converged=bool(conv.value))

    def green_real(self, iorb, ispin, maxnstep, omega, eta):
        """G(w + i eta) of green_diag on real frequencies; A(w) = -Im G / pi."""
        omega = _f64(omega)
        g = np.zeros(2 * omega.size)
        self._check(self._L.edzt_green_real(self._h, iorb, ispin, maxnstep, omega.size, _ptr(omega), float(eta),
                                            _ptr(g)))
        return g[0::2] + 1j * g[1::2]

    def gs_occupancy(self, nspin=2):
        """<n_{iorb,ispin}> [ispin][iorb] and double occupancies [iorb] of the
        resident ground state (post_process.f90:62-112)."""
        norb = self.model.norb
        occ = np.zeros(norb * nspin)
        docc = np.zeros(norb)
        self._check(self._L.edzt_gs_occupancy(self._h, nspin, _ptr(occ), _ptr(docc)))
        return occ.reshape(nspin, norb), docc

    def cluster_green_matrix(self, nspin, maxnstep, omega):
        """Full G_ab on the resident ground state (edzt_cluster_green_matrix),
        returned as G[ispin, a, b, iw]."""
        omega = _f64(omega)
        nw = omega.size
        norb = self.model.norb
        G = np.zeros(2 * nw * norb * norb * nspin)
        self._check(self._L.edzt_cluster_green_matrix(self._h, nspin, maxnstep, nw, _ptr(omega), _ptr(G)))
        Gc = (G[0::2] + 1j * G[1::2]).reshape(nspin, norb, norb, nw)   # [s, b, a, iw]
        return Gc.transpose(0, 2, 1, 3)

    def tune_sector(self, ne_up, ne_dn, steps=12):
        """Autotune the persistent kernel's tile shape for a sector shape
        (edzt_tune_sector): returns dict(cols_per_slab, rows_per_tile, block,
        ms_per_step) of the fastest shape, recorded on the context."""
        wc, r, blk = C.c_int(), C.c_int(), C.c_int()
        ms = C.c_double()
        self._check(self._L.edzt_tune_sector(self._h, ne_up, ne_dn, steps, C.byref(wc), C.byref(r), C.byref(blk),
                                             C.byref(ms)))
        return dict(cols_per_slab=wc.value, rows_per_tile=r.value, block=blk.value, ms_per_step=ms.value)

    def clear_tuning(self):
        self._check(self._L.edzt_clear_tuning(self._h))

    def set_fault_test(self, pass_cap=0, wait_seconds=0.0, stall_cta=-1):
        """Fault tests of the persistent kernel (edzt_set_fault_test); all
        defaults restore normal operation."""
        self._check(self._L.edzt_set_fault_test(self._h, int(pass_cap), float(wait_seconds), int(stall_cta)))

    def footprint(self, inst) -> int:
        """Device bytes a request holds at its peak (edzt_instance_footprint)."""
        keep = []
        rec = _instance(inst, keep)
        b = C.c_longlong()
        self._check(self._L.edzt_instance_footprint(C.byref(rec), C.byref(b)))
        return b.value

    def solve_batch(self, instances, maxnstep, omega, hbm_budget=0):
        """Many independent solves in batched persistent launches
        (edzt_solve_batch).  instances: dicts with model, sectors, nspin (1),
        seed (0).  Returns isector, e0 ([n]) and the per-instance G_cl arrays,
        shaped (nspin, norb, nw) like solve()."""
        omega = _f64(omega)
        nw = omega.size
        n = len(instances)
        keep = []
        arr = (Instance * max(n, 1))()
        for i, inst in enumerate(instances):
            arr[i] = _instance(inst, keep)
        sizes = [2 * nw * inst["model"].norb * int(inst.get("nspin", 1)) for inst in instances]
        G = np.zeros(max(sum(sizes), 1))
        isec = np.zeros(max(n, 1), dtype=np.int32)
        e0 = np.zeros(max(n, 1))
        self._check(self._L.edzt_solve_batch(self._h, n, C.addressof(arr), maxnstep, nw, _ptr(omega), _ptr(isec),
                                             _ptr(e0), _ptr(G), int(hbm_budget)))
        out, off = [], 0
        for inst, sz in zip(instances, sizes):
            g = G[off:off + sz]
            off += sz
            out.append((g[0::2] + 1j * g[1::2]).reshape(int(inst.get("nspin", 1)), inst["model"].norb, nw))
        return dict(isector=isec[:n], e0=e0[:n], G_cl=out)

    def solve(self, sectors, maxnstep, omega, nspin=1, seed=0):
        """ground_state + cluster_green_ftn in one call (src/dmft.f90:76-78)."""
        sec = np.ascontiguousarray(np.asarray(sectors, dtype=np.int32).reshape(-1, 2))
        omega = _f64(omega)
        nw = omega.size
        norb = self.model.norb
        G = np.zeros(2 * nw * norb * nspin)
        isec, e0 = C.c_int(), C.c_double()
        self._check(self._L.edzt_solve(self._h, len(sec), _ptr(sec), maxnstep, C.c_uint64(seed), nspin, nw,
                                       _ptr(omega), C.byref(isec), C.byref(e0), _ptr(G), None))
        return dict(isector=isec.value, e0=e0.value, G_cl=(G[0::2] + 1j * G[1::2]).reshape(nspin, norb, nw))


class Server:
    """Served form (edzt_server_*): continuous batching of impurity solves on
    one solver context.  submit() queues a request (a dict like solve_batch's
    instances), step() admits what fits in device memory and advances every
    admitted request by one phase in one persistent launch, result() returns
    a finished request's isector, e0 and G_cl (nspin, norb, nw), else None."""

    def __init__(self, solver: "Solver", maxnstep: int, omega, hbm_budget: int = 0):
        self.solver = solver
        self._L = solver._L
        self.omega = _f64(omega)
        self.nw = self.omega.size
        self.maxnstep = maxnstep
        h = C.c_void_p()
        solver._check(self._L.edzt_server_create(solver._h, maxnstep, self.nw, _ptr(self.omega), int(hbm_budget),
                                                 C.byref(h)))
        self._h = h
        self._shape = {}

    def submit(self, inst) -> int:
        keep = []
        rec = _instance(inst, keep)
        rid = C.c_longlong()
        self.solver._check(self._L.edzt_server_submit(self._h, C.byref(rec), C.byref(rid)))
        self._shape[rid.value] = (int(inst.get("nspin", 1)), inst["model"].norb)
        return rid.value

    def step(self):
        na, nq, nf = C.c_int(), C.c_int(), C.c_int()
        self.solver._check(self._L.edzt_server_step(self._h, C.byref(na), C.byref(nq), C.byref(nf)))
        return na.value, nq.value, nf.value

    def result(self, rid: int):
        nspin, norb = self._shape[rid]
        G = np.zeros(2 * self.nw * norb * nspin)
        done, isec, e0 = C.c_int(), C.c_int(), C.c_double()
        self.solver._check(self._L.edzt_server_result(self._h, rid, C.byref(done), C.byref(isec), C.byref(e0),
                                                      _ptr(G)))
        if not done.value:
            return None
        del self._shape[rid]
        return dict(isector=isec.value, e0=e0.value, G_cl=(G[0::2] + 1j * G[1::2]).reshape(nspin, norb, self.nw))

    def cancel(self, rid: int):
        self.solver._check(self._L.edzt_server_cancel(self._h, rid))

    def set_step_ms(self, ms: float):
        """Time budget of one step (edzt_server_set_step_ms)."""
        self.solver._check(self._L.edzt_server_set_step_ms(self._h, C.c_double(ms)))

    def close(self):
        if self._h:
            self._L.edzt_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve(server: Server, requests, arrivals):
    """Request loop of the served form: request i is submitted once the wall
    clock passes arrivals[i] (seconds from the start); the server steps while
    work is queued or running and idles until the next arrival otherwise.
    Returns (results in request order, latency of each request in seconds
    from its arrival to the end of the step that finished it, total seconds)."""
    import time
    order = np.argsort(np.asarray(arrivals, dtype=float), kind="stable")
    ids = [None] * len(requests)
    done = [None] * len(requests)
    lat = np.zeros(len(requests))
    t0 = time.perf_counter()
    nxt = 0
    pending = set()
    while nxt < len(order) or pending:
        now = time.perf_counter() - t0
        while nxt < len(order) and arrivals[order[nxt]] <= now:
            i = int(order[nxt])
            ids[i] = server.submit(requests[i])
            pending.add(i)
            nxt += 1
        if not pending:
            time.sleep(max(0.0, arrivals[order[nxt]] - now))
            continue
        server.step()
        t = time.perf_counter() - t0
        for i in list(pending):
            r = server.result(ids[i])
            if r is not None:
                done[i] = r
                lat[i] = t - arrivals[i]
                pending.discard(i)
    return done, lat, time.perf_counter() - t0
