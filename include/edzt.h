/*
 * edzt.h — C ABI of the B200 (sm_100a) zero-temperature ED impurity solver.
 *
 * Drop-in boundary for the hot path of yw-choi/DMFT-ED-ZT.  Each entry point
 * replaces one Fortran procedure of the reference (cited per function); a
 * Fortran host binds them through an iso_c_binding interface module with
 * one bind(C) interface per function.  The reference's DMFT loop, lattice,
 * grid and bath fit can stay on the host unchanged; the library also
 * carries a Bethe-lattice DMFT loop of its own (edzt_dmft_bethe).
 *
 * Conventions
 *  - Every function returns EDZT_OK (0) or an error code; edzt_last_error()
 *    gives the message.  The reference aborts through die()/stop instead; a
 *    Fortran shim calls die() on a non-zero status.
 *  - Arrays are FP64, laid out as the reference's Fortran arrays:
 *      em(norb,2)        em[iorb + norb*ispin]
 *      ek(nbath,2)       ek[jbath + nbath*ispin]
 *      vmk(norb,nbath,2) vmk[iorb + norb*(jbath + nbath*ispin)]
 *    (0-based here).  A sector vector of (ne_up, ne_dn) has
 *    C(nsite,ne_up)*C(nsite,ne_dn) entries, index idn*nup + iup
 *    (src/ed_basis.f90:132-135).  Complex arrays are interleaved (re, im).
 *  - Vector arguments may be host or device pointers (CUDA unified
 *    addressing tells them apart); host buffers are staged through the device.
 *  - One host thread per context.  A context owns one GPU, one stream and the
 *    device-resident state between calls (the ground state vector stays on
 *    the device for the Green's-function runs).
 *  - Electron counts, orbital and spin indices follow the reference
 *    (iorb, ispin are 1-based; pm = 1 creates, pm = 2 annihilates).
 */
#ifndef EDZT_H
#define EDZT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDZT_OK 0
#define EDZT_ERR_ARG 1      /* invalid argument (sector, index, size)            */
#define EDZT_ERR_CUDA 2     /* CUDA runtime error                                */
#define EDZT_ERR_OOM 3      /* device allocation failed                          */
#define EDZT_ERR_STATE 4    /* call out of order (no model / no ground state)    */
#define EDZT_ERR_TIMEOUT 5  /* a bounded device-side wait ran out                */
#define EDZT_ERR_NUMERIC 6  /* non-finite result / tridiagonal solve failed      */

/* Lanczos engine selector (edzt_set_engine). */
#define EDZT_ENGINE_FUSED 0 /* persistent batched kernel (default)               */
#define EDZT_ENGINE_PLAIN 1 /* one kernel per BLAS-1 step, host-driven: the plain */
                            /* one-solve-at-a-time GPU Lanczos of the reference  */

typedef struct edzt_ctx edzt_ctx;

/* Context on CUDA device `device`.  Replaces mpi_setup (src/mpi.f90:16-30):
 * the GPU path has no MPI decomposition. */
int edzt_ctx_create(int device, edzt_ctx **out);
void edzt_ctx_destroy(edzt_ctx *ctx);
const char *edzt_last_error(const edzt_ctx *ctx);
/* Library version string. */
const char *edzt_version(void);

/* Impurity model: the dmft_params globals (src/dmft_params.f90:7-50) plus the
 * (em, ek, vmk) arguments every reference routine carries.  Up and Jp are the
 * final values (the reference defaults Up = U - 2J, Jp = J when the input is
 * negative, src/dmft_params.f90:90-96; the caller applies that rule).
 * nsite = norb + nbath <= 20, norb <= 4. */
int edzt_set_model(edzt_ctx *ctx, int norb, int nbath, const double *em, const double *ek,
                   const double *vmk, double U, double Up, double Jex, double Jp, double mu);

/* Selects the Lanczos engine (EDZT_ENGINE_*). */
int edzt_set_engine(edzt_ctx *ctx, int engine);

/* generate_basis (src/ed_basis.f90:42-114): the ascending up and down bit
 * strings of sector (ne_up, ne_dn).  nup/ndn receive C(nsite, ne_up/dn);
 * up/dn (nullable, host or device) receive the strings.  Bit-exact hook. */
int edzt_basis(edzt_ctx *ctx, int ne_up, int ne_dn, int *nup, int *ndn, uint32_t *up, uint32_t *dn);

/* Rank table of one spin species (idx_up/idx_down of basis_t,
 * src/ed_basis.f90:32-33,106-109), 0-based, -1 for strings outside the
 * sector: rank[0 .. 2^nsite). */
int edzt_basis_rank(edzt_ctx *ctx, int ne, int32_t *rank);

/* Dimension C(nsite,ne_up)*C(nsite,ne_dn) of a sector (0 if empty). */
long long edzt_sector_dim(edzt_ctx *ctx, int ne_up, int ne_dn);

/* hx (src/impurity_hamiltonian.f90:77-247): y = H x, or y = y + H x when
 * accumulate != 0 (the `py` flag).  x, y: sector vectors. */
int edzt_hx(edzt_ctx *ctx, int ne_up, int ne_dn, const double *x, double *y, int accumulate);

/* apply_c (src/ed_operator.f90:13-57): vec_out = c^+_{iorb,ispin} vec (pm=1)
 * or c_{iorb,ispin} vec (pm=2).  vec is in sector (ne_up, ne_dn); vec_out in
 * the N+-1 sector chosen as green_diag does (src/dmft_green.f90:204-210,
 * 232-238).  Returns EDZT_ERR_ARG if that sector is empty. */
int edzt_apply_c(edzt_ctx *ctx, int ne_up, int ne_dn, const double *vec, int pm, int iorb, int ispin,
                 double *vec_out);

/* lanczos_iteration (src/lanczos_solver.f90:92-173): three-term Lanczos from
 * v_init without re-orthogonalisation.  a, b: [maxnstep] (host or device),
 * zeroed then filled; b[0] = 0.  *nstep = steps taken.  Breakdown
 * (b(k) < 1e-16) is tested before dividing and stops with nstep = k-1. */
int edzt_lanczos_iteration(edzt_ctx *ctx, int ne_up, int ne_dn, const double *v_init, int maxnstep,
                           int *nstep, double *a, double *b);

/* edzt_lanczos_iteration without any device allocation.  No counterpart in
 * the reference (its lanczos_iteration allocates its work vectors on every
 * call).  For callers that cannot call cudaMalloc/cudaFree: device memory
 * owned entirely by another allocator, or a latency-critical loop that must
 * not take the device-wide synchronisation an allocation can cause.  Same
 * arguments and results as edzt_lanczos_iteration, always on the persistent
 * kernel, whose scratch is one static device array of about 13.1 MiB that
 * every GPU loading the library holds until exit.  Limits: sector dimension
 * <= EDZT_NOALLOC_MAX_DIM, maxnstep <= EDZT_NOALLOC_MAX_STEPS (EDZT_ERR_ARG
 * beyond).  The sector's tables must already exist on the context (built by
 * any earlier allocating call on that sector after edzt_set_model, e.g.
 * edzt_hx or edzt_lanczos_iteration), else EDZT_ERR_STATE.  The first call
 * on each device looks the scratch array up with that device current and
 * should come before any stream capture; the address is kept until exit,
 * so cudaDeviceReset is not supported while the library is loaded.  The
 * array is shared by all contexts of a device: calls whose GPU work
 * overlaps race.  v_init may be host memory, or device memory of the
 * context's GPU (device memory of another GPU: EDZT_ERR_ARG). */
#define EDZT_NOALLOC_MAX_DIM 262144
#define EDZT_NOALLOC_MAX_STEPS 2048
int edzt_lanczos_iteration_noalloc(edzt_ctx *ctx, int ne_up, int ne_dn, const double *v_init, int maxnstep,
                                   int *nstep, double *a, double *b);

/* diag_lanczos (src/lanczos_solver.f90:20-90) with a reproducible start
 * vector (U[0,1) from (seed, stream)): lowest eigenvalue of the sector, its
 * eigenvector (nullable) and the residual |H g - E g|^2 (nullable). */
int edzt_diag_lanczos(edzt_ctx *ctx, int ne_up, int ne_dn, int maxnstep, uint64_t seed, uint64_t stream,
                      double *eigval, double *eigvec, double *residual);

/* diag_arpack (src/arpack_solver.f90:19-124): lowest eigenvalue and
 * eigenvector of a sector by a restarted Lanczos with the reference's ARPACK
 * settings (nev 3, ncv 6, which 'SA', tol 0 = machine precision, exact
 * shifts, at most 20000 restarts), kept by thick restart, which spans the
 * same subspace as ARPACK's implicit restart with exact shifts.  The start
 * vector is U[0,1) from (seed, stream) where ARPACK draws its own.  eigvec
 * (nullable, host or device) [dim] is normalised; its sign is arbitrary, as
 * ARPACK's.  ritz (nullable) [3]: the three lowest Ritz values; resid
 * (nullable) [3]: their direct residuals |H x - theta x| (the reference's
 * printed d(:,2)), three more H.v; nmult (nullable): H.v count (multcount).
 * Sector dimension < ncv = 6: EDZT_ERR_ARG (pdsaupd rejects it); not
 * converged in 20000 restarts: EDZT_ERR_NUMERIC (the reference dies). */
int edzt_diag_arpack(edzt_ctx *ctx, int ne_up, int ne_dn, uint64_t seed, uint64_t stream, double *eigval,
                     double *eigvec, double *ritz, double *resid, int *nmult);

/* ground_state's diag_solver (src/ground_state.f90:53-60): 1 = diag_lanczos
 * (default), 2 = diag_arpack on every sector; anything else EDZT_ERR_ARG
 * ("invalid diag solver").  Applies to edzt_ground_state and edzt_solve;
 * edzt_diag_lanczos, the batched and the served forms always use Lanczos. */
#define EDZT_DIAG_LANCZOS 1
#define EDZT_DIAG_ARPACK 2
int edzt_set_diag_solver(edzt_ctx *ctx, int diag_solver);

/* Whether ground_state's fused scan keeps every step's Lanczos vectors for
 * the eigenvector (edzt_ground_state): 1 (default) when they fit in half of
 * the device memory free at context creation, 0 never (the winner's recurrence is run again, as
 * src/lanczos_solver.f90:213-300 does).  Anything else EDZT_ERR_ARG. */
int edzt_set_keep_vectors(edzt_ctx *ctx, int keep);

/* ground_state (src/ground_state.f90:1-81): scans sectors[nsector][2] =
 * (ne_up, ne_dn), keeps the lowest energy (a later sector wins only if lower
 * by more than 1e-10*max(1,|E|)), and keeps its normalised vector resident
 * on the device for edzt_cluster_green_ftn.  Sector i starts Lanczos from
 * stream i of `seed`.  gsvec (nullable, host or device) receives the vector
 * (gs%vec, src/eigpair.f90:5-9); e_sector (nullable) [nsector] the per-sector
 * lowest energies.  Device memory: when (maxnstep + 1) * 16 bytes per state
 * of all sectors fit in half of the device memory that was free when the
 * context was created, the scan keeps every
 * step's Lanczos vectors and the ground-state vector is their sum (one pass);
 * otherwise the winner's recurrence is run again, as the reference's
 * lanczos_ground_state does.  Both form the same sum; the rerun sums
 * ||v_init|| again, so the two agree to rounding. */
int edzt_ground_state(edzt_ctx *ctx, int nsector, const int *sectors, int maxnstep, uint64_t seed,
                      int *isector, double *e0, double *gsvec, double *e_sector);

/* Dimension of the resident ground-state vector (0 if none). */
long long edzt_gs_dim(edzt_ctx *ctx);

/* green_diag (src/dmft_green.f90:177-260) on the resident ground state:
 * c^+ and c Lanczos runs of maxnstep steps in the N+-1 sectors,
 * b(1) = |c^(+)|gs>|, and g(iw) = CF_p(E0 + i w) + CF_m(-E0 + i w)
 * (src/numeric_utils.f90:11-44).  ap, bp, am, bm: [maxnstep]; g: complex [nw]. */
int edzt_green_diag(edzt_ctx *ctx, int iorb, int ispin, int maxnstep, int nw, const double *omega,
                    double *ap, double *bp, double *am, double *bm, double *g);

/* cluster_green_ftn (src/dmft_green.f90:47-126) on the resident ground
 * state: G_cl(nw, norb, nspin) complex (column-major, interleaved) and,
 * nullable, coeffs[norb][2][4][maxnstep] = (ap, bp, am, bm) per (orbital,
 * spin): the rows the reference writes to g_coeffs.dat.  All c/c^+ runs of
 * all orbitals and spins go to the device in one batched launch. */
int edzt_cluster_green_ftn(edzt_ctx *ctx, int nspin, int maxnstep, int nw, const double *omega,
                           double *G_cl, double *coeffs);

/* green_diag on the real axis: g(w) = CF_p(E0 + w + i eta) + CF_m(-E0 + w +
 * i eta) at the real frequencies omega[nw] (complex [nw]); the spectral
 * function is A(w) = -Im g(w) / pi (utils/spectral_ftn.py:35-44, which passes
 * the c^+ coefficients to CF_m as well; here each fraction gets its own). */
int edzt_green_real(edzt_ctx *ctx, int iorb, int ispin, int maxnstep, int nw, const double *omega, double eta,
                    double *g);

/* Occupancies of the resident ground state (src/post_process.f90:62-112):
 * occ(norb, nspin) (column-major, nullable) = <n_{iorb,ispin}>, docc(norb)
 * (nullable) = <n_{iorb,up} n_{iorb,down}>, summed on the device. */
int edzt_gs_occupancy(edzt_ctx *ctx, int nspin, double *occ, double *docc);

/* Full cluster Green's function matrix on the resident ground state:
 * G(nw, norb, norb, nspin) complex (column-major, interleaved).  No
 * counterpart in the reference, which computes the diagonal only
 * (src/dmft_green.f90:71-121): G_ab = (G_(a+b) - G_aa - G_bb) / 2 with
 * G_(a+b) green_diag's construction for c_a + c_b (c^+ and c runs from
 * (c_a^+ + c_b^+)|gs> and (c_a + c_b)|gs>), diagonal and spin rules as
 * edzt_cluster_green_ftn. */
int edzt_cluster_green_matrix(edzt_ctx *ctx, int nspin, int maxnstep, int nw, const double *omega, double *G);

/* One impurity solve: edzt_ground_state followed by edzt_cluster_green_ftn
 * (the calls at src/dmft.f90:76-78).  G_cl and coeffs nullable. */
int edzt_solve(edzt_ctx *ctx, int nsector, const int *sectors, int maxnstep, uint64_t seed, int nspin,
               int nw, const double *omega, int *isector, double *e0, double *G_cl, double *coeffs);

/* One impurity instance of a batch: the arguments of edzt_set_model, of
 * edzt_ground_state and of edzt_cluster_green_ftn for one solve.  Arrays are
 * host memory in the layouts above; sectors is [nsector][2] (ne_up, ne_dn);
 * sector i starts Lanczos from stream i of seed. */
typedef struct edzt_instance {
    int norb, nbath;
    const double *em, *ek, *vmk;
    double U, Up, Jex, Jp, mu;
    int nsector;
    const int *sectors;
    int nspin;
    uint64_t seed;
} edzt_instance;

/* Batched form of edzt_solve (the ground_state + cluster_green_ftn pair of
 * src/dmft.f90:76-78) for ninst independent instances of uneven Fock
 * dimension: the sector scans of all instances run in one persistent launch,
 * then all eigenvector passes, then all c / c^+ runs, in waves whose device
 * memory stays within hbm_budget bytes (0: 80% of the free memory).  Each
 * instance's results are those of edzt_solve on it alone, to rounding.
 * isector, e0: [ninst] (nullable); G_cl (nullable, host or device): the
 * instances' G_cl(nw, norb, nspin) complex arrays, concatenated in order. */
int edzt_solve_batch(edzt_ctx *ctx, int ninst, const edzt_instance *inst, int maxnstep, int nw,
                     const double *omega, int *isector, double *e0, double *G_cl, size_t hbm_budget);

/* Served form: continuous batching of impurity solves on one context.
 * Requests (edzt_instance, copied at submit) wait in a queue and are
 * admitted by their device-memory footprint (the sector scan's 40 B per
 * state, or the Green's runs') while the admitted ones fit hbm_budget (0: 80%
 * of the free memory; a request is always admitted when nothing else runs).
 * A request goes through three phases -- sector scan, eigenvector pass, c / c^+
 * runs plus continued fractions -- whose Lanczos runs live on the device
 * across launches.  Requests fall in size classes (by nsite; up to nsite 11
 * in one class).  Every edzt_server_step serves the next class in turn: it
 * runs persistent launches of a budget of Lanczos phases over that class's
 * runs (each launch ends with the unfinished runs' next step opened, and a
 * later launch resumes them) and moves requests on as their phase's runs
 * finish, until the step's time budget (edzt_server_set_step_ms, default 25
 * ms) is spent or the class has nothing left to run.  Requests submitted
 * meanwhile join at the next step.  A request's result is the same as
 * edzt_solve's on it alone, to rounding.  maxnstep, nw, omega are fixed per
 * server; destroy the server before its context. */
typedef struct edzt_server edzt_server;
int edzt_server_create(edzt_ctx *ctx, int maxnstep, int nw, const double *omega, size_t hbm_budget,
                       edzt_server **out);
/* Queues one request; *id identifies it. */
int edzt_server_submit(edzt_server *srv, const edzt_instance *inst, long long *id);
/* Admits what fits and serves the next size class for up to the step's time
 * budget (blocks until the step's GPU work is done).  nactive, nqueued,
 * nfinished nullable. */
int edzt_server_step(edzt_server *srv, int *nactive, int *nqueued, int *nfinished);
/* Time budget of one step in milliseconds (> 0; at least one launch of two
 * Lanczos phases runs per step whatever the budget). */
int edzt_server_set_step_ms(edzt_server *srv, double ms);
/* *done = 1 and the results (isector, e0, G_cl(nw, norb, nspin) complex; all
 * nullable) once request id has finished, which also releases it; *done = 0
 * while it runs. */
int edzt_server_result(edzt_server *srv, long long id, int *done, int *isector, double *e0, double *G_cl);
/* Removes a queued request, or marks a running one to leave at the next step
 * (its memory is released then); its result call reports EDZT_ERR_NUMERIC
 * "cancelled".  edzt_server_submit rejects a request whose device-memory
 * footprint exceeds the server's budget with EDZT_ERR_OOM. */
int edzt_server_cancel(edzt_server *srv, long long id);
void edzt_server_destroy(edzt_server *srv);
/* Device-memory footprint (bytes) a request holds at its peak in the batched
 * and served forms: the sector scan's pair and down-hop buffers (40 B per
 * state of every sector) or its Green's runs', whichever is larger, plus its
 * ground state. */
int edzt_instance_footprint(const edzt_instance *inst, long long *bytes);

/* Autotuner (north_star's tuned stripe width; no counterpart in the
 * reference): times short Lanczos runs (`steps` steps, 2..1000) of the
 * context's model on sector (ne_up, ne_dn) for every tile shape of the
 * persistent kernel that fits -- columns per slab of the column phase (the
 * stripe width: 2, 4, 8 or 16), rows per tile of the row phase (1, 2, 4 or
 * 8), one CTA of 512 or two of 256 threads per SM -- and records the fastest
 * on the context for that sector shape; later launches on the context use it
 * for every run of that shape (results unchanged but for rounding).
 * Outputs (nullable): the chosen shape and its time per Lanczos step.
 * edzt_clear_tuning forgets every recorded shape. */
int edzt_tune_sector(edzt_ctx *ctx, int ne_up, int ne_dn, int steps, int *cols_per_slab, int *rows_per_tile,
                     int *block, double *ms_per_step);
int edzt_clear_tuning(edzt_ctx *ctx);

/* Fault tests (no counterpart in the reference; no GPU fault is involved):
 * pass_cap > 0 caps the passes of a persistent launch (a run that needs more
 * fails with EDZT_ERR_NUMERIC); wait_seconds > 0 shortens the grid-barrier
 * wait limit (default 5 s); stall_cta >= 0 makes that CTA leave the launch
 * without arriving at the next grid barrier, so the others' bounded wait runs
 * out and the call returns EDZT_ERR_TIMEOUT.  All zero / -1: normal
 * operation.  The context stays usable after either error. */
int edzt_set_fault_test(edzt_ctx *ctx, int pass_cap, double wait_seconds, int stall_cta);

/* ---- the DMFT loop around the solver (host code, dmft_loop.cpp) ----------
 * The caller of the path, restated so that a whole DMFT run needs no
 * Fortran: the Bethe-lattice loop of src/dmft.f90:38-137 with the bath fit
 * of src/ed_projection.f90 and the output files of src/dump_data.f90 and
 * src/dmft_green.f90:66-109.  Arrays in the reference's Fortran layouts:
 * em(norb,2), ek(nbath,2), vmk(norb,nbath,2) and complex (nw,norb,nspin),
 * column-major, real and imaginary parts interleaved. */

/* D_cl = sum_l vmk^2 / (i w - ek) (cluster_hybridization_ftn,
 * src/dmft_green.f90:24-45).  No device needed. */
int edzt_hybridization(int norb, int nbath, int nspin, int nw, const double *omega, const double *ek,
                       const double *vmk, double *D);

/* local_green_ftn (src/dmft_green.f90:128-170): G_loc of the Bethe lattice
 * (semicircle, half-bandwidth 1) by the reference's 10000-point quadrature.
 * No device needed. */
int edzt_local_green_bethe(int norb, int nspin, int nw, const double *em, double hfield, const double *D,
                           const double *G_cl, double *G_loc);

/* fit_h_imp_params (src/ed_projection.f90:23-101): new (em, ek, vmk), in
 * place, minimising sum_{a,w} |em - em_old + D(ek,vmk) - D_old + 1/G_loc -
 * 1/G_cl|^2 / w / (norb nw) per spin by Polak-Ribiere conjugate gradients
 * (relative stop ftol; the reference's is 1e-6); nspin 1 copies spin up to
 * spin down.  cost (nullable) [nspin]: the final cost.  No device needed. */
int edzt_fit_bath(int norb, int nbath, int nspin, int nw, const double *omega, double *em, double *ek, double *vmk,
                  const double *D, const double *G_cl, const double *G_loc, double ftol, double *cost);

typedef struct edzt_dmft_params {
    int norb, nbath, nspin;
    double U, Up, Jex, Jp, mu, hfield;
    int nsector;
    const int *sectors;     /* [nsector][2]: (ne_up, ne_dn) */
    int maxnstep;           /* LanczosSteps */
    uint64_t seed;          /* start vectors, as edzt_ground_state */
    int nw;
    const double *omega;    /* [nw] Matsubara frequencies */
    int nloop;              /* at most this many iterations */
    double scf_tol;         /* stop when sum |G_cl - G_loc|^2 / (norb nbath nw) < scf_tol */
    double mixing;          /* (0, 1]: new = mixing * fitted + (1 - mixing) * previous; 1 = the reference */
    double fit_ftol;        /* bath-fit stop; 1e-6 = the reference */
    const char *outdir;     /* nullable: write h_imp.dat, green.dat.<o>.<s>, g_coeffs.dat every
                             * iteration and sigma.dat.<o>.<s> at the end, into this directory */
} edzt_dmft_params;

/* The DMFT loop (src/dmft.f90:55-98) with this library as the impurity
 * solver: em, ek, vmk (in/out) start as the initial bath and return the
 * last iteration's; D_cl, G_cl, G_loc (nullable) complex (nw,norb,nspin) of
 * the last iteration; Z (nullable) (norb,nspin) the quasiparticle weight
 * 1/(1 - Im Sigma(i w_1)/w_1) (src/post_process.f90:39-57, for every
 * orbital and spin); history (nullable) [nloop] the convergence measure of
 * each iteration; *iterations, *converged.  Errors of the solver calls are
 * returned as they come (edzt_last_error(ctx) has the message). */
int edzt_dmft_bethe(edzt_ctx *ctx, const edzt_dmft_params *p, double *em, double *ek, double *vmk, double *D_cl,
                    double *G_cl, double *G_loc, double *Z, int *iterations, double *history, int *converged);

/* Kernel launches issued by this context since creation (instrumentation). */
long long edzt_launch_count(const edzt_ctx *ctx);

/* The cudaStream_t every kernel of this context runs on (for event timing). */
int edzt_get_stream(edzt_ctx *ctx, void **stream);

/* Persistent Lanczos kernel statistics since the last reset: launches, total
 * device time (CUDA events around each launch, ms) and algorithmic HBM bytes
 * (24 B per state per coefficient step, 40 B per state per eigenvector step,
 * 8 B per state for a generated start vector, 16 B per state for a copied or
 * c/c^+-projected one). */
int edzt_kernel_stats(edzt_ctx *ctx, long long *launches, double *ms, double *bytes);
int edzt_reset_stats(edzt_ctx *ctx);
/* The same per launch, in launch order since the last reset (at most the
 * first 256 launches): device ms, algorithmic bytes and the states (sum of
 * the runs' sector dimensions) of each; *n receives the count returned (at
 * most max).  ms, bytes, states nullable. */
int edzt_kernel_launch_log(edzt_ctx *ctx, int max, int *n, double *ms, double *bytes, double *states);

#ifdef __cplusplus
}
#endif
#endif /* EDZT_H */
