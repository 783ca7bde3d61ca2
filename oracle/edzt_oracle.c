/*
 * edzt_oracle.c — CPU oracle for the zero-temperature ED impurity-solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
 * its reference arm) load the shared library built from it.  The product path
 * (dmft-ed-zt_b200/csrc) never links, loads or calls it.
 *
 * It restates, in plain C, the algorithm of the Fortran reference
 * (yw-choi/DMFT-ED-ZT) for the hot path, line by line where the reference is
 * explicit.  Every function cites the reference file:line it follows.
 *
 * Parity status: PINNED to the reference's own source.  The reference ships
 * no tests, golden vectors or fixtures, and it cannot be compiled in this
 * image (no Fortran compiler, MPI, MKL or ARPACK; its module graph is also
 * cyclic: dmft_green -> lanczos_solver -> impurity_hamiltonian ->
 * ed_projection -> dmft_green).  oracle/f90run.py instead translates the
 * reference's hot-path procedures statement by statement and runs them;
 * tests/golden/make_ref_golden.py records their outputs (with the SHA-256 of
 * every reference file read) in tests/golden/ref_golden.npz, and
 * tests/test_ref_golden.py holds this oracle to them: basis strings, hx (both
 * py forms, one to three orbitals, spin-flip and pair hopping) and apply_c
 * bit for bit, Lanczos coefficients, the ground state and G(i w) within 1e-12.
 * It is further checked against independent known-answer tests (dense
 * diagonalisation, the U=0 free-fermion limit, the atomic limit, sum rules,
 * particle-hole and spin symmetry, Hermiticity) and a literal pure-Python
 * transliteration (oracle/ref_literal.py).
 *
 * Deliberate, documented deviations from the reference (all also made by the
 * product so that both agree):
 *   - Fock states are held as 64-bit integers `up | down << nsite` instead of
 *     the reference's default 32-bit integer (src/ed_basis.f90:16-17,135),
 *     which overflows at nsite = 16.
 *   - The Lanczos start vector is a seeded counter-based hash (splitmix64,
 *     Steele/Lea/Flood 2014) instead of the unseeded `random_seed` /
 *     `random_number` of src/lanczos_solver.f90:42-46.  Entries are U[0,1)
 *     as in the reference.
 *   - Lanczos breakdown: the reference divides by b(k) before testing
 *     b(k) < 1e-16 (src/lanczos_solver.f90:152-161), which gives NaN for a
 *     one-dimensional sector.  Here the test comes first; on breakdown at
 *     step k the run stops with nstep = k-1 and a(k..), b(k..) = 0.
 *   - A zero start vector (an excitation that annihilates the ground state)
 *     or an empty sector returns nstep = 0 instead of NaN.
 *   - Sector selection keeps the first sector whose energy is lower by more
 *     than 1e-10*max(1,|E|) (src/ground_state.f90:62 uses a bare strict `<`,
 *     so 1e-15 rounding noise would pick among degenerate sectors).
 *   - Dot products (src/numeric_utils.f90:159-170, `sum(A*B)` whose order is
 *     compiler-defined) are summed in fixed chunks of ORACLE_CHUNK elements,
 *     chunks in ascending order, so the result does not depend on the number
 *     of OpenMP threads.
 *   - dstevx (MKL, src/lanczos_solver.f90:197) is replaced by Sturm-sequence
 *     bisection for the lowest eigenvalue plus inverse iteration for its
 *     eigenvector; only the lowest pair is ever used (src/lanczos_solver.f90:67-68).
 *   - green_diag builds z = cmplx(gs%val, omega(iw)) without a kind argument
 *     (src/dmft_green.f90:223,253), which Fortran evaluates in single
 *     precision; here z keeps E0 and w in double precision, as the product
 *     does.  Run literally, the reference's G(i w) differs from the double-
 *     precision one by about 1e-7 (tests/test_ref_golden.py records it).
 *
 * Layout conventions follow the reference's Fortran column-major arrays:
 *   em(norb,2)        -> em[iorb + norb*ispin]
 *   ek(nbath,2)       -> ek[jbath + nbath*ispin]
 *   vmk(norb,nbath,2) -> vmk[iorb + norb*(jbath + nbath*ispin)]
 * (all indices 0-based here).  A sector vector is indexed
 * i = idown*nup + iup (src/ed_basis.f90:132-135): the up rank is the fast index.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_CHUNK 4096
#define MAXSITE 20

typedef struct {
    int norb, nbath, nsite;
    double *em, *ek, *vmk;
    double U, Up, Jex, Jp, mu;
    /* per electron count n: ascending strings and dense 1-based rank table */
    int *str[MAXSITE + 1];
    int *idx[MAXSITE + 1];
    int cnt[MAXSITE + 1];
} or_ctx;

typedef struct {
    int ne_up, ne_dn;
    int nup, ndn;
    long long ntot;
    const int *up, *dn;
    const int *idx_up, *idx_dn;
} or_sector;

/* ------------------------------------------------------------------------- */
/* numeric_utils.f90:181-222  (icom via iP/ifact, int32 like the reference)   */
/* ------------------------------------------------------------------------- */
static int ifact(int n) { int f = 1; for (int i = 1; i <= n; i++) f *= i; return f; }
static int iP(int n, int m) { int p = 1; for (int i = n - m + 1; i <= n; i++) p *= i; return p; }

int or_icom(int n, int m)
{
    if (n == m || m == 0) return 1;
    if (m < 0 || m > n) return 0;           /* reference is undefined here */
    if (m > n / 2) { int k = n - m; return iP(n, k) / ifact(k); }
    return iP(n, m) / ifact(m);
}

/* ------------------------------------------------------------------------- */
/* ed_basis.f90:76-113: ascending enumeration of popcount-n strings over     */
/* [minrange, maxrange] and the dense rank table idx(minrange:maxrange).     */
/* ------------------------------------------------------------------------- */
int or_generate_spin_basis(int nsite, int n, int *strings, int *idx)
{
    int minrange = 0, maxrange = 0, counts = 0;
    if (n < 0 || n > nsite) return 0;
    for (int i = 1; i <= n; i++) {                       /* :81-84 */
        minrange += 1 << (i - 1);
        maxrange += 1 << (nsite - i);
    }
    if (idx) memset(idx, 0, sizeof(int) * ((size_t)1 << nsite));
    for (int i = minrange; i <= maxrange; i++) {         /* :94-112 */
        int nbit = 0;
        for (int j = 0; j < nsite; j++)
            if ((i >> j) & 1) nbit++;
        if (nbit == n) {
            counts++;
            if (strings) strings[counts - 1] = i;
            if (idx) idx[i] = counts;
        }
    }
    return counts;
}

static int ensure_spin(or_ctx *c, int n)
{
    if (n < 0 || n > c->nsite) return 0;
    if (!c->str[n]) {
        int C = or_icom(c->nsite, n);
        c->str[n] = (int *)malloc(sizeof(int) * (size_t)(C > 0 ? C : 1));
        c->idx[n] = (int *)malloc(sizeof(int) * ((size_t)1 << c->nsite));
        c->cnt[n] = or_generate_spin_basis(c->nsite, n, c->str[n], c->idx[n]);
    }
    return c->cnt[n];
}

/* generate_basis (ed_basis.f90:42-114), single rank: nloc = ntot. */
static int make_sector(or_ctx *c, int ne_up, int ne_dn, or_sector *s)
{
    memset(s, 0, sizeof(*s));
    s->ne_up = ne_up; s->ne_dn = ne_dn;
    if (ne_up < 0 || ne_dn < 0 || ne_up > c->nsite || ne_dn > c->nsite) return 0;
    s->nup = ensure_spin(c, ne_up);
    s->ndn = ensure_spin(c, ne_dn);
    s->ntot = (long long)s->nup * s->ndn;
    s->up = c->str[ne_up]; s->dn = c->str[ne_dn];
    s->idx_up = c->idx[ne_up]; s->idx_dn = c->idx[ne_dn];
    return 1;
}

/* ed_basis_get (ed_basis.f90:122-136), with a 64-bit state. */
static inline uint64_t basis_get(const or_ctx *c, const or_sector *s, long long b)
{
    long long iup = b % s->nup, idn = b / s->nup;
    return (uint64_t)(unsigned)s->up[iup] | ((uint64_t)(unsigned)s->dn[idn] << c->nsite);
}

/* ed_basis_idx (ed_basis.f90:139-151), 0-based result. */
static inline long long basis_idx(const or_ctx *c, const or_sector *s, uint64_t st)
{
    uint64_t mask = ((uint64_t)1 << c->nsite) - 1;
    int u = (int)(st & mask), d = (int)(st >> c->nsite);
    return (long long)(s->idx_dn[d] - 1) * s->nup + (s->idx_up[u] - 1);
}

#define BTEST(s, k) ((int)(((s) >> (k)) & 1u))
#define IBSET(s, k) ((s) | ((uint64_t)1 << (k)))
#define IBCLR(s, k) ((s) & ~((uint64_t)1 << (k)))

/* impurity_hamiltonian.f90:249-260: (-1)^{sum_{k=i}^{j-1} n_k}, 1-based k. */
static inline int sgn_h(uint64_t st, int i, int j)
{
    int s = 1;
    for (int k = i; k <= j - 1; k++) if (BTEST(st, k - 1)) s = -s;
    return s;
}

/* impurity_hamiltonian.f90:262-276 */
static inline int sgn2_h(uint64_t st, int i, int j, int nsite)
{
    int s = 1;
    for (int k = i; k <= j - 1; k++) {
        if (BTEST(st, k - 1)) s = -s;
        if (BTEST(st, nsite + k - 1)) s = -s;
    }
    return s;
}

/* ed_operator.f90:59-76: (-1)^{sum_{k=i}^{j} n_k}, 1-based k. */
static inline int sgn_op(uint64_t st, int i, int j)
{
    int sum = 0;
    for (int k = i; k <= j; k++) if (BTEST(st, k - 1)) sum++;
    return (sum % 2) ? -1 : 1;
}

/* ------------------------------------------------------------------------- */
/* context                                                                    */
/* ------------------------------------------------------------------------- */
or_ctx *or_create(int norb, int nbath, const double *em, const double *ek, const double *vmk,
                  double U, double Up, double Jex, double Jp, double mu)
{
    if (norb < 1 || nbath < 0 || norb + nbath > MAXSITE) return NULL;
    or_ctx *c = (or_ctx *)calloc(1, sizeof(or_ctx));
    c->norb = norb; c->nbath = nbath; c->nsite = norb + nbath;
    c->em = (double *)malloc(sizeof(double) * 2 * norb);
    c->ek = (double *)malloc(sizeof(double) * 2 * (nbath > 0 ? nbath : 1));
    c->vmk = (double *)malloc(sizeof(double) * 2 * norb * (nbath > 0 ? nbath : 1));
    memcpy(c->em, em, sizeof(double) * 2 * norb);
    if (nbath > 0) {
        memcpy(c->ek, ek, sizeof(double) * 2 * nbath);
        memcpy(c->vmk, vmk, sizeof(double) * 2 * norb * nbath);
    }
    c->U = U; c->Up = Up; c->Jex = Jex; c->Jp = Jp; c->mu = mu;
    return c;
}

void or_destroy(or_ctx *c)
{
    if (!c) return;
    for (int n = 0; n <= MAXSITE; n++) { free(c->str[n]); free(c->idx[n]); }
    free(c->em); free(c->ek); free(c->vmk); free(c);
}

long long or_sector_dim(or_ctx *c, int ne_up, int ne_dn)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s)) return 0;
    return s.ntot;
}

/* Copies the ascending up/down strings of a sector (generate_basis output). */
int or_basis(or_ctx *c, int ne_up, int ne_dn, int *up, int *dn)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s)) return -1;
    if (up) memcpy(up, s.up, sizeof(int) * (size_t)s.nup);
    if (dn) memcpy(dn, s.dn, sizeof(int) * (size_t)s.ndn);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* hx: impurity_hamiltonian.f90:77-247, row loop restated term by term.      */
/* ------------------------------------------------------------------------- */
#define EM(i, s) c->em[(i) + c->norb * (s)]
#define EK(j, s) c->ek[(j) + c->nbath * (s)]
#define VMK(i, j, s) c->vmk[(i) + c->norb * ((j) + c->nbath * (s))]

static void hx_range(const or_ctx *c, const or_sector *s, const double *x, double *y, int py,
                     long long r0, long long r1)
{
    const int norb = c->norb, nbath = c->nbath, nsite = c->nsite;
    const double U = c->U, Up = c->Up, Jex = c->Jex, Jp = c->Jp, mu = c->mu;
#pragma omp parallel for schedule(static)
    for (long long b = r0; b < r1; b++) {                               /* :98 */
        uint64_t bra = basis_get(c, s, b);                              /* :99 */
        double rowsum = 0.0;                                            /* :100 */
        int ni[2], nj[2];
        for (int iorb = 1; iorb <= norb; iorb++) {                      /* :102 */
            ni[0] = BTEST(bra, iorb - 1);                               /* :103-107 */
            ni[1] = BTEST(bra, nsite + iorb - 1);                       /* :109-113 */
            /* 1. onsite energies, 2. intra-orbital density-density :119-121 */
            rowsum = rowsum + ((EM(iorb - 1, 0) - mu) * ni[0]
                               + (EM(iorb - 1, 1) - mu) * ni[1]
                               + U * ni[0] * ni[1]) * x[b];
            /* 3. inter-orbital density-density :126-141 */
            for (int jorb = iorb + 1; jorb <= norb; jorb++) {
                nj[0] = BTEST(bra, jorb - 1);
                nj[1] = BTEST(bra, nsite + jorb - 1);
                rowsum = rowsum + ((Up - Jex) * (ni[0] * nj[0] + ni[1] * nj[1])
                                   + Up * (ni[0] * nj[1] + ni[1] * nj[0])) * x[b];
            }
            /* 4. hybridization :146-174 */
            for (int ispin = 1; ispin <= 2; ispin++) {
                for (int jbath = 1; jbath <= nbath; jbath++) {
                    double v = VMK(iorb - 1, jbath - 1, ispin - 1);
                    if (fabs(v) < 1.0e-16) continue;                    /* :148 */
                    int isite = (ispin - 1) * nsite + iorb;             /* :152 */
                    int jsite = (ispin - 1) * nsite + norb + jbath;     /* :153 */
                    int jb = BTEST(bra, jsite - 1);                     /* :155 */
                    if (ni[ispin - 1] == 0 && jb) {                     /* :157-163 */
                        uint64_t ket = IBSET(IBCLR(bra, jsite - 1), isite - 1);
                        long long a = basis_idx(c, s, ket);
                        rowsum = rowsum + (double)sgn_h(bra, isite, jsite) * v * x[a];
                    } else if (ni[ispin - 1] != 0 && !jb) {             /* :165-171 */
                        uint64_t ket = IBSET(IBCLR(bra, isite - 1), jsite - 1);
                        long long a = basis_idx(c, s, ket);
                        rowsum = rowsum - (double)sgn_h(bra, isite, jsite) * v * x[a];
                    }
                }
            }
            /* 5. spin-flip and pair-hopping :179-226 */
            for (int jorb = 1; jorb <= norb; jorb++) {
                if (iorb == jorb) continue;
                nj[0] = BTEST(bra, jorb - 1);
                nj[1] = BTEST(bra, nsite + jorb - 1);
                int imin = iorb < jorb ? iorb : jorb;
                int imax = iorb < jorb ? jorb : iorb;
                if (ni[0] == 0 && nj[0] != 0 && nj[1] == 0 && ni[1] != 0) {   /* :201-211 */
                    uint64_t ket = IBCLR(bra, nsite + iorb - 1);
                    ket = IBSET(ket, nsite + jorb - 1);
                    ket = IBCLR(ket, jorb - 1);
                    ket = IBSET(ket, iorb - 1);
                    long long a = basis_idx(c, s, ket);
                    rowsum = rowsum - (double)sgn2_h(bra, imin, imax, nsite) * Jp * x[a];
                }
                if (ni[0] == 0 && ni[1] == 0 && nj[0] != 0 && nj[1] != 0) {   /* :215-225 */
                    uint64_t ket = IBCLR(bra, nsite + jorb - 1);
                    ket = IBSET(ket, nsite + iorb - 1);
                    ket = IBCLR(ket, jorb - 1);
                    ket = IBSET(ket, iorb - 1);
                    long long a = basis_idx(c, s, ket);
                    rowsum = rowsum + (double)sgn2_h(bra, imin, imax, nsite) * Jp * x[a];
                }
            }
        }
        /* 6. bath onsite :232-239 */
        for (int jbath = 1; jbath <= nbath; jbath++) {
            if (BTEST(bra, norb + jbath - 1)) rowsum = rowsum + EK(jbath - 1, 0) * x[b];
            if (BTEST(bra, nsite + norb + jbath - 1)) rowsum = rowsum + EK(jbath - 1, 1) * x[b];
        }
        if (py) y[b] = y[b] + rowsum;                                   /* :241-245 */
        else y[b] = rowsum;
    }
}

static void hx_rows(const or_ctx *c, const or_sector *s, const double *x, double *y, int py)
{
    hx_range(c, s, x, y, py, 0, s->ntot);
}

/* Rows [r0, r1) of H x only (y indexed globally); spot checks of large sectors. */
int or_hx_rows(or_ctx *c, int ne_up, int ne_dn, const double *x, double *y, long long r0, long long r1)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s)) return -1;
    if (r0 < 0) r0 = 0;
    if (r1 > s.ntot) r1 = s.ntot;
    hx_range(c, &s, x, y, 0, r0, r1);
    return 0;
}

int or_hx(or_ctx *c, int ne_up, int ne_dn, const double *x, double *y, int py)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s)) return -1;
    hx_rows(c, &s, x, y, py);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* apply_c: ed_operator.f90:13-57, written row-wise over the output basis.    */
/* ------------------------------------------------------------------------- */
static void apply_c_rows(const or_ctx *c, const or_sector *sin, const double *vec, int pm,
                         int iorb, int ispin, const or_sector *sout, double *vec_out)
{
    const int nsite = c->nsite;
    long long nout = sout->ntot;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nout; i++) {                              /* :31 */
        vec_out[i] = 0.0;                                               /* :24 */
        uint64_t basis_i = basis_get(c, sout, i);                       /* :32 */
        int isite = (ispin - 1) * nsite + iorb;                         /* :33 */
        int sgntot = sgn_op(basis_i, 1, isite - 1);                     /* :34 */
        uint64_t basis_j;
        if (pm == 1) {                                                  /* :36-40 */
            if (!BTEST(basis_i, isite - 1)) sgntot = 0;
            basis_j = IBCLR(basis_i, isite - 1);
        } else {                                                        /* :41-46 */
            if (BTEST(basis_i, isite - 1)) sgntot = 0;
            basis_j = IBSET(basis_i, isite - 1);
        }
        if (sgntot == 0) continue;                                      /* :48-50 */
        long long j = basis_idx(c, sin, basis_j);                       /* :52 */
        vec_out[i] = vec_out[i] + vec[j] * sgntot;                      /* :53 */
    }
}

/* Output sector of apply_c as chosen by green_diag (dmft_green.f90:204-210,232-238). */
static void excitation_sector(int ne_up, int ne_dn, int pm, int ispin, int *oup, int *odn)
{
    int d = (pm == 1) ? 1 : -1;
    *oup = ne_up + (ispin == 1 ? d : 0);
    *odn = ne_dn + (ispin == 2 ? d : 0);
}

int or_apply_c(or_ctx *c, int ne_up, int ne_dn, const double *vec, int pm, int iorb, int ispin,
               double *vec_out)
{
    or_sector sin, sout;
    int oup, odn;
    if (pm != 1 && pm != 2) return -1;
    if (iorb < 1 || iorb > c->norb || ispin < 1 || ispin > 2) return -1;
    if (!make_sector(c, ne_up, ne_dn, &sin)) return -1;
    excitation_sector(ne_up, ne_dn, pm, ispin, &oup, &odn);
    if (!make_sector(c, oup, odn, &sout)) return 1;   /* empty output sector */
    apply_c_rows(c, &sin, vec, pm, iorb, ispin, &sout, vec_out);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* mpi_dot_product / mpi_norm: numeric_utils.f90:159-179 (single rank).      */
/* ------------------------------------------------------------------------- */
double or_dot(const double *A, const double *B, long long n)
{
    long long nch = (n + ORACLE_CHUNK - 1) / ORACLE_CHUNK;
    double *part = (double *)malloc(sizeof(double) * (size_t)(nch > 0 ? nch : 1));
#pragma omp parallel for schedule(static)
    for (long long ch = 0; ch < nch; ch++) {
        long long i0 = ch * ORACLE_CHUNK, i1 = i0 + ORACLE_CHUNK;
        if (i1 > n) i1 = n;
        double s = 0.0;
        for (long long i = i0; i < i1; i++) s = s + A[i] * B[i];
        part[ch] = s;
    }
    double dab = 0.0;
    for (long long ch = 0; ch < nch; ch++) dab = dab + part[ch];
    free(part);
    return dab;
}

static double or_norm(const double *A, long long n) { return sqrt(or_dot(A, A, n)); }

/* daxpy: y = y + a*x (lanczos_solver.f90:143,166,...). */
static void axpy(long long n, double a, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; i++) y[i] = y[i] + a * x[i];
}

/* ------------------------------------------------------------------------- */
/* start vector: replaces random_seed/random_number (lanczos_solver.f90:42-46)*/
/* splitmix64 (Steele, Lea, Flood, OOPSLA 2014) as a counter-based hash.      */
/* ------------------------------------------------------------------------- */
static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void or_start_vector(uint64_t seed, uint64_t stream, long long n, double *v)
{
    uint64_t key = mix64(seed ^ mix64(stream));
    for (long long i = 0; i < n; i++)
        v[i] = (double)(mix64(key + (uint64_t)i) >> 11) * 0x1.0p-53;
}

/* ------------------------------------------------------------------------- */
/* lanczos_iteration: lanczos_solver.f90:92-173                               */
/* Returns nstep; a, b have maxnstep entries.                                 */
/* ------------------------------------------------------------------------- */
static int lanczos_iteration_s(const or_ctx *c, const or_sector *s, const double *v_init,
                               int maxnstep, double *a, double *b, double *norm_out)
{
    long long nloc = s->ntot;
    for (int i = 0; i < maxnstep; i++) { a[i] = 0.0; b[i] = 0.0; }   /* :116-117 */
    if (norm_out) *norm_out = 0.0;
    if (nloc <= 0 || maxnstep < 1) return 0;
    double *v = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *w = (double *)malloc(sizeof(double) * (size_t)nloc);
    double norm_v = or_norm(v_init, nloc);                              /* :128 */
    if (norm_out) *norm_out = norm_v;
    if (!(norm_v > 0.0)) { free(v); free(w); return 0; }
    for (long long i = 0; i < nloc; i++) w[i] = v_init[i] / norm_v;     /* :130 */
    hx_rows(c, s, w, v, 0);                                             /* :132 */
    a[0] = or_dot(w, v, nloc);                                          /* :134 */
    b[0] = 0.0;                                                         /* :135 */
    int nstep;
    if (maxnstep == 1) { free(v); free(w); return 1; }                  /* :137-141 */
    axpy(nloc, -a[0], w, v);                                            /* :143 */
    b[1] = or_norm(v, nloc);                                            /* :144 */
    int k = 2;                                                          /* :146 */
    for (;;) {
        if (b[k - 1] < 1.0e-16) {          /* breakdown test moved before the divide */
            nstep = k - 1;
            b[k - 1] = 0.0;
            break;
        }
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < nloc; i++) {                          /* :152-156 */
            double t = w[i];
            w[i] = v[i] / b[k - 1];
            v[i] = -b[k - 1] * t;
        }
        hx_rows(c, s, w, v, 1);                                         /* :158 */
        a[k - 1] = or_dot(w, v, nloc);                                  /* :159 */
        if (k >= maxnstep) { nstep = k; break; }                        /* :161-164 */
        axpy(nloc, -a[k - 1], w, v);                                    /* :166 */
        b[k] = or_norm(v, nloc);                                        /* :167 */
        k = k + 1;
    }
    free(v); free(w);
    return nstep;
}

int or_lanczos_iteration(or_ctx *c, int ne_up, int ne_dn, const double *v_init, int maxnstep,
                         int *nstep, double *a, double *b)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s)) return -1;
    *nstep = lanczos_iteration_s(c, &s, v_init, maxnstep, a, b, NULL);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* lanczos_diagonalize replacement (lanczos_solver.f90:175-211, MKL dstevx):  */
/* lowest eigenpair of the tridiagonal with d = a(1:n), e = b(2:n).           */
/* ------------------------------------------------------------------------- */
/* Number of eigenvalues strictly below x (Sturm sequence, LDL^T pivots).     */
static int sturm_count(int n, const double *d, const double *e2, double x, double pivmin)
{
    int cnt = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) cnt++;
    for (int i = 1; i < n; i++) {
        q = d[i] - x - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0) cnt++;
    }
    return cnt;
}

int or_tridiag_lowest(int n, const double *a, const double *b, double *e0, double *z)
{
    if (n < 1) return -1;
    if (n == 1) { *e0 = a[0]; if (z) z[0] = 1.0; return 0; }
    double *e2 = (double *)malloc(sizeof(double) * (size_t)n);
    double lo = a[0], hi = a[0], emax2 = 0.0, tnorm = 0.0;
    for (int i = 0; i < n; i++) {
        double r = 0.0;
        if (i > 0) r += fabs(b[i]);
        if (i < n - 1) r += fabs(b[i + 1]);
        if (a[i] - r < lo) lo = a[i] - r;
        if (a[i] + r > hi) hi = a[i] + r;
        if (fabs(a[i]) + r > tnorm) tnorm = fabs(a[i]) + r;
    }
    for (int i = 0; i < n - 1; i++) { e2[i] = b[i + 1] * b[i + 1]; if (e2[i] > emax2) emax2 = e2[i]; }
    double pivmin = 2.2250738585072014e-308 * (emax2 > 1.0 ? emax2 : 1.0);
    lo -= 2.0 * 2.220446049250313e-16 * tnorm + pivmin;
    hi += 2.0 * 2.220446049250313e-16 * tnorm + pivmin;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(n, a, e2, mid, pivmin) >= 1) hi = mid; else lo = mid;
    }
    double lam = 0.5 * (lo + hi);
    *e0 = lam;
    free(e2);
    if (!z) return 0;
    /* inverse iteration: (T - lam I) x = rhs by Gaussian elimination with
     * partial pivoting on the tridiagonal (three bands + one fill-in band) */
    double *dl = (double *)malloc(sizeof(double) * (size_t)n);
    double *dd = (double *)malloc(sizeof(double) * (size_t)n);
    double *du = (double *)malloc(sizeof(double) * (size_t)n);
    double *du2 = (double *)malloc(sizeof(double) * (size_t)n);
    int *piv = (int *)malloc(sizeof(int) * (size_t)n);
    double shift = lam;
    double eps = 2.220446049250313e-16;
    for (int i = 0; i < n; i++) {
        dd[i] = a[i] - shift;
        du[i] = (i < n - 1) ? b[i + 1] : 0.0;
        dl[i] = (i < n - 1) ? b[i + 1] : 0.0;
        du2[i] = 0.0;
    }
    for (int i = 0; i < n - 1; i++) {
        if (fabs(dd[i]) >= fabs(dl[i])) {
            piv[i] = 0;
            if (dd[i] == 0.0) dd[i] = eps * tnorm;
            double f = dl[i] / dd[i];
            dl[i] = f;
            dd[i + 1] -= f * du[i];
            du2[i] = 0.0;
        } else {
            piv[i] = 1;
            double f = dd[i] / dl[i];
            dd[i] = dl[i];
            dl[i] = f;
            double t = du[i];
            du[i] = dd[i + 1];
            dd[i + 1] = t - f * dd[i + 1];
            if (i < n - 2) { du2[i] = du[i + 1]; du[i + 1] = -f * du[i + 1]; }
        }
    }
    if (dd[n - 1] == 0.0) dd[n - 1] = eps * tnorm;
    for (int i = 0; i < n; i++) z[i] = 1.0;
    for (int it = 0; it < 3; it++) {
        /* forward: apply L^{-1} with row interchanges */
        for (int i = 0; i < n - 1; i++) {
            if (piv[i] == 0) z[i + 1] -= dl[i] * z[i];
            else { double t = z[i]; z[i] = z[i + 1]; z[i + 1] = t - dl[i] * z[i]; }
        }
        /* backward: U x = z */
        z[n - 1] /= dd[n - 1];
        if (n > 1) z[n - 2] = (z[n - 2] - du[n - 2] * z[n - 1]) / dd[n - 2];
        for (int i = n - 3; i >= 0; i--) z[i] = (z[i] - du[i] * z[i + 1] - du2[i] * z[i + 2]) / dd[i];
        double nrm = 0.0, big = 0.0;
        for (int i = 0; i < n; i++) { nrm += z[i] * z[i]; if (fabs(z[i]) > fabs(big)) big = z[i]; }
        nrm = sqrt(nrm);
        if (big < 0) nrm = -nrm;           /* sign: largest component positive */
        for (int i = 0; i < n; i++) z[i] /= nrm;
    }
    free(dl); free(dd); free(du); free(du2); free(piv);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* lanczos_ground_state: lanczos_solver.f90:213-300                           */
/* ------------------------------------------------------------------------- */
static void lanczos_ground_state_s(const or_ctx *c, const or_sector *s, const double *v_init, int nstep,
                                   const double *a, const double *b, const double *coeff,
                                   double eigval, double *eigvec, double *residual)
{
    long long nloc = s->ntot;
    double *v = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *w = (double *)malloc(sizeof(double) * (size_t)nloc);
    double norm_v = or_norm(v_init, nloc);                              /* :249 */
    for (long long i = 0; i < nloc; i++) w[i] = v_init[i] / norm_v;     /* :251 */
    for (long long i = 0; i < nloc; i++) eigvec[i] = 0.0;              /* :254 */
    axpy(nloc, coeff[0], w, eigvec);                                    /* :255 */
    hx_rows(c, s, w, v, 0);                                             /* :257 */
    if (nstep > 1) {                                                    /* :259-262 */
        axpy(nloc, -a[0], w, v);                                        /* :264 */
        int k = 2;
        for (;;) {
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < nloc; i++) {                      /* :272-276 */
                double t = w[i];
                w[i] = v[i] / b[k - 1];
                v[i] = -b[k - 1] * t;
            }
            axpy(nloc, coeff[k - 1], w, eigvec);                        /* :279 */
            hx_rows(c, s, w, v, 1);                                     /* :281 */
            if (k >= nstep || b[k - 1] < 1.0e-16) break;                /* :283-285 */
            axpy(nloc, -a[k - 1], w, v);                                /* :287 */
            k = k + 1;
        }
    }
    /* The reference returns before normalising when nstep == 1 (:259-262),
     * leaving eigvec = coeff(1)*w = w, already normalised; normalising
     * unconditionally is the same up to rounding. */
    double nrm = or_norm(eigvec, nloc);                                 /* :291 */
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nloc; i++) eigvec[i] = eigvec[i] / nrm;
    hx_rows(c, s, eigvec, v, 0);                                        /* :294 */
    axpy(nloc, -eigval, eigvec, v);                                     /* :295 */
    if (residual) *residual = or_dot(v, v, nloc);                       /* :297 */
    free(v); free(w);
}

/* diag_lanczos: lanczos_solver.f90:20-90 with a seeded start vector. */
static int diag_lanczos_s(const or_ctx *c, const or_sector *s, int maxnstep, uint64_t seed,
                          uint64_t stream, double *eigval, double *eigvec, double *residual,
                          int *nstep_out, double *a_out, double *b_out)
{
    long long nloc = s->ntot;
    double *v_init = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *a = (double *)malloc(sizeof(double) * (size_t)maxnstep);
    double *b = (double *)malloc(sizeof(double) * (size_t)maxnstep);
    or_start_vector(seed, stream, nloc, v_init);                        /* :42-46 */
    int nstep = lanczos_iteration_s(c, s, v_init, maxnstep, a, b, NULL);/* :49 */
    if (nstep_out) *nstep_out = nstep;
    if (a_out) memcpy(a_out, a, sizeof(double) * (size_t)maxnstep);
    if (b_out) memcpy(b_out, b, sizeof(double) * (size_t)maxnstep);
    double *coeff = (double *)malloc(sizeof(double) * (size_t)(nstep > 0 ? nstep : 1));
    int rc = 0;
    if (nstep < 1) rc = -1;
    else {
        or_tridiag_lowest(nstep, a, b, eigval, coeff);                  /* :64-68 */
        if (eigvec)
            lanczos_ground_state_s(c, s, v_init, nstep, a, b, coeff, *eigval, eigvec, residual); /* :80 */
    }
    free(coeff); free(v_init); free(a); free(b);
    return rc;
}

int or_diag_lanczos(or_ctx *c, int ne_up, int ne_dn, int maxnstep, uint64_t seed, uint64_t stream,
                    double *eigval, double *eigvec, double *residual, int *nstep, double *a, double *b)
{
    or_sector s;
    if (!make_sector(c, ne_up, ne_dn, &s) || s.ntot == 0) return -1;
    return diag_lanczos_s(c, &s, maxnstep, seed, stream, eigval, eigvec, residual, nstep, a, b);
}

/* ------------------------------------------------------------------------- */
/* ground_state: ground_state.f90:1-81                                        */
/* sectors: [nsector][2] (ne_up, ne_dn).  gsvec must hold the largest sector.  */
/* e_sector (nullable): per-sector lowest energies.                           */
/* ------------------------------------------------------------------------- */
int or_ground_state(or_ctx *c, int nsector, const int *sectors, int maxnstep, uint64_t seed,
                    int *isector, double *e0, double *gsvec, double *e_sector, double *residual_out)
{
    double best = HUGE_VAL;                                             /* :28 */
    int best_i = -1;
    long long maxdim = 0;
    for (int is = 0; is < nsector; is++) {
        long long d = or_sector_dim(c, sectors[2 * is], sectors[2 * is + 1]);
        if (d > maxdim) maxdim = d;
    }
    double *vec = (double *)malloc(sizeof(double) * (size_t)(maxdim > 0 ? maxdim : 1));
    for (int is = 0; is < nsector; is++) {                              /* :30 */
        or_sector s;
        double ev = HUGE_VAL, res = 0.0;
        if (e_sector) e_sector[is] = NAN;
        if (!make_sector(c, sectors[2 * is], sectors[2 * is + 1], &s) || s.ntot == 0) continue;
        if (diag_lanczos_s(c, &s, maxnstep, seed, (uint64_t)is, &ev, vec, &res, NULL, NULL, NULL) != 0)
            continue;                                                   /* :55 */
        if (e_sector) e_sector[is] = ev;
        double tie = 1.0e-10 * (fabs(best) > 1.0 ? fabs(best) : 1.0);
        if (best_i < 0 || ev < best - tie) {                            /* :62-68 */
            best = ev; best_i = is;
            if (gsvec) memcpy(gsvec, vec, sizeof(double) * (size_t)s.ntot);
            if (residual_out) *residual_out = res;
        }
    }
    free(vec);
    *isector = best_i;
    *e0 = best;
    return best_i >= 0 ? 0 : -1;
}

/* ------------------------------------------------------------------------- */
/* continued fractions: numeric_utils.f90:11-44 (complex z = zr + i zi)       */
/* ------------------------------------------------------------------------- */
static inline void cdiv(double ar, double ai, double br, double bi, double *cr, double *ci)
{
    /* (ar + i ai) / (br + i bi), Smith's algorithm */
    if (fabs(br) >= fabs(bi)) {
        double r = bi / br, den = br + bi * r;
        *cr = (ar + ai * r) / den;
        *ci = (ai - ar * r) / den;
    } else {
        double r = br / bi, den = bi + br * r;
        *cr = (ar * r + ai) / den;
        *ci = (ai * r - ar) / den;
    }
}

/* sign = -1: continued_fraction_p (z - a), sign = +1: continued_fraction_m (z + a) */
void or_continued_fraction(double zr, double zi, int n, const double *a, const double *b, int sign,
                           double *fr, double *fi)
{
    double xr, xi;
    cdiv(b[n - 1] * b[n - 1], 0.0, zr + sign * a[n - 1], zi, &xr, &xi);         /* :18 / :39 */
    for (int i = n - 1; i >= 2; i--)                                           /* :19-21 */
        cdiv(b[i - 1] * b[i - 1], 0.0, zr + sign * a[i - 1] - xr, zi - xi, &xr, &xi);
    cdiv(b[0] * b[0], 0.0, zr + sign * a[0] - xr, zi - xi, &xr, &xi);         /* :22 / :43 */
    *fr = xr; *fi = xi;
}

/* Number of continued-fraction levels used for a run that returned nstep:
 * a breakdown after the first vector (nstep == 1 < maxnstep) is evaluated
 * with a zero second level, which is exactly b(1)^2/(z - a(1)). */
static int cf_levels(int nstep, int maxnstep) { return (nstep == 1 && maxnstep >= 2) ? 2 : nstep; }

/* ------------------------------------------------------------------------- */
/* green_diag: dmft_green.f90:177-260                                         */
/* g: complex [nw] as interleaved (re, im); ap..bm: [maxnstep]                */
/* nstep_out (nullable): [2] = nstep of the c^+ and c runs                    */
/* ------------------------------------------------------------------------- */
int or_green_diag(or_ctx *c, int ne_up, int ne_dn, const double *gsvec, double e0, int iorb, int ispin,
                  int maxnstep, int nw, const double *omega, double *ap, double *bp, double *am,
                  double *bm, double *g, int *nstep_out)
{
    or_sector sgs;
    if (!make_sector(c, ne_up, ne_dn, &sgs)) return -1;
    for (int iw = 0; iw < nw; iw++) { g[2 * iw] = 0.0; g[2 * iw + 1] = 0.0; }   /* :200 */
    for (int pm = 1; pm <= 2; pm++) {
        double *aa = (pm == 1) ? ap : am, *bb = (pm == 1) ? bp : bm;
        int oup, odn;
        or_sector sout;
        for (int i = 0; i < maxnstep; i++) { aa[i] = 0.0; bb[i] = 0.0; }
        if (nstep_out) nstep_out[pm - 1] = 0;
        excitation_sector(ne_up, ne_dn, pm, ispin, &oup, &odn);         /* :204-210, :232-238 */
        if (!make_sector(c, oup, odn, &sout) || sout.ntot == 0) continue;
        double *v_init = (double *)malloc(sizeof(double) * (size_t)sout.ntot);
        apply_c_rows(c, &sgs, gsvec, pm, iorb, ispin, &sout, v_init);  /* :215 / :245 */
        double nrm = 0.0;
        int nstep = lanczos_iteration_s(c, &sout, v_init, maxnstep, aa, bb, &nrm); /* :218 / :248 */
        if (nstep_out) nstep_out[pm - 1] = nstep;
        free(v_init);
        if (nstep < 1) continue;
        bb[0] = nrm;                                                    /* :219 / :249 */
        int nl = cf_levels(nstep, maxnstep);
        for (int iw = 0; iw < nw; iw++) {                               /* :222-226 / :252-257 */
            double fr, fi;
            if (pm == 1) or_continued_fraction(e0, omega[iw], nl, aa, bb, -1, &fr, &fi);
            else or_continued_fraction(-e0, omega[iw], nl, aa, bb, +1, &fr, &fi);
            g[2 * iw] += fr;
            g[2 * iw + 1] += fi;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* cluster_green_ftn: dmft_green.f90:47-126                                   */
/* G_cl: complex (nw, norb, nspin) column-major, interleaved (re, im).         */
/* coeffs (nullable): [norb][2][4][maxnstep] = ap, bp, am, bm per (orb, spin), */
/* the rows that g_coeffs.dat receives (dmft_green.f90:89-109).               */
/* ------------------------------------------------------------------------- */
int or_cluster_green_ftn(or_ctx *c, int nspin, int ne_up, int ne_dn, const double *gsvec, double e0,
                         int maxnstep, int nw, const double *omega, double *G_cl, double *coeffs)
{
    int norb = c->norb;
    int even = !(nspin == 2 || ne_up != ne_dn);                         /* :76-80 */
    double *g1 = (double *)malloc(sizeof(double) * 2 * (size_t)nw);
    double *g2 = (double *)malloc(sizeof(double) * 2 * (size_t)nw);
    double *ap = (double *)malloc(sizeof(double) * (size_t)maxnstep * 4);
    double *bp = ap + maxnstep, *am = bp + maxnstep, *bm = am + maxnstep;
    memset(G_cl, 0, sizeof(double) * 2 * (size_t)nw * norb * nspin);  /* :62 */
    for (int iorb = 1; iorb <= norb; iorb++) {                          /* :71 */
        or_green_diag(c, ne_up, ne_dn, gsvec, e0, iorb, 1, maxnstep, nw, omega, ap, bp, am, bm, g1, NULL);
        if (coeffs) memcpy(coeffs + ((size_t)(iorb - 1) * 2 + 0) * 4 * maxnstep, ap, sizeof(double) * 4 * maxnstep);
        if (!even)                                                      /* :96-100 */
            or_green_diag(c, ne_up, ne_dn, gsvec, e0, iorb, 2, maxnstep, nw, omega, ap, bp, am, bm, g2, NULL);
        if (coeffs) memcpy(coeffs + ((size_t)(iorb - 1) * 2 + 1) * 4 * maxnstep, ap, sizeof(double) * 4 * maxnstep);
        for (int iw = 0; iw < nw; iw++) {                               /* :111-118 */
            size_t o1 = 2 * ((size_t)iw + (size_t)nw * ((iorb - 1) + (size_t)norb * 0));
            size_t o2 = 2 * ((size_t)iw + (size_t)nw * ((iorb - 1) + (size_t)norb * 1));
            if (nspin == 1 && even) {
                G_cl[o1] = g1[2 * iw]; G_cl[o1 + 1] = g1[2 * iw + 1];
            } else if (nspin == 1) {
                G_cl[o1] = 0.5 * (g1[2 * iw] + g2[2 * iw]);
                G_cl[o1 + 1] = 0.5 * (g1[2 * iw + 1] + g2[2 * iw + 1]);
            } else {
                G_cl[o1] = g1[2 * iw]; G_cl[o1 + 1] = g1[2 * iw + 1];
                G_cl[o2] = g2[2 * iw]; G_cl[o2 + 1] = g2[2 * iw + 1];
            }
        }
    }
    free(g1); free(g2); free(ap);
    return 0;
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
