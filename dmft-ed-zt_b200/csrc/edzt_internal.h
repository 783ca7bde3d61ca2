// edzt_internal.h — host-side declarations shared by the CUDA translation
// units of libedzt (not part of the public C ABI; see include/edzt.h).
#pragma once
#include <atomic>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "edzt_device.cuh"

// Impurity model as the kernels see it.  Shapes follow the reference's
// Fortran arrays em(norb,2), ek(nbath,2), vmk(norb,nbath,2)
// (src/impurity_hamiltonian.f90:80-84), stored here with the spin index last.
struct DevModel {
    int norb, nbath, nsite;
    double em[EDZT_MAX_NORB][2];
    double ek[EDZT_MAX_NSITE][2];
    double vmk[EDZT_MAX_NORB][EDZT_MAX_NSITE][2];
    double U, Up, Jex, Jp, mu;
};

// True the first time it is called for the current device with this set of
// flags: per-device one-time set-up such as a kernel's shared-memory
// attribute, which cudaFuncSetAttribute sets for the current device only.
inline bool edzt_once_per_device(std::atomic<unsigned long long>& done)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
    const unsigned long long bit = 1ull << dev;
    return (done.fetch_or(bit) & bit) == 0;
}

// ---- tables.cu -------------------------------------------------------------
void edzt_init_binomials(int device);
uint64_t edzt_binom(int n, int k);
// Fills str[C(nsite,n)] (ascending) and rank[2^nsite] on the device.
void launch_build_strings(int nsite, int n, uint32_t* str, int32_t* rank, cudaStream_t s);
// Per-string tables of one spin species (sigma = 0 up, 1 down) for a model.
// hpk: [hw/4][count] uint4 (packed hop entries, see edzt_hop_pack); amp:
// [2*norb*nbath] (at least 2) amplitude slots.
void launch_build_spin_ops(const DevModel& m, int sigma, int count, const uint32_t* str, const int32_t* rank,
                           int hw, double* e1, uint8_t* hcnt, uint32_t* hpk, double* amp, uint8_t* imp,
                           int32_t* sub, cudaStream_t s);
// Largest number of allowed hops of any string with n electrons of spin sigma.
int edzt_max_hops(const DevModel& m, int sigma, int n);

// ---- kernels.cu: standalone (non-persistent) kernels ------------------------
// Ground-state vector from the kept pairs of a coefficient run: out =
// sum_{k=1..nstep} coeff[k-1] w_k, w_k the second value of step k's pair,
// accumulated in step order as the eigenvector pass does.
void launch_keep_combine(const double2* keep, long long dim, int nstep, const double* coeff, double* out,
                         cudaStream_t s);
// H.v in two phases (hv_phase.cuh); scratch: hx_scratch_size doubles of
// device memory (the down-hop part, slab-major, slabs of up to 16 columns).
void launch_hx(const DevSector& S, const double* x, double* y, int accumulate, double* scratch, cudaStream_t s);
inline long long hx_scratch_size(int nup, int ndn) { return (long long)((nup + 15) / 16) * 16 * ndn; }
// Whether a sector's staged row and column slab fit in shared memory.
bool hx_fits(int nup, int ndn);
// Deterministic dot product: result written to *out (device).  partials needs
// dot_partials_size() doubles.
int dot_partials_size();
void launch_dot(const double* a, const double* b, long long n, double* partials, double* out, cudaStream_t s);
// Scalars come from *p when p is non-null, else from the value argument.
void launch_swap_scale(double* w, double* v, long long n, const double* bk_p, double bk, cudaStream_t s);
void launch_axpy(double* y, const double* x, long long n, const double* alpha_p, double alpha, double sign,
                 cudaStream_t s);
void launch_scale_inv_sqrt(double* x, long long n, const double* nrm2, cudaStream_t s);
void launch_fill_start(double* v, long long n, uint64_t key, cudaStream_t s);
void launch_copy(double* dst, const double* src, long long n, cudaStream_t s);

void launch_apply_c(const ApplyCArgs& A, const double* in, double* out, cudaStream_t s);
// Per-block partial sums [occ_partials_size()] = [block][12]: occupation of
// orbital a by up (q = a), down (q = 4 + a) and both spins (q = 8 + a).
int occ_partials_size();
void launch_gs_occ(const double* x, const uint32_t* up, const uint32_t* dn, int nup, long long dim, int norb,
                   double* part, cudaStream_t s);

// Continued fractions (src/numeric_utils.f90:11-44) for many runs at once.
struct CFJob {
    const double* a;      // [levels]
    const double* b;      // [levels], b[0] unused
    double b1;            // b(1) = ||c^(+)|gs>|| (dmft_green.f90:219,249)
    int levels;           // number of CF levels (0: contributes nothing)
    double zr_shift;      // real part of z: +E0 for c^+, -E0 for c
    double sign;          // -1: z - a (continued_fraction_p), +1: z + a (continued_fraction_m)
    double* g;            // [nw] complex interleaved, written (levels >= 1)
};
// omega: Matsubara frequencies, or real frequencies with real_axis (z = w + i eta).
void launch_cf(const CFJob* jobs_dev, int njobs, const double* omega, int nw, cudaStream_t s, int real_axis = 0,
               double eta = 0.0);

// ---- arpack.cu: vector kernels of the restarted Lanczos (diag_arpack) ------
#define EDZT_RL_MAXV 8
struct RlVecs { const double* p[EDZT_RL_MAXV]; };
struct RlOut { double* p[EDZT_RL_MAXV]; };
int rl_partials_size();
// out[q] = <V_q, w> for q < nv (device, deterministic); partials: rl_partials_size() doubles.
void launch_rl_mdot(const RlVecs& V, int nv, const double* w, long long n, double* partials, double* out,
                    cudaStream_t s);
// w -= sum_q h[q] V_q (h on the device).
void launch_rl_project_out(double* w, const RlVecs& V, int nv, const double* h, long long n, cudaStream_t s);
// O_i = sum_{j<m} Y[j*k + i] V_j for i < k (Y on the device, m, k <= EDZT_RL_MAXV).
void launch_rl_combine(const RlOut& O, int k, const RlVecs& V, int m, const double* Y, long long n, cudaStream_t s);
void launch_rl_div(double* out, const double* w, double beta, long long n, cudaStream_t s);

// ---- lanczos.cu: persistent fused Lanczos over a batch of jobs ------------
enum LzMode { LZ_COEFF = 0, LZ_EIGVEC = 1 };
enum LzInit { LZ_INIT_HASH = 0, LZ_INIT_APPLYC = 1, LZ_INIT_COPY = 2 };

// The tiles of one job in one phase (0: column phase, 1: row phase): tiles
// [tile0, tile0 + ntiles) of that phase's list; its participants are CTAs
// (tile0 + q) mod G, q < npart, and participant q owns partial-sum slot
// slot0 + q.
struct LzPhase {
    long long tile0;      // first tile in the launch's tile list of the phase
    long long slot0;      // first partial-sum slot
    int ntiles;
    int npart;            // participating CTAs: part0, part0 + 1, ..., one slot each
    int width;            // columns per slab (column phase) or rows per tile (row phase)
    int part0;
};

// Recurrence state of one run between phases (every participating CTA
// derives the same value; the first participant also stores it).
struct LzState {
    int k;                // the step in progress: opened by a column phase, finished by the row phase
    int active;           // 1 while the run is going
    int nstep;            // result: number of valid Lanczos steps
    int opened;           // step k already opened (a_{k-1} derived) by the closing pass of a slice
    double a_prev;        // a_{k-1}
    double b_cur;         // b_k, the normaliser of the step (||v_init|| for k = 1)
    double norm0;         // ||v_init||
    double spare;
};

// The Lanczos vectors of a run live as interleaved pairs (y_k, w_k), one
// 16-byte access each: step k writes YW[k & 1] and reads YW[(k - 1) & 1].
struct LzJob {
    DevSector S;
    double2* YW[2];       // ping-pong pair buffers [dim]; keep: YW[0] holds every step's pair, step k at k * dim
    double* D;            // [lz_d_size] down-hop part of H v_k, column phase -> row phase, slab-major:
                          // the slab of columns [c0, c0 + WC) is the block [ndn][WC] at c0 * ndn
    double* eig;          // EIGVEC: output eigenvector (unnormalised)
    const double* coeff;  // EIGVEC: ground eigenvector of the tridiagonal [nstep]
    double* a;            // [maxnstep] a(1..), written as steps are accepted
    double* b;            // [maxnstep] b(1..)
    int maxnstep;         // COEFF: LanczosSteps; EIGVEC: nstep of the coefficient pass
    int mode;
    int init;
    int keep;             // 1: the pairs of every step are kept ([maxnstep + 1][dim] at YW[0])
    LzPhase ph[2];
    LzState* st;          // [2] the run's state by phase parity (kept across launches of a sliced run)
    uint64_t key;         // LZ_INIT_HASH
    ApplyCArgs ac;        // LZ_INIT_APPLYC
    const double* src;    // LZ_INIT_APPLYC: the ground state; LZ_INIT_COPY: the start vector
};

// The pair buffer step k of a run writes (and step k + 1 reads).
__host__ __device__ inline double2* lz_pairs(const LzJob& J, int k)
{
    return J.keep ? J.YW[0] + (long long)k * J.S.dim : J.YW[k & 1];
}

// Doubles of a job's D buffer (slabs of up to 8 columns).
inline long long lz_d_size(int nup, int ndn) { return (long long)((nup + 7) / 8) * 8 * ndn; }

struct LzBatch {
    int njobs;
    int grid;
    int block;
    int max_phases;               // phase budget of the launch (even for a slice)
    size_t smem;
    long long total[2];           // tiles of the column and the row phase
    unsigned long long wait_ns;   // grid-barrier wait limit (0: the default 5 s)
    int stall_cta;                // fault test: this CTA leaves without arriving (-1: none)
    int slice;                    // 1: a slice of longer runs; at the end of the budget every run
                                  // still going opens its next step, so a later launch resumes it
};

// Largest dynamic shared memory of one persistent CTA.
constexpr size_t kLzSmemMax = 220 * 1024;
// CTAs of block threads that can be resident with smem bytes each.
int lz_grid_size(int device, size_t smem, int block);
// jobs[j].st: the job's state by phase parity; prefix: [2][njobs + 1] tile
// prefix sums of the column and row phases; slots: [slots][2] partial sums
// by step parity.
cudaError_t launch_lanczos_persistent(const LzBatch& B, const LzJob* jobs, const long long* prefix, double* slots,
                                      unsigned* sync_words, int* status, cudaStream_t s);
// Shared memory of a row tile of R rows, of a column slab of WC columns, and
// of the fixed tables.
size_t lz_row_smem(int nup, int R);
size_t lz_col_smem(int ndn, int WC);
size_t lz_fixed_smem();
// Sync-word buffer size (bytes) for a grid of G CTAs.
size_t lz_sync_bytes(int G);
// Tile shapes of the jobs of one launch: every job's rows per tile and
// columns per slab (a nonzero jobs[j].ph[].width on entry is a preset, kept
// when it fits), the launch's block size (prefer_block 512: one CTA of 512
// threads per SM; 256: two of 256 whenever they fit; 0: two of 256 unless a
// job has long lines or needs more shared memory), grid and shared memory;
// the phases' tile lists, participants and slots are filled in.  prefix
// receives, per phase, the jobs' first tiles [njobs + 1], then per phase
// every CTA's first tile [grid + 1] (CTA b takes the contiguous tiles
// [range[b], range[b + 1]), cut by tile cost so the CTAs finish together),
// then the slab of each column-phase tile position [total[0]].
struct LzPlan {
    int block = 256;
    int grid = 0;
    size_t smem = 0;
    long long total[2] = {0, 0};
    long long slots = 0;
};
LzPlan lz_plan(int device, LzJob* jobs, int njobs, std::vector<long long>& prefix, int prefer_block = 0);
// The device-free part of lz_plan: given every job's widths (ph[].width) and
// the grid G, the phases' tile lists, CTA ranges, participants and the column
// phase's slab order (prefix as lz_plan describes it), the tiles per phase
// (total) and the number of partial-sum slots (returned).
long long lz_cut(LzJob* jobs, int njobs, int G, std::vector<long long>& prefix, long long total[2]);

// ---- edzt_host.cu: context accessors (no table building, no allocation) -----
struct edzt_ctx;
int edzt_ctx_device(const edzt_ctx* c);
cudaStream_t edzt_ctx_stream(const edzt_ctx* c);
void edzt_ctx_set_error(edzt_ctx* c, const char* msg);
void edzt_count_launches(edzt_ctx* c, long long n);
// The sector of (nu, nd) when its tables already exist; else an error code
// with the reason in *why.
int edzt_ctx_ready_sector(edzt_ctx* c, int nu, int nd, DevSector* S, const char** why);

#ifdef EDZT_DEVICE_CHECKS
int lz_debug_bad(long long* out4);
int kernels_debug_bad(long long* out4);
int tables_debug_bad(long long* out4);
#endif
