// lanczos.cu — kernel (c): persistent, batched, fused Lanczos.
//
// One cooperative launch runs every step of many independent Lanczos runs
// ("jobs": sectors of the ground-state search, the eigenvector pass of the
// winning sector, c / c^+ excitation runs of the Green's function).  A step of
// every active job is one phase over a global list of tiles (job, block of
// full rows); phases are separated by a grid barrier with a bounded wait.
//
// The recurrence is the reference's (src/lanczos_solver.f90:92-173):
//   w_k = v_k / b_k,  y_k = H w_k - b_k w_{k-1},  a_k = <w_k, y_k>,
//   v_{k+1} = y_k - a_k w_k,  b_{k+1} = ||v_{k+1}||.
// Fusion: phase k stores y_k and w_k; the next phase forms
// w_{k+1}(j) = (y_k(j) - a_k w_k(j)) * (1/b_{k+1}) on the fly wherever it is
// read (staging rows in shared memory, gathering down-spin neighbours), so a
// step is one sweep: gather y_k, w_k; write y_{k+1}, w_{k+1}.  The three sums
// <w,y>, <y,y>, <w,w> are reduced together and
// b_{k+1}^2 = <y,y> - 2a<w,y> + a^2<w,w>.  When that difference cancels
// (b^2 < 1e-5 <y,y>, e.g. an exhausted Krylov space in a tiny sector) the
// step takes one extra phase that sums (y - a w)^2 exactly, as the reference
// does.  Reductions are deterministic: per-CTA partials in fixed slots, summed
// in a fixed order by the last CTA to finish each job.  The first step
// divides v_init by its norm exactly as the reference does (w = v/|v|), so a
// one-dimensional sector breaks down with b(2) = 0 exactly.
#include <cuda_runtime.h>
#include "edzt_internal.h"
#include "hv_row.cuh"

static constexpr int kLzThreads = 256;
static constexpr int kLzTargetElems = 2048;
static constexpr double kExactFrac = 1.0e-5;
static constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000ull * 1000ull * 1000ull;

// sync words
#define SW_COUNT 0
#define SW_GEN 1
#define SW_ACTIVE 2
#define SW_EXACT 3
#define SW_SNAP_ACTIVE 4
#define SW_SNAP_EXACT 5

int lz_rows_per_tile(int nup, int ndn)
{
    int r = kLzTargetElems / (nup > 0 ? nup : 1);
    if (r < 1) r = 1;
    if (r > ndn) r = ndn;
    return r;
}

size_t lz_smem_bytes(int nup, int rows_per_tile)
{
    return (size_t)(96 + (size_t)rows_per_tile * nup) * sizeof(double);
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier with a bounded wait.  The last CTA to arrive snapshots
// the job counters, so every CTA takes the same branch after the barrier.
__device__ bool grid_barrier(unsigned* sw, int* status)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_u32(sw + SW_GEN);
        __threadfence();
        const unsigned prev = atomicAdd(sw + SW_COUNT, 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(sw + SW_COUNT, 0u);
            atomicExch(sw + SW_SNAP_ACTIVE, atomicAdd(sw + SW_ACTIVE, 0u));
            atomicExch(sw + SW_SNAP_EXACT, atomicAdd(sw + SW_EXACT, 0u));
            __threadfence();
            atomicAdd(sw + SW_GEN, 1u);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            unsigned it = 0;
            while (ld_acquire_u32(sw + SW_GEN) == gen) {
                if (ld_acquire_s32(status) != EDZT_DEV_OK) { ok = 0; break; }
                if ((++it & 255u) == 0u && globaltimer_ns() - t0 > kBarrierTimeoutNs) {
                    atomicCAS(status, EDZT_DEV_OK, EDZT_DEV_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
        s_ok = ok && (ld_acquire_s32(status) == EDZT_DEV_OK);
    }
    __syncthreads();
    return s_ok != 0;
}

struct Tile {
    int r0, rows, n;
    long long g0;
};

__device__ __forceinline__ Tile tile_geom(const LzJob& J, long long t)
{
    Tile T;
    const int nup = J.S.up.count, ndn = J.S.dn.count;
    const int R = J.rows_per_tile;
    T.r0 = (int)(t - J.tile0) * R;
    T.rows = min(R, ndn - T.r0);
    T.n = T.rows * nup;
    T.g0 = (long long)T.r0 * nup;
    return T;
}

__device__ __forceinline__ int find_job(const long long* __restrict__ prefix, int njobs, long long t)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// finishers: run by the last participating CTA of a job, thread 0 only
// ---------------------------------------------------------------------------
__device__ void finish_init(const LzJob& J, LzState* st, unsigned* sw, double svv)
{
    const double nrm = sqrt(svv);
    st->norm0 = nrm;
    st->need_exact = 0;
    if (!(nrm > 0.0)) {                     // zero start vector: nothing to do
        st->active = 0;
        st->nstep = 0;
        if (J.mode == LZ_COEFF) atomicSub(sw + SW_ACTIVE, 1u);
        return;
    }
    st->a_prev = 0.0;
    st->b_cur = nrm;
    st->k = 0;
}

__device__ void end_run(const LzJob& J, LzState* st, unsigned* sw, int nstep)
{
    st->active = 0;
    st->nstep = nstep;
    atomicSub(sw + SW_ACTIVE, 1u);
    (void)J;
}

// b_{k+1} known (exact or from the identity): apply the reference's stopping rules.
__device__ void accept_b(const LzJob& J, LzState* st, unsigned* sw, int k, double bnext)
{
    if (bnext < 1.0e-16) {                  // breakdown before dividing (see header)
        J.b[k] = 0.0;
        end_run(J, st, sw, k);
        return;
    }
    J.b[k] = bnext;
    st->b_cur = bnext;
}

__device__ void finish_step(const LzJob& J, LzState* st, unsigned* sw, int k, double swy, double syy,
                            double sww)
{
    const double a = swy;                   // a(k) = <w, y>   (lanczos_solver.f90:134,159)
    J.a[k - 1] = a;
    if (k == 1) J.b[0] = 0.0;               // :135
    st->k = k;
    st->a_prev = a;
    if (k >= J.maxnstep) {                  // :137-141, :161-164
        end_run(J, st, sw, k);
        return;
    }
    const double bb2 = syy - 2.0 * a * swy + a * a * sww;
    if (bb2 > kExactFrac * syy) {
        accept_b(J, st, sw, k, sqrt(bb2));
    } else {                                // cancellation: sum (y - a w)^2 exactly next phase
        st->need_exact = 1;
        atomicAdd(sw + SW_EXACT, 1u);
    }
}

__device__ void finish_exact(const LzJob& J, LzState* st, unsigned* sw, double svv)
{
    st->need_exact = 0;
    atomicSub(sw + SW_EXACT, 1u);
    accept_b(J, st, sw, st->k, sqrt(svv));
}

// ---------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------
enum { PH_INIT = 0, PH_STEP = 1, PH_EXACT = 2 };

__global__ void __launch_bounds__(kLzThreads) k_lanczos(LzBatch B, const LzJob* __restrict__ jobs,
                                                        LzState* __restrict__ state,
                                                        const long long* __restrict__ prefix,
                                                        double* __restrict__ partials,
                                                        unsigned* __restrict__ arrive,
                                                        unsigned* __restrict__ sw, int* __restrict__ status)
{
    extern __shared__ double smem[];
    double* red = smem;          // 96 doubles of reduction scratch
    double* xs = smem + 96;      // staged rows of the current tile
    __shared__ LzJob sJ;
    __shared__ LzState sS;
    __shared__ int s_last, s_run;

    const int G = gridDim.x;

    auto load_job = [&](int j) {
        __syncthreads();
        const int* src = reinterpret_cast<const int*>(jobs + j);
        int* dst = reinterpret_cast<int*>(&sJ);
        for (int i = threadIdx.x; i < (int)(sizeof(LzJob) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
        const int* ss = reinterpret_cast<const int*>(state + j);
        int* sd = reinterpret_cast<int*>(&sS);
        for (int i = threadIdx.x; i < (int)(sizeof(LzState) / sizeof(int)); i += blockDim.x) sd[i] = __ldcg(ss + i);
        __syncthreads();
    };

    // Flush this CTA's partial sums of job j; the last participant reduces them.
    auto flush = [&](int j, int phase, int step, double (&acc)[3]) {
        block_sum<3>(acc, red);
        if (threadIdx.x == 0) {
            const int q = (int)(((long long)blockIdx.x - (sJ.tile0 % G) + G) % G);
            double* slot = partials + (sJ.slot0 + q) * 3;
            slot[0] = acc[0]; slot[1] = acc[1]; slot[2] = acc[2];
            __threadfence();
            const unsigned prev = atomicAdd(arrive + j, 1u);
            s_last = (prev == (unsigned)sJ.npart - 1u);
            if (s_last) {
                atomicExch(arrive + j, 0u);
                __threadfence();
            }
        }
        __syncthreads();
        if (!s_last) return;
        double v[3] = {0.0, 0.0, 0.0};
        for (int i = threadIdx.x; i < sJ.npart; i += blockDim.x) {
            const double* p = partials + (sJ.slot0 + i) * 3;
            v[0] += __ldcg(p); v[1] += __ldcg(p + 1); v[2] += __ldcg(p + 2);
        }
        block_sum<3>(v, red);
        if (threadIdx.x == 0) {
            LzState* st = state + j;
            if (phase == PH_INIT) finish_init(sJ, st, sw, v[1]);
            else if (phase == PH_STEP) finish_step(sJ, st, sw, step, v[0], v[1], v[2]);
            else finish_exact(sJ, st, sw, v[1]);
            __threadfence();
        }
        __syncthreads();
    };

    // One phase over the global tile list.
    auto run_phase = [&](int phase, int step) {
        int cur = -1;
        bool act = false;
        double acc[3] = {0.0, 0.0, 0.0};
        for (long long t = blockIdx.x; t < B.total_tiles; t += G) {
            if (cur < 0 || t >= __ldg(prefix + cur + 1)) {
                if (cur >= 0 && act && (phase != PH_STEP || sJ.mode == LZ_COEFF)) flush(cur, phase, step, acc);
                cur = find_job(prefix, B.njobs, t);
                load_job(cur);
                acc[0] = acc[1] = acc[2] = 0.0;
                if (phase == PH_INIT) act = true;
                else if (phase == PH_EXACT) act = (sJ.mode == LZ_COEFF) && sS.active && sS.need_exact;
                else if (sJ.mode == LZ_COEFF) act = sS.active && !sS.need_exact;
                else act = sS.active && step <= sJ.maxnstep;
            }
            if (!act) continue;
            const Tile T = tile_geom(sJ, t);
            const int nup = sJ.S.up.count;
            if (phase == PH_INIT) {
                double* Y1 = sJ.Y[1];
                for (int e = threadIdx.x; e < T.n; e += blockDim.x) {
                    const long long g = T.g0 + e;
                    double v;
                    if (sJ.init == LZ_INIT_HASH) v = edzt_u01(sJ.key, (uint64_t)g);
                    else if (sJ.init == LZ_INIT_APPLYC) v = apply_c_value(sJ.ac, sJ.ac_src, g);
                    else v = __ldg(sJ.ac_src + g);
                    Y1[g] = v;
                    acc[1] = fma(v, v, acc[1]);
                }
                continue;
            }
            const int p = step & 1;
            if (phase == PH_EXACT) {
                const double* Yn = sJ.Y[p ^ 1];
                const double* Wn = sJ.W[p ^ 1];
                const double am = -sS.a_prev;
                for (int e = threadIdx.x; e < T.n; e += blockDim.x) {
                    const long long g = T.g0 + e;
                    const double v = fma(am, __ldcg(Wn + g), __ldcg(Yn + g));
                    acc[1] = fma(v, v, acc[1]);
                }
                continue;
            }
            // ---- PH_STEP -----------------------------------------------------
            const double* Yp = sJ.Y[p];
            const double* Wp = sJ.W[p];
            double* Yn = sJ.Y[p ^ 1];
            double* Wn = sJ.W[p ^ 1];
            double a_prev, b_cur;
            if (sJ.mode == LZ_COEFF) { a_prev = sS.a_prev; b_cur = sS.b_cur; }
            else {
                a_prev = (step >= 2) ? sJ.a[step - 2] : 0.0;
                b_cur = (step >= 2) ? sJ.b[step - 1] : sS.norm0;
            }
            const double rb = 1.0 / b_cur;
            const double am = -a_prev;
            const bool first = (step == 1);
            for (int e = threadIdx.x; e < T.n; e += blockDim.x) {
                const long long g = T.g0 + e;
                const double yv = __ldcg(Yp + g);
                xs[e] = first ? yv / b_cur : fma(am, __ldcg(Wp + g), yv) * rb;
            }
            __syncthreads();
            auto gather = [&](long long idx) -> double {
                const double yv = __ldcg(Yp + idx);
                return first ? yv / b_cur : fma(am, __ldcg(Wp + idx), yv) * rb;
            };
            const double ck = (sJ.mode == LZ_EIGVEC) ? sJ.coeff[step - 1] : 0.0;
            int r = threadIdx.x / nup, iu = threadIdx.x - r * nup;
            for (int e = threadIdx.x; e < T.n; e += blockDim.x) {
                const long long g = T.g0 + e;
                const int id = T.r0 + r;
                const double xe = xs[e];
                const double hv = hv_row_element(sJ.S, iu, id, xs + r * nup, xe, gather);
                const double y = first ? hv : fma(-b_cur, __ldcg(Wp + g), hv);
                __stcg(Yn + g, y);
                __stcg(Wn + g, xe);
                if (sJ.mode == LZ_COEFF) {
                    acc[0] = fma(xe, y, acc[0]);
                    acc[1] = fma(y, y, acc[1]);
                    acc[2] = fma(xe, xe, acc[2]);
                } else {
                    double* eg = sJ.eig + g;
                    *eg = first ? ck * xe : fma(ck, xe, *eg);
                }
                iu += blockDim.x;
                while (iu >= nup) { iu -= nup; ++r; }
            }
            __syncthreads();
        }
        if (cur >= 0 && act && (phase != PH_STEP || sJ.mode == LZ_COEFF)) flush(cur, phase, step, acc);
    };

    // init: materialise each start vector and its norm
    run_phase(PH_INIT, 0);
    if (!grid_barrier(sw, status)) return;
    for (int step = 1; step <= B.max_steps; step++) {
        if (threadIdx.x == 0)
            s_run = (ld_acquire_u32(sw + SW_SNAP_ACTIVE) > 0u) || (step <= B.max_eig_steps);
        __syncthreads();
        if (!s_run) break;
        run_phase(PH_STEP, step);
        if (!grid_barrier(sw, status)) return;
        if (threadIdx.x == 0) s_run = ld_acquire_u32(sw + SW_SNAP_EXACT) > 0u;
        __syncthreads();
        if (s_run) {
            run_phase(PH_EXACT, step);
            if (!grid_barrier(sw, status)) return;
        }
    }
}

int lz_grid_size(int device, size_t smem, int* block_out)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_lanczos, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr = true;
    }
    int per_sm = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos, kLzThreads, smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (block_out) *block_out = kLzThreads;
    return per_sm * nsm;
}

cudaError_t launch_lanczos_persistent(const LzBatch& B, const LzJob* jobs, LzState* state,
                                      const long long* tile_prefix, double* partials, unsigned* arrive,
                                      unsigned* sync_words, int* status, cudaStream_t s)
{
    LzBatch b = B;
    void* args[] = {(void*)&b, (void*)&jobs, (void*)&state, (void*)&tile_prefix, (void*)&partials,
                    (void*)&arrive, (void*)&sync_words, (void*)&status};
    return cudaLaunchCooperativeKernel((const void*)k_lanczos, dim3(B.grid), dim3(B.block), args, B.smem, s);
}
