// lanczos.cu — kernel (c): persistent, batched, fused Lanczos.
//
// One cooperative launch runs every step of many independent Lanczos runs
// ("jobs": sectors of the ground-state search, the eigenvector pass of the
// winning sector, c / c^+ excitation runs of the Green's function).  The
// jobs' elements are concatenated and CTA b owns the contiguous range
// [b*E/G, (b+1)*E/G) in every phase, so the work is balanced to one element.
// Phases are separated by a grid barrier with a bounded wait.
//
// The recurrence is the reference's (src/lanczos_solver.f90:92-173):
//   w_k = v_k / b_k,  y_k = H w_k - b_k w_{k-1},  a_k = <w_k, y_k>,
//   v_{k+1} = y_k - a_k w_k,  b_{k+1} = ||v_{k+1}||.
// Fusion: phase k stores the pair (y_k, w_k); the next phase forms
// w_{k+1}(j) = (y_k(j) - a_k w_k(j)) * (1/b_{k+1}) wherever it reads it
// (rows staged in shared memory for the up-spin hops, down-spin neighbours
// gathered as one 16-byte pair per hop), so a step is one sweep.  The norm
// needs a_k before it can be summed, so the pass sums around a predicted
// shift instead: with t = y - a_{k-1} w it reduces <w,t>, <t,t>, <w,w>
// together, then a_k = a_{k-1}<w,w> + <w,t> and, with d = a_k - a_{k-1},
// b_{k+1}^2 = <t,t> - 2d<w,t> + d^2<w,w>.  The cancellation in that
// difference scales with d^2/b^2 (consecutive a differ by O(b)) rather than
// a^2/b^2.  When it is still too large (b^2 < 1e-2 <t,t>, e.g. an exhausted
// Krylov space in a tiny sector) the step takes one extra phase that sums
// (y - a w)^2 exactly, as the reference does.  The first step divides v_init by its norm exactly as the reference
// does (w = v/|v|), so a one-dimensional sector breaks down with b(2) = 0.
// Reductions are deterministic: per-CTA partials in fixed slots, summed in a
// fixed order by the last CTA to finish each job.
#include <cuda_runtime.h>
#include "edzt_internal.h"
#include "hv_row.cuh"

static constexpr int kLzThreads = 256;
static constexpr size_t kLzSmemTarget = 24 * 1024;
static constexpr double kExactFrac = 1.0e-2;
static constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000ull * 1000ull * 1000ull;
static constexpr int kFixedDoubles = 96 + 2 * EDZT_MAX_COEF;   // reduction scratch + amplitude tables

// sync words
#define SW_COUNT 0
#define SW_GEN 1
#define SW_ACTIVE 2
#define SW_EXACT 3
#define SW_SNAP_ACTIVE 4
#define SW_SNAP_EXACT 5

size_t lz_smem_budget(int max_nup, int max_hw_dn)
{
    const size_t one = staged_row_bytes(max_nup, max_hw_dn);
    return one > kLzSmemTarget ? one : kLzSmemTarget;
}

int lz_rows_per_chunk(int nup, int ndn, int hw_dn, size_t budget)
{
    int r = (int)(budget / staged_row_bytes(nup, hw_dn));
    if (r < 1) r = 1;
    if (r > ndn) r = ndn;
    return r;
}

size_t lz_smem_bytes(int nup, int hw_dn, int rmax)
{
    return kFixedDoubles * sizeof(double) + (size_t)rmax * staged_row_bytes(nup, hw_dn) + 16;
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
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok && (ld_acquire_s32(status) == EDZT_DEV_OK);
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ int find_job(const long long* __restrict__ prefix, int njobs, long long e)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= e) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ long long cta_lo(long long E, int G, int b)
{
    // floor(E * b / G) without 128-bit arithmetic on the device
    const long long q = E / G, r = E % G;
    return q * b + (r * b) / G;
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

__device__ void end_run(LzState* st, unsigned* sw, int nstep)
{
    st->active = 0;
    st->nstep = nstep;
    atomicSub(sw + SW_ACTIVE, 1u);
}

// b_{k+1} known: apply the reference's stopping rule (breakdown tested before
// the next division, see the file header).
__device__ void accept_b(const LzJob& J, LzState* st, unsigned* sw, int k, double bnext)
{
    if (bnext < 1.0e-16) {
        J.b[k] = 0.0;
        end_run(st, sw, k);
        return;
    }
    J.b[k] = bnext;
    st->b_cur = bnext;
}

// ah: the shift the pass used (a_{k-1}, 0 at k = 1); swt = <w,t>, stt = <t,t>.
__device__ void finish_step(const LzJob& J, LzState* st, unsigned* sw, int k, double ah, double swt, double stt,
                            double sww)
{
    const double a = fma(ah, sww, swt);     // a(k) = <w, y>   (lanczos_solver.f90:134,159)
    J.a[k - 1] = a;
    if (k == 1) J.b[0] = 0.0;               // :135
    st->k = k;
    st->a_prev = a;
    if (k >= J.maxnstep) {                  // :137-141, :161-164
        end_run(st, sw, k);
        return;
    }
    const double d = a - ah;
    const double bb2 = stt - 2.0 * d * swt + d * d * sww;
    if (bb2 > kExactFrac * stt) {
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

__global__ void __launch_bounds__(kLzThreads, 4) k_lanczos(LzBatch B, const LzJob* __restrict__ jobs,
                                                           LzState* __restrict__ state,
                                                           const long long* __restrict__ prefix,
                                                           double* __restrict__ partials,
                                                           unsigned* __restrict__ arrive,
                                                           unsigned* __restrict__ sw, int* __restrict__ status)
{
    extern __shared__ double smem[];
    double* red = smem;                                  // 96 doubles of reduction scratch
    double* cu = smem + 96;                              // up-spin hop amplitudes
    double* cd = cu + EDZT_MAX_COEF;                     // down-spin hop amplitudes
    double* xs = smem + kFixedDoubles;                   // staged rows of w
    __shared__ LzJob sJ;
    __shared__ LzState sS;
    __shared__ int s_last, s_run;

    const int G = gridDim.x;
    const long long E = B.total_elems;
    const long long my_lo = cta_lo(E, G, blockIdx.x), my_hi = cta_lo(E, G, blockIdx.x + 1);

    auto load_job = [&](int j, bool coefs) {
        __syncthreads();
        const int* src = reinterpret_cast<const int*>(jobs + j);
        int* dst = reinterpret_cast<int*>(&sJ);
        for (int i = threadIdx.x; i < (int)(sizeof(LzJob) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
        const int* ss = reinterpret_cast<const int*>(state + j);
        int* sd = reinterpret_cast<int*>(&sS);
        for (int i = threadIdx.x; i < (int)(sizeof(LzState) / sizeof(int)); i += blockDim.x) sd[i] = __ldcg(ss + i);
        __syncthreads();
        if (coefs) stage_coefs(sJ.S, cu, cd);
    };

    // Flush this CTA's partial sums of job j; the last participant reduces them.
    auto flush = [&](int j, int phase, int step, double (&acc)[3]) {
        block_sum<3>(acc, red);
        if (threadIdx.x == 0) {
            const int q = (int)blockIdx.x - sJ.first_cta;
            EDZT_OK_OR(q >= 0 && q < sJ.nspan, 24, blockIdx.x, sJ.first_cta, sJ.nspan, return)
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
        // sum the slots of the CTAs of the span that own elements, in CTA order
        double v[3] = {0.0, 0.0, 0.0};
        for (int i = threadIdx.x; i < sJ.nspan; i += blockDim.x) {
            const int b = sJ.first_cta + i;
            if (cta_lo(E, G, b) >= cta_lo(E, G, b + 1)) continue;
            const double* p = partials + (sJ.slot0 + i) * 3;
            v[0] += __ldcg(p); v[1] += __ldcg(p + 1); v[2] += __ldcg(p + 2);
        }
        block_sum<3>(v, red);
        if (threadIdx.x == 0) {
            LzState* st = state + j;
            if (phase == PH_INIT) finish_init(sJ, st, sw, v[1]);
            else if (phase == PH_STEP) finish_step(sJ, st, sw, step, step == 1 ? 0.0 : sS.a_prev, v[0], v[1], v[2]);
            else finish_exact(sJ, st, sw, v[1]);
            __threadfence();
        }
        __syncthreads();
    };

    // One Lanczos step of the current job over its local elements [lo, hi).
    auto step_range = [&](long long lo, long long hi, int step, double (&acc)[3]) {
        const int nup = sJ.S.up.count, hwd = sJ.S.dn.hw;
        const int p = step & 1;
        const double2* YWp = sJ.YW[p];
        double2* YWn = sJ.YW[p ^ 1];
        double a_prev, b_cur;
        if (sJ.mode == LZ_COEFF) { a_prev = sS.a_prev; b_cur = sS.b_cur; }
        else {
            a_prev = (step >= 2) ? sJ.a[step - 2] : 0.0;
            b_cur = (step >= 2) ? sJ.b[step - 1] : sS.norm0;
        }
        const double rb = 1.0 / b_cur, am = -a_prev, mb = -b_cur;
        const bool first = (step == 1);
        const double ah = first ? 0.0 : am;                 // minus the predicted shift
        const double ck = (sJ.mode == LZ_EIGVEC) ? sJ.coeff[step - 1] : 0.0;
        auto wval = [&](double2 pr) { return first ? pr.x / b_cur : fma(am, pr.y, pr.x) * rb; };
        auto fetch = [&](long long idx) {
            EDZT_OK_OR(idx >= 0 && idx < sJ.S.dim, 21, idx, sJ.S.dim, step, return 0.0)
            return wval(__ldcg(YWp + idx));
        };
        const int rmax = sJ.rmax;
        uint32_t* dw = reinterpret_cast<uint32_t*>(xs + (size_t)rmax * nup);
        int* dc = reinterpret_cast<int*>(dw + (size_t)rmax * hwd);
        const int ra = (int)(lo / nup), rend = (int)((hi - 1) / nup) + 1;
        for (int r0 = ra; r0 < rend; r0 += rmax) {
            const int r1 = min(r0 + rmax, rend);
            const long long g0 = (long long)r0 * nup;
            const int nst = (r1 - r0) * nup;
            EDZT_OK_OR(r1 - r0 <= rmax && r1 <= sJ.S.dn.count && g0 + nst <= sJ.S.dim, 22, r0, r1, rmax, break)
            for (int e = threadIdx.x; e < nst; e += blockDim.x) xs[e] = wval(__ldcg(YWp + g0 + e));
            stage_down_hops(sJ.S.dn, r0, r1 - r0, dw, dc);
            __syncthreads();
            const int c0 = (int)(max(lo, g0) - g0), c1 = (int)(min(hi, (long long)r1 * nup) - g0);
            int el = c0 + threadIdx.x;
            int r = el / nup, iu = el - r * nup;
            for (; el < c1; el += blockDim.x) {
                const long long g = g0 + el;
                EDZT_OK_OR(r >= 0 && r < r1 - r0 && iu >= 0 && iu < nup && g < sJ.S.dim, 23, g, r, iu, break)
                const double xe = xs[el];
                const double hv = hv_element(sJ.S, iu, r0 + r, xs + (size_t)r * nup, xe, dw + (size_t)r * hwd,
                                             dc[r], cu, cd, fetch);
                const double y = first ? hv : fma(mb, __ldcg(YWp + g).y, hv);
                __stcg(YWn + g, make_double2(y, xe));
                if (sJ.mode == LZ_COEFF) {
                    const double t = fma(ah, xe, y);         // y - a_{k-1} w
                    acc[0] = fma(xe, t, acc[0]);
                    acc[1] = fma(t, t, acc[1]);
                    acc[2] = fma(xe, xe, acc[2]);
                } else {
                    double* eg = sJ.eig + g;
                    __stcg(eg, first ? ck * xe : fma(ck, xe, __ldcg(eg)));
                }
                iu += blockDim.x;
                while (iu >= nup) { iu -= nup; ++r; }
            }
            __syncthreads();
        }
    };

    // One phase over this CTA's element range.
    auto run_phase = [&](int phase, int step) {
        if (my_lo >= my_hi) return;
        int j = find_job(prefix, B.njobs, my_lo);
        for (; j < B.njobs; j++) {
            const long long pj = __ldg(prefix + j), pj1 = __ldg(prefix + j + 1);
            if (pj >= my_hi) break;
            load_job(j, phase == PH_STEP);
            bool act, red_needed;
            if (phase == PH_INIT) { act = true; red_needed = true; }
            else if (phase == PH_EXACT) {
                act = (sJ.mode == LZ_COEFF) && sS.active && sS.need_exact;
                red_needed = true;
            } else if (sJ.mode == LZ_COEFF) {
                act = sS.active && !sS.need_exact;
                red_needed = true;
            } else {
                act = sS.active && step <= sJ.maxnstep;
                red_needed = false;
            }
            if (!act) continue;
            const long long lo = max(my_lo, pj) - pj, hi = min(my_hi, pj1) - pj;
            double acc[3] = {0.0, 0.0, 0.0};
            if (phase == PH_INIT) {
                double2* Y1 = sJ.YW[1];
                for (long long g = lo + threadIdx.x; g < hi; g += blockDim.x) {
                    EDZT_OK_OR(g < sJ.S.dim, 25, g, sJ.S.dim, j, break)
                    double v;
                    if (sJ.init == LZ_INIT_HASH) v = edzt_u01(sJ.key, (uint64_t)g);
                    else if (sJ.init == LZ_INIT_APPLYC) v = apply_c_value(sJ.ac, sJ.src, g);
                    else v = __ldg(sJ.src + g);
                    __stcg(Y1 + g, make_double2(v, 0.0));
                    acc[1] = fma(v, v, acc[1]);
                }
            } else if (phase == PH_EXACT) {
                const double2* YWn = sJ.YW[(step & 1) ^ 1];
                const double am = -sS.a_prev;
                for (long long g = lo + threadIdx.x; g < hi; g += blockDim.x) {
                    const double2 pr = __ldcg(YWn + g);
                    const double v = fma(am, pr.y, pr.x);
                    acc[1] = fma(v, v, acc[1]);
                }
            } else {
                step_range(lo, hi, step, acc);
            }
            if (red_needed) flush(j, phase, step, acc);
        }
    };

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

#ifdef EDZT_DEVICE_CHECKS
int lz_debug_bad(long long* out4)
{
    return cudaMemcpyFromSymbol(out4, g_edzt_bad, 4 * sizeof(long long)) == cudaSuccess ? 0 : 2;
}
#endif

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
                                      const long long* elem_prefix, double* partials, unsigned* arrive,
                                      unsigned* sync_words, int* status, cudaStream_t s)
{
    LzBatch b = B;
    void* args[] = {(void*)&b, (void*)&jobs, (void*)&state, (void*)&elem_prefix, (void*)&partials,
                    (void*)&arrive, (void*)&sync_words, (void*)&status};
    return cudaLaunchCooperativeKernel((const void*)k_lanczos, dim3(B.grid), dim3(B.block), args, B.smem, s);
}
