// lanczos.cu — kernel (c): persistent, batched, fused Lanczos.
//
// One cooperative launch runs every step of many independent Lanczos runs
// ("jobs": sectors of the ground-state search, the eigenvector pass of the
// winning sector, c / c^+ excitation runs of the Green's function).
//
// The recurrence is the reference's (src/lanczos_solver.f90:92-173):
//   v_1 = v_init,  v_k = y_{k-1} - a_{k-1} w_{k-1}  (k >= 2),
//   b_k = ||v_k||,  w_k = v_k / b_k,
//   y_k = H w_k - b_k w_{k-1},  a_k = <w_k, y_k>,
// with a(1..), b(1) = 0, b(k) = ||v_k|| (k >= 2) stored as they are accepted.
//
// A step is two phases of the whole grid, separated by grid barriers; H.v
// is split as in hv_phase.cuh:
//   column phase  each CTA stages slabs of whole columns of v_k (formed from
//                 the stored pair (y_{k-1}, w_{k-1}) element by element),
//                 sums ||v_k||^2 exactly and writes D = the down-hop part of
//                 H v_k (not yet normalised);
//   row phase     with b_k known from those sums, each CTA stages tiles of
//                 whole rows of w_k = v_k / b_k, adds the diagonal, up-hop and
//                 exchange parts to D / b_k, subtracts b_k w_{k-1}, stores the
//                 pair (y_k, w_k) and sums <w_k, y_k> exactly.
// Every neighbour value comes from shared memory, every global access is a
// coalesced stream (pair buffers, D, the eigenvector), and both reductions
// are exact sums, as in the reference.  The tiles of all jobs of a phase
// form one list, cut into one contiguous range per CTA at equal modelled
// cost (lz_plan); within a job the column slabs are numbered by round, so
// the CTAs stage neighbouring slabs at the same time.  A job's participants
// in a phase (the CTAs whose range meets its tiles) write one partial sum
// each into their slot (double-buffered by step parity).  Every
// participating CTA re-derives a job's scalars from the slots in a fixed
// order, so all of them get the same bits; the first participant also
// stores them.
//
// The pairs of a run are ping-pong buffers, or (LzJob::keep) one slot per
// step, so that the eigenvector can be summed from them afterwards.  The
// eigenvector pass (LZ_EIGVEC) instead reruns the recurrence with the stored
// a, b (src/lanczos_solver.f90:213-300) and accumulates sum_k coeff_k w_k.
//
// A launch may be a slice of longer runs (LzBatch::slice): when its phase
// budget runs out, a closing pass opens every unfinished run's next step
// (derives a(k-1) and the finish test) and stores the state marked opened,
// so a later launch, with any mix of other runs, resumes it.
#include <algorithm>
#include <type_traits>
#include <cuda_runtime.h>
#include "edzt_internal.h"
#include "hv_phase.cuh"

static constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000ull * 1000ull * 1000ull;
static constexpr int kRedDoubles = 64;
static constexpr int kWintDoubles = EDZT_MAX_P * EDZT_MAX_P;
static constexpr int kFixedDoubles = kRedDoubles + kWintDoubles + 2 * EDZT_MAX_AMP;
static constexpr int kBarGroup = 16;                    // CTAs per barrier group
static constexpr int kStageDepth = 16;                  // pair loads a thread keeps in flight when staging

// sync words (unsigned), each counter on its own 128-byte line; SW_GEN is a
// 64-bit word (barrier count << 32 | runs still going)
#define SW_GEN 0
#define SW_TOP 32
#define SW_ACTIVE 64
#define SW_GROUP(g) (128 + 32 * (g))

size_t lz_sync_bytes(int G) { return sizeof(unsigned) * (128 + 32 * (size_t)((G + kBarGroup - 1) / kBarGroup)); }

size_t lz_row_smem(int nup, int R) { return (size_t)nup * phase_stride(R) * sizeof(double); }
size_t lz_col_smem(int ndn, int WC) { return (size_t)ndn * phase_stride(WC) * sizeof(double); }
size_t lz_fixed_smem() { return kFixedDoubles * sizeof(double); }

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Hierarchical grid barrier with a bounded wait.  Counters only grow: the
// k-th barrier of a launch is complete on a group counter at k * (group
// size) arrivals and on the top counter at k * (number of groups), so no
// counter is read before arriving or reset after.  CTAs arrive on the counter
// of their group of 16, the last of each group on the top counter, and the
// last of all publishes (k << 32 | runs still going) in the 64-bit
// generation word, which the others wait for.  Returns false (and the kernel
// stops) when the wait ran out or another CTA reported an error; snap
// receives the number of runs still going.
__device__ bool grid_barrier(unsigned* sw, int* status, unsigned& nbar, unsigned& snap, const LzBatch& B)
{
    if ((int)blockIdx.x == B.stall_cta) return false;   // fault test: leave without arriving
    const unsigned long long limit = B.wait_ns ? B.wait_ns : kBarrierTimeoutNs;
    __shared__ int s_ok;
    __shared__ unsigned s_snap;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned k1 = nbar + 1u;
        const int G = gridDim.x;
        const int g = blockIdx.x / kBarGroup;
        const unsigned ngroups = (unsigned)((G + kBarGroup - 1) / kBarGroup);
        const unsigned gsize = (unsigned)min(kBarGroup, G - g * kBarGroup);
        unsigned long long* genw = reinterpret_cast<unsigned long long*>(sw + SW_GEN);
        __threadfence();                                  // this CTA's sums and states before its arrival
        bool last = false;
        if (atomicAdd(sw + SW_GROUP(g), 1u) == k1 * gsize - 1u)
            last = atomicAdd(sw + SW_TOP, 1u) == k1 * ngroups - 1u;
        unsigned long long w;
        if (last) {
            const unsigned act = atomicAdd(sw + SW_ACTIVE, 0u);   // every arrival's decrements are in
            w = ((unsigned long long)k1 << 32) | act;
            st_release_u64(genw, w);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            unsigned it = 0;
            while ((unsigned)((w = ld_acquire_u64(genw)) >> 32) < k1) {
                if (ld_acquire_s32(status) != EDZT_DEV_OK) { ok = 0; break; }
                if ((++it & 255u) == 0u && globaltimer_ns() - t0 > limit) {
                    atomicCAS(status, EDZT_DEV_OK, EDZT_DEV_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        s_snap = (unsigned)w;
        s_ok = ok && (ld_acquire_s32(status) == EDZT_DEV_OK);
    }
    __syncthreads();
    nbar++;
    snap = s_snap;
    return s_ok != 0;
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

// Element e of the start vector of a job.
__device__ __forceinline__ double init_value(const LzJob& J, long long e)
{
    if (J.init == LZ_INIT_HASH) return edzt_u01(J.key, (uint64_t)e);
    if (J.init == LZ_INIT_APPLYC) return apply_c_value(J.ac, J.src, e);
    return __ldg(J.src + e);
}

// v_k at element e: the start vector for k = 1, else y_{k-1} - a_{k-1} w_{k-1}
// from the stored pair.  Every phase and every CTA forms it with this one
// expression, so all get the same bits.
__device__ __forceinline__ double form_v(const LzJob& J, int k, const double2* __restrict__ pin, double am,
                                         long long e)
{
    if (k == 1) return init_value(J, e);
    const double2 pr = __ldcg(pin + e);
    return fma(am, pr.y, pr.x);
}

// ---------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_lanczos(LzBatch B, const LzJob* __restrict__ jobs,
                                                 const long long* __restrict__ prefix, double* __restrict__ slots,
                                                 unsigned* __restrict__ sw, int* __restrict__ status)
{
    extern __shared__ __align__(16) double smem[];
    double* red = smem;                                  // reduction scratch
    double* wint = red + kRedDoubles;                    // interaction energies by impurity patterns
    double* amp_up = wint + kWintDoubles;                // up-spin hop amplitudes by slot
    double* amp_dn = amp_up + EDZT_MAX_AMP;              // down-spin hop amplitudes by slot
    double* chunk = smem + kFixedDoubles;                // the staged row tile or column slab
    __shared__ LzJob sJ;
    __shared__ LzState sS;
    __shared__ int s_job;
    __shared__ int s_resumed;

    const int G = gridDim.x;
    const int T = blockDim.x;
    unsigned nbar = 0u;                                  // grid barriers this CTA has passed
    if (threadIdx.x == 0) s_job = -1;
    __syncthreads();

    // participant index of this CTA in phase ph of the current job
    auto my_q = [&](int ph) { return (int)blockIdx.x - sJ.ph[ph].part0; };
    // this CTA's tiles of phase ph: [range[0], range[1])
    auto my_range = [&](int ph) { return prefix + 2 * (size_t)(B.njobs + 1) + (size_t)ph * (G + 1) + blockIdx.x; };
    // the slab that column-phase tile position t stages
    const long long* __restrict__ slab_of = prefix + 2 * (size_t)(B.njobs + 1) + 2 * (size_t)(G + 1);


    // Enter job j in phase p: load it if needed and derive its state.  The
    // closing pass of a slice (closing) opens the next step only: it derives
    // a(k-1) and the finish test of a column phase and stores the state,
    // marked opened, under both parities for the launch that resumes it.
    auto begin_job = [&](int j, int p, bool closing) {
        __syncthreads();
        if (j != s_job) {
            const int* src = reinterpret_cast<const int*>(jobs + j);
            int* dst = reinterpret_cast<int*>(&sJ);
            for (int i = threadIdx.x; i < (int)(sizeof(LzJob) / sizeof(int)); i += T) dst[i] = __ldg(src + i);
            __syncthreads();
            stage_table(sJ.S.wint, sJ.S.P * sJ.S.P, wint);
            stage_table(sJ.S.up.amp, sJ.S.up.namp, amp_up);
            stage_table(sJ.S.dn.amp, sJ.S.dn.namp, amp_dn);
            if (threadIdx.x == 0) s_job = j;
        }
        const int ph = p & 1;
        // The sums of the other phase's partial-sum slots, both parities, in
        // participant order (every thread gets them), loaded while thread 0
        // loads the run's state: which parity applies depends on the step.
        double ps2[2] = {0.0, 0.0};
        {
            const LzPhase& O = sJ.ph[ph ^ 1];
            const double2* sl = reinterpret_cast<const double2*>(slots) + O.slot0;
            for (int i = threadIdx.x; i < O.npart; i += T) {
                const double2 q = __ldcg(sl + i);
                ps2[0] += q.x;
                ps2[1] += q.y;
            }
        }
        if (threadIdx.x == 0) {
            const int* ss = reinterpret_cast<const int*>(sJ.st + ((p + 1) & 1));
            int* sd = reinterpret_cast<int*>(&sS);
            for (int i = 0; i < (int)(sizeof(LzState) / sizeof(int)); i++) sd[i] = __ldcg(ss + i);
            s_resumed = (ph == 0 && sS.opened);          // step already opened by a closing pass
            if (ph == 0 && !sS.opened) sS.k += 1;        // the column phase opens the next step
            sS.opened = 0;
        }
        block_sum<2>(ps2, red);                          // ends with a CTA barrier: sS is visible
        if (s_resumed) {
            if (threadIdx.x == 0 && my_q(0) == 0) sJ.st[p & 1] = sS;
            __syncthreads();
            return;
        }
        const int k = sS.k;
        const bool coeff = (sJ.mode == LZ_COEFF);
        // sums needed: a(k-1) before a column phase, ||v_k||^2 before a row
        // phase (the eigenvector pass takes a and b from the coefficient pass
        // but sums ||v_init|| itself)
        double sum = 0.0;
        if (sS.active && ((ph == 0 && k >= 2 && coeff) || (ph == 1 && (coeff || k == 1))))
            sum = (ph == 0) ? ps2[(k - 1) & 1] : ps2[k & 1];
        if (threadIdx.x == 0) {
            const bool out = (my_q(ph) == 0);
            LzState n = sS;
            auto finish = [&](int nstep) {
                n.active = 0;
                n.nstep = nstep;
                if (out) atomicSub(sw + SW_ACTIVE, 1u);
            };
            if (n.active) {
                if (ph == 0) {
                    if (k >= 2) {                        // a(k-1) = <w, y> of the last row phase (:134,159)
                        const double a = coeff ? sum : sJ.a[k - 2];
                        if (out && coeff) sJ.a[k - 2] = a;
                        n.a_prev = a;
                        if (k - 1 >= sJ.maxnstep) finish(k - 1);          // :137-141, :161-164
                    } else {
                        n.a_prev = 0.0;
                    }
                } else if (k == 1) {                     // ||v_init|| (:128-130); b(1) = 0 (:135)
                    const double nrm = sqrt(sum);
                    n.norm0 = nrm;
                    n.b_cur = nrm;
                    if (out && coeff) sJ.b[0] = 0.0;
                    if (!(nrm > 0.0)) finish(0);         // zero start vector
                } else {                                 // b(k) = ||v_k|| (:144,167), breakdown (:161)
                    const double bk = coeff ? sqrt(sum) : sJ.b[k - 1];
                    if (coeff && bk < 1.0e-16) {
                        if (out) sJ.b[k - 1] = 0.0;
                        finish(k - 1);
                    } else {
                        if (out && coeff) sJ.b[k - 1] = bk;
                        n.b_cur = bk;
                    }
                }
            }
            if (closing && n.active) n.opened = 1;
            if (out) {                                   // published by the barrier's fence (or the launch's end)
                sJ.st[p & 1] = n;
                if (closing) sJ.st[(p + 1) & 1] = n;
            }
            sS = n;
        }
        __syncthreads();
    };

    auto flush = [&](int ph, double acc) {
        double v[1] = {acc};
        block_sum<1>(v, red);
        if (threadIdx.x == 0) {
            EDZT_OK_OR(my_q(ph) < sJ.ph[ph].npart, 24, blockIdx.x, sJ.ph[ph].tile0, sJ.ph[ph].npart, return)
            slots[(sJ.ph[ph].slot0 + my_q(ph)) * 2 + (sS.k & 1)] = v[0];
        }
    };

    // Column phase of step k on slab tl: stage v_k on columns [c0, c0 + WC)
    // of every row, sum v^2, write the down-hop part of H v_k into D.
    auto col_tile = [&](auto wc_tag, int tl, double& acc) {
        constexpr int WC = decltype(wc_tag)::value;
        constexpr int WS = phase_stride(WC);
        const int nup = sJ.S.up.count, ndn = sJ.S.dn.count, k = sS.k;
        const double2* __restrict__ pin = lz_pairs(sJ, k - 1);
        const double am = -sS.a_prev;
        const int c0 = tl * WC;
        double* ws = chunk;
        const int n = ndn * WC;
        if (k == 1) {
            for (int i = threadIdx.x; i < n; i += T) {
                const int id = i / WC, c = i - id * WC;
                const double v = (c0 + c < nup) ? init_value(sJ, (long long)id * nup + c0 + c) : 0.0;
                ws[id * WS + c] = v;
                acc = fma(v, v, acc);
            }
        } else {
            // kStageDepth pair loads in flight per thread before the first is used
            for (int i0 = threadIdx.x; i0 < n; i0 += kStageDepth * T) {
                double2 pr[kStageDepth];
#pragma unroll
                for (int q = 0; q < kStageDepth; q++) {
                    const int i = i0 + q * T;
                    const int id = i / WC, c = i - id * WC;
                    pr[q] = (i < n && c0 + c < nup) ? __ldcg(pin + (long long)id * nup + c0 + c) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int q = 0; q < kStageDepth; q++) {
                    const int i = i0 + q * T;
                    const int id = i / WC, c = i - id * WC;
                    if (i < n) {
                        const double v = fma(am, pr[q].y, pr[q].x);   // form_v of the stored pair
                        ws[id * WS + c] = v;
                        acc = fma(v, v, acc);
                    }
                }
            }
        }
        __syncthreads();
        HopList nxt{};
        if ((int)threadIdx.x < ndn) nxt = hop_list(sJ.S.dn, threadIdx.x);
        for (int id = threadIdx.x; id < ndn; id += T) {
            const HopList cur = nxt;                     // this row's hop list; the next one's in flight
            if (id + T < ndn) nxt = hop_list(sJ.S.dn, id + T);
            double d[WC];
            col_part<WC, WS>(sJ.S, ws, amp_dn, id, cur, d);
            store_slab_row<WC>(sJ.D, c0, ndn, id, d);   // columns past nup hold 0 (staged as 0)
        }
        __syncthreads();
    };

    // Row phase of step k on tile tl: stage w_k = v_k / b_k (and w_{k-1}) on
    // rows [r0, r0 + R), finish y_k = H w_k - b_k w_{k-1}, store (y_k, w_k),
    // sum <w_k, y_k> (or accumulate the eigenvector).
    auto row_tile = [&](auto r_tag, int tl, double& acc) {
        constexpr int R = decltype(r_tag)::value;
        constexpr int RS = phase_stride(R);
        const int nup = sJ.S.up.count, ndn = sJ.S.dn.count, k = sS.k;
        const double2* __restrict__ pin = lz_pairs(sJ, k - 1);
        double2* __restrict__ pout = lz_pairs(sJ, k);
        const double am = -sS.a_prev, bk = sS.b_cur, rb = 1.0 / bk, n0 = sS.norm0;
        const bool first = (k == 1);
        const bool coeff = (sJ.mode == LZ_COEFF);
        const double ck = coeff ? 0.0 : sJ.coeff[k - 1];
        const int r0 = tl * R, nr = min(R, ndn - r0);
        const int wsh = __ffs(sJ.ph[0].width) - 1;       // D's slab width, log2
        double* xs = chunk;                              // [nup][RS] w_k
        const double2* prev = first ? nullptr : pin;     // w_{k-1}: read with each column's data
        // w at a global index, as its owner forms it (exchange terms)
        auto fetch_w = [&](long long idx) {
            EDZT_OK_OR(idx >= 0 && idx < sJ.S.dim, 21, idx, sJ.S.dim, k, return 0.0)
            const double v = form_v(sJ, k, pin, am, idx);
            return first ? v / n0 : v * rb;
        };
        if (first) {
            for (int iu = threadIdx.x; iu < nup; iu += T) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const long long e = (long long)(r0 + r) * nup + iu;
                    xs[iu * RS + r] = (r < nr) ? init_value(sJ, e) / n0 : 0.0;   // the reference divides (:130)
                }
            }
        } else {
            // U columns of R rows per thread: U * R pair loads in flight before the first is used
            constexpr int U = (kStageDepth / R) > 0 ? kStageDepth / R : 1;
            for (int iu0 = threadIdx.x; iu0 < nup; iu0 += U * T) {
                double2 pr[U][R];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int iu = iu0 + u * T;
#pragma unroll
                    for (int r = 0; r < R; r++)
                        pr[u][r] = (iu < nup && r < nr) ? __ldcg(pin + (long long)(r0 + r) * nup + iu)
                                                        : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int iu = iu0 + u * T;
                    if (iu >= nup) break;
#pragma unroll
                    for (int r = 0; r < R; r++) xs[iu * RS + r] = fma(am, pr[u][r].y, pr[u][r].x) * rb;
                }
            }
        }
        double e1d[R];
        int pd[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int id = min(r0 + r, ndn - 1);
            e1d[r] = __ldg(sJ.S.dn.e1 + id);
            pd[r] = __ldg(sJ.S.dn.imp + id);
        }
        __syncthreads();
        RowCol<R> nxt{};
        if ((int)threadIdx.x < nup) nxt = row_col<R>(sJ.S, sJ.D, wsh, threadIdx.x, r0, nr, prev);
        for (int iu = threadIdx.x; iu < nup; iu += T) {
            const RowCol<R> cur = nxt;                   // this column's data; the next one's in flight
            if (iu + T < nup) nxt = row_col<R>(sJ.S, sJ.D, wsh, iu + T, r0, nr, prev);
            double hv[R];
            row_part<R, RS>(sJ.S, xs, wint, amp_up, iu, cur, e1d, pd, hv);
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (r >= nr) break;
                const long long e = (long long)(r0 + r) * nup + iu;
                double y = hv[r] + (first ? cur.dd[r] / n0 : cur.dd[r] * rb);
                if (sJ.S.has_j) y = exchange_part(sJ.S, r0 + r, iu, cur.pu, pd[r], y, fetch_w);
                const double w = xs[iu * RS + r];
                if (!first) y = fma(-bk, cur.wp[r], y);
                __stcg(pout + e, make_double2(y, w));
                if (coeff) {
                    acc = fma(w, y, acc);
                } else {
                    double* ep = sJ.eig + e;
                    __stcg(ep, first ? ck * w : fma(ck, w, __ldcg(ep)));
                }
            }
        }
        __syncthreads();
    };

    unsigned running = 1u;
    int p = 0;
    for (; p < B.max_phases; p++) {
        const int ph = p & 1;
        const long long* pre = prefix + (size_t)ph * (B.njobs + 1);
        const long long* rg = my_range(ph);
        const long long t_end = __ldg(rg + 1);
        int cur = -1;
        double acc = 0.0;
        for (long long t = __ldg(rg); t < t_end; t++) {
            if (cur < 0 || t >= __ldg(pre + cur + 1)) {
                if (cur >= 0 && sS.active) flush(ph, acc);
                cur = find_job(pre, B.njobs, t);
                begin_job(cur, p, false);
                acc = 0.0;
            }
            if (!sS.active) continue;
            const int tl = (ph == 0) ? (int)__ldg(slab_of + t) : (int)(t - sJ.ph[ph].tile0);
            const int wdt = sJ.ph[ph].width;
            if (ph == 0) {
                switch (wdt) {
                case 8: col_tile(std::integral_constant<int, 8>{}, tl, acc); break;
                case 4: col_tile(std::integral_constant<int, 4>{}, tl, acc); break;
                default: col_tile(std::integral_constant<int, 2>{}, tl, acc); break;
                }
            } else {
                switch (wdt) {
                case 4: row_tile(std::integral_constant<int, 4>{}, tl, acc); break;
                case 2: row_tile(std::integral_constant<int, 2>{}, tl, acc); break;
                default: row_tile(std::integral_constant<int, 1>{}, tl, acc); break;
                }
            }
        }
        if (cur >= 0 && sS.active) flush(ph, acc);
        if (!grid_barrier(sw, status, nbar, running, B)) return;
        if (running == 0u) break;
    }
    if (B.slice && running != 0u && p == B.max_phases) {  // budget spent: open every run's next step
        const long long* pre = prefix;
        const long long* rg = my_range(0);
        const long long t_end = __ldg(rg + 1);
        int cur = -1;
        for (long long t = __ldg(rg); t < t_end; t++) {
            if (cur < 0 || t >= __ldg(pre + cur + 1)) {
                cur = find_job(pre, B.njobs, t);
                begin_job(cur, p, true);
            }
        }
    }
}

#ifdef EDZT_DEVICE_CHECKS
int lz_debug_bad(long long* out4)
{
    return cudaMemcpyFromSymbol(out4, g_edzt_bad, 4 * sizeof(long long)) == cudaSuccess ? 0 : 2;
}
#endif

int lz_grid_size(int device, size_t smem, int block)
{
    static std::atomic<unsigned long long> attr{0};
    if (edzt_once_per_device(attr))
        cudaFuncSetAttribute(k_lanczos, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLzSmemMax);
    int per_sm = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos, block, smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    return per_sm * nsm;
}

cudaError_t launch_lanczos_persistent(const LzBatch& B, const LzJob* jobs, const long long* prefix, double* slots,
                                      unsigned* sync_words, int* status, cudaStream_t s)
{
    LzBatch b = B;
    void* args[] = {(void*)&b, (void*)&jobs, (void*)&prefix, (void*)&slots, (void*)&sync_words, (void*)&status};
    return cudaLaunchCooperativeKernel((const void*)k_lanczos, dim3(B.grid), dim3(B.block), args, B.smem, s);
}

// ---------------------------------------------------------------------------
// launch plan
// ---------------------------------------------------------------------------
// Per-CTA dynamic shared memory: two CTAs of 256 threads per SM when every
// job fits, else one CTA of 512 threads per SM.
static constexpr size_t kLzSmemTwoPerSm = 108 * 1024;
static constexpr int kLzLongLine = 1500;
// Fixed cost of a tile in states, for cutting the tile list into CTA ranges
static constexpr double kLzTileCost = 1024.0;

// Width (of opts, descending) for `count` lines, each tile needing need(w)
// bytes of the budget: with few tiles in the launch, the one that minimises
// the lines one CTA sweeps when the job runs alone, ceil(tiles / G) * w
// (ties to the wider); with many, the widest that fits.
template <class Need>
static int pick_width(const int* opts, int nopt, int count, size_t budget, int G, bool many, Need need)
{
    int best = -1;
    long long best_cost = -1;
    for (int i = 0; i < nopt; i++) {
        const int w = opts[i];
        if (need(w) > budget) continue;
        if (many) return w;
        const long long tiles = (count + w - 1) / w;
        const long long cost = ((tiles + G - 1) / G) * w;
        if (best < 0 || cost < best_cost) { best = w; best_cost = cost; }
    }
    return best < 0 ? opts[nopt - 1] : best;
}

LzPlan lz_plan(int device, LzJob* jobs, int nj, std::vector<long long>& prefix, int prefer_block)
{
    LzPlan P;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const size_t fixed = lz_fixed_smem();
    size_t need_min = 0;
    long long lines8 = 0;
    int longest = 0;
    for (int j = 0; j < nj; j++) {
        const int nup = jobs[j].S.up.count, ndn = jobs[j].S.dn.count;
        need_min = std::max(need_min, std::max(lz_row_smem(nup, 1), lz_col_smem(ndn, 2)));
        lines8 += (ndn + 7) / 8 + (nup + 15) / 16;
        longest = std::max(longest, std::max(nup, ndn));
    }
    // Lines of kLzLongLine strings or more (nsite >= 13 near half filling)
    // run faster as one 512-thread CTA per SM with twice the shared memory
    // for wider tiles (measured with the tuner: 5-35% per step at nsite
    // 13-15, equal at 16); shorter lines as two 256-thread CTAs.
    const bool two = fixed + need_min <= kLzSmemTwoPerSm &&
                     (prefer_block == 256 || (longest < kLzLongLine && prefer_block != 512));
    P.block = two ? 256 : 512;
    const size_t budget = (two ? kLzSmemTwoPerSm : kLzSmemMax) - fixed;
    const int G_est = (two ? 2 : 1) * nsm;
    const bool many = lines8 >= 4LL * G_est;
    const int ropts[3] = {4, 2, 1}, copts[3] = {8, 4, 2};
    size_t chunk = 0;
    for (int j = 0; j < nj; j++) {
        LzJob& J = jobs[j];
        const int nup = J.S.up.count, ndn = J.S.dn.count;
        // a width preset by the tuner is kept when it fits this launch's budget
        const int wc = J.ph[0].width, r = J.ph[1].width;
        J.ph[0].width = (wc > 0 && lz_col_smem(ndn, wc) <= budget)
                            ? wc : pick_width(copts, 3, nup, budget, G_est, many, [&](int w) { return lz_col_smem(ndn, w); });
        J.ph[1].width = (r > 0 && lz_row_smem(nup, r) <= budget)
                            ? r : pick_width(ropts, 3, ndn, budget, G_est, many, [&](int w) { return lz_row_smem(nup, w); });
        chunk = std::max(chunk, std::max(lz_col_smem(ndn, J.ph[0].width), lz_row_smem(nup, J.ph[1].width)));
    }
    P.smem = fixed + chunk;
    P.grid = lz_grid_size(device, P.smem, P.block);
    if (P.grid <= 0) return P;
    P.slots = lz_cut(jobs, nj, P.grid, prefix, P.total);
    return P;
}

long long lz_cut(LzJob* jobs, int nj, int G, std::vector<long long>& prefix, long long total[2])
{
    long long slots = 0;
    prefix.assign(2 * (size_t)(nj + 1) + 2 * (size_t)(G + 1), 0);
    std::vector<long long> slab_order;
    for (int ph = 0; ph < 2; ph++) {
        long long* pre = prefix.data() + (size_t)ph * (nj + 1);
        for (int j = 0; j < nj; j++) {
            LzPhase& Q = jobs[j].ph[ph];
            const int count = (ph == 0) ? jobs[j].S.up.count : jobs[j].S.dn.count;
            Q.ntiles = (count + Q.width - 1) / Q.width;
            Q.tile0 = pre[j];
            pre[j + 1] = pre[j] + Q.ntiles;
        }
        const long long T = pre[nj];
        total[ph] = T;
        // CTA ranges: with no more tiles than CTAs, CTA b takes tile b; else
        // the list is cut where the running cost crosses b/G of the total
        // (a tile costs its states plus a fixed amount for its staging round
        // and barriers), every CTA keeping at least one tile.
        long long* range = prefix.data() + 2 * (size_t)(nj + 1) + (size_t)ph * (G + 1);
        if (T <= G) {
            for (int b = 0; b <= G; b++) range[b] = std::min<long long>(b, T);
        } else {
            std::vector<double> cum((size_t)T + 1, 0.0);
            for (int j = 0; j < nj; j++) {
                const LzPhase& Q = jobs[j].ph[ph];
                const long long lines = (ph == 0) ? jobs[j].S.dn.count : jobs[j].S.up.count;
                const int count = (ph == 0) ? jobs[j].S.up.count : jobs[j].S.dn.count;
                for (int i = 0; i < Q.ntiles; i++) {
                    const int w = std::min(Q.width, count - i * Q.width);
                    cum[Q.tile0 + i + 1] = cum[Q.tile0 + i] + (double)lines * w + kLzTileCost;
                }
            }
            range[0] = 0;
            range[G] = T;
            long long t = 0;
            for (int b = 1; b < G; b++) {
                const double target = cum[T] * b / G;
                while (t < T && cum[t + 1] <= target) t++;
                range[b] = std::min(std::max(t, range[b - 1] + 1), T - (G - b));
                t = range[b];
            }
        }
        // participants of a job: the CTAs whose range meets its tiles (a contiguous run)
        auto owner = [&](long long tile) {
            return (int)(std::upper_bound(range, range + G + 1, tile) - range) - 1;
        };
        for (int j = 0; j < nj; j++) {
            LzPhase& Q = jobs[j].ph[ph];
            Q.part0 = owner(Q.tile0);
            Q.npart = owner(Q.tile0 + Q.ntiles - 1) - Q.part0 + 1;
            Q.slot0 = slots;
            slots += Q.npart;
        }
        // Column phase: the slab each tile position stages.  A participant
        // takes its positions in order; numbering the slabs by round (the
        // r-th tile of every participant, participants in order) makes the
        // participants stage neighbouring slabs at the same time, so the
        // rows they read sit side by side in DRAM.
        if (ph == 0) {
            slab_order.assign((size_t)T, 0);
            for (int j = 0; j < nj; j++) {
                const LzPhase& Q = jobs[j].ph[0];
                const long long lo = Q.tile0, hi = Q.tile0 + Q.ntiles;
                long long next = 0;
                for (long long r = 0; next < Q.ntiles; r++)
                    for (int q = 0; q < Q.npart; q++) {
                        const long long s0 = std::max(range[Q.part0 + q], lo), s1 = std::min(range[Q.part0 + q + 1], hi);
                        if (s0 + r < s1) slab_order[(size_t)(s0 + r)] = next++;
                    }
            }
        }
    }
    prefix.insert(prefix.end(), slab_order.begin(), slab_order.end());
    return slots;
}
