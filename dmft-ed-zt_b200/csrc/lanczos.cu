// lanczos.cu — kernel (c): persistent, batched, fused Lanczos.
//
// One cooperative launch runs every step of many independent Lanczos runs
// ("jobs": sectors of the ground-state search, the eigenvector pass of the
// winning sector, c / c^+ excitation runs of the Green's function).  Each
// job is cut into tiles of whole rows; the tiles of all jobs form one list
// and CTA b takes tiles b, b+G, b+2G, ... in every pass, so the CTAs sweep
// the vectors together (the rows a sweep gathers from stay in L2) and the
// same CTAs meet the same job every pass.  Passes are separated by a
// hierarchical grid barrier with a bounded wait.
//
// The recurrence is the reference's (src/lanczos_solver.f90:92-173):
//   w_k = v_k / b_k,  v_k = y_{k-1} - a_{k-1} w_{k-1},
//   y_k = H w_k - b_k w_{k-1},  a_k = <w_k, y_k>,  b_{k+1} = ||y_k - a_k w_k||.
// Fusion: a pass stores the pair (y_k, w_k); the next pass forms w_{k+1}
// wherever it reads it (rows staged in shared memory for the up-spin hops,
// down-spin neighbours gathered as one 16-byte pair per hop), so a step is
// one sweep.  Its sums are taken around the shift a_{k-1}: with
// t = y - a_{k-1} w it reduces <w,t>, <t,t>, <w,w>, so a_k = a_{k-1}<w,w> +
// <w,t> and, with d = a_k - a_{k-1}, b_{k+1}^2 = <t,t> - 2d<w,t> + d^2<w,w>.
// The next pass, which forms v_{k+1} element by element anyway, also sums
// ||v_{k+1}||^2 exactly; when that disagrees with the b_{k+1} it used (by
// more than 1e-12 relative, e.g. in an exhausted Krylov space of a tiny
// sector) the job repeats that step with the exact norm, as the reference
// computes it.  The first step divides v_init by its norm exactly as the
// reference does, so a one-dimensional sector breaks down with b(2) = 0.
//
// Between passes every participating CTA of a job re-derives the job's
// scalars from the partial sums of the previous pass (slots in a fixed order,
// so all of them get the same bits) and the first participant also stores
// them; partial sums and states are double-buffered by pass parity, so no
// per-job atomics are needed.
#include <cuda_runtime.h>
#include <type_traits>
#include "edzt_internal.h"
#include "hv_row.cuh"

static constexpr int kLzThreads = 256;
// CTAs per SM the register allocation is sized for
#ifndef EDZT_LZ_MINBLOCKS
#define EDZT_LZ_MINBLOCKS 2
#endif
static constexpr size_t kLzTileTarget = 24 * 1024;
static constexpr double kVerifyTol = 1.0e-12;
static constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000ull * 1000ull * 1000ull;
static constexpr int kFixedDoubles = 128 + EDZT_MAX_P * EDZT_MAX_P + EDZT_MAX_AMP;   // reduction scratch, wint, amp
static constexpr int kBarGroup = 16;                                  // CTAs per barrier group

// sync words (unsigned), each counter on its own 128-byte line; SW_GEN is a
// 64-bit word (barrier count << 32 | runs still going)
#define SW_GEN 0
#define SW_TOP 32
#define SW_ACTIVE 64

#define SW_GROUP(g) (128 + 32 * (g))

size_t lz_sync_bytes(int G) { return sizeof(unsigned) * (128 + 32 * (size_t)((G + kBarGroup - 1) / kBarGroup)); }

int lz_rows_per_tile(int nup, int ndn, int hw_dn)
{
    int r = (int)(kLzTileTarget / staged_row_bytes(nup, hw_dn));
    if (r < 1) r = 1;
    if (r > ndn) r = ndn;
    return r;
}

int lz_rows_balanced(int ndn, int rows_max, int G)
{
    // rows per tile <= rows_max minimising the rows one CTA sweeps when the
    // job runs alone, ceil(tiles / G) * rows; ties go to fewer, larger tiles
    int best = rows_max;
    long long best_cost = -1;
    for (int r = rows_max; r >= 1; r--) {
        const long long tiles = (ndn + r - 1) / r;
        const long long cost = ((tiles + G - 1) / G) * r;
        if (best_cost < 0 || cost < best_cost) { best = r; best_cost = cost; }
    }
    return best;
}

size_t lz_smem_bytes(int nup, int hw_dn, int rows)
{
    return kFixedDoubles * sizeof(double) + (size_t)rows * staged_row_bytes(nup, hw_dn);
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Hierarchical grid barrier with a bounded wait.  Counters only grow: the
// k-th barrier of a launch is complete on a group counter at k * (group
// size) arrivals and on the top counter at k * (number of groups), so no
// counter is read before arriving or reset after.  CTAs arrive on the counter
// of their group of 16, the last of each group on the top counter, and the
// last of all publishes (k << 32 | runs still going) in the 64-bit
// generation word, which the others wait for.  Returns false (and the kernel
// stops) when the wait ran out or another CTA reported an error; *snap
// receives the number of runs still going.
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

// ---------------------------------------------------------------------------
// scalar recurrence between passes (same on every participating CTA)
// ---------------------------------------------------------------------------
struct Sums {
    double wt, tt, ww, vv;
};

// State of the pass after `prev`, from the sums of the pass that used `prev`.
// `out` marks the first participant: it stores a(k), b(k) as they are
// accepted and counts finished runs.
__device__ LzState advance(const LzJob& J, const LzState& prev, const Sums& s, bool out, unsigned* sw)
{
    LzState n = prev;
    n.retry = 0;
    if (!prev.active) return n;
    auto finish = [&](int nstep) {
        n.active = 0;
        n.nstep = nstep;
        if (out) atomicSub(sw + SW_ACTIVE, 1u);
    };
    if (prev.k == 0) {                                  // after the start-vector pass
        const double nrm = sqrt(s.vv);
        n.norm0 = nrm;
        if (!(nrm > 0.0)) { finish(0); return n; }      // zero start vector
        n.k = 1;
        n.a_prev = 0.0;
        n.b_cur = nrm;
        return n;
    }
    const int k = prev.k;
    if (J.mode == LZ_EIGVEC) {                          // stored coefficients, no sums
        if (k >= J.maxnstep) { finish(k); return n; }
        n.k = k + 1;
        n.a_prev = J.a[k - 1];
        n.b_cur = J.b[k];
        return n;
    }
    if (k >= 2) {                                       // verify the b_k the step used
        const double bex = sqrt(s.vv);
        if (bex < 1.0e-16) {                            // breakdown (lanczos_solver.f90:161)
            if (out) J.b[k - 1] = 0.0;
            finish(k - 1);
            return n;
        }
        if (!(fabs(bex - prev.b_cur) <= kVerifyTol * bex)) {
            if (out) J.b[k - 1] = bex;
            n.b_cur = bex;
            n.retry = 1;
            return n;
        }
    }
    const double ah = (k == 1) ? 0.0 : prev.a_prev;
    const double a = fma(ah, s.ww, s.wt);               // a(k) = <w, y>  (lanczos_solver.f90:134,159)
    if (out) {
        J.a[k - 1] = a;
        if (k == 1) J.b[0] = 0.0;                       // :135
    }
    if (k >= J.maxnstep) { finish(k); return n; }       // :137-141, :161-164
    const double d = a - ah;
    const double bb2 = s.tt - 2.0 * d * s.wt + d * d * s.ww;
    // an ill-conditioned or non-positive estimate is repaired by the next
    // pass's exact norm (one repeated step)
    const double bn = sqrt(fmax(bb2, 1.0e-300));
    if (out) J.b[k] = bn;
    n.k = k + 1;
    n.a_prev = a;
    n.b_cur = bn;
    return n;
}

// ---------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kLzThreads, EDZT_LZ_MINBLOCKS)
    k_lanczos(LzBatch B, const LzJob* __restrict__ jobs, LzState* __restrict__ state,
              const long long* __restrict__ prefix, double* __restrict__ partials, unsigned* __restrict__ sw,
              int* __restrict__ status)
{
    extern __shared__ __align__(16) double smem[];
    double* red = smem;                                  // 128 doubles of reduction scratch
    double* wint = smem + 128;                           // interaction energies by impurity patterns
    double* amp = wint + EDZT_MAX_P * EDZT_MAX_P;        // up-spin hop amplitudes by slot
    double* chunk_base = smem + kFixedDoubles;           // staged rows of the current tile
    __shared__ LzJob sJ;
    __shared__ LzState sS;
    __shared__ int s_job;

    const int G = gridDim.x;
    unsigned nbar = 0u;                                  // grid barriers this CTA has passed
    if (threadIdx.x == 0) s_job = -1;
    __syncthreads();

    // slot of this CTA in the current job (participants: CTAs (tile0 + q) mod G, q < npart)
    auto my_q = [&]() { return (int)(((long long)blockIdx.x - sJ.tile0 % G + G) % G); };

    // Enter job j in pass `pass`: load it if needed and derive its state.
    auto begin_job = [&](int j, int pass) {
        __syncthreads();
        if (j != s_job) {
            const int* src = reinterpret_cast<const int*>(jobs + j);
            int* dst = reinterpret_cast<int*>(&sJ);
            for (int i = threadIdx.x; i < (int)(sizeof(LzJob) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
            __syncthreads();
            stage_wint(sJ.S, wint);
            stage_amp(sJ.S.up, amp);
            if (threadIdx.x == 0) s_job = j;
        }
        if (pass == 0) {
            if (threadIdx.x == 0) {
                const int* ss = reinterpret_cast<const int*>(state + 2 * (size_t)j);
                int* sd = reinterpret_cast<int*>(&sS);
                for (int i = 0; i < (int)(sizeof(LzState) / sizeof(int)); i++) sd[i] = __ldcg(ss + i);
            }
            __syncthreads();
            return;
        }
        // sum the previous pass's slots in participant order
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        const int par = (pass - 1) & 1;
        for (int i = threadIdx.x; i < sJ.npart; i += blockDim.x) {
            const double* p = partials + ((sJ.slot0 + i) * 2 + par) * 4;
            v[0] += __ldcg(p); v[1] += __ldcg(p + 1); v[2] += __ldcg(p + 2); v[3] += __ldcg(p + 3);
        }
        block_sum<4>(v, red);
        if (threadIdx.x == 0) {
            LzState prev;
            const int* ss = reinterpret_cast<const int*>(state + 2 * (size_t)j + par);
            int* sd = reinterpret_cast<int*>(&prev);
            for (int i = 0; i < (int)(sizeof(LzState) / sizeof(int)); i++) sd[i] = __ldcg(ss + i);
            const bool first = (my_q() == 0);
            Sums s{v[0], v[1], v[2], v[3]};
            sS = advance(sJ, prev, s, first, sw);
            if (first) state[2 * (size_t)j + (pass & 1)] = sS;   // published by the barrier's fence
        }
        __syncthreads();
    };

    auto flush = [&](int pass, double (&acc)[4]) {
        block_sum<4>(acc, red);
        if (threadIdx.x == 0) {
            EDZT_OK_OR(my_q() < sJ.npart, 24, blockIdx.x, sJ.tile0, sJ.npart, return)
            double* p = partials + ((sJ.slot0 + my_q()) * 2 + (pass & 1)) * 4;
            p[0] = acc[0]; p[1] = acc[1]; p[2] = acc[2]; p[3] = acc[3];
        }
    };

    // Start vector rows of tile tl: materialise (v, 0) pairs, sum v^2.
    auto init_tile = [&](int tl, double (&acc)[4]) {
        const int nup = sJ.S.up.count;
        const int r0 = tl * sJ.rows, rows = min(sJ.rows, sJ.S.dn.count - r0);
        const long long g0 = (long long)r0 * nup, n = (long long)rows * nup;
        double2* Y1 = sJ.YW[1];
        for (long long e = threadIdx.x; e < n; e += blockDim.x) {
            const long long g = g0 + e;
            EDZT_OK_OR(g < sJ.S.dim, 25, g, sJ.S.dim, tl, break)
            double v;
            if (sJ.init == LZ_INIT_HASH) v = edzt_u01(sJ.key, (uint64_t)g);
            else if (sJ.init == LZ_INIT_APPLYC) v = apply_c_value(sJ.ac, sJ.src, g);
            else v = __ldg(sJ.src + g);
            __stcg(Y1 + g, make_double2(v, 0.0));
            acc[3] = fma(v, v, acc[3]);
        }
    };

    // One Lanczos step (k = sS.k) on the rows of tile tl.  The first step
    // (FIRST) divides by the start vector's norm exactly; later steps
    // multiply by 1/b_k, so no division sits in their loops.
    auto step_tile = [&](auto first_tag, int tl, double (&acc)[4]) {
        constexpr bool FIRST = decltype(first_tag)::value;
        const int nup = sJ.S.up.count, hwd = sJ.S.dn.hw;
        const int k = sS.k;
        const int p = k & 1;
        const double2* __restrict__ YWp = sJ.YW[p];
        double2* __restrict__ YWn = sJ.YW[p ^ 1];
        const double b_cur = sS.b_cur, rb = 1.0 / b_cur, am = -sS.a_prev, mb = -b_cur;
        const bool coeff = (sJ.mode == LZ_COEFF);
        const double ck = coeff ? 0.0 : sJ.coeff[k - 1];
        auto fetch = [&](long long idx) {
            EDZT_OK_OR(idx >= 0 && idx < sJ.S.dim, 21, idx, sJ.S.dim, k, return 0.0)
            const double2 pr = __ldcg(YWp + idx);
            if (FIRST) return pr.x / b_cur;
            return fma(am, pr.y, pr.x) * rb;
        };
        const int r0 = tl * sJ.rows, rows = min(sJ.rows, sJ.S.dn.count - r0);
        Chunk C = chunk_layout(chunk_base, sJ.rows, nup, hwd);
        const int n = rows * nup;
        EDZT_OK_OR(rows >= 1 && (long long)r0 * nup + n <= sJ.S.dim, 22, r0, rows, n, return)
        const double2* __restrict__ Yt = YWp + (long long)r0 * nup;
        double2* __restrict__ Ot = YWn + (long long)r0 * nup;
        double* __restrict__ Et = coeff ? nullptr : sJ.eig + (long long)r0 * nup;
        for (int e0 = threadIdx.x; e0 < n; e0 += 4 * blockDim.x) {
            double2 pr[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int e = e0 + q * blockDim.x;
                pr[q] = (e < n) ? __ldcg(Yt + e) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int e = e0 + q * blockDim.x;
                if (e >= n) break;
                if (FIRST) {
                    C.xs[e] = pr[q].x / b_cur;
                } else {
                    const double v = fma(am, pr[q].y, pr[q].x);
                    acc[3] = fma(v, v, acc[3]);      // exact ||v_k||^2: verifies b_k
                    C.xs[e] = v * rb;
                }
            }
        }
        stage_rows(sJ.S.dn, C, r0, rows);
        __syncthreads();
        // Warps take (row, column segment) items; a row's down hops, energy and
        // impurity bits are loaded once per item into registers, and the warp
        // walks its segment 32 columns at a time.
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        const int W = max(32, ((nup + nwarps - 1) / nwarps + 31) & ~31);
        const int nseg = (nup + W - 1) / W;
        const uint4* __restrict__ hpk = sJ.S.up.hpk;
        const bool two = sJ.S.up.hw > 4;
        for (int item = warp; item < rows * nseg; item += nwarps) {
            const int r = item / nseg, c0 = (item - r * nseg) * W, c1 = min(nup, c0 + W);
            const int hd = C.dcnt[r];
            EDZT_OK_OR(hd >= 0 && hd <= C.hw, 13, r, hd, C.hw, continue)
            const DHop* __restrict__ rec = C.dh + r * C.hw;
            unsigned off[8];                                         // amplitudes stay in shared memory
#pragma unroll
            for (int q = 0; q < 8; q++) off[q] = (q < hd) ? (unsigned)rec[q].off : 0u;
            const double rowe = C.de1[r];
            const double* __restrict__ wrow = wint + C.dimp[r];
            const double* __restrict__ xrow = C.xs + r * nup;
            for (int iu = c0 + lane; iu < c1; iu += 32) {
                const int e = r * nup + iu;
                const double2* __restrict__ col = YWp + iu;
                // every load of the element first
                const uint4 q0 = __ldg(hpk + iu);
                const uint4 q1 = two ? __ldg(hpk + nup + iu) : make_uint4(0u, 0u, 0u, 0u);
                const int hu = __ldg(sJ.S.up.hcnt + iu);
                const int pu = __ldg(sJ.S.up.imp + iu);
                const double e1u = __ldg(sJ.S.up.e1 + iu);
                const double wprev = FIRST ? 0.0 : __ldcg(reinterpret_cast<const double*>(Yt + e) + 1);
                const double eprev = (coeff || FIRST) ? 0.0 : __ldcg(Et + e);
                double2 g[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    EDZT_OK_OR(q >= hd || (long long)off[q] + iu < sJ.S.dim, 21, off[q], iu, sJ.S.dim, g[q] = make_double2(0.0, 0.0); continue)
                    g[q] = (q < hd) ? __ldcg(col + off[q]) : make_double2(0.0, 0.0);
                }
                // diagonal and up hops from the staged row
                const double xe = xrow[iu];
                double hv = (e1u + rowe + wrow[pu * sJ.S.P]) * xe;
                const uint32_t eu[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    if (c < hu) {
                        EDZT_OK_OR(edzt_hop_rank(eu[c]) < nup && edzt_hop_slot(eu[c]) < sJ.S.up.namp, 11, iu, c,
                                   (long long)eu[c], continue)
                        hv = fma(amp[edzt_hop_slot(eu[c])], xrow[edzt_hop_rank(eu[c])], hv);
                    }
                }
                for (int h0 = 8; h0 < hu; h0 += 4) {                 // hop lists longer than 8
                    const uint4 q = __ldg(hpk + (size_t)(h0 >> 2) * nup + iu);
                    const uint32_t f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (h0 + c < hu) hv = fma(amp[edzt_hop_slot(f[c])], xrow[edzt_hop_rank(f[c])], hv);
                }
                // down hops: v = y - a w at each neighbour, as its owner forms it
                double dv = 0.0;
#pragma unroll
                for (int q = 0; q < 8; q++)
                    if (q < hd) dv = fma(rec[q].val, fma(am, g[q].y, g[q].x), dv);
                for (int h = 8; h < hd; h++) {
                    const double2 gg = __ldcg(col + rec[h].off);
                    dv = fma(rec[h].val, fma(am, gg.y, gg.x), dv);
                }
                hv += FIRST ? dv / b_cur : dv * rb;                   // sum c * w_k(id', iu)
                if (sJ.S.has_j) hv = hv_exchange(sJ.S, C, r, iu, hv, fetch);
                const double y = FIRST ? hv : fma(mb, wprev, hv);
                __stcg(Ot + e, make_double2(y, xe));
                if (coeff) {
                    const double t = fma(am, xe, y);         // y - a_{k-1} w (a_0 = 0)
                    acc[0] = fma(xe, t, acc[0]);
                    acc[1] = fma(t, t, acc[1]);
                    acc[2] = fma(xe, xe, acc[2]);
                } else {
                    __stcg(Et + e, FIRST ? ck * xe : fma(ck, xe, eprev));
                }
            }
        }
        __syncthreads();
    };

    for (int pass = 0; pass < B.max_passes; pass++) {
        int cur = -1;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (long long t = blockIdx.x; t < B.total_tiles; t += G) {
            if (cur < 0 || t >= __ldg(prefix + cur + 1)) {
                if (cur >= 0 && sS.active) flush(pass, acc);
                cur = find_job(prefix, B.njobs, t);
                begin_job(cur, pass);
                acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
            }
            if (!sS.active) continue;
            const int tl = (int)(t - sJ.tile0);
            if (pass == 0) init_tile(tl, acc);
            else if (sS.k == 1) step_tile(std::true_type{}, tl, acc);
            else step_tile(std::false_type{}, tl, acc);
        }
        if (cur >= 0 && sS.active) flush(pass, acc);
        unsigned running = 0u;
        if (!grid_barrier(sw, status, nbar, running, B)) return;
        if (running == 0u) break;
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
    static std::atomic<unsigned long long> attr{0};
    if (edzt_once_per_device(attr))
        cudaFuncSetAttribute(k_lanczos, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    int per_sm = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos, kLzThreads, smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (block_out) *block_out = kLzThreads;
    return per_sm * nsm;
}

cudaError_t launch_lanczos_persistent(const LzBatch& B, const LzJob* jobs, LzState* state, const long long* tile_prefix,
                                      double* partials, unsigned* sync_words, int* status, cudaStream_t s)
{
    LzBatch b = B;
    void* args[] = {(void*)&b, (void*)&jobs, (void*)&state, (void*)&tile_prefix, (void*)&partials,
                    (void*)&sync_words, (void*)&status};
    return cudaLaunchCooperativeKernel((const void*)k_lanczos, dim3(B.grid), dim3(B.block), args, B.smem, s);
}
