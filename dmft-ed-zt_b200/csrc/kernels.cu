// kernels.cu — standalone (one launch per operation) sm_100a kernels:
// H.v, the BLAS-1 steps of the plain Lanczos drop-in, apply_c and the
// continued fractions.  The fused persistent Lanczos lives in lanczos.cu.
#include <algorithm>
#include <cuda_runtime.h>
#include "edzt_internal.h"
#include "hv_phase.cuh"
#include "hv_gather.cuh"

static constexpr int kWintDoubles = EDZT_MAX_P * EDZT_MAX_P;
static constexpr int kAmpDoubles = EDZT_MAX_AMP;

#ifdef EDZT_DEVICE_CHECKS
int kernels_debug_bad(long long* out4)
{
    return cudaMemcpyFromSymbol(out4, g_edzt_bad, 4 * sizeof(long long)) == cudaSuccess ? 0 : 2;
}
#endif

// ---------------------------------------------------------------------------
// H.v: y = H x (accumulate = 0) or y = y + H x (accumulate = 1), the `py`
// flag of src/impurity_hamiltonian.f90:241-245, in the two phases of
// hv_phase.cuh: k_hx_col writes the down-hop part of every element into a
// scratch vector D, then k_hx_row adds the diagonal, up-hop and exchange
// parts.  Both stream their data once; all neighbour values come from
// shared memory.
// ---------------------------------------------------------------------------
static constexpr int kHxThreads = 256;
static constexpr int kHxThreadsLong = 1024;          // lines of kHxLongLine strings or more
static constexpr int kHxLongLine = 1500;
static constexpr int kHxGatherLine = 3000;            // single-pass form from here (nsite >= 14 near half filling)
static constexpr size_t kHxSmemSoft = 100 * 1024;    // two CTAs per SM
static constexpr size_t kHxSmemHard = 210 * 1024;    // one CTA per SM

// Column phase: CTA b stages columns [b*WC, b*WC + WC) of every row.
template <int WC, int NT>
__global__ void __launch_bounds__(NT) k_hx_col(DevSector S, const double* __restrict__ x,
                                                      double* __restrict__ D)
{
    constexpr int WS = phase_stride(WC);
    extern __shared__ __align__(16) double smem[];
    double* amp = smem;                                    // down-hop amplitudes
    double* ws = smem + kAmpDoubles;                       // [ndn][WS]
    const int nup = S.up.count, ndn = S.dn.count;
    const int c0 = blockIdx.x * WC;
    stage_table(S.dn.amp, S.dn.namp, amp);
    const int n = ndn * WC;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {   // the whole slab in flight at once
        const int id = i / WC, c = i - id * WC;
        const bool in = c0 + c < nup;
        copy_async8(ws + id * WS + c, x + (in ? (size_t)id * nup + c0 + c : 0), in);
    }
    copy_async_wait_all();
    __syncthreads();
    HopList nxt{};
    if ((int)threadIdx.x < ndn) nxt = hop_list(S.dn, threadIdx.x);
    for (int id = threadIdx.x; id < ndn; id += blockDim.x) {
        const HopList cur = nxt;
        if (id + (int)blockDim.x < ndn) nxt = hop_list(S.dn, id + blockDim.x);
        double d[WC];
        col_part<WC, WS>(S, ws, amp, id, cur, d);
        store_slab_row<WC>(D, c0, ndn, id, d);          // columns past nup hold 0 (staged as 0)
    }
}

// Row phase: CTA b stages rows [b*R, b*R + R), thread per column.
template <bool ACC, int R, int NT>
__global__ void __launch_bounds__(NT) k_hx_row(DevSector S, const double* __restrict__ x,
                                                      const double* __restrict__ D, int wsh, double* __restrict__ y)
{
    constexpr int RS = phase_stride(R);
    extern __shared__ __align__(16) double smem[];
    double* wint = smem;
    double* amp = smem + kWintDoubles;
    double* xs = amp + kAmpDoubles;                        // [nup][RS]
    const int nup = S.up.count, ndn = S.dn.count;
    const int r0 = blockIdx.x * R;
    const int nr = min(R, ndn - r0);
    stage_table(S.wint, S.P * S.P, wint);
    stage_table(S.up.amp, S.up.namp, amp);
    for (int iu = threadIdx.x; iu < nup; iu += blockDim.x) {   // the whole tile in flight at once
#pragma unroll
        for (int r = 0; r < R; r++)
            copy_async8(xs + iu * RS + r, x + (r < nr ? (size_t)(r0 + r) * nup + iu : 0), r < nr);
    }
    double e1d[R];
    int pd[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int id = min(r0 + r, ndn - 1);
        e1d[r] = __ldg(S.dn.e1 + id);
        pd[r] = __ldg(S.dn.imp + id);
    }
    copy_async_wait_all();
    __syncthreads();
    auto fetch = [&](long long idx) {
        EDZT_OK_OR(idx >= 0 && idx < S.dim, 61, idx, S.dim, blockIdx.x, return 0.0)
        return __ldg(x + idx);
    };
    RowCol<R> nxt{};
    if ((int)threadIdx.x < nup) nxt = row_col<R>(S, D, wsh, threadIdx.x, r0, nr);
    for (int iu = threadIdx.x; iu < nup; iu += blockDim.x) {
        const RowCol<R> cur = nxt;                          // this column's data; the next one's in flight
        if (iu + (int)blockDim.x < nup) nxt = row_col<R>(S, D, wsh, iu + blockDim.x, r0, nr);
        double acc[R];
        row_part<R, RS>(S, xs, wint, amp, iu, cur, e1d, pd, acc);
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (r >= nr) break;
            const size_t g = (size_t)(r0 + r) * nup + iu;
            double v = acc[r] + cur.dd[r];
            if (S.has_j) v = exchange_part(S, r0 + r, iu, cur.pu, pd[r], v, fetch);
            y[g] = ACC ? y[g] + v : v;
        }
    }
}

// Rows per tile: the most (of 8, 4, 2, 1) that fit two CTAs per SM and still
// give every SM two tiles; columns per slab likewise (16, 8, 4, 2).  A
// sector too large for that takes one CTA per SM.
static int hx_rows_of(int nup, int ndn, int nsm)
{
    const int opts[4] = {8, 4, 2, 1};
    for (int R : opts) {
        const size_t sm = (kWintDoubles + kAmpDoubles + (size_t)nup * phase_stride(R)) * sizeof(double);
        if (sm <= kHxSmemSoft && (ndn + R - 1) / R >= 2 * nsm) return R;
    }
    for (int R : {2, 1}) {
        const size_t sm = (kWintDoubles + kAmpDoubles + (size_t)nup * phase_stride(R)) * sizeof(double);
        if (sm <= kHxSmemSoft) return R;
    }
    return 1;
}

static int hx_cols_of(int nup, int ndn, int nsm)
{
    const int opts[4] = {16, 8, 4, 2};
    for (int W : opts) {
        const size_t sm = (kAmpDoubles + (size_t)ndn * phase_stride(W)) * sizeof(double);
        if (sm <= kHxSmemSoft && (nup + W - 1) / W >= 2 * nsm) return W;
    }
    return 2;
}

bool hx_fits(int nup, int ndn)
{
    const size_t row = (kWintDoubles + kAmpDoubles + (size_t)nup * phase_stride(1)) * sizeof(double);
    const size_t col = (kAmpDoubles + (size_t)ndn * phase_stride(2)) * sizeof(double);
    return row <= kHxSmemHard && col <= kHxSmemHard;
}

template <int R, int NT>
static void launch_hx_row(const DevSector& S, const double* x, const double* D, int wc, double* y, int accumulate,
                          cudaStream_t s)
{
    const int wsh = __builtin_ctz((unsigned)wc);
    static std::atomic<unsigned long long> attr_set{0};
    if (edzt_once_per_device(attr_set)) {
        cudaFuncSetAttribute(k_hx_row<false, R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHxSmemHard);
        cudaFuncSetAttribute(k_hx_row<true, R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHxSmemHard);
    }
    const int tiles = (S.dn.count + R - 1) / R;
    const size_t sm = (kWintDoubles + kAmpDoubles + (size_t)S.up.count * phase_stride(R)) * sizeof(double);
    if (accumulate) k_hx_row<true, R, NT><<<tiles, NT, sm, s>>>(S, x, D, wsh, y);
    else k_hx_row<false, R, NT><<<tiles, NT, sm, s>>>(S, x, D, wsh, y);
}

template <int W, int NT>
static void launch_hx_col(const DevSector& S, const double* x, double* D, cudaStream_t s)
{
    static std::atomic<unsigned long long> attr_set{0};
    if (edzt_once_per_device(attr_set))
        cudaFuncSetAttribute(k_hx_col<W, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHxSmemHard);
    const int slabs = (S.up.count + W - 1) / W;
    const size_t sm = (kAmpDoubles + (size_t)S.dn.count * phase_stride(W)) * sizeof(double);
    k_hx_col<W, NT><<<slabs, NT, sm, s>>>(S, x, D);
}

// ---------------------------------------------------------------------------
// Single-pass H.v for long lines (hv_gather.cuh): one CTA per tile of R full
// rows staged in shared memory with their down-hop records; the up hops read
// the staged rows, the down hops gather coalesced slices of other rows from
// global memory.  T threads per CTA, 64 registers (32 warps per SM).
// ---------------------------------------------------------------------------
static constexpr size_t kGatherTileBytes = 24 * 1024;

template <bool ACC, int T>
__global__ void __launch_bounds__(T, T == 512 ? 2 : 1) k_hx_gather(DevSector S, const double* __restrict__ x,
                                                                  double* __restrict__ y, int R)
{
    extern __shared__ __align__(16) double smem[];
    double* wint = smem;
    double* amp = smem + kWintDoubles;
    const int nup = S.up.count, ndn = S.dn.count;
    Chunk C = chunk_layout(smem + kWintDoubles + kAmpDoubles, R, nup, S.dn.hw);
    const int r0 = blockIdx.x * R;
    const int rows = min(R, ndn - r0);
    const int n = rows * nup;
    const long long g0 = (long long)r0 * nup;
    for (int e = threadIdx.x; e < n; e += blockDim.x) C.xs[e] = __ldg(x + g0 + e);
    stage_rows(S.dn, C, r0, rows);
    stage_table(S.wint, S.P * S.P, wint);
    stage_table(S.up.amp, S.up.namp, amp);
    __syncthreads();
    auto fetch = [&](long long idx) {
        EDZT_OK_OR(idx >= 0 && idx < S.dim, 61, idx, S.dim, blockIdx.x, return 0.0)
        return __ldg(x + idx);
    };
    const SrcVec src{x};
    int r = threadIdx.x / nup, iu = threadIdx.x - r * nup;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        double du, dn;
        hv_elem(S, C, wint, amp, src, r, iu, C.xs[e], du, dn);
        double acc = du + dn;
        if (S.has_j) acc = hv_exchange(S, C, r, iu, acc, fetch);
        const long long g = g0 + e;
        y[g] = ACC ? y[g] + acc : acc;
        iu += blockDim.x;
        while (iu >= nup) { iu -= nup; ++r; }
    }
}

template <int T>
static void launch_hx_gather(const DevSector& S, const double* x, double* y, int accumulate, cudaStream_t s)
{
    static std::atomic<unsigned long long> attr_set{0};
    if (edzt_once_per_device(attr_set)) {
        cudaFuncSetAttribute(k_hx_gather<false, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHxSmemHard);
        cudaFuncSetAttribute(k_hx_gather<true, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHxSmemHard);
    }
    const int nup = S.up.count, ndn = S.dn.count;
    const size_t row = staged_row_bytes(nup, S.dn.hw);
    const int R = std::max(1, std::min(ndn, (int)(kGatherTileBytes / row)));
    const int tiles = (ndn + R - 1) / R;
    const size_t smem = (kWintDoubles + kAmpDoubles) * sizeof(double) + (size_t)R * row;
    if (accumulate) k_hx_gather<true, T><<<tiles, T, smem, s>>>(S, x, y, R);
    else k_hx_gather<false, T><<<tiles, T, smem, s>>>(S, x, y, R);
}

// Whether H.v of a sector takes the single-pass form: lines of
// kHxGatherLine strings or more (measured faster there: the two-phase
// slabs and tiles are too narrow).
bool hx_single_pass(int nup, int ndn) { return std::max(nup, ndn) >= kHxGatherLine; }

void launch_hx(const DevSector& S, const double* x, double* y, int accumulate, double* scratch, cudaStream_t s)
{
    const int nup = S.up.count, ndn = S.dn.count;
    if (nup <= 0 || ndn <= 0) return;
    if (hx_single_pass(nup, ndn)) {
        // 1024 threads from 32 M states, else 512 (two CTAs per SM)
        if (S.dim >= (32LL << 20)) launch_hx_gather<1024>(S, x, y, accumulate, s);
        else launch_hx_gather<512>(S, x, y, accumulate, s);
        return;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // long lines (1500 strings or more) take 1024-thread CTAs, so the SM has
    // 32 or more warps to overlap the hop lists' and neighbours' latency
    // (measured: 17% faster at nsite 13, 6% at 14)
    const int wc = (ndn > kHxLongLine) ? (hx_cols_of(nup, ndn, nsm) == 4 ? 4 : 2) : hx_cols_of(nup, ndn, nsm);
    if (ndn > kHxLongLine) {
        if (wc == 4) launch_hx_col<4, kHxThreadsLong>(S, x, scratch, s);
        else launch_hx_col<2, kHxThreadsLong>(S, x, scratch, s);
    } else {
        switch (wc) {
        case 16: launch_hx_col<16, kHxThreads>(S, x, scratch, s); break;
        case 8: launch_hx_col<8, kHxThreads>(S, x, scratch, s); break;
        case 4: launch_hx_col<4, kHxThreads>(S, x, scratch, s); break;
        default: launch_hx_col<2, kHxThreads>(S, x, scratch, s); break;
        }
    }
    if (nup > kHxLongLine) {
        const int r = hx_rows_of(nup, ndn, nsm);
        if (r >= 4) launch_hx_row<4, kHxThreadsLong>(S, x, scratch, wc, y, accumulate, s);
        else if (r == 2) launch_hx_row<2, kHxThreadsLong>(S, x, scratch, wc, y, accumulate, s);
        else launch_hx_row<1, kHxThreadsLong>(S, x, scratch, wc, y, accumulate, s);
    } else {
        switch (hx_rows_of(nup, ndn, nsm)) {
        case 8: launch_hx_row<8, kHxThreads>(S, x, scratch, wc, y, accumulate, s); break;
        case 4: launch_hx_row<4, kHxThreads>(S, x, scratch, wc, y, accumulate, s); break;
        case 2: launch_hx_row<2, kHxThreads>(S, x, scratch, wc, y, accumulate, s); break;
        default: launch_hx_row<1, kHxThreads>(S, x, scratch, wc, y, accumulate, s); break;
        }
    }
}

// ---------------------------------------------------------------------------
// Ground-state vector from kept Lanczos pairs (the eigenvector pass's sum,
// src/lanczos_solver.f90:213-300, without rerunning the recurrence).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_keep_combine(const double2* __restrict__ keep, long long dim, int nstep,
                                                      const double* __restrict__ coeff, double* __restrict__ out)
{
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < dim; e += (long long)gridDim.x * blockDim.x) {
        const double* w = reinterpret_cast<const double*>(keep + dim + e) + 1;   // w_1
        double acc = __ldg(coeff) * __ldcs(w);
#pragma unroll 8
        for (int k = 2; k <= nstep; k++) acc = fma(__ldg(coeff + k - 1), __ldcs(w + 2 * (k - 1) * dim), acc);
        out[e] = acc;
    }
}

void launch_keep_combine(const double2* keep, long long dim, int nstep, const double* coeff, double* out,
                         cudaStream_t s)
{
    if (dim <= 0 || nstep <= 0) return;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = std::min<long long>((dim + 255) / 256, 8LL * nsm);
    k_keep_combine<<<(unsigned)blocks, 256, 0, s>>>(keep, dim, nstep, coeff, out);
}

// ---------------------------------------------------------------------------
// Deterministic dot product (mpi_dot_product, src/numeric_utils.f90:159-170):
// fixed grid of partial sums, then one block sums the partials in order.
// ---------------------------------------------------------------------------
static constexpr int kDotBlocks = 592;
static constexpr int kDotThreads = 256;

int dot_partials_size() { return kDotBlocks; }

__global__ void __launch_bounds__(kDotThreads) k_dot_partial(const double* __restrict__ a,
                                                             const double* __restrict__ b, long long n,
                                                             double* __restrict__ partials)
{
    __shared__ double scratch[32];
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v[0] = fma(a[i], b[i], v[0]);
    block_sum<1>(v, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(kDotThreads) k_dot_final(const double* __restrict__ partials, int np,
                                                           double* __restrict__ out)
{
    __shared__ double scratch[32];
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < np; i += blockDim.x) v[0] += partials[i];
    block_sum<1>(v, scratch);
    if (threadIdx.x == 0) *out = v[0];
}

void launch_dot(const double* a, const double* b, long long n, double* partials, double* out, cudaStream_t s)
{
    k_dot_partial<<<kDotBlocks, kDotThreads, 0, s>>>(a, b, n, partials);
    k_dot_final<<<1, kDotThreads, 0, s>>>(partials, kDotBlocks, out);
}

// w = v / b_k ; v = -b_k * w_old  (src/lanczos_solver.f90:152-156); *bk holds b_k.
__global__ void k_swap_scale(double* __restrict__ w, double* __restrict__ v, long long n,
                             const double* __restrict__ bk_p, double bk)
{
    const double b = bk_p ? *bk_p : bk;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double t = w[i];
        w[i] = v[i] / b;
        v[i] = -b * t;
    }
}

void launch_swap_scale(double* w, double* v, long long n, const double* bk_p, double bk, cudaStream_t s)
{
    k_swap_scale<<<592, 256, 0, s>>>(w, v, n, bk_p, bk);
}

// y = y + (sign * alpha) * x  (daxpy with a device scalar)
__global__ void k_axpy(double* __restrict__ y, const double* __restrict__ x, long long n,
                       const double* __restrict__ alpha_p, double alpha, double sign)
{
    const double al = sign * (alpha_p ? *alpha_p : alpha);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = fma(al, x[i], y[i]);
}

void launch_axpy(double* y, const double* x, long long n, const double* alpha_p, double alpha, double sign,
                 cudaStream_t s)
{
    k_axpy<<<592, 256, 0, s>>>(y, x, n, alpha_p, alpha, sign);
}

// x = x / sqrt(*nrm2)
__global__ void k_scale_inv_sqrt(double* __restrict__ x, long long n, const double* __restrict__ nrm2)
{
    const double nrm = sqrt(*nrm2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = x[i] / nrm;
}

void launch_scale_inv_sqrt(double* x, long long n, const double* nrm2, cudaStream_t s)
{
    k_scale_inv_sqrt<<<592, 256, 0, s>>>(x, n, nrm2);
}

__global__ void k_fill_start(double* __restrict__ v, long long n, uint64_t key)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v[i] = edzt_u01(key, (uint64_t)i);
}

void launch_fill_start(double* v, long long n, uint64_t key, cudaStream_t s)
{
    k_fill_start<<<592, 256, 0, s>>>(v, n, key);
}

void launch_copy(double* dst, const double* src, long long n, cudaStream_t s)
{
    cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s);
}

// ---------------------------------------------------------------------------
// apply_c (src/ed_operator.f90:13-57), row-wise over the output sector.
// ---------------------------------------------------------------------------
__global__ void k_apply_c(ApplyCArgs A, const double* __restrict__ in, double* __restrict__ out)
{
    const long long n = (long long)A.out_nup * A.out_ndn;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = apply_c_value(A, in, i);
}

void launch_apply_c(const ApplyCArgs& A, const double* in, double* out, cudaStream_t s)
{
    const long long n = (long long)A.out_nup * A.out_ndn;
    if (n <= 0) return;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_apply_c<<<(int)blocks, 256, 0, s>>>(A, in, out);
}

// ---------------------------------------------------------------------------
// Continued fractions (src/numeric_utils.f90:11-44): one thread per (run, w).
//   f = b_n^2/(z -/+ a_n);  f = b_i^2/(z -/+ a_i - f), i = n-1..1
// Complex division by Smith's method.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cdiv_real(double num, double br, double bi, double* cr, double* ci)
{
    if (fabs(br) >= fabs(bi)) {
        const double r = bi / br, den = br + bi * r;
        *cr = num / den;
        *ci = (-num * r) / den;
    } else {
        const double r = br / bi, den = bi + br * r;
        *cr = (num * r) / den;
        *ci = (-num) / den;
    }
}

__global__ void k_cf(const CFJob* __restrict__ jobs, int njobs, const double* __restrict__ omega, int nw,
                     int real_axis, double eta)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= njobs * nw) return;
    const int jb = t / nw, iw = t - jb * nw;
    const CFJob J = jobs[jb];
    const int n = J.levels;
    if (n < 1) return;
    // z = (+-E0) + i w_n on the Matsubara axis, (+-E0) + w + i eta on the real axis
    const double zr = J.zr_shift + (real_axis ? omega[iw] : 0.0), zi = real_axis ? eta : omega[iw];
    auto bk = [&](int i) { return i == 0 ? J.b1 : J.b[i]; };   // b(1) = ||c^(+)|gs>|
    // the reference's recursion literally (numeric_utils.f90:18-22 / :39-43),
    // including its final level with b(1) when n == 1
    double xr, xi;
    cdiv_real(bk(n - 1) * bk(n - 1), zr + J.sign * J.a[n - 1], zi, &xr, &xi);
    for (int i = n - 1; i >= 2; i--)
        cdiv_real(bk(i - 1) * bk(i - 1), zr + J.sign * J.a[i - 1] - xr, zi - xi, &xr, &xi);
    cdiv_real(J.b1 * J.b1, zr + J.sign * J.a[0] - xr, zi - xi, &xr, &xi);
    J.g[2 * iw] = xr;
    J.g[2 * iw + 1] = xi;
}

void launch_cf(const CFJob* jobs_dev, int njobs, const double* omega, int nw, cudaStream_t s, int real_axis,
               double eta)
{
    const int n = njobs * nw;
    if (n <= 0) return;
    k_cf<<<(n + 127) / 128, 128, 0, s>>>(jobs_dev, njobs, omega, nw, real_axis, eta);
}

// ---------------------------------------------------------------------------
// Occupancies of the ground state (post_process.f90:62-112):
// occ(iorb, ispin) = sum |x_i|^2 over states with orbital iorb of spin ispin
// filled, docc(iorb) = sum |x_i|^2 over states with both spins filled.
// Fixed grid of per-block partial sums, summed in block order by the host.
// ---------------------------------------------------------------------------
static constexpr int kOccBlocks = 592;

__global__ void __launch_bounds__(256) k_gs_occ(const double* __restrict__ x, const uint32_t* __restrict__ up,
                                                const uint32_t* __restrict__ dn, int nup, long long dim, int norb,
                                                double* __restrict__ part)
{
    __shared__ double scratch[12 * 32];
    double acc[12];
#pragma unroll
    for (int q = 0; q < 12; q++) acc[q] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += (long long)gridDim.x * blockDim.x) {
        const long long id = i / nup;
        const int iu = (int)(i - id * nup);
        const double w = x[i] * x[i];
        const uint32_t u = __ldg(up + iu), d = __ldg(dn + id);
#pragma unroll
        for (int a = 0; a < EDZT_MAX_NORB; a++) {
            if (a < norb) {
                const bool bu = (u >> a) & 1u, bd = (d >> a) & 1u;
                acc[a] += bu ? w : 0.0;
                acc[4 + a] += bd ? w : 0.0;
                acc[8 + a] += (bu && bd) ? w : 0.0;
            }
        }
    }
    block_sum<12>(acc, scratch);
    if (threadIdx.x == 0)
        for (int q = 0; q < 12; q++) part[(size_t)blockIdx.x * 12 + q] = acc[q];
}

int occ_partials_size() { return kOccBlocks * 12; }

void launch_gs_occ(const double* x, const uint32_t* up, const uint32_t* dn, int nup, long long dim, int norb,
                   double* part, cudaStream_t s)
{
    k_gs_occ<<<kOccBlocks, 256, 0, s>>>(x, up, dn, nup, dim, norb, part);
}
