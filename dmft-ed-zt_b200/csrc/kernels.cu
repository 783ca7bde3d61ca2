// kernels.cu — standalone (one launch per operation) sm_100a kernels:
// H.v, the BLAS-1 steps of the plain Lanczos drop-in, apply_c and the
// continued fractions.  The fused persistent Lanczos lives in lanczos.cu.
#include <cuda_runtime.h>
#include "edzt_internal.h"
#include "hv_row.cuh"

static constexpr size_t kHxSmemTarget = 24 * 1024;
static constexpr int kWintDoubles = EDZT_MAX_P * EDZT_MAX_P;
static constexpr int kAmpDoubles = EDZT_MAX_AMP;

#ifdef EDZT_DEVICE_CHECKS
int kernels_debug_bad(long long* out4)
{
    return cudaMemcpyFromSymbol(out4, g_edzt_bad, 4 * sizeof(long long)) == cudaSuccess ? 0 : 2;
}
#endif

int hx_rows_per_tile(int nup, int ndn, int hw_dn)
{
    const size_t row = staged_row_bytes(nup, hw_dn);
    int r = (int)(kHxSmemTarget / row);
    if (r < 1) r = 1;
    if (r > ndn) r = ndn;
    return r;
}

// ---------------------------------------------------------------------------
// H.v: y = H x (accumulate = 0) or y = y + H x (accumulate = 1), the `py`
// flag of src/impurity_hamiltonian.f90:241-245.  One CTA per block of R full
// rows; the rows and their per-row hop data are staged in shared memory.
// T threads per CTA: 256, or for large sectors 512 (two CTAs per SM) and
// 1024 (one), both at 64 registers, 32 warps per SM.
// ---------------------------------------------------------------------------
template <bool ACC, int T>
__global__ void __launch_bounds__(T, T == 512 ? 2 : 1) k_hx(DevSector S, const double* __restrict__ x,
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
    stage_wint(S, wint);
    stage_amp(S.up, amp);
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

// Threads per CTA of k_hx by sector dimension.  Measured on B200 (y = H x on
// the half-filled sector of a single-orbital impurity): at nsite 16 (1.66e8
// states) 4.45 / 3.10 / 2.85 ms with 256 / 512 / 1024 threads, at nsite 14
// (1.18e7) 0.228 / 0.212 / 0.254 ms, at nsite 12 (8.5e5) 0.039 / 0.040 /
// 0.042 ms.  Large sectors wait on the latency of their down-hop gathers,
// which more warps per SM hide; small ones have too few row tiles to fill
// 148 SMs with large CTAs.
int hx_threads(long long dim)
{
    return dim >= (32LL << 20) ? 1024 : dim >= (4LL << 20) ? 512 : 256;
}

template <int T>
static void launch_hx_t(const DevSector& S, const double* x, double* y, int accumulate, int tiles, int R,
                        size_t smem, cudaStream_t s)
{
    static std::atomic<unsigned long long> attr_set{0};
    if (edzt_once_per_device(attr_set)) {
        cudaFuncSetAttribute(k_hx<false, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_hx<true, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    }
    if (accumulate) k_hx<true, T><<<tiles, T, smem, s>>>(S, x, y, R);
    else k_hx<false, T><<<tiles, T, smem, s>>>(S, x, y, R);
}

void launch_hx(const DevSector& S, const double* x, double* y, int accumulate, cudaStream_t s)
{
    const int nup = S.up.count, ndn = S.dn.count;
    if (nup <= 0 || ndn <= 0) return;
    const int R = hx_rows_per_tile(nup, ndn, S.dn.hw);
    const int tiles = (ndn + R - 1) / R;
    const size_t smem = (kWintDoubles + kAmpDoubles) * sizeof(double) + (size_t)R * staged_row_bytes(nup, S.dn.hw);
    switch (hx_threads(S.dim)) {
    case 1024: launch_hx_t<1024>(S, x, y, accumulate, tiles, R, smem, s); break;
    case 512: launch_hx_t<512>(S, x, y, accumulate, tiles, R, smem, s); break;
    default: launch_hx_t<256>(S, x, y, accumulate, tiles, R, smem, s); break;
    }
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
