// arpack.cu — vector kernels of the restarted Lanczos eigensolver that takes
// the place of ARPACK's pdsaupd/pdseupd in diag_arpack
// (src/arpack_solver.f90:19-124).
//
// The solver keeps at most EDZT_RL_MAXV basis vectors of one sector on the
// device.  Each Lanczos step orthogonalises H v_j against all of them
// (classical Gram-Schmidt, two passes), and a restart replaces the basis by
// the kept Ritz vectors.  These are streaming kernels over the sector
// vector: every basis vector is read once per pass, in the same
// grid-stride order, with the block partial sums of the dot products
// reduced in a fixed order so that results do not depend on timing.
#include <cuda_runtime.h>
#include "edzt_internal.h"

static constexpr int kRlBlocks = 592;      // 4 x 148 SMs
static constexpr int kRlThreads = 256;

int rl_partials_size() { return kRlBlocks * EDZT_RL_MAXV; }

// partials[block][q] = sum over the block's indices of V_q[i] * w[i], q < nv.
__global__ void __launch_bounds__(kRlThreads) k_rl_mdot(RlVecs V, int nv, const double* __restrict__ w,
                                                        long long n, double* __restrict__ partials)
{
    __shared__ double red[kRlThreads / 32][EDZT_RL_MAXV];
    double acc[EDZT_RL_MAXV];
#pragma unroll
    for (int q = 0; q < EDZT_RL_MAXV; q++) acc[q] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int q = 0; q < EDZT_RL_MAXV; q++)
            if (q < nv) acc[q] = fma(V.p[q][i], wi, acc[q]);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < EDZT_RL_MAXV; q++) {
        double s = acc[q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double s = 0.0;
        for (int k = 0; k < kRlThreads / 32; k++) s += red[k][threadIdx.x];
        partials[(size_t)blockIdx.x * EDZT_RL_MAXV + threadIdx.x] = s;
    }
}

// out[q] = sum over blocks of partials[block][q], in a fixed order.
__global__ void __launch_bounds__(kRlThreads) k_rl_mdot_final(const double* __restrict__ partials, int nblocks,
                                                              int nv, double* __restrict__ out)
{
    __shared__ double red[kRlThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nv; q++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * EDZT_RL_MAXV + q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < kRlThreads / 32; k++) t += red[k];
            out[q] = t;
        }
        __syncthreads();
    }
}

void launch_rl_mdot(const RlVecs& V, int nv, const double* w, long long n, double* partials, double* out,
                    cudaStream_t s)
{
    k_rl_mdot<<<kRlBlocks, kRlThreads, 0, s>>>(V, nv, w, n, partials);
    k_rl_mdot_final<<<1, kRlThreads, 0, s>>>(partials, kRlBlocks, nv, out);
}

// w = w - sum_q h[q] V_q  (h on the device: the projections just computed).
__global__ void __launch_bounds__(kRlThreads) k_rl_project_out(double* __restrict__ w, RlVecs V, int nv,
                                                               const double* __restrict__ h, long long n)
{
    double hq[EDZT_RL_MAXV];
#pragma unroll
    for (int q = 0; q < EDZT_RL_MAXV; q++) hq[q] = q < nv ? h[q] : 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double t = w[i];
#pragma unroll
        for (int q = 0; q < EDZT_RL_MAXV; q++)
            if (q < nv) t = fma(-hq[q], V.p[q][i], t);
        w[i] = t;
    }
}

void launch_rl_project_out(double* w, const RlVecs& V, int nv, const double* h, long long n, cudaStream_t s)
{
    k_rl_project_out<<<kRlBlocks, kRlThreads, 0, s>>>(w, V, nv, h, n);
}

// out_i = sum_{j < m} Y[j * k + i] V_j for i < k: the Ritz vectors of the
// projected problem (Y its eigenvectors, row j, column i), every V_j read once.
__global__ void __launch_bounds__(kRlThreads) k_rl_combine(RlOut O, int k, RlVecs V, int m,
                                                           const double* __restrict__ Y, long long n)
{
    __shared__ double ys[EDZT_RL_MAXV * EDZT_RL_MAXV];
    for (int t = threadIdx.x; t < m * k; t += blockDim.x) ys[t] = Y[t];
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double v[EDZT_RL_MAXV];
#pragma unroll
        for (int j = 0; j < EDZT_RL_MAXV; j++) v[j] = j < m ? V.p[j][i] : 0.0;
#pragma unroll
        for (int c = 0; c < EDZT_RL_MAXV; c++) {
            if (c < k) {
                double t = 0.0;
#pragma unroll
                for (int j = 0; j < EDZT_RL_MAXV; j++)
                    if (j < m) t = fma(ys[j * k + c], v[j], t);
                O.p[c][i] = t;
            }
        }
    }
}

void launch_rl_combine(const RlOut& O, int k, const RlVecs& V, int m, const double* Y, long long n, cudaStream_t s)
{
    k_rl_combine<<<kRlBlocks, kRlThreads, 0, s>>>(O, k, V, m, Y, n);
}

// out = w / beta
__global__ void __launch_bounds__(kRlThreads) k_rl_div(double* __restrict__ out, const double* __restrict__ w,
                                                       double beta, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = w[i] / beta;
}

void launch_rl_div(double* out, const double* w, double beta, long long n, cudaStream_t s)
{
    k_rl_div<<<kRlBlocks, kRlThreads, 0, s>>>(out, w, beta, n);
}
