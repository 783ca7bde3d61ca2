// edzt_device.cuh — device-side data structures and helpers shared by the
// sm_100a kernels of the ED hot path.
//
// Layout of a sector vector in HBM (same convention as the reference,
// src/ed_basis.f90:132-135): element (iup, idn) lives at idn*nup + iup, so
// the up-string rank is the fast index and a sector vector is a row-major
// matrix X[ndn][nup].  All arithmetic is FP64; all indices and signs are
// exact integers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define EDZT_MAX_NSITE 20
#define EDZT_MAX_NORB 4
#define EDZT_MAX_P (1 << EDZT_MAX_NORB)
#define EDZT_MAX_JT 12  // norb*(norb-1) spin-flip/pair-hop transitions per pattern pair

// One spin species of one sector: strings with a fixed electron count and
// the per-string tables derived from the impurity model.
struct DevSpin {
    int count;              // C(nsite, n)
    int hw;                 // packed hop slots per string: a multiple of 4, >= every string's hop count
    int namp;               // amplitude slots: 2 * norb * nbath
    const uint32_t* str;    // [count] ascending bit strings (ed_basis.f90:94-112)
    const int32_t* rank;    // [2^nsite] rank of a string, -1 if popcount != n
    const double* e1;       // [count] one-body energy: sum (em-mu) n_imp + sum ek n_bath
    const uint8_t* hcnt;    // [count] number of allowed impurity<->bath hops
    const uint4* hpk;       // [hw/4][count] hops of a string, four per uint4: target rank | slot << 20
    const double* amp;      // [namp] amplitude of a slot: +V at 2c, -V at 2c+1, c = iorb*nbath + jbath
    const uint8_t* imp;     // [count] impurity bits (sites 1..norb)
    const int32_t* sub;     // [count][P] rank after replacing the impurity bits (norb > 1)
};

// Packed hop entry: target rank in the low 20 bits (C(20,10) < 2^20), the
// amplitude slot (sign folded in) above.
#define EDZT_HOP_RANK_BITS 20
#define EDZT_MAX_AMP (2 * EDZT_MAX_NORB * EDZT_MAX_NSITE)
__host__ __device__ __forceinline__ uint32_t edzt_hop_pack(int rank, int slot)
{
    return (uint32_t)rank | ((uint32_t)slot << EDZT_HOP_RANK_BITS);
}
__device__ __forceinline__ int edzt_hop_rank(uint32_t e) { return (int)(e & ((1u << EDZT_HOP_RANK_BITS) - 1u)); }
__device__ __forceinline__ int edzt_hop_slot(uint32_t e) { return (int)(e >> EDZT_HOP_RANK_BITS); }

// Spin-flip / pair-hop transition between impurity patterns (pu, pd) -> (pu2, pd2).
struct JTrans {
    int pu2, pd2;
    double c;
};

struct DevSector {
    DevSpin up, dn;
    long long dim;          // nup * ndn
    int P;                  // 2^norb
    int has_j;              // any spin-flip / pair-hop terms
    const double* wint;     // [P*P] density-density interaction energy by impurity patterns
    const int* jcnt;        // [P*P]
    const JTrans* jt;       // [P*P][EDZT_MAX_JT]
};

// ---------------------------------------------------------------------------
// Counter-based start vector: splitmix64 (Steele, Lea, Flood, OOPSLA 2014)
// used as a hash of (seed, stream, index) -> U[0,1).  Replaces the unseeded
// random_number of src/lanczos_solver.f90:42-46 with a reproducible stream.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t edzt_mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t edzt_stream_key(uint64_t seed, uint64_t stream)
{
    return edzt_mix64(seed ^ edzt_mix64(stream));
}
__host__ __device__ __forceinline__ double edzt_u01(uint64_t key, uint64_t i)
{
    return (double)(edzt_mix64(key + i) >> 11) * 0x1.0p-53;
}

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values; result valid in every thread.  scratch needs
// NV*32 doubles of shared memory.  Fixed order: deterministic.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) scratch[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double t = (lane < nw) ? scratch[q * 32 + lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) scratch[q * 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = scratch[q * 32];
    __syncthreads();
}

// ---------------------------------------------------------------------------
// memory-model helpers for the persistent kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Optional device-side bounds checks (compiled in with -DEDZT_DEVICE_CHECKS):
// the first failed check records (code, a, b, c) and the access is skipped.
#ifdef EDZT_DEVICE_CHECKS
static __device__ long long g_edzt_bad[4];
static __device__ __noinline__ void edzt_record_bad(long long code, long long a, long long b, long long c)
{
    if (atomicCAS(reinterpret_cast<unsigned long long*>(&g_edzt_bad[0]), 0ull, (unsigned long long)code) == 0ull) {
        g_edzt_bad[1] = a;
        g_edzt_bad[2] = b;
        g_edzt_bad[3] = c;
    }
}
#define EDZT_OK_OR(cond, code, a, b, c, skip) \
    if (!(cond)) { edzt_record_bad((code), (long long)(a), (long long)(b), (long long)(c)); skip; }
#else
#define EDZT_OK_OR(cond, code, a, b, c, skip)
#endif

// apply_c (src/ed_operator.f90:13-57) from sector `in` to sector `out`.
struct ApplyCArgs {
    int pm, iorb, ispin;       // 1-based iorb/ispin as in the reference; pm 1 = c^+, 2 = c
    int nsite;
    int out_nup, out_ndn;
    const uint32_t* out_up_str;
    const uint32_t* out_dn_str;
    int in_nup;
    const int32_t* in_up_rank;
    const int32_t* in_dn_rank;
};

// Element i of apply_c's output, row-wise over the output sector
// (ed_operator.f90:31-54).  The bit of the full state is
// q = (ispin-1)*nsite + iorb - 1 and the sign is (-1)^{popcount of the output
// state's bits 0..q-1} (ed_operator.f90:34,59-76); for a down-spin operator
// that count includes every up electron.
__device__ __forceinline__ double apply_c_value(const ApplyCArgs& A, const double* __restrict__ in,
                                                long long i)
{
    const int iu = (int)(i % A.out_nup), id = (int)(i / A.out_nup);
    const uint32_t u = __ldg(A.out_up_str + iu), d = __ldg(A.out_dn_str + id);
    const uint32_t bit = 1u << (A.iorb - 1);
    int par;
    long long j;
    if (A.ispin == 1) {
        if ((A.pm == 1) != ((u & bit) != 0u)) return 0.0;
        par = __popc(u & (bit - 1u));
        j = (long long)id * A.in_nup + __ldg(A.in_up_rank + (u ^ bit));   // down rank unchanged
        EDZT_OK_OR(__ldg(A.in_up_rank + (u ^ bit)) >= 0, 41, i, u, bit, return 0.0)
    } else {
        if ((A.pm == 1) != ((d & bit) != 0u)) return 0.0;
        par = __popc(u) + __popc(d & (bit - 1u));
        j = (long long)__ldg(A.in_dn_rank + (d ^ bit)) * A.in_nup + iu;   // up rank unchanged
        EDZT_OK_OR(__ldg(A.in_dn_rank + (d ^ bit)) >= 0, 42, i, d, bit, return 0.0)
    }
    const double v = __ldg(in + j);
    return (par & 1) ? -v : v;
}

// Error codes written by kernels into a device status word.
#define EDZT_DEV_OK 0
#define EDZT_DEV_BARRIER_TIMEOUT 1
#define EDZT_DEV_BAD_INDEX 2
