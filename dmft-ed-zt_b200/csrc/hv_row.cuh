// hv_row.cuh — one element of the matrix-free Fock-space H.v (kernel (b)).
//
// Restates the row sum of src/impurity_hamiltonian.f90:98-246 with the work
// split by what it touches:
//   diagonal      (e1_up[iu] + e1_dn[id] + wint[imp_up, imp_dn]) * x(id, iu)
//   up hops       sum_h c * x(id, iu')    -- same row: read from shared memory
//   down hops     sum_h c * x(id', iu)    -- same column: a warp over
//                                            consecutive iu reads a contiguous,
//                                            coalesced slice of row id'
//   spin-flip / pair-hop (norb > 1)        sum c * x(id', iu')
// The terms are the reference's; only the floating-point summation order
// differs (diagonal first, then up hops, down hops, exchange terms).  Hops
// are processed four at a time so that their loads are in flight together.
#pragma once
#include "edzt_device.cuh"

// xrow: shared-memory copy of row id (nup values).  dn/hd: shared-memory copy
// of row id's down-hop words.  cu/cd: shared-memory amplitude tables of the
// up and down spin.  fetch(idx) returns the vector value at global index
// idx = id'*nup + iu' for rows that are not in shared memory.
template <class Fetch>
__device__ __forceinline__ double hv_element(const DevSector& S, int iu, int id, const double* __restrict__ xrow,
                                             double xe, const uint32_t* __restrict__ dn, int hd,
                                             const double* __restrict__ cu, const double* __restrict__ cd,
                                             Fetch fetch)
{
    const int nup = S.up.count;
    const int P = S.P;
    const int pu = __ldg(S.up.imp + iu), pd = __ldg(S.dn.imp + id);
    double acc = (__ldg(S.up.e1 + iu) + __ldg(S.dn.e1 + id) + __ldg(S.wint + pu * P + pd)) * xe;
    // up-spin hybridisation hops: targets in the same row
    const int hu = __ldg(S.up.hcnt + iu);
    const uint32_t* __restrict__ hp = S.up.hop + iu;
    int h = 0;
    for (; h + 4 <= hu; h += 4) {
        const uint32_t p0 = __ldg(hp + (size_t)(h + 0) * nup);
        const uint32_t p1 = __ldg(hp + (size_t)(h + 1) * nup);
        const uint32_t p2 = __ldg(hp + (size_t)(h + 2) * nup);
        const uint32_t p3 = __ldg(hp + (size_t)(h + 3) * nup);
        EDZT_OK_OR((p0 & HOP_RANK_MASK) < (uint32_t)nup && (p1 & HOP_RANK_MASK) < (uint32_t)nup &&
                   (p2 & HOP_RANK_MASK) < (uint32_t)nup && (p3 & HOP_RANK_MASK) < (uint32_t)nup,
                   11, iu, id, p0, continue)
        acc = fma(hop_coef(p0, cu), xrow[p0 & HOP_RANK_MASK], acc);
        acc = fma(hop_coef(p1, cu), xrow[p1 & HOP_RANK_MASK], acc);
        acc = fma(hop_coef(p2, cu), xrow[p2 & HOP_RANK_MASK], acc);
        acc = fma(hop_coef(p3, cu), xrow[p3 & HOP_RANK_MASK], acc);
    }
    for (; h < hu; h++) {
        const uint32_t p0 = __ldg(hp + (size_t)h * nup);
        EDZT_OK_OR((p0 & HOP_RANK_MASK) < (uint32_t)nup, 12, iu, id, p0, continue)
        acc = fma(hop_coef(p0, cu), xrow[p0 & HOP_RANK_MASK], acc);
    }
    // down-spin hybridisation hops: same column of other rows (warp-uniform lists)
    EDZT_OK_OR(hd >= 0 && hd <= S.dn.hw, 13, iu, id, hd, hd = 0)
    h = 0;
    for (; h + 4 <= hd; h += 4) {
        const uint32_t p0 = dn[h], p1 = dn[h + 1], p2 = dn[h + 2], p3 = dn[h + 3];
        EDZT_OK_OR((p0 & HOP_RANK_MASK) < (uint32_t)S.dn.count && (p3 & HOP_RANK_MASK) < (uint32_t)S.dn.count &&
                   ((p0 >> HOP_CIDX_SHIFT) & HOP_CIDX_MASK) < (uint32_t)S.dn.ncoef, 14, iu, id, p0, continue)
        const double v0 = fetch((long long)(p0 & HOP_RANK_MASK) * nup + iu);
        const double v1 = fetch((long long)(p1 & HOP_RANK_MASK) * nup + iu);
        const double v2 = fetch((long long)(p2 & HOP_RANK_MASK) * nup + iu);
        const double v3 = fetch((long long)(p3 & HOP_RANK_MASK) * nup + iu);
        acc = fma(hop_coef(p0, cd), v0, acc);
        acc = fma(hop_coef(p1, cd), v1, acc);
        acc = fma(hop_coef(p2, cd), v2, acc);
        acc = fma(hop_coef(p3, cd), v3, acc);
    }
    for (; h < hd; h++) {
        const uint32_t p0 = dn[h];
        acc = fma(hop_coef(p0, cd), fetch((long long)(p0 & HOP_RANK_MASK) * nup + iu), acc);
    }
    // spin-flip and pair-hopping (impurity_hamiltonian.f90:179-226)
    if (S.has_j) {
        const int pp = pu * P + pd;
        const int nj = __ldg(S.jcnt + pp);
        for (int q = 0; q < nj; q++) {
            const JTrans tr = S.jt[pp * EDZT_MAX_JT + q];
            const int iu2 = __ldg(S.up.sub + (size_t)iu * P + tr.pu2);
            const int id2 = __ldg(S.dn.sub + (size_t)id * P + tr.pd2);
            EDZT_OK_OR(iu2 >= 0 && iu2 < nup && id2 >= 0 && id2 < S.dn.count, 15, iu2, id2, pp, continue)
            acc = fma(tr.c, fetch((long long)id2 * nup + iu2), acc);
        }
    }
    return acc;
}

// Stage the down-hop words of rows [r0, r0+nr) into shared memory:
// words[r*hw + h], counts[r].
__device__ __forceinline__ void stage_down_hops(const DevSpin& dn, int r0, int nr, uint32_t* words, int* counts)
{
    const int hw = dn.hw, ndn = dn.count;
    for (int i = threadIdx.x; i < nr * hw; i += blockDim.x) {
        const int r = i / hw, h = i - r * hw;
        EDZT_OK_OR(r0 + r < ndn && r0 >= 0, 31, r0, r, ndn, continue)
        words[i] = __ldg(dn.hop + (size_t)h * ndn + r0 + r);
    }
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        EDZT_OK_OR(r0 + r < ndn, 32, r0, r, ndn, continue)
        counts[r] = __ldg(dn.hcnt + r0 + r);
    }
}

__device__ __forceinline__ void stage_coefs(const DevSector& S, double* cu, double* cd)
{
    for (int i = threadIdx.x; i < S.up.ncoef; i += blockDim.x) cu[i] = __ldg(S.up.coef + i);
    for (int i = threadIdx.x; i < S.dn.ncoef; i += blockDim.x) cd[i] = __ldg(S.dn.coef + i);
}

// Bytes of shared memory one staged row needs (values + down-hop words + count).
__host__ __device__ __forceinline__ size_t staged_row_bytes(int nup, int hw_dn)
{
    return (size_t)nup * sizeof(double) + (size_t)hw_dn * sizeof(uint32_t) + sizeof(int);
}
