// hv_row.cuh — one row of the matrix-free Fock-space H.v (kernel (b)).
//
// Restates the row sum of src/impurity_hamiltonian.f90:98-246 with the
// per-row work split by what it touches:
//   diagonal      (e1_up[iu] + e1_dn[id] + wint[imp_up, imp_dn]) * x(id, iu)
//   up hops       sum_h c * x(id, iu')    -- same row: read from shared memory
//   down hops     sum_h c * x(id', iu)    -- same column: a warp over
//                                            consecutive iu reads a contiguous,
//                                            coalesced slice of row id'
//   spin-flip / pair-hop (norb > 1)        sum c * x(id', iu')
// The terms are the reference's; only the floating-point summation order
// differs (diagonal first, then up hops, down hops, exchange terms).
#pragma once
#include "edzt_device.cuh"

// xrow: shared-memory copy of row id (nup values).  gather(idx) returns the
// vector value at global index idx = id'*nup + iu'.
template <class Gather>
__device__ __forceinline__ double hv_row_element(const DevSector& S, int iu, int id, const double* xrow,
                                                 double xe, Gather gather)
{
    const int nup = S.up.count, ndn = S.dn.count;
    const int P = S.P;
    const int pu = __ldg(S.up.imp + iu), pd = __ldg(S.dn.imp + id);
    double acc = (__ldg(S.up.e1 + iu) + __ldg(S.dn.e1 + id) + __ldg(S.wint + pu * P + pd)) * xe;
    // up-spin hybridisation hops: targets in the same row
    const int hu = __ldg(S.up.hcnt + iu);
    for (int h = 0; h < hu; h++) {
        const int j = __ldg(S.up.hidx + (size_t)h * nup + iu);
        const double c = __ldg(S.up.hval + (size_t)h * nup + iu);
        acc = fma(c, xrow[j], acc);
    }
    // down-spin hybridisation hops: targets in the same column (warp-uniform lists)
    const int hd = __ldg(S.dn.hcnt + id);
    for (int h = 0; h < hd; h++) {
        const int j = __ldg(S.dn.hidx + (size_t)h * ndn + id);
        const double c = __ldg(S.dn.hval + (size_t)h * ndn + id);
        acc = fma(c, gather((long long)j * nup + iu), acc);
    }
    // spin-flip and pair-hopping (impurity_hamiltonian.f90:179-226)
    if (S.has_j) {
        const int pp = pu * P + pd;
        const int nj = __ldg(S.jcnt + pp);
        for (int q = 0; q < nj; q++) {
            const JTrans tr = S.jt[pp * EDZT_MAX_JT + q];
            const int iu2 = __ldg(S.up.sub + (size_t)iu * P + tr.pu2);
            const int id2 = __ldg(S.dn.sub + (size_t)id * P + tr.pd2);
            acc = fma(tr.c, gather((long long)id2 * nup + iu2), acc);
        }
    }
    return acc;
}
