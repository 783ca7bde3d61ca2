// hv_row.cuh — the matrix-free Fock-space H.v of kernel (b), by column item.
//
// Restates the row sum of src/impurity_hamiltonian.f90:98-246 with the work
// split by what it touches.  A sector vector is the matrix X[ndn][nup] (up
// rank fast); element (id, iu):
//   diagonal      (e1_up[iu] + e1_dn[id] + wint[imp_up, imp_dn]) * x(id, iu)
//   up hops       sum_h c * x(id, iu')    -- same row, read from shared memory
//   down hops     sum_h c * x(id', iu)    -- same column of other rows: a warp
//                                            over consecutive iu reads a
//                                            contiguous slice of row id'
//   spin-flip / pair-hop (norb > 1)        sum c * x(id', iu')
// Work is handed out as column items: one thread takes column iu of up to
// EDZT_ROW_GROUP staged rows, loads the up-hop list of iu once and applies it
// to every row of the group, then gathers the down hops of each row (lists
// staged in shared memory per row).  The terms are the reference's; only the
// floating-point summation order differs (diagonal, up hops, down hops,
// exchange terms).
#pragma once
#include "edzt_device.cuh"

#define EDZT_ROW_GROUP 4

// Shared-memory view of a chunk of staged rows [r0, r0 + rows).
struct Chunk {
    double* xs;       // [rows][nup]  the vector on the chunk's rows
    int* doff;        // [rows][hw]   down-hop target offsets id'*nup
    double* dval;     // [rows][hw]   down-hop amplitudes (signed)
    int* dcnt;        // [rows]       number of down hops of the row
    double* de1;      // [rows]       e1_dn of the row
    int* dimp;        // [rows]       impurity pattern of the row's down string
    int r0, rows, nup, hw;
};

// Shared-memory bytes of one staged row.
__host__ __device__ __forceinline__ size_t staged_row_bytes(int nup, int hw_dn)
{
    return (size_t)nup * sizeof(double) + (size_t)hw_dn * (sizeof(int) + sizeof(double)) + 2 * sizeof(double);
}

// Carve the chunk arrays for `rmax` rows out of shared memory at `base` (8-byte aligned).
__device__ __forceinline__ Chunk chunk_layout(double* base, int rmax, int nup, int hw)
{
    Chunk C;
    C.xs = base;
    C.dval = base + (size_t)rmax * nup;
    C.de1 = C.dval + (size_t)rmax * hw;
    C.doff = reinterpret_cast<int*>(C.de1 + rmax);
    C.dcnt = C.doff + (size_t)rmax * hw;
    C.dimp = C.dcnt + rmax;
    C.nup = nup;
    C.hw = hw;
    C.r0 = 0;
    C.rows = 0;
    return C;
}

// Stage the per-row data of rows [r0, r0+nr) (everything but xs).
__device__ __forceinline__ void stage_rows(const DevSpin& dn, Chunk& C, int r0, int nr)
{
    const int hw = C.hw, ndn = dn.count;
    C.r0 = r0;
    C.rows = nr;
    for (int i = threadIdx.x; i < nr * hw; i += blockDim.x) {
        const int r = i / hw, h = i - r * hw;
        EDZT_OK_OR(r0 + r < ndn && r0 >= 0, 31, r0, r, ndn, continue)
        C.doff[i] = __ldg(dn.hidx + (size_t)h * ndn + r0 + r) * C.nup;
        C.dval[i] = __ldg(dn.hval + (size_t)h * ndn + r0 + r);
    }
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        EDZT_OK_OR(r0 + r < ndn, 32, r0, r, ndn, continue)
        C.dcnt[r] = __ldg(dn.hcnt + r0 + r);
        C.de1[r] = __ldg(dn.e1 + r0 + r);
        C.dimp[r] = __ldg(dn.imp + r0 + r);
    }
}

// Column iu of chunk rows [ra, rz) (rz - ra <= EDZT_ROW_GROUP).  fetch(idx)
// returns the vector at global index idx (rows outside shared memory); the
// epilogue epi(r, iu, x, hx) receives each element's x(id, iu) and (H x)(id, iu).
template <class Fetch, class Epi>
__device__ __forceinline__ void hv_column(const DevSector& S, const Chunk& C, const double* __restrict__ wint, int iu,
                                          int ra, int rz, Fetch fetch, Epi epi)
{
    const int nup = C.nup;
    const int P = S.P;
    const int pu = __ldg(S.up.imp + iu);
    const double e1u = __ldg(S.up.e1 + iu);
    double acc[EDZT_ROW_GROUP], xe[EDZT_ROW_GROUP];
#pragma unroll
    for (int q = 0; q < EDZT_ROW_GROUP; q++) {
        acc[q] = 0.0;
        xe[q] = 0.0;
        if (ra + q < rz) {
            const int r = ra + q;
            xe[q] = C.xs[(size_t)r * nup + iu];
            acc[q] = (e1u + C.de1[r] + wint[pu * P + C.dimp[r]]) * xe[q];
        }
    }
    // up-spin hops: the list of iu, loaded once, applied to every row of the group
    const int hu = __ldg(S.up.hcnt + iu);
    for (int h = 0; h < hu; h++) {
        const int j = __ldg(S.up.hidx + (size_t)h * nup + iu);
        const double c = __ldg(S.up.hval + (size_t)h * nup + iu);
        EDZT_OK_OR(j >= 0 && j < nup, 11, iu, h, j, continue)
#pragma unroll
        for (int q = 0; q < EDZT_ROW_GROUP; q++)
            if (ra + q < rz) acc[q] = fma(c, C.xs[(size_t)(ra + q) * nup + j], acc[q]);
    }
    // down-spin hops: per row, four gathers in flight at a time
#pragma unroll
    for (int q = 0; q < EDZT_ROW_GROUP; q++) {
        if (ra + q < rz) {
            const int r = ra + q;
            const int hd = C.dcnt[r];
            const int* off = C.doff + (size_t)r * C.hw;
            const double* val = C.dval + (size_t)r * C.hw;
            EDZT_OK_OR(hd >= 0 && hd <= C.hw, 13, iu, r, hd, continue)
            double a = acc[q];
            int h = 0;
            for (; h + 4 <= hd; h += 4) {
                const double v0 = fetch(off[h] + iu), v1 = fetch(off[h + 1] + iu);
                const double v2 = fetch(off[h + 2] + iu), v3 = fetch(off[h + 3] + iu);
                a = fma(val[h], v0, a);
                a = fma(val[h + 1], v1, a);
                a = fma(val[h + 2], v2, a);
                a = fma(val[h + 3], v3, a);
            }
            for (; h < hd; h++) a = fma(val[h], fetch(off[h] + iu), a);
            acc[q] = a;
        }
    }
    // spin-flip and pair-hopping (impurity_hamiltonian.f90:179-226)
    if (S.has_j) {
#pragma unroll
        for (int q = 0; q < EDZT_ROW_GROUP; q++) {
            if (ra + q < rz) {
                const int id = C.r0 + ra + q;
                const int pp = pu * P + C.dimp[ra + q];
                const int nj = __ldg(S.jcnt + pp);
                for (int t = 0; t < nj; t++) {
                    const JTrans tr = S.jt[pp * EDZT_MAX_JT + t];
                    const int iu2 = __ldg(S.up.sub + (size_t)iu * P + tr.pu2);
                    const int id2 = __ldg(S.dn.sub + (size_t)id * P + tr.pd2);
                    EDZT_OK_OR(iu2 >= 0 && iu2 < nup && id2 >= 0 && id2 < S.dn.count, 15, iu2, id2, pp, continue)
                    acc[q] = fma(tr.c, fetch(id2 * nup + iu2), acc[q]);
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < EDZT_ROW_GROUP; q++)
        if (ra + q < rz) epi(ra + q, iu, xe[q], acc[q]);
}

// Items of a chunk: (iu, row group) with iu fastest, so consecutive threads
// take consecutive columns.  Calls body(iu, ra, rz) for this thread's items.
template <class Body>
__device__ __forceinline__ void for_column_items(const Chunk& C, Body body)
{
    const int ngroups = (C.rows + EDZT_ROW_GROUP - 1) / EDZT_ROW_GROUP;
    const int nitems = ngroups * C.nup;
    for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
        const int g = it / C.nup;
        const int iu = it - g * C.nup;
        const int ra = g * EDZT_ROW_GROUP;
        body(iu, ra, min(ra + EDZT_ROW_GROUP, C.rows));
    }
}

__device__ __forceinline__ void stage_wint(const DevSector& S, double* w)
{
    for (int i = threadIdx.x; i < S.P * S.P; i += blockDim.x) w[i] = __ldg(S.wint + i);
}
