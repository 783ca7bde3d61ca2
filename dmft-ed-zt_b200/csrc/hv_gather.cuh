// hv_gather.cuh — the single-pass H.v of k_hx_gather, by element.
//
// Restates the row sum of src/impurity_hamiltonian.f90:98-246 for sectors
// with long lines, where the two phases of hv_phase.cuh leave only narrow
// slabs and tiles.  A sector vector is the matrix X[ndn][nup] (up rank
// fast); element (id, iu):
//   diagonal      (e1_up[iu] + e1_dn[id] + wint[imp_up, imp_dn]) * x(id, iu)
//   up hops       sum_h c * x(id, iu')    -- same row, read from shared memory
//   down hops     sum_h c * x(id', iu)    -- same column of other rows: a warp
//                                            over consecutive iu reads a
//                                            contiguous slice of row id'
//   spin-flip / pair-hop (norb > 1)        sum c * x(id', iu')
// A CTA stages a tile of whole rows in shared memory: the vector on the rows
// and, per row, its down hops as 16-byte records (amplitude, target offset).
// Threads take the tile's elements in order (consecutive threads, consecutive
// iu).  An up-hop list is read as packed 4-byte entries, four per 16-byte
// load, with the amplitude looked up by slot in shared memory.  The terms are
// the reference's; only the floating-point summation order differs
// (diagonal, up hops, down hops, exchange terms).
#pragma once
#include "edzt_device.cuh"

// A staged down hop of a row: signed amplitude and the target row's offset id'*nup.
struct __align__(16) DHop {
    double val;
    long long off;
};

// Shared-memory view of a tile of staged rows [r0, r0 + rows).
struct Chunk {
    DHop* dh;         // [rows][hw]   down hops of each row
    double* xs;       // [rows][nup]  the vector on the tile's rows
    double* de1;      // [rows]       e1_dn of the row
    int* dcnt;        // [rows]       number of down hops of the row
    int* dimp;        // [rows]       impurity pattern of the row's down string
    int r0, rows, nup, hw;
};

// Shared-memory bytes of one staged row (hw_dn: down hop slots per string).
__host__ __device__ __forceinline__ size_t staged_row_bytes(int nup, int hw_dn)
{
    return (size_t)hw_dn * sizeof(DHop) + (size_t)nup * sizeof(double) + sizeof(double) + 2 * sizeof(int);
}

// Carve the chunk arrays for `rmax` rows out of shared memory at `base` (16-byte aligned).
__device__ __forceinline__ Chunk chunk_layout(void* base, int rmax, int nup, int hw)
{
    Chunk C;
    C.dh = reinterpret_cast<DHop*>(base);
    C.xs = reinterpret_cast<double*>(C.dh + (size_t)rmax * hw);
    C.de1 = C.xs + (size_t)rmax * nup;
    C.dcnt = reinterpret_cast<int*>(C.de1 + rmax);
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
    const uint32_t* __restrict__ hp = reinterpret_cast<const uint32_t*>(dn.hpk);
    C.r0 = r0;
    C.rows = nr;
    for (int i = threadIdx.x; i < nr * hw; i += blockDim.x) {
        const int r = i / hw, h = i - r * hw;
        EDZT_OK_OR(r0 + r < ndn && r0 >= 0, 31, r0, r, ndn, continue)
        const uint32_t e = __ldg(hp + ((size_t)(h >> 2) * ndn + r0 + r) * 4 + (h & 3));
        EDZT_OK_OR(edzt_hop_rank(e) < ndn && edzt_hop_slot(e) < dn.namp, 33, r0 + r, h, (long long)e, continue)
        DHop d;
        d.val = __ldg(dn.amp + edzt_hop_slot(e));
        d.off = (long long)edzt_hop_rank(e) * C.nup;
        C.dh[i] = d;
    }
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        EDZT_OK_OR(r0 + r < ndn, 32, r0, r, ndn, continue)
        C.dcnt[r] = __ldg(dn.hcnt + r0 + r);
        C.de1[r] = __ldg(dn.e1 + r0 + r);
        C.dimp[r] = __ldg(dn.imp + r0 + r);
    }
}

// Source of the down-spin gathers: a plain vector.
struct SrcVec {
    const double* __restrict__ x;
    using raw = double;
    __device__ __forceinline__ raw load(long long i) const { return __ldg(x + i); }
    __device__ __forceinline__ raw zero() const { return 0.0; }
    __device__ __forceinline__ double value(raw v) const { return v; }
};

// Element (row r of the chunk, column iu): returns the diagonal plus up-hop
// part (on the staged, already normalised row) in `du` and the raw down-hop
// sum (on the source, not normalised) in `dn`.  Every load of the element is
// issued before the first one is consumed: the up-hop list as two 16-byte
// loads without waiting for the hop count, and the down gathers eight at a
// time, so an element costs one L1 and one L2 round trip while hop counts are
// <= 8 (nsite <= 14 near half filling); longer lists continue in a loop.
template <class Src>
__device__ __forceinline__ void hv_elem(const DevSector& S, const Chunk& C, const double* __restrict__ wint,
                                        const double* __restrict__ amp_up, const Src& src, int r, int iu, double xe,
                                        double& du, double& dn)
{
    const int nup = C.nup;
    const uint4* __restrict__ hp = S.up.hpk + iu;
    const int hu = __ldg(S.up.hcnt + iu);
    const int pu = __ldg(S.up.imp + iu);
    const double e1u = __ldg(S.up.e1 + iu);
    const uint4 q0 = __ldg(hp);
    const uint4 q1 = (S.up.hw > 4) ? __ldg(hp + nup) : make_uint4(0u, 0u, 0u, 0u);
    int hd = C.dcnt[r];
    EDZT_OK_OR(hd >= 0 && hd <= C.hw, 13, iu, r, hd, hd = 0)
    const DHop* __restrict__ rec = C.dh + r * C.hw;
    double val[8];
    typename Src::raw g[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        val[q] = 0.0;
        g[q] = src.zero();
        if (q < hd) {
            const DHop d = rec[q];
            EDZT_OK_OR(d.off >= 0 && d.off + iu < S.dim, 21, d.off, iu, S.dim, continue)
            val[q] = d.val;
            g[q] = src.load(d.off + iu);
        }
    }
    // diagonal and up hops
    const double* __restrict__ xrow = C.xs + r * nup;
    double acc = (e1u + C.de1[r] + wint[pu * S.P + C.dimp[r]]) * xe;
    const uint32_t e[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int c = 0; c < 8; c++) {
        if (c < hu) {
            EDZT_OK_OR(edzt_hop_rank(e[c]) < nup && edzt_hop_slot(e[c]) < S.up.namp, 11, iu, c, (long long)e[c],
                       continue)
            acc = fma(amp_up[edzt_hop_slot(e[c])], xrow[edzt_hop_rank(e[c])], acc);
        }
    }
    for (int h0 = 8; h0 < hu; h0 += 4) {                     // hop lists longer than 8
        const uint4 q = __ldg(hp + (h0 >> 2) * nup);
        const uint32_t f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (h0 + c < hu) acc = fma(amp_up[edzt_hop_slot(f[c])], xrow[edzt_hop_rank(f[c])], acc);
    }
    du = acc;
    // down hops
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) s = fma(val[q], src.value(g[q]), s);
    for (int h = 8; h < hd; h++) {
        const DHop d = rec[h];
        s = fma(d.val, src.value(src.load(d.off + iu)), s);
    }
    dn = s;
}

// Spin-flip and pair-hopping terms (impurity_hamiltonian.f90:179-226) of
// element (id, iu); fetch(idx) returns the vector at a global index.
template <class Fetch>
__device__ __forceinline__ double hv_exchange(const DevSector& S, const Chunk& C, int r, int iu, double acc,
                                              Fetch fetch)
{
    const int P = S.P;
    const int id = C.r0 + r;
    const int pp = __ldg(S.up.imp + iu) * P + C.dimp[r];
    const int nj = __ldg(S.jcnt + pp);
    for (int t = 0; t < nj; t++) {
        const JTrans tr = S.jt[pp * EDZT_MAX_JT + t];
        const int iu2 = __ldg(S.up.sub + iu * P + tr.pu2);
        const int id2 = __ldg(S.dn.sub + id * P + tr.pd2);
        EDZT_OK_OR(iu2 >= 0 && iu2 < C.nup && id2 >= 0 && id2 < S.dn.count, 15, iu2, id2, pp, continue)
        acc = fma(tr.c, fetch((long long)id2 * C.nup + iu2), acc);
    }
    return acc;
}
