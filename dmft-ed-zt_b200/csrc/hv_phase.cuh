// hv_phase.cuh — the matrix-free Fock-space H.v in two streaming phases.
//
// Restates the row sum of src/impurity_hamiltonian.f90:98-246 with the work
// split by the spin whose string a term changes.  A sector vector is the
// matrix X[ndn][nup] (up rank fast).  Then
//
//   (H x)(id, iu) = diag(id, iu) x(id, iu)                       diagonal
//                 + sum_h up_amp_h(iu)  x(id, up_rank_h(iu))     up hops: same row
//                 + sum_h dn_amp_h(id)  x(dn_rank_h(id), iu)     down hops: same column
//                 + sum_t c_t x(id2_t, iu2_t)                    spin-flip / pair hop
//
// A whole row is closed under the up hops and a whole column under the down
// hops.  So the row phase stages tiles of R whole rows in shared memory and
// computes the diagonal and up-hop part there, and the column phase stages
// slabs of WC whole columns (every row of the sector, WC columns wide) and
// computes the down-hop part there: every neighbour value comes from shared
// memory, every global access is a coalesced stream, and no neighbour value
// is gathered from L2 or DRAM.  The exchange terms of a multi-orbital model
// change both strings and are gathered from global memory in the row phase.
//
// Shared-memory layouts are transposed so that a hop's neighbour values for
// two consecutive rows (row phase) or columns (column phase) are one 16-byte
// load: the row tile is xs[iu][RS] and the column slab ws[id][WS], with the
// strides RS and WS = 2 (mod 4) doubles so that the 16-byte loads of a warp,
// at scattered neighbours, spread over all eight bank quads.
//
// The terms are the reference's; only the floating-point summation order
// differs (diagonal, up hops in table order, then the down-hop sum, then
// the exchange terms).
#pragma once
#include "edzt_device.cuh"

// Padded stride of a staged line of n doubles: n rounded up to 2 (mod 4)
// (n = 1 stays 1: a single value, loaded as a scalar).
__host__ __device__ constexpr int phase_stride(int n) { return n <= 1 ? 1 : ((n + 1) / 4) * 4 + 2; }

// Hop entry h of string t in a packed table [hw/4][count] of uint4
__device__ __forceinline__ uint32_t hop_entry(const DevSpin& sp, int t, int h)
{
    const uint32_t* hp = reinterpret_cast<const uint32_t*>(sp.hpk);
    return __ldg(hp + ((size_t)(h >> 2) * sp.count + t) * 4 + (h & 3));
}

__device__ __forceinline__ void stage_table(const double* __restrict__ src, int n, double* dst)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// acc[q] += a * line[q] for q < N, two at a time (16-byte shared loads).
template <int N>
__device__ __forceinline__ void axpy_line(double a, const double* __restrict__ line, double (&acc)[N])
{
    if constexpr (N == 1) {
        acc[0] = fma(a, line[0], acc[0]);
    } else {
#pragma unroll
        for (int q = 0; q < N; q += 2) {
            const double2 v = *reinterpret_cast<const double2*>(line + q);
            acc[q] = fma(a, v.x, acc[q]);
            acc[q + 1] = fma(a, v.y, acc[q + 1]);
        }
    }
}

// Row phase, column iu of a tile of R staged rows: the diagonal and up-hop
// part of (H x)(r0 + r, iu) into acc[r].  xs: [nup][RS] staged values,
// wint: [P*P], amp: up-hop amplitudes by slot, e1d/pd: the rows' down-string
// energies and impurity patterns.
template <int R, int RS>
__device__ __forceinline__ void row_part(const DevSector& S, const double* __restrict__ xs,
                                         const double* __restrict__ wint, const double* __restrict__ amp, int iu,
                                         const double (&e1d)[R], const int (&pd)[R], double (&acc)[R])
{
    const double* __restrict__ own = xs + iu * RS;
    const double e1u = __ldg(S.up.e1 + iu);
    const int pu = __ldg(S.up.imp + iu) * S.P;
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = (e1u + e1d[r] + wint[pu + pd[r]]) * own[r];
    const int hu = __ldg(S.up.hcnt + iu);
    for (int h = 0; h < hu; h++) {
        const uint32_t e = hop_entry(S.up, iu, h);
        EDZT_OK_OR(edzt_hop_rank(e) < S.up.count && edzt_hop_slot(e) < S.up.namp, 71, iu, h, (long long)e, continue)
        axpy_line<R>(amp[edzt_hop_slot(e)], xs + edzt_hop_rank(e) * RS, acc);
    }
}

// Column phase, row id of a slab of WC staged columns: the down-hop part of
// (H x)(id, c0 + c) into d[c].  ws: [ndn][WS] staged values, amp: down-hop
// amplitudes by slot.
template <int WC, int WS>
__device__ __forceinline__ void col_part(const DevSector& S, const double* __restrict__ ws,
                                         const double* __restrict__ amp, int id, double (&d)[WC])
{
#pragma unroll
    for (int c = 0; c < WC; c++) d[c] = 0.0;
    const int hd = __ldg(S.dn.hcnt + id);
    for (int h = 0; h < hd; h++) {
        const uint32_t e = hop_entry(S.dn, id, h);
        EDZT_OK_OR(edzt_hop_rank(e) < S.dn.count && edzt_hop_slot(e) < S.dn.namp, 72, id, h, (long long)e, continue)
        axpy_line<WC>(amp[edzt_hop_slot(e)], ws + edzt_hop_rank(e) * WS, d);
    }
}

// Spin-flip and pair-hopping terms (impurity_hamiltonian.f90:179-226) of
// element (id, iu) with up impurity pattern pu and down pattern pd;
// fetch(index) returns the vector at a global index.
template <class Fetch>
__device__ __forceinline__ double exchange_part(const DevSector& S, int id, int iu, int pu, int pd, double acc,
                                                Fetch fetch)
{
    const int P = S.P, nup = S.up.count;
    const int pp = pu * P + pd;
    const int nj = __ldg(S.jcnt + pp);
    for (int t = 0; t < nj; t++) {
        const JTrans tr = S.jt[pp * EDZT_MAX_JT + t];
        const int iu2 = __ldg(S.up.sub + iu * P + tr.pu2);
        const int id2 = __ldg(S.dn.sub + id * P + tr.pd2);
        EDZT_OK_OR(iu2 >= 0 && iu2 < nup && id2 >= 0 && id2 < S.dn.count, 73, iu2, id2, pp, continue)
        acc = fma(tr.c, fetch((long long)id2 * nup + iu2), acc);
    }
    return acc;
}
