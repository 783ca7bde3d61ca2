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

__device__ __forceinline__ void stage_table(const double* __restrict__ src, int n, double* dst)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Asynchronous 8-byte copy global -> shared (cp.async, no register holds the
// value in flight, so a thread can have its whole share of a tile in flight
// at once); when `valid` is false nothing is read and the destination gets 0.
__device__ __forceinline__ void copy_async8(double* dst, const double* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

// Wait for every asynchronous copy this thread issued (the caller then syncs the CTA).
__device__ __forceinline__ void copy_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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

// The packed hop list of string t (table [hw/4][count] of uint4): its count
// and first eight entries, loaded as one byte and two 16-byte words.  A
// loop over strings loads the next string's list before it uses the current
// one, so the table's latency overlaps the current string's arithmetic.
struct HopList {
    int hc;
    uint4 q0, q1;
};

__device__ __forceinline__ HopList hop_list(const DevSpin& sp, int t)
{
    HopList L;
    const uint4* __restrict__ hp = sp.hpk + t;
    L.hc = __ldg(sp.hcnt + t);
    L.q0 = (sp.hw > 0) ? __ldg(hp) : make_uint4(0u, 0u, 0u, 0u);
    L.q1 = (sp.hw > 4) ? __ldg(hp + sp.count) : make_uint4(0u, 0u, 0u, 0u);
    return L;
}

// Hop sum of string t over staged lines: acc[q] += amp(h) * lines[rank(h) *
// STRIDE + q] over the string's hops h, in table order.  The eight terms of
// the loaded entries are issued without waiting on one another (lanes past
// their string's hop count are predicated off); longer lists continue four
// at a time.
template <int N, int STRIDE>
__device__ __forceinline__ void hop_sum(const DevSpin& sp, int t, const HopList& L, const double* __restrict__ amp,
                                        const double* __restrict__ lines, double (&acc)[N], int code)
{
    const int hc = L.hc;
    const uint32_t e[8] = {L.q0.x, L.q0.y, L.q0.z, L.q0.w, L.q1.x, L.q1.y, L.q1.z, L.q1.w};
#pragma unroll
    for (int h = 0; h < 8; h++) {
        if (h < hc) {
            EDZT_OK_OR(edzt_hop_rank(e[h]) < sp.count && edzt_hop_slot(e[h]) < sp.namp, code, t, h, (long long)e[h],
                       continue)
            axpy_line<N>(amp[edzt_hop_slot(e[h])], lines + edzt_hop_rank(e[h]) * STRIDE, acc);
        }
    }
    for (int h0 = 8; h0 < hc; h0 += 4) {
        const uint4 q = __ldg(sp.hpk + t + (size_t)(h0 >> 2) * sp.count);
        const uint32_t f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int h = 0; h < 4; h++) {
            if (h0 + h < hc) {
                EDZT_OK_OR(edzt_hop_rank(f[h]) < sp.count && edzt_hop_slot(f[h]) < sp.namp, code, t, h0 + h,
                           (long long)f[h], continue)
                axpy_line<N>(amp[edzt_hop_slot(f[h])], lines + edzt_hop_rank(f[h]) * STRIDE, acc);
            }
        }
    }
}

// The down-hop part D written by the column phase is slab-major: the slab
// of columns [c0, c0 + WC) is one contiguous block [ndn][WC] at c0 * ndn, so
// a CTA writes its slab as one stream of 16-byte stores.  Element (id, iu)
// with WC = 2^wsh:
__device__ __forceinline__ long long slab_index(int id, int iu, int ndn, int wsh)
{
    return ((long long)(iu >> wsh) * ndn + id) * (1 << wsh) + (iu & ((1 << wsh) - 1));
}

// Store the WC values of row id of the slab starting at column c0 (16-byte
// stores; c0 and WC are even, so every pair is 16-byte aligned).
template <int WC>
__device__ __forceinline__ void store_slab_row(double* __restrict__ D, int c0, int ndn, int id, const double (&d)[WC])
{
    double2* out = reinterpret_cast<double2*>(D + (long long)c0 * ndn + (long long)id * WC);
#pragma unroll
    for (int c = 0; c < WC; c += 2) __stcg(out + c / 2, make_double2(d[c], d[c + 1]));
}

// What the row phase reads from global memory for column iu of a tile of R
// rows: the column's up string (energy, impurity bits, hop list), the
// down-hop part D of its R elements (slabs of 2^wsh columns) and, in the
// Lanczos kernel, w_{k-1} of those elements (the second value of each stored
// (y, w) pair; prev null: none); loaded one column ahead.
template <int R>
struct RowCol {
    double e1u;
    int pu;
    HopList L;
    double dd[R];
    double wp[R];
};

template <int R>
__device__ __forceinline__ RowCol<R> row_col(const DevSector& S, const double* __restrict__ D, int wsh, int iu,
                                             int r0, int nr, const double2* __restrict__ prev = nullptr)
{
    RowCol<R> c;
    c.e1u = __ldg(S.up.e1 + iu);
    c.pu = __ldg(S.up.imp + iu);
    c.L = hop_list(S.up, iu);
#pragma unroll
    for (int r = 0; r < R; r++) {
        c.dd[r] = (r < nr) ? __ldcg(D + slab_index(r0 + r, iu, S.dn.count, wsh)) : 0.0;
        c.wp[r] = (prev != nullptr && r < nr)
                      ? __ldcg(reinterpret_cast<const double*>(prev + (long long)(r0 + r) * S.up.count + iu) + 1)
                      : 0.0;
    }
    return c;
}

// Row phase, column iu of a tile of R staged rows: the diagonal and up-hop
// part of (H x)(r0 + r, iu) into acc[r].  xs: [nup][RS] staged values,
// wint: [P*P], amp: up-hop amplitudes by slot, e1d/pd: the rows' down-string
// energies and impurity patterns, c: the column's prefetched data.
template <int R, int RS>
__device__ __forceinline__ void row_part(const DevSector& S, const double* __restrict__ xs,
                                         const double* __restrict__ wint, const double* __restrict__ amp, int iu,
                                         const RowCol<R>& c, const double (&e1d)[R], const int (&pd)[R],
                                         double (&acc)[R])
{
    const double* __restrict__ own = xs + iu * RS;
    const int pu = c.pu * S.P;
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = (c.e1u + e1d[r] + wint[pu + pd[r]]) * own[r];
    hop_sum<R, RS>(S.up, iu, c.L, amp, xs, acc, 71);
}

// Column phase, row id of a slab of WC staged columns: the down-hop part of
// (H x)(id, c0 + c) into d[c].  ws: [ndn][WS] staged values, amp: down-hop
// amplitudes by slot, L: the row's prefetched hop list.
template <int WC, int WS>
__device__ __forceinline__ void col_part(const DevSector& S, const double* __restrict__ ws,
                                         const double* __restrict__ amp, int id, const HopList& L, double (&d)[WC])
{
#pragma unroll
    for (int c = 0; c < WC; c++) d[c] = 0.0;
    hop_sum<WC, WS>(S.dn, id, L, amp, ws, d, 72);
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
