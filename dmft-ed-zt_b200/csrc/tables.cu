// tables.cu — kernel (a): sector basis enumeration, combinadic ranking and
// the per-string sign/hop tables, all as exact integer work on the device.
//
// Reference behaviour restated (src/ed_basis.f90:76-113): the strings of one
// spin with popcount n are enumerated in ascending integer order and each
// gets a 1-based rank.  Ascending order of fixed-popcount integers is colex
// order, so the rank of the string with set bits p_1 < ... < p_n is
// sum_k C(p_k, k) (0-based here) and the r-th string is recovered greedily
// from the top bit down.  The fermion signs of src/impurity_hamiltonian.f90:
// 251-260 are popcounts of the bits strictly between the two sites.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <set>
#include "edzt_internal.h"

__constant__ uint32_t c_binom[EDZT_MAX_NSITE + 2][EDZT_MAX_NSITE + 2];

static uint64_t h_binom[EDZT_MAX_NSITE + 2][EDZT_MAX_NSITE + 2];
static std::once_flag h_binom_once;

static void fill_host_binom()
{
    for (int n = 0; n <= EDZT_MAX_NSITE + 1; n++)
        for (int k = 0; k <= EDZT_MAX_NSITE + 1; k++) {
            if (k == 0) h_binom[n][k] = 1;
            else if (n == 0) h_binom[n][k] = 0;
            else h_binom[n][k] = h_binom[n - 1][k - 1] + h_binom[n - 1][k];
        }
}

uint64_t edzt_binom(int n, int k)
{
    std::call_once(h_binom_once, fill_host_binom);
    if (n < 0 || k < 0 || n > EDZT_MAX_NSITE + 1 || k > EDZT_MAX_NSITE + 1) return 0;
    return h_binom[n][k];
}

void edzt_init_binomials(int device)
{
    static std::mutex mu;
    static std::set<int> done;
    std::lock_guard<std::mutex> g(mu);
    if (done.count(device)) return;
    std::call_once(h_binom_once, fill_host_binom);
    uint32_t t[EDZT_MAX_NSITE + 2][EDZT_MAX_NSITE + 2];
    for (int n = 0; n < EDZT_MAX_NSITE + 2; n++)
        for (int k = 0; k < EDZT_MAX_NSITE + 2; k++) t[n][k] = (uint32_t)h_binom[n][k];
    cudaMemcpyToSymbol(c_binom, t, sizeof(t));
    done.insert(device);
}

// r-th (0-based) string of popcount n on nsite bits in ascending order.
__device__ __forceinline__ uint32_t unrank_colex(uint32_t r, int n, int nsite)
{
    uint32_t s = 0;
    int top = nsite;  // positions available: [0, top)
    for (int k = n; k >= 1; --k) {
        int p = k - 1;
        while (p + 1 < top && c_binom[p + 1][k] <= r) ++p;
        s |= 1u << p;
        r -= c_binom[p][k];
        top = p;
    }
    return s;
}

__device__ __forceinline__ int32_t rank_colex(uint32_t s)
{
    int32_t r = 0;
    int k = 0;
    while (s) {
        int p = __ffs(s) - 1;
        ++k;
        r += (int32_t)c_binom[p][k];
        s &= s - 1;
    }
    return r;
}

__global__ void k_build_strings(int nsite, int n, int count, uint32_t* __restrict__ str)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) str[t] = unrank_colex((uint32_t)t, n, nsite);
}

__global__ void k_build_rank(int nsite, int n, int32_t* __restrict__ rank)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < (1u << nsite)) rank[s] = (__popc(s) == n) ? rank_colex(s) : -1;
}

// Per string of one spin species: one-body energy, hop list, impurity bits
// and the rank of every impurity-pattern substitution.
__global__ void k_build_spin_ops(DevModel m, int sigma, int count, const uint32_t* __restrict__ str,
                                 const int32_t* __restrict__ rank, int hw, double* __restrict__ e1,
                                 uint8_t* __restrict__ hcnt, uint32_t* __restrict__ hpk,
                                 double* __restrict__ amp, uint8_t* __restrict__ imp, int32_t* __restrict__ sub)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {   // amplitude slots: +V at 2c, -V at 2c+1, c = iorb*nbath + jbath
        for (int a = 0; a < m.norb; a++)
            for (int l = 0; l < m.nbath; l++) {
                amp[2 * (a * m.nbath + l)] = m.vmk[a][l][sigma];
                amp[2 * (a * m.nbath + l) + 1] = -m.vmk[a][l][sigma];
            }
        if (m.nbath == 0) amp[0] = amp[1] = 0.0;
    }
    if (t >= count) return;
    const uint32_t u = str[t];
    const int norb = m.norb, nbath = m.nbath;
    // one-body diagonal (impurity_hamiltonian.f90:119-120 em-mu terms, :232-239 ek terms)
    double e = 0.0;
    for (int a = 0; a < norb; a++)
        if ((u >> a) & 1u) e += m.em[a][sigma] - m.mu;
    for (int l = 0; l < nbath; l++)
        if ((u >> (norb + l)) & 1u) e += m.ek[l][sigma];
    e1[t] = e;
    // hybridisation hops (impurity_hamiltonian.f90:146-174), loop order iorb, jbath;
    // entry h of string t sits at uint32 index ((h/4)*count + t)*4 + h%4
    auto slot_at = [&](int h) -> uint32_t& { return hpk[((size_t)(h >> 2) * count + t) * 4 + (h & 3)]; };
    int h = 0;
    for (int a = 0; a < norb; a++) {
        for (int l = 0; l < nbath; l++) {
            const double v = m.vmk[a][l][sigma];
            if (fabs(v) < 1.0e-16) continue;                    // :148
            const int i = a, j = norb + l;                       // i < j
            const uint32_t bi = (u >> i) & 1u, bj = (u >> j) & 1u;
            if (bi == bj) continue;
            // bits strictly between i and j; for bi == 1 the reference's
            // sgn() also counts bit i and subtracts, which cancels (:161-171)
            const uint32_t between = ((1u << j) - 1u) & ~((2u << i) - 1u);
            const uint32_t u2 = u ^ (1u << i) ^ (1u << j);
            EDZT_OK_OR(h < hw && rank[u2] >= 0, 51, t, h, u2, continue)
            const int neg = __popc(u & between) & 1;
            slot_at(h) = edzt_hop_pack(rank[u2], 2 * (a * nbath + l) + neg);
            ++h;
        }
    }
    for (int q = h; q < hw; q++) slot_at(q) = 0u;
    hcnt[t] = (uint8_t)h;
    const uint32_t P = 1u << norb;
    imp[t] = (uint8_t)(u & (P - 1u));
    if (sub) {
        for (uint32_t p = 0; p < P; p++) sub[(size_t)t * P + p] = rank[(u & ~(P - 1u)) | p];
    }
}

#ifdef EDZT_DEVICE_CHECKS
int tables_debug_bad(long long* out4)
{
    return cudaMemcpyFromSymbol(out4, g_edzt_bad, 4 * sizeof(long long)) == cudaSuccess ? 0 : 2;
}
#endif

void launch_build_strings(int nsite, int n, uint32_t* str, int32_t* rank, cudaStream_t s)
{
    int count = (int)edzt_binom(nsite, n);
    if (count > 0) k_build_strings<<<(count + 255) / 256, 256, 0, s>>>(nsite, n, count, str);
    int nst = 1 << nsite;
    k_build_rank<<<(nst + 255) / 256, 256, 0, s>>>(nsite, n, rank);
}

void launch_build_spin_ops(const DevModel& m, int sigma, int count, const uint32_t* str, const int32_t* rank,
                           int hw, double* e1, uint8_t* hcnt, uint32_t* hpk, double* amp, uint8_t* imp,
                           int32_t* sub, cudaStream_t s)
{
    const int n = count > 0 ? count : 1;   // the amplitude slots are written even for an empty table
    k_build_spin_ops<<<(n + 127) / 128, 128, 0, s>>>(m, sigma, count, str, rank, hw, e1, hcnt, hpk, amp, imp, sub);
}

int edzt_max_hops(const DevModel& m, int sigma, int n)
{
    const int ns = m.nsite;
    if (n < 0 || n > ns) return 0;
    int best = 0;
    // every string with popcount n (Gosper's hack; the empty and full strings directly)
    uint64_t u = (n == 0) ? 0ull : ((1ull << n) - 1ull);
    const uint64_t end = 1ull << ns;
    while (u < end) {
        int h = 0;
        for (int a = 0; a < m.norb; a++)
            for (int l = 0; l < m.nbath; l++)
                if (std::fabs(m.vmk[a][l][sigma]) >= 1.0e-16 && (((u >> a) ^ (u >> (m.norb + l))) & 1ull)) h++;
        if (h > best) best = h;
        if (n == 0) break;
        const uint64_t c = u & (0ull - u), r = u + c;
        u = (((r ^ u) >> 2) / c) | r;
    }
    return best;
}
