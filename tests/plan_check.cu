// Host-only check of lz_cut (the device-free part of the persistent kernel's
// launch plan, dmft-ed-zt_b200/csrc/lanczos.cu): on seeded random job sets
// and grid sizes it verifies the tile lists, the CTA ranges, every job's run
// of participating CTAs, the partial-sum slots and the column phase's slab
// order.  Built and run by tests/test_plan_cpu.py; makes no CUDA call.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>
#include "edzt_internal.h"

static int fails = 0;
#define CHECK(c, ...)                                                   \
    do {                                                                \
        if (!(c)) {                                                     \
            if (fails < 20) std::printf("FAIL %s: ", #c), std::printf(__VA_ARGS__), std::printf("\n"); \
            fails++;                                                    \
        }                                                               \
    } while (0)

int main()
{
    std::mt19937_64 rng(20260);
    const int grids[] = {1, 2, 7, 148, 296, 512};
    long long cases = 0;
    for (int trial = 0; trial < 3000; trial++) {
        const int G = grids[trial % 6];
        const int nj = 1 + (int)(rng() % 24);
        std::vector<LzJob> jobs(nj);
        for (auto& J : jobs) {
            std::memset(&J, 0, sizeof(J));
            J.S.up.count = 1 + (int)(rng() % 3000);
            J.S.dn.count = 1 + (int)(rng() % 3000);
            J.ph[0].width = 2 << (rng() % 3);      // 2, 4, 8 columns per slab
            J.ph[1].width = 1 << (rng() % 3);      // 1, 2, 4 rows per tile
        }
        std::vector<long long> prefix;
        long long total[2] = {0, 0};
        const long long slots = lz_cut(jobs.data(), nj, G, prefix, total);
        CHECK(prefix.size() == 2 * (size_t)(nj + 1) + 2 * (size_t)(G + 1) + (size_t)total[0], "prefix size");
        if (prefix.size() != 2 * (size_t)(nj + 1) + 2 * (size_t)(G + 1) + (size_t)total[0]) continue;
        long long slot_sum = 0;
        for (int ph = 0; ph < 2; ph++) {
            const long long* pre = prefix.data() + (size_t)ph * (nj + 1);
            const long long* range = prefix.data() + 2 * (size_t)(nj + 1) + (size_t)ph * (G + 1);
            const long long T = total[ph];
            // tile lists
            CHECK(pre[0] == 0 && pre[nj] == T, "phase %d tile list ends", ph);
            for (int j = 0; j < nj; j++) {
                const LzPhase& Q = jobs[j].ph[ph];
                const int count = ph == 0 ? jobs[j].S.up.count : jobs[j].S.dn.count;
                CHECK(Q.ntiles == (count + Q.width - 1) / Q.width, "ntiles");
                CHECK(Q.tile0 == pre[j] && pre[j + 1] == pre[j] + Q.ntiles, "tile0");
            }
            // CTA ranges: monotone, cover [0, T), non-empty when T >= G
            CHECK(range[0] == 0 && range[G] == T, "range ends");
            for (int b = 0; b < G; b++) {
                CHECK(range[b] <= range[b + 1], "monotone");
                if (T >= G) CHECK(range[b] < range[b + 1], "every CTA has a tile");
                else CHECK(range[b + 1] - range[b] == (b < T ? 1 : 0), "one tile per CTA");
            }
            // participants: exactly the CTAs whose range meets the job's tiles
            for (int j = 0; j < nj; j++) {
                const LzPhase& Q = jobs[j].ph[ph];
                const long long lo = Q.tile0, hi = Q.tile0 + Q.ntiles;
                for (int b = 0; b < G; b++) {
                    const bool meets = std::max(range[b], lo) < std::min(range[b + 1], hi);
                    const bool in = b >= Q.part0 && b < Q.part0 + Q.npart;
                    CHECK(meets == in, "participants of job %d phase %d CTA %d", j, ph, b);
                }
                CHECK(Q.npart >= 1 && Q.npart <= G, "npart");
                CHECK(Q.slot0 == slot_sum, "slots consecutive");
                slot_sum += Q.npart;
            }
            // slab order: a bijection per job; the r-th tile of every
            // participant, in participant order, gets consecutive slabs
            if (ph == 0) {
                const long long* slab = prefix.data() + 2 * (size_t)(nj + 1) + 2 * (size_t)(G + 1);
                for (int j = 0; j < nj; j++) {
                    const LzPhase& Q = jobs[j].ph[0];
                    const long long lo = Q.tile0, hi = Q.tile0 + Q.ntiles;
                    std::vector<char> seen((size_t)Q.ntiles, 0);
                    long long expect = 0;
                    for (long long r = 0; expect < Q.ntiles && r <= Q.ntiles; r++)
                        for (int q = 0; q < Q.npart; q++) {
                            const long long s0 = std::max(range[Q.part0 + q], lo);
                            const long long s1 = std::min(range[Q.part0 + q + 1], hi);
                            if (s0 + r < s1) {
                                const long long v = slab[s0 + r];
                                CHECK(v == expect, "slab order job %d round %lld", j, r);
                                if (v >= 0 && v < Q.ntiles) seen[(size_t)v]++;
                                expect++;
                            }
                        }
                    for (long long i = 0; i < Q.ntiles; i++) CHECK(seen[(size_t)i] == 1, "slab %lld of job %d", i, j);
                }
            }
        }
        CHECK(slots == slot_sum, "slot count");
        cases++;
    }
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("ok %lld job sets\n", cases);
    return 0;
}
