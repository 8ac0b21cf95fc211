// Checks of the host copy pool (illuminaprt_b200/csrc/hostpool.h), built and
// run by test_hostpool.py: every part of a job runs exactly once, jobs of
// different sizes follow one another on one pool, and pool_copy moves every
// byte of segments of any length, whatever the split.
#include "hostpool.h"

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

using ilg::CopySeg;
using ilg::HostPool;

static int fails = 0;
#define CHECK(c)                                                            \
    do {                                                                    \
        if (!(c)) {                                                         \
            std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
            fails++;                                                        \
        }                                                                   \
    } while (0)

int main()
{
    std::mt19937_64 rng(7);
    {
        HostPool pool;
        for (unsigned parts : {1u, 2u, 16u, 3u, 1u, 9u, 16u, 5u}) {
            std::vector<std::atomic<int>> hits(parts);
            for (auto &h : hits) h = 0;
            pool.run(parts, [&](unsigned k) { hits[k]++; });
            for (unsigned k = 0; k < parts; k++) CHECK(hits[k] == 1);
        }
        CHECK(pool.threads() == 15u);
        // many small jobs in a row on the same threads
        std::atomic<long> sum{0};
        for (int rep = 0; rep < 2000; rep++) pool.run(1 + rep % 16, [&](unsigned k) { sum += k + 1; });
        long want = 0;
        for (int rep = 0; rep < 2000; rep++) {
            const int p = 1 + rep % 16;
            want += (long)p * (p + 1) / 2;
        }
        CHECK(sum == want);
    }
    {
        HostPool pool;
        for (int rep = 0; rep < 200; rep++) {
            const int nseg = 1 + (int)(rng() % 6);
            std::vector<std::vector<uint8_t>> src(nseg), dst(nseg);
            CopySeg seg[6];
            for (int i = 0; i < nseg; i++) {
                const size_t len = (rng() % 4 == 0) ? 0 : (size_t)(rng() % (3u << 20));
                src[i].resize(len);
                dst[i].assign(len, 0xEE);
                for (auto &b : src[i]) b = (uint8_t)rng();
                seg[i] = {dst[i].data(), src[i].data(), len};
            }
            const unsigned max_parts = 1 + (unsigned)(rng() % 16);
            const size_t min_part = (rng() % 2) ? size_t(1) << 20 : 1 + rng() % 4096;
            ilg::pool_copy(pool, seg, nseg, max_parts, min_part);
            for (int i = 0; i < nseg; i++) CHECK(dst[i] == src[i]);
        }
    }
    if (fails) return 1;
    std::printf("hostpool ok\n");
    return 0;
}
