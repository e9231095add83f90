// Randomised check of the serving loop's frontier range allocator (host-only bookkeeping)
// against a byte-map model: grants never overlap, stay inside the range, respect the granule
// and the least/want bounds, and freed ranges merge back to one range.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "frontier_arena.h"

int main() {
    using csm::kGranule;
    std::mt19937_64 rng(12345);
    for (int round = 0; round < 200; round++) {
        const uint64_t size = kGranule * (1 + rng() % 4096);
        csm::RangeAllocator ra;
        ra.reset(size);
        std::vector<uint8_t> owner(size / kGranule, 0);
        struct Grant {
            uint64_t off, len;
        };
        std::vector<Grant> live;
        for (int step = 0; step < 400; step++) {
            if (!live.empty() && (rng() % 3 == 0)) {
                const size_t i = rng() % live.size();
                for (uint64_t g = live[i].off / kGranule; g < (live[i].off + live[i].len) / kGranule; g++) owner[g] = 0;
                ra.give(live[i].off, live[i].len);
                live.erase(live.begin() + i);
                continue;
            }
            const uint64_t want = 1 + rng() % (size / 2 + 1);
            const uint64_t least = rng() % 2 ? 0 : 1 + rng() % (want + 1);
            const uint64_t largest = ra.largest_free();
            uint64_t off = ~0ull;
            const uint64_t got = ra.take(want, least, &off);
            const uint64_t want_r = (want + kGranule - 1) / kGranule * kGranule;
            const uint64_t expect = std::min(want_r, largest);
            if (expect == 0 || expect < least) {
                if (got != 0) return std::printf("granted %llu below least\n", (unsigned long long)got), 1;
                continue;
            }
            if (got != expect) return std::printf("grant %llu expected %llu\n", (unsigned long long)got, (unsigned long long)expect), 1;
            if (off % kGranule || off + got > size) return std::printf("grant out of range\n"), 1;
            for (uint64_t g = off / kGranule; g < (off + got) / kGranule; g++) {
                if (owner[g]) return std::printf("overlapping grants\n"), 1;
                owner[g] = 1;
            }
            live.push_back({off, got});
        }
        uint64_t used = 0;
        for (auto &g : live) used += g.len;
        if (used != ra.used()) return std::printf("used mismatch\n"), 1;
        for (auto &g : live) ra.give(g.off, g.len);
        if (ra.used() != 0 || ra.free_ranges() != 1 || ra.largest_free() != ra.size())
            return std::printf("ranges did not merge back\n"), 1;
    }
    std::printf("ok\n");
    return 0;
}
