// The serving loop's staging ring (cgbdsm_b200/csrc/staging_ring.h) under
// random FIFO traffic: allocations of random sizes while they fit, releases
// of the oldest block; live blocks must lie inside the ring, never overlap,
// and an empty ring must take any block up to its capacity.
#include <cstdio>
#include <deque>
#include <random>

#include "staging_ring.h"

int main() {
    std::mt19937_64 rng(12345);
    unsigned long long bad = 0, allocs = 0, wraps = 0;
    for (int trial = 0; trial < 200; ++trial) {
        cgb::StagingRing ring;
        ring.cap = 1000 + rng() % 100000;
        std::deque<std::pair<uint64_t, uint64_t>> live;
        for (int step = 0; step < 5000; ++step) {
            const bool try_alloc = live.empty() || (rng() % 3) != 0;
            if (try_alloc) {
                const uint64_t len = 1 + rng() % (ring.cap / (1 + rng() % 8) + 1);
                uint64_t off = 0;
                if (ring.alloc(len, &off)) {
                    ++allocs;
                    if (off + len > ring.cap) ++bad;
                    for (auto& b : live)
                        if (off < b.first + b.second && b.first < off + len) ++bad;  // overlap
                    if (!live.empty() && off < live.back().first) ++wraps;
                    live.emplace_back(off, len);
                } else if (live.empty()) {
                    ++bad;  // an empty ring must take any block up to its capacity
                }
            } else {
                ring.release(live.front().first, live.front().second);
                live.pop_front();
            }
            uint64_t sum = 0;
            for (auto& b : live) sum += b.second;
            if (ring.used < sum || ring.used > ring.cap) ++bad;
        }
        while (!live.empty()) {
            ring.release(live.front().first, live.front().second);
            live.pop_front();
        }
        if (ring.used != 0) ++bad;
        uint64_t off = 0;
        if (!ring.alloc(ring.cap, &off) || off != 0) ++bad;  // the whole ring, once empty
    }
    std::printf("allocs=%llu wraps=%llu bad=%llu\n", allocs, wraps, bad);
    return bad ? 1 : 0;
}
