// Back-to-back jobs of varied sizes on the producer's worker pool: every
// task of every job runs exactly once and before its job returns.  A late
// worker that ran a task of the next job early, or ran one twice, shows up
// as a count other than 1.
#include "calig.h"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char** argv) {
    const int jobs = argc > 1 ? std::atoi(argv[1]) : 20000;
    std::vector<std::atomic<int>> hits(64);
    long bad = 0;
    for (int it = 0; it < jobs; ++it) {
        const uint32_t n = 2 + (uint32_t)(it * 7919u) % 37;
        for (uint32_t i = 0; i < n; ++i) hits[i].store(0, std::memory_order_relaxed);
        std::function<void(uint32_t)> fn = [&hits](uint32_t t) { hits[t].fetch_add(1, std::memory_order_relaxed); };
        cgb::pool_run(n, fn);
        for (uint32_t i = 0; i < n; ++i) bad += hits[i].load(std::memory_order_relaxed) != 1;
    }
    std::printf("jobs=%d bad=%ld\n", jobs, bad);
    return bad != 0;
}
