// insert_run / erase_run (the producer's batched sorted-set edits) against
// std::set_union / std::set_difference on random sets: short and long lists,
// sparse and dense edits, repeated values in an insert run; and the task
// queue dedupe (serial and range-parallel) against sort + unique, on uniform
// and skewed vertex ids and on key ranges of 11 bits or fewer.  The
// producer's source is compiled into this file so its internal functions
// are visible.
#include "calig.cpp"

#include <random>

int main() {
    std::mt19937_64 g(7);
    long bad = 0;
    for (int it = 0; it < 100000; ++it) {
        const size_t n = g() % (it % 10 == 0 ? 5000 : 40), k = 2 + g() % (it % 7 == 0 ? 3000 : 20);
        const uint32_t range = 1 + (uint32_t)(g() % (it % 3 ? 100 : 100000));
        std::vector<uint32_t> L(n), x(k);
        for (auto& v : L) v = (uint32_t)(g() % range);
        std::sort(L.begin(), L.end());
        L.erase(std::unique(L.begin(), L.end()), L.end());
        for (auto& v : x) v = (uint32_t)(g() % range);
        std::sort(x.begin(), x.end());

        std::vector<uint32_t> want, got = L;
        std::set_union(L.begin(), L.end(), x.begin(), x.end(), std::back_inserter(want));
        want.erase(std::unique(want.begin(), want.end()), want.end());
        cgb::insert_run(got, x.data(), x.size());
        bad += got != want;

        x.erase(std::unique(x.begin(), x.end()), x.end());
        want.clear();
        std::set_difference(L.begin(), L.end(), x.begin(), x.end(), std::back_inserter(want));
        std::vector<uint8_t> hit(x.size());
        got = L;
        cgb::erase_run(got, x.data(), x.size(), hit.data());
        bad += got != want;
        for (size_t j = 0; j < x.size(); ++j) bad += hit[j] != (uint8_t)std::binary_search(L.begin(), L.end(), x[j]);
    }
    struct Tk { uint32_t u, v; };
    for (int it = 0; it < 3000; ++it) {
        const size_t n = it % 50 == 0 ? 200000 : 1 + g() % 5000;
        const uint32_t vr = it % 4 == 0 ? 1u + (uint32_t)(g() % 40) : 1u + (uint32_t)(g() % 2000000);
        const bool skew = it % 3 == 0;
        std::vector<Tk> q(n);
        std::vector<uint64_t> want(n);
        for (size_t i = 0; i < n; ++i) {
            uint32_t v = (uint32_t)(g() % vr);
            if (skew) v = (uint32_t)((uint64_t)v * (g() % 1024) / 1023 / (1 + g() % 64));
            q[i] = {(uint32_t)(g() % 12), v};
            want[i] = (uint64_t)q[i].v << 5 | q[i].u;
        }
        std::sort(want.begin(), want.end());
        want.erase(std::unique(want.begin(), want.end()), want.end());
        for (uint32_t T : {1u, 3u, 8u}) {
            std::vector<Tk> d = q;
            cgb::dedupe(d, T);
            bool ok = d.size() == want.size();
            for (size_t i = 0; ok && i < d.size(); ++i) ok = ((uint64_t)d[i].v << 5 | d[i].u) == want[i];
            bad += !ok;
        }
    }
    std::printf("bad=%ld\n", bad);
    return bad != 0;
}
