// insert_run / erase_run (the producer's batched sorted-set edits) against
// std::set_union / std::set_difference on random sets: short and long lists,
// sparse and dense edits, repeated values in an insert run.  The producer's
// source is compiled into this file so its internal functions are visible.
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
    std::printf("bad=%ld\n", bad);
    return bad != 0;
}
