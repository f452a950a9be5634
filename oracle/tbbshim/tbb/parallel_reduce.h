// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include <mutex>
#include "tbb/blocked_range.h"
#include "tbb/detail_pool.h"
namespace tbb {
template <typename T, typename V, typename F, typename R>
V parallel_reduce(const blocked_range<T>& r, const V& identity, const F& f, const R& reduce) {
    V total = identity;
    std::mutex m;
    shim::chunked(r.begin(), r.end(), r.grainsize(), [&](T s, T e) {
        V part = f(blocked_range<T>(s, e, r.grainsize()), identity);
        std::lock_guard<std::mutex> lk(m);
        total = reduce(total, part);
    });
    return total;
}
}  // namespace tbb
