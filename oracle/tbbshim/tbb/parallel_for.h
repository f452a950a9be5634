// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include "tbb/blocked_range.h"
#include "tbb/detail_pool.h"
#include "tbb/task_arena.h"
namespace tbb {
struct static_partitioner {};
struct auto_partitioner {};
struct simple_partitioner {};

template <typename I, typename F>
void parallel_for(I first, I last, const F& f) {
    shim::chunked(first, last, 1, [&](I s, I e) { for (I i = s; i < e; ++i) f(i); });
}
template <typename T, typename F>
void parallel_for(const blocked_range<T>& r, const F& f) {
    shim::chunked(r.begin(), r.end(), r.grainsize(),
                  [&](T s, T e) { f(blocked_range<T>(s, e, r.grainsize())); });
}
template <typename T, typename F, typename P>
void parallel_for(const blocked_range<T>& r, const F& f, const P&) {
    parallel_for(r, f);
}
}  // namespace tbb
