// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include <algorithm>
namespace tbb {
template <typename It> void parallel_sort(It b, It e) { std::sort(b, e); }
template <typename It, typename C> void parallel_sort(It b, It e, const C& c) { std::sort(b, e, c); }
}  // namespace tbb
