// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include <cstddef>
namespace tbb {
template <typename T>
class blocked_range {
public:
    blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), g_(grain ? grain : 1) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    size_t size() const { return (size_t)(e_ - b_); }
    bool empty() const { return !(b_ < e_); }
    size_t grainsize() const { return g_; }
private:
    T b_, e_;
    size_t g_;
};
}  // namespace tbb
