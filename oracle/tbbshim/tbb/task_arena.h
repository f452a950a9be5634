// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include "tbb/detail_pool.h"
namespace tbb {
namespace this_task_arena {
inline int current_thread_index() { return shim::tls_index(); }
inline int max_concurrency() { return shim::Pool::get().size(); }
}  // namespace this_task_arena
class task_arena {
public:
    struct constraints {
        constraints& set_max_concurrency(int) { return *this; }
        constraints& set_numa_id(int) { return *this; }
    };
    task_arena() {}
    explicit task_arena(const constraints&) {}
    explicit task_arena(int) {}
    template <typename F> void execute(const F& f) { f(); }
};
}  // namespace tbb
