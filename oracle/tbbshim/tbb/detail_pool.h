// Minimal oneTBB-API stand-in used ONLY to compile the reference's CPU sources
// (index/calig.cpp, index/cpu_dfs.cpp, index/cpu_index_mirror.cpp) for the
// oracle under oracle/_ref.  oneTBB is not installed in this image.
//
// This is test infrastructure: nothing in the product links it.
//
// Semantics kept from oneTBB that the reference relies on:
//   * this_task_arena::current_thread_index() is in [0, concurrency) and is
//     stable for the duration of one body invocation (the reference indexes
//     per-thread vectors with it);
//   * parallel_for / parallel_reduce return only after every body finished;
//   * a nested parallel call runs serially on the calling thread.
// Thread count: CGB_REF_THREADS (default: std::thread::hardware_concurrency()).
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace tbb {
namespace shim {

inline int& tls_index() { static thread_local int idx = 0; return idx; }
inline bool& tls_busy() { static thread_local bool busy = false; return busy; }

class Pool {
public:
    static Pool& get() { static Pool p; return p; }
    int size() const { return n_; }

    // Runs fn(tid) once on every pool thread (the caller is tid 0) and waits.
    void run_all(const std::function<void(int)>& fn) {
        if (n_ == 1 || tls_busy()) { fn(tls_index()); return; }
        {
            std::unique_lock<std::mutex> lk(m_);
            job_ = &fn;
            pending_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        tls_busy() = true;
        fn(0);
        tls_busy() = false;
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

    ~Pool() {
        {
            std::unique_lock<std::mutex> lk(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

private:
    Pool() {
        int n = (int)std::thread::hardware_concurrency();
        if (const char* e = std::getenv("CGB_REF_THREADS")) n = std::atoi(e);
        if (n < 1) n = 1;
        int hw = (int)std::thread::hardware_concurrency();
        if (hw > 0 && n > hw) n = hw;  // the reference sizes per-thread state by hw concurrency
        n_ = n;
        for (int t = 1; t < n_; ++t) workers_.emplace_back([this, t] { loop(t); });
    }
    void loop(int tid) {
        tls_index() = tid;
        tls_busy() = true;
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
            }
            (*job)(tid);
            std::unique_lock<std::mutex> lk(m_);
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
    int n_ = 1;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* job_ = nullptr;
    int pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// Dynamic chunked loop over [first, last): every pool thread pulls chunks.
template <class I, class F>
void chunked(I first, I last, size_t grain, F&& body_chunk) {
    if (!(first < last)) return;
    const size_t n = (size_t)(last - first);
    Pool& p = Pool::get();
    if (p.size() == 1 || tls_busy() || n <= grain) { body_chunk(first, last); return; }
    size_t chunk = std::max<size_t>(grain, n / ((size_t)p.size() * 16));
    if (chunk == 0) chunk = 1;
    std::atomic<size_t> next{0};
    p.run_all([&](int) {
        for (;;) {
            size_t s = next.fetch_add(chunk);
            if (s >= n) break;
            size_t e = std::min(n, s + chunk);
            body_chunk((I)(first + (I)s), (I)(first + (I)e));
        }
    });
}

}  // namespace shim
}  // namespace tbb
