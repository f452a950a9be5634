#include "calig.h"

#include <algorithm>
#include <unistd.h>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>
#include <thread>
#include <unordered_map>

namespace cgb {

namespace {

// Workers wait on a generation counter: a job bumps it, and tasks are
// claimed from `claim_` = generation << 32 | next index by compare-and-swap,
// so a worker only ever claims tasks of the generation it woke for, while
// that generation is current.  Before a new job replaces (fn_, ntasks_), the
// old generation is closed in `claim_` (index field all ones); a late worker
// that reads the new ntasks_ is therefore ordered after the close and its
// compare-and-swap on the old value fails.  The caller takes tasks too and
// returns when every task has finished.  Workers spin briefly before
// sleeping, so back-to-back phases do not pay a wake-up.
class WorkerPool {
public:
    explicit WorkerPool(uint32_t n) {
        for (uint32_t i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~WorkerPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_.store(true, std::memory_order_relaxed);
            gen_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    void run(uint32_t n, const std::function<void(uint32_t)>& fn) {
        std::lock_guard<std::mutex> job(job_m_);
        const uint32_t g = (uint32_t)gen_.load(std::memory_order_relaxed) + 1u;
        claim_.store((uint64_t)(g - 1u) << 32 | kClosed, std::memory_order_relaxed);
        fn_ = &fn;
        ntasks_.store(n, std::memory_order_release);
        done_.store(0, std::memory_order_relaxed);
        {
            std::lock_guard<std::mutex> lk(m_);
            claim_.store((uint64_t)g << 32, std::memory_order_release);
            gen_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        work(g);
        while (done_.load(std::memory_order_acquire) < n) std::this_thread::yield();
    }
    static thread_local bool in_job;

private:
    std::vector<std::thread> workers_;
    std::mutex m_, job_m_;
    std::condition_variable cv_;
    std::atomic<uint64_t> gen_{0};
    std::atomic<uint64_t> claim_{0};
    std::atomic<uint32_t> done_{0};
    std::atomic<bool> stop_{false};
    std::atomic<uint32_t> ntasks_{0};
    const std::function<void(uint32_t)>* fn_ = nullptr;
    static constexpr uint32_t kClosed = 0xffffffffu;

    void work(uint32_t g) {
        in_job = true;
        for (;;) {
            uint64_t c = claim_.load(std::memory_order_acquire);
            if ((uint32_t)(c >> 32) != g || (uint32_t)c >= ntasks_.load(std::memory_order_acquire)) break;
            if (!claim_.compare_exchange_weak(c, c + 1, std::memory_order_acq_rel, std::memory_order_acquire))
                continue;
            (*fn_)((uint32_t)c);
            done_.fetch_add(1, std::memory_order_release);
        }
        in_job = false;
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            uint64_t g = gen_.load(std::memory_order_acquire);
            for (int spin = 0; g == seen && spin < 20000; ++spin) {
                std::this_thread::yield();
                g = gen_.load(std::memory_order_acquire);
            }
            if (g == seen) {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_.load(std::memory_order_acquire) != seen; });
                g = gen_.load(std::memory_order_acquire);
            }
            seen = g;
            if (stop_.load(std::memory_order_relaxed)) return;
            work((uint32_t)g);
        }
    }
};
thread_local bool WorkerPool::in_job = false;

WorkerPool& worker_pool() {
    static WorkerPool pool(std::max(1u, std::thread::hardware_concurrency()) - 1);
    return pool;
}
const pid_t g_pool_pid = getpid();  // a forked child has no workers: it runs jobs inline

// Whole-file reader + integer tokenizer (the reference streams with >>).
bool slurp(const std::string& path, std::vector<char>& buf) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize((size_t)sz + 1);
    size_t got = std::fread(buf.data(), 1, (size_t)sz, f);
    std::fclose(f);
    buf[got] = 0;
    buf.resize(got + 1);
    return true;
}

struct Tok {
    const char* p;
    const char* e;
    bool skip_ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
        return p < e && *p;
    }
    bool ch(char& c) {
        if (!skip_ws()) return false;
        c = *p++;
        return true;
    }
    bool num(long long& x) {
        if (!skip_ws()) return false;
        bool neg = false;
        if (*p == '-' || *p == '+') { neg = *p == '-'; ++p; }
        if (p >= e || *p < '0' || *p > '9') return false;
        long long v = 0;
        while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
        x = neg ? -v : v;
        return true;
    }
};

// The C library's rand() from its default state (seed 1, no srand call):
// glibc's additive feedback generator of degree 31 and separation 3.  The
// state r[0..30] comes from the Lehmer sequence r[i] = 16807 r[i-1] mod
// (2^31 - 1) started at the seed; r[31..33] repeat r[0..2]; afterwards
// r[i] = r[i-31] + r[i-3] (mod 2^32) and the k-th output is r[k+344] >> 1.
// Restated from the published description of the generator so the label
// sequence does not depend on other users of rand() in the process.
class LibcRand {
public:
    LibcRand() {
        int32_t r[34];
        r[0] = 1;
        for (int i = 1; i < 31; ++i) {
            const int64_t v = (16807LL * r[i - 1]) % 2147483647LL;
            r[i] = (int32_t)(v < 0 ? v + 2147483647LL : v);
        }
        for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
        for (int i = 0; i < 34; ++i) ring_[i % 34] = (uint32_t)r[i];
        n_ = 34;
        for (int i = 34; i < 344; ++i) step();
    }
    int next() { return (int)(step() >> 1); }

private:
    uint32_t ring_[34];
    uint64_t n_ = 0;  // index of the next value r[n_]
    uint32_t step() {
        const uint32_t v = ring_[(n_ - 31) % 34] + ring_[(n_ - 3) % 34];
        ring_[n_ % 34] = v;
        ++n_;
        return v;
    }
};

inline bool sorted_insert(std::vector<uint32_t>& v, uint32_t x) {
    auto it = std::lower_bound(v.begin(), v.end(), x);
    if (it != v.end() && *it == x) return false;
    v.insert(it, x);
    return true;
}

inline bool sorted_erase(std::vector<uint32_t>& v, uint32_t x) {
    auto it = std::lower_bound(v.begin(), v.end(), x);
    if (it == v.end() || *it != x) return false;
    v.erase(it);
    return true;
}
inline bool sorted_has(const std::vector<uint32_t>& v, uint32_t x) {
    return std::binary_search(v.begin(), v.end(), x);
}

// First index p >= r of the ascending d[0..n) with d[p] >= x, found by
// galloping from r (exponential steps, then a binary search).
inline size_t gallop_lb(const uint32_t* d, size_t n, size_t r, uint32_t x) {
    size_t lo = r, hi = r, step = 1;
    while (hi < n && d[hi] < x) {
        lo = hi + 1;
        hi += step;
        step <<= 1;
    }
    if (hi > n) hi = n;
    return (size_t)(std::lower_bound(d + lo, d + hi, x) - d);
}

// Adds the ascending values x[0..k) to the sorted set L: the result is the
// set union, as k sorted_insert calls give (a hub's list takes many values
// per batch; one memmove each would be quadratic).  Each value's insertion
// point is found by galloping from the previous one; then L grows once and
// the old stretches between the points move right with memmove, from the
// back, so a long list that gains a few values is not walked element by
// element.
void insert_run(std::vector<uint32_t>& L, const uint32_t* x, size_t k) {
    if (k == 1) { sorted_insert(L, x[0]); return; }
    thread_local std::vector<size_t> pos;
    thread_local std::vector<uint32_t> val;
    pos.clear();
    val.clear();
    const size_t n = L.size();
    size_t r = 0;
    for (size_t j = 0; j < k; ++j) {
        if (j && x[j] == x[j - 1]) continue;
        const size_t p = gallop_lb(L.data(), n, r, x[j]);
        r = p;
        if (p < n && L[p] == x[j]) continue;
        pos.push_back(p);
        val.push_back(x[j]);
    }
    if (pos.empty()) return;
    const size_t m = pos.size();
    L.resize(n + m);
    uint32_t* d = L.data();
    // old entries [pos[i], end) have i + 1 new values before them
    size_t end = n;
    for (size_t i = m; i-- > 0;) {
        const size_t p = pos[i];
        if (end > p) std::memmove(d + p + i + 1, d + p, (end - p) * sizeof(uint32_t));
        d[p + i] = val[i];
        end = p;
    }
}

// Removes the ascending distinct values x[0..k) from the sorted set L;
// hit[i] = 1 when x[i] was present (what sorted_erase would return).  Each
// value is found by galloping from the previous one and the kept stretches
// between them move left with memmove.
void erase_run(std::vector<uint32_t>& L, const uint32_t* x, size_t k, uint8_t* hit) {
    if (k == 1) { hit[0] = sorted_erase(L, x[0]); return; }
    uint32_t* d = L.data();
    const size_t n = L.size();
    size_t r = 0, w = 0;
    for (size_t j = 0; j < k; ++j) {
        const size_t p = gallop_lb(d, n, r, x[j]);
        if (p > r) {
            if (w != r) std::memmove(d + w, d + r, (p - r) * sizeof(uint32_t));
            w += p - r;
        }
        r = p;
        if (p < n && d[p] == x[j]) { hit[j] = 1; ++r; }
        else hit[j] = 0;
    }
    if (n > r) {
        if (w != r) std::memmove(d + w, d + r, (n - r) * sizeof(uint32_t));
        w += n - r;
    }
    L.resize(w);
}

// Thread that owns data vertex v among T: a multiplicative hash, since
// R-MAT-like ids concentrate degree on ids with many zero bits (v % T would
// hand most of the work to thread 0).
inline uint32_t owner(uint32_t v, uint32_t T) {
    return (uint32_t)(((uint64_t)(v * 0x9E3779B1u) * T) >> 32);
}

template <typename T>
void concat(std::vector<T>& dst, std::vector<std::vector<T>>& parts) {
    size_t n = dst.size();
    for (auto& p : parts) n += p.size();
    dst.reserve(n);
    for (auto& p : parts) dst.insert(dst.end(), p.begin(), p.end());
}

// LSD radix sort of keys by their low `bits` bits, 11 bits per pass.
void radix_sort(std::vector<uint64_t>& a, int bits) {
    std::vector<uint64_t> b(a.size());
    std::vector<size_t> cnt(2049);
    for (int shift = 0; shift < bits; shift += 11) {
        std::fill(cnt.begin(), cnt.end(), 0);
        for (uint64_t x : a) ++cnt[((x >> shift) & 2047) + 1];
        for (int i = 0; i < 2048; ++i) cnt[i + 1] += cnt[i];
        for (uint64_t x : a) b[cnt[(x >> shift) & 2047]++] = x;
        a.swap(b);
    }
}

// LSD radix sort of a[0..n) by the low `bits` bits, 11 bits per pass, with
// buf[0..n) as scratch; the result is left in a.
void radix_sort_range(uint64_t* a, uint64_t* buf, size_t n, int bits) {
    size_t cnt[2049];
    uint64_t *src = a, *dst = buf;
    for (int shift = 0; shift < bits; shift += 11) {
        std::fill(cnt, cnt + 2049, 0);
        for (size_t i = 0; i < n; ++i) ++cnt[((src[i] >> shift) & 2047) + 1];
        for (int i = 0; i < 2048; ++i) cnt[i + 1] += cnt[i];
        for (size_t i = 0; i < n; ++i) dst[cnt[(src[i] >> shift) & 2047]++] = src[i];
        std::swap(src, dst);
    }
    if (src != a) std::copy(src, src + n, a);
}

// Sorts a task queue by (v, u) and drops repeats.  Repeated tasks in the
// reference's queues only redo inserts that fail and checks guarded by the
// checked bit, so processing each distinct task once yields the same index
// and deltas.  Keys v << 5 | u (query vertices < 32), radix-sorted.  With
// T > 1 threads the keys are split by their top (up to) 11 bits into ranges,
// counted and scattered by T slices, and each range is sorted and
// deduplicated on its own: many more ranges than threads, so the ranges of
// low ids that skewed graphs crowd do not serialise the sort.
template <typename Q>
void dedupe(std::vector<Q>& q, uint32_t T) {
    const size_t n = q.size();
    if (n < 2) return;
    std::vector<uint64_t> key(n);
    if (T <= 1) {
        uint64_t top = 0;
        for (size_t i = 0; i < n; ++i) {
            key[i] = (uint64_t)q[i].v << 5 | q[i].u;
            top |= key[i];
        }
        radix_sort(key, 64 - __builtin_clzll(top | 1));
        key.erase(std::unique(key.begin(), key.end()), key.end());
        q.resize(key.size());
        for (size_t i = 0; i < key.size(); ++i) q[i] = {(uint32_t)(key[i] & 31u), (uint32_t)(key[i] >> 5)};
        return;
    }
    std::vector<uint64_t> tops(T, 0);
    run_threads(T, [&](uint32_t s) {
        uint64_t top = 0;
        for (size_t i = n * s / T; i < n * (s + 1) / T; ++i) {
            key[i] = (uint64_t)q[i].v << 5 | q[i].u;
            top |= key[i];
        }
        tops[s] = top;
    });
    uint64_t top = 0;
    for (uint64_t t : tops) top |= t;
    const int bits = 64 - __builtin_clzll(top | 1);
    const int hb = std::min(bits, 11), shift = bits - hb;
    const size_t B = (size_t)1 << hb;
    std::vector<size_t> at((size_t)T * B, 0);  // [slice * B + range]: count, then write position
    run_threads(T, [&](uint32_t s) {
        size_t* c = &at[(size_t)s * B];
        for (size_t i = n * s / T; i < n * (s + 1) / T; ++i) ++c[key[i] >> shift];
    });
    std::vector<size_t> rs(B + 1);  // range starts
    size_t run = 0;
    for (size_t r = 0; r < B; ++r) {
        rs[r] = run;
        for (uint32_t s = 0; s < T; ++s) {
            const size_t c = at[(size_t)s * B + r];
            at[(size_t)s * B + r] = run;
            run += c;
        }
    }
    rs[B] = run;
    std::vector<uint64_t> tmp(n);
    run_threads(T, [&](uint32_t s) {
        size_t* w = &at[(size_t)s * B];
        for (size_t i = n * s / T; i < n * (s + 1) / T; ++i) tmp[w[key[i] >> shift]++] = key[i];
    });
    // ranges in groups of 16 per task; keys of one range agree above `shift`
    constexpr size_t G = 16;
    const uint32_t ntask = (uint32_t)((B + G - 1) / G);
    std::vector<size_t> uniq(B);
    run_threads(ntask, [&](uint32_t g) {
        for (size_t r = g * G; r < std::min(B, (g + 1) * G); ++r) {
            uint64_t* a = tmp.data() + rs[r];
            const size_t m = rs[r + 1] - rs[r];
            if (m < 64) std::sort(a, a + m);
            else radix_sort_range(a, key.data() + rs[r], m, shift);
            uniq[r] = (size_t)(std::unique(a, a + m) - a);
        }
    });
    std::vector<size_t> uo(B + 1, 0);
    for (size_t r = 0; r < B; ++r) uo[r + 1] = uo[r] + uniq[r];
    q.resize(uo[B]);
    run_threads(ntask, [&](uint32_t g) {
        for (size_t r = g * G; r < std::min(B, (g + 1) * G); ++r)
            for (size_t j = 0; j < uniq[r]; ++j) {
                const uint64_t x = tmp[rs[r] + j];
                q[uo[r] + j] = {(uint32_t)(x & 31u), (uint32_t)(x >> 5)};
            }
    });
}

}  // namespace

void pool_run(uint32_t n, const std::function<void(uint32_t)>& fn) {
    if (n <= 1 || WorkerPool::in_job || getpid() != g_pool_pid) {
        for (uint32_t k = 0; k < n; ++k) fn(k);
        return;
    }
    worker_pool().run(n, fn);
}

// calig.cpp:111-164: 'v id label' lines (label -1 -> 0), then 'e a b label'.
std::string CaLiGIndex::load_query(const std::string& path) {
    std::vector<char> buf;
    if (!slurp(path, buf)) return "cannot open query file " + path;
    Tok t{buf.data(), buf.data() + buf.size() - 1};
    qlabel_.clear();
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    char c;
    long long a, b, l;
    while (t.ch(c)) {
        if (c == 'v') {
            if (!t.num(a) || !t.num(l)) return "bad query vertex line";
            if (l == -1) l = 0;
            qlabel_.push_back((int)l);
        } else if (c == 'e') {
            if (!t.num(a) || !t.num(b) || !t.num(l)) return "bad query edge line";
            edges.emplace_back((uint32_t)a, (uint32_t)b);
        } else {
            // other record types ('t ...'): skip the rest of the line
            while (t.p < t.e && *t.p != '\n') ++t.p;
        }
    }
    qn_ = (uint32_t)qlabel_.size();
    if (qn_ == 0 || qn_ > 32) return "query must have 1..32 vertices";
    qnei_.assign(qn_, {});
    for (auto& [x, y] : edges) {
        if (x >= qn_ || y >= qn_) return "query edge out of range";
        sorted_insert(qnei_[x], y);
        sorted_insert(qnei_[y], x);
    }
    // dense label slots for the query's labels (calig.cpp:144-163 labels map)
    std::unordered_map<int, int> slot;
    qlist_.clear();
    for (uint32_t u = 0; u < qn_; ++u) {
        auto it = slot.find(qlabel_[u]);
        if (it == slot.end()) {
            slot[qlabel_[u]] = (int)qlist_.size();
            qlist_.push_back({});
        }
        qlist_[slot[qlabel_[u]]].push_back(u);
    }
    int maxl = 0;
    for (int l2 : qlabel_) maxl = std::max(maxl, l2);
    label_slot_.assign((size_t)maxl + 1, -1);
    for (auto& [l2, s] : slot) label_slot_[l2] = s;
    // per ui: block offset of its lists inside a vertex block of its label
    block_off_.assign(qn_, 0);
    block_size_.assign(qlist_.size(), 0);
    for (size_t s = 0; s < qlist_.size(); ++s) {
        uint32_t off = 0;
        for (uint32_t u : qlist_[s]) { block_off_[u] = off; off += (uint32_t)qnei_[u].size(); }
        block_size_[s] = off;
    }
    npos_.assign((size_t)qn_ * qn_, -1);
    for (uint32_t u = 0; u < qn_; ++u)
        for (size_t k = 0; k < qnei_[u].size(); ++k) npos_[u * qn_ + qnei_[u][k]] = (int)k;
    // rep_nei: neighbour groups sharing a label, size > 1 (calig.cpp:145-162)
    rep_.assign(qn_, {});
    rep_of_label_.assign(qn_, std::vector<int>(qlist_.size(), -1));
    for (uint32_t u = 0; u < qn_; ++u) {
        std::vector<std::vector<uint32_t>> by(qlist_.size());
        for (uint32_t w : qnei_[u]) by[label_slot_[qlabel_[w]]].push_back(w);
        for (size_t s = 0; s < by.size(); ++s)
            if (by[s].size() > 1) {
                rep_of_label_[u][s] = (int)rep_[u].size();
                rep_[u].push_back(by[s]);
            }
    }
    return "";
}

// calig.cpp:166-216: vertices with labels outside the query are pruned (-1);
// edges are kept only between unpruned vertices that existed at the first edge.
std::string CaLiGIndex::load_graph(const std::string& path) {
    std::vector<char> buf;
    if (!slurp(path, buf)) return "cannot open graph file " + path;
    Tok t{buf.data(), buf.data() + buf.size() - 1};
    glabel_.clear();
    char c;
    long long a, b, l;
    size_t gsize = 0;
    bool edges_started = false;
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    while (t.ch(c)) {
        if (!edges_started && c == 'v') {
            if (!t.num(a) || !t.num(l)) return "bad vertex line";
            while ((long long)glabel_.size() < a) glabel_.push_back(-1);
            int s = (l >= 0 && (size_t)l < label_slot_.size()) ? label_slot_[l] : -1;
            glabel_.push_back(s);
        } else {
            if (!edges_started) { edges_started = true; gsize = glabel_.size(); }
            if (!t.num(a) || !t.num(b) || !t.num(l)) break;
            if (a >= 0 && b >= 0 && (size_t)a < gsize && (size_t)b < gsize && glabel_[a] >= 0 && glabel_[b] >= 0)
                edges.emplace_back((uint32_t)a, (uint32_t)b);
        }
    }
    const uint32_t n = (uint32_t)glabel_.size();
    std::vector<uint32_t> deg(n, 0);
    for (auto& [x, y] : edges) { deg[x]++; deg[y]++; }
    nei_.assign(n, {});
    for (uint32_t v = 0; v < n; ++v) nei_[v].reserve(deg[v]);
    for (auto& [x, y] : edges) { nei_[x].push_back(y); nei_[y].push_back(x); }
    for (auto& v : nei_) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    li_.assign(n, 0);
    checked_.assign(n, 0);
    return "";
}

std::string CaLiGIndex::load_graph_bin(const std::string& prefix) {
    std::ifstream meta(prefix + ".meta.txt");
    if (!meta) return "cannot open " + prefix + ".meta.txt";
    uint64_t n_edges = 0;
    uint32_t n = 0, vsize = 0, esize = 0, vlbl = 0, elbl = 0, maxdeg = 0, feat = 0, nvcls = 0, necls = 0;
    meta >> n >> n_edges >> vsize >> esize >> vlbl >> elbl >> maxdeg >> feat >> nvcls >> necls;
    if (!meta) return "bad meta file " + prefix + ".meta.txt";
    if (vsize != 4 || esize != 8) return "unsupported id sizes in meta (expected vertex 4, edge 8)";
    if (nvcls == 0) return "meta gives zero vertex classes";
    std::vector<uint64_t> row(n + 1ull, 0);
    FILE* f = std::fopen((prefix + ".vertex.bin").c_str(), "rb");
    if (!f) return "cannot open " + prefix + ".vertex.bin";
    const size_t got_r = std::fread(row.data(), sizeof(uint64_t), row.size(), f);
    std::fclose(f);
    if (got_r != row.size()) return "short read of " + prefix + ".vertex.bin";
    std::vector<uint32_t> adj(n_edges, 0);
    f = std::fopen((prefix + ".edge.bin").c_str(), "rb");
    if (!f) return "cannot open " + prefix + ".edge.bin";
    const size_t got_e = n_edges ? std::fread(adj.data(), sizeof(uint32_t), adj.size(), f) : 0;
    std::fclose(f);
    if (got_e != adj.size()) return "short read of " + prefix + ".edge.bin";
    for (uint32_t v = 0; v < n; ++v)
        if (row[v] > row[v + 1] || row[v + 1] > n_edges) return "row pointers out of order or range";
    LibcRand rnd;
    glabel_.assign(n, -1);
    for (uint32_t v = 0; v < n; ++v) {
        const int lb = rnd.next() % (int)nvcls;
        glabel_[v] = (size_t)lb < label_slot_.size() ? label_slot_[lb] : -1;
    }
    // an edge is an update edge iff hash(min, max) % 10 == 0; each such
    // pair is listed once, from its smaller endpoint's row, as (max, min)
    auto is_update = [](uint32_t a, uint32_t b) {
        const uint64_t key = ((uint64_t)std::min(a, b) << 32) | std::max(a, b);
        return (key * 0x9e3779b97f4a7c15ULL) % 10ULL == 0;
    };
    nei_.assign(n, {});
    std::vector<int> upd;
    for (uint32_t v = 0; v < n; ++v) {
        auto& nv = nei_[v];
        for (uint64_t i = row[v]; i < row[v + 1]; ++i) {
            const uint32_t u = adj[i];
            if (is_update(v, u)) {
                if (v < u) { upd.push_back((int)u); upd.push_back((int)v); }
            } else {
                nv.push_back(u);
            }
        }
        std::sort(nv.begin(), nv.end());
        nv.erase(std::unique(nv.begin(), nv.end()), nv.end());
    }
    const size_t pairs = upd.size() / 2;
    std::vector<int> idx(pairs);
    std::iota(idx.begin(), idx.end(), 0);
    std::mt19937 rng(42);
    std::shuffle(idx.begin(), idx.end(), rng);
    update_.assign(upd.size(), 0);
    for (size_t i = 0; i < pairs; ++i) {
        update_[2 * i] = upd[2 * (size_t)idx[i]];
        update_[2 * i + 1] = upd[2 * (size_t)idx[i] + 1];
    }
    li_.assign(n, 0);
    checked_.assign(n, 0);
    return "";
}

// calig.cpp:719-733: "<char> v1 v2 w" per line.
std::string CaLiGIndex::load_updates(const std::string& path) {
    std::vector<char> buf;
    if (!slurp(path, buf)) return "cannot open update file " + path;
    Tok t{buf.data(), buf.data() + buf.size() - 1};
    update_.clear();
    char c;
    long long a, b, w;
    while (t.ch(c) && t.num(a) && t.num(b) && t.num(w)) {
        update_.push_back((int)a);
        update_.push_back((int)b);
    }
    return "";
}

const std::vector<uint32_t>* CaLiGIndex::cand(uint32_t v, uint32_t ui, uint32_t uj) const {
    if (v >= glabel_.size() || ui >= qn_ || uj >= qn_) return nullptr;
    if (!(glabel_[v] >= 0 && glabel_[v] == label_slot_[qlabel_[ui]])) return nullptr;
    int p = npos_[ui * qn_ + uj];
    if (p < 0) return nullptr;
    return &lists_[cbase_[v] + block_off_[ui] + (uint32_t)p];
}

void CaLiGIndex::set_threads(uint32_t n) {
    if (n == 0) n = std::max(1u, std::thread::hardware_concurrency());
    threads_ = std::min<uint32_t>(n, 64);
    // CGB_PRODUCER_MIN_PARALLEL: the smallest phase (items, pairs or tasks)
    // that runs on threads; smaller ones run inline.  Default 4096.
    if (const char* e = std::getenv("CGB_PRODUCER_MIN_PARALLEL")) par_min_ = std::strtoull(e, nullptr, 10);
}

void EdgeSet::reset(size_t max_edges) {
    size_t cap = 1024;
    while (cap < max_edges + max_edges / 2) cap <<= 1;
    slots_.assign(cap, kEmpty);
    bits_ = __builtin_ctzll(cap);
    count_ = 0;
}

void EdgeSet::reserve(size_t more) {
    if ((count_ + more) * 4 <= slots_.size() * 3) return;
    std::vector<uint64_t> old;
    old.swap(slots_);
    reset(count_ + more);
    for (uint64_t k : old)
        if (k != kEmpty) insert((uint32_t)(k >> 32), (uint32_t)k);
}

bool EdgeSet::has(uint32_t a, uint32_t b) const {
    const uint64_t k = key(a, b);
    for (size_t i = slot(k);; i = (i + 1) & (slots_.size() - 1)) {
        const uint64_t s = __atomic_load_n(&slots_[i], __ATOMIC_RELAXED);
        if (s == k) return true;
        if (s == kEmpty) return false;
    }
}

void EdgeSet::insert(uint32_t a, uint32_t b) {
    const uint64_t k = key(a, b);
    for (size_t i = slot(k);; i = (i + 1) & (slots_.size() - 1)) {
        uint64_t s = __atomic_load_n(&slots_[i], __ATOMIC_RELAXED);
        if (s == k) return;
        if (s == kEmpty) {
            if (__atomic_compare_exchange_n(&slots_[i], &s, k, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                __atomic_fetch_add(&count_, 1, __ATOMIC_RELAXED);
                return;
            }
            if (s == k) return;  // another thread put the same key here
        }
    }
}

// calig.cpp:325-356 constructCand, then 705-717 staticFilter.  Vertices are
// independent in both (each writes its own lists and LI), so they run on
// slices of the vertex range.
void CaLiGIndex::construct() {
    const uint32_t n = (uint32_t)glabel_.size();
    cbase_.assign(n + 1, 0);
    uint64_t total = 0;
    size_t adj = 0;
    for (uint32_t v = 0; v < n; ++v) {
        cbase_[v] = total;
        if (glabel_[v] >= 0) total += block_size_[glabel_[v]];
        adj += nei_[v].size();
    }
    cbase_[n] = total;
    lists_.assign(total, {});
    edges_.reset(adj / 2 + update_.size() / 2);
    li_.assign(n, 0);
    words_ = (n + 63) / 64;
    litbits_.assign((size_t)qn_ * words_, 0);
    const uint32_t T = n >= par_min_ ? threads_ : 1u;
    std::vector<std::vector<Task>> delp(T);
    run_threads(T, [&](uint32_t s) {
        const uint32_t v0 = (uint32_t)((uint64_t)n * s / T), v1 = (uint32_t)((uint64_t)n * (s + 1) / T);
        for (uint32_t v = v0; v < v1; ++v) {
            checked_[v] = 0;
            for (uint32_t y : nei_[v])
                if (v <= y) edges_.insert(v, y);
            const int sl = glabel_[v];
            if (sl < 0) continue;
            for (uint32_t ui : qlist_[sl]) {
                for (uint32_t vj : nei_[v]) {
                    const int lj = glabel_[vj];
                    if (lj < 0) continue;
                    for (uint32_t uj : qnei_[ui])
                        if (label_slot_[qlabel_[uj]] == lj) C(v, ui, uj).push_back(vj);  // nei_ sorted -> lists sorted
                }
                light(v, ui);
            }
        }
        // staticFilter: turnOff every lit (v, ui) failing checkNei (v's own lists only)
        for (uint32_t v = v0; v < v1; ++v) {
            const int sl = glabel_[v];
            if (sl < 0) continue;
            for (uint32_t ui : qlist_[sl]) {
                if (!lit(v, ui)) continue;
                if (!check_nei(v, ui)) {
                    unlight(v, ui);
                    delp[s].push_back({ui, v});
                }
            }
        }
    });
    std::vector<std::vector<uint32_t>>().swap(nei_);
    // then delAndCheck to the fix-point
    std::vector<Task> del;
    concat(del, delp);
    delta_del.clear();
    while (!del.empty()) del_and_check(del);
    delta_del.clear();
}

// calig.cpp:358-408
bool CaLiGIndex::try_nei(uint32_t v, uint32_t u, const std::vector<uint32_t>& group, size_t th,
                         std::vector<uint32_t>& used) {
    if (th == group.size()) return true;
    const uint32_t uj = group[th];
    for (uint32_t vj : C(v, u, uj)) {
        if (std::find(used.begin(), used.end(), vj) != used.end()) continue;
        used.push_back(vj);
        if (try_nei(v, u, group, th + 1, used)) return true;
        used.pop_back();
    }
    return false;
}

bool CaLiGIndex::check_nei(uint32_t v, uint32_t u) {
    for (uint32_t uj : qnei_[u])
        if (C(v, u, uj).empty()) return false;
    for (auto& g : rep_[u]) {
        std::vector<uint32_t> used;
        if (!try_nei(v, u, g, 0, used)) return false;
    }
    return true;
}

// Both fix-points below run on threads_ threads (large rounds), thread k
// owning every data vertex v with owner(v, T) == k: the candidate lists of v,
// its LI and checked bits.  A round first scans the task queue read-only in
// T slices of equal item count, thread s dropping each item into the bucket
// of its target vertex's owner; then each owner takes its buckets in
// slice order (so it sees its items in the reference's queue order) and
// edits only the lists it owns.  The sequential round reads the pre-round
// lists and LI while building its work list, and its set results (list
// contents, deltas, the next queue) do not depend on the order of the edits;
// the one order-dependent step — which same-label group a checked (u, v) is
// tested against — depends on the order of v's own items only, which the
// owner keeps.

// The items of a round are the entries of the lists C(t.v, t.u, uj) of every
// task t and every uj in qnei_[t.u], in queue order.  item_offsets() sets
// first[i] to the index of task i's first item (first[n] = the item count,
// returned); scan_items() visits items [lo, hi) in order, so T threads can
// take equal shares even when one hub task holds most of a round.
size_t CaLiGIndex::item_offsets(const std::vector<Task>& q, std::vector<size_t>& first) {
    // the list headers are cache misses: counts in T index slices, then one
    // prefix pass over the tasks
    const uint32_t n = (uint32_t)q.size();
    const uint32_t T = n >= par_min_ / 8 ? threads_ : 1u;
    first.resize((size_t)n + 1);
    first[0] = 0;
    run_threads(T, [&](uint32_t s) {
        for (uint32_t i = (uint32_t)((uint64_t)n * s / T); i < (uint32_t)((uint64_t)n * (s + 1) / T); ++i) {
            size_t c = 0;
            for (uint32_t uj : qnei_[q[i].u]) c += C(q[i].v, q[i].u, uj).size();
            first[(size_t)i + 1] = c;
        }
    });
    for (uint32_t i = 0; i < n; ++i) first[(size_t)i + 1] += first[i];
    return first[n];
}

template <class Fn>
void CaLiGIndex::scan_items(const std::vector<Task>& q, const std::vector<size_t>& first, size_t lo, size_t hi,
                            Fn&& fn) {
    if (lo >= hi) return;
    size_t i = (size_t)(std::upper_bound(first.begin(), first.end(), lo) - first.begin()) - 1;
    for (size_t at = lo; at < hi && i < q.size(); ++i) {
        const Task& t = q[i];
        size_t base = first[i];
        for (uint32_t uj : qnei_[t.u]) {
            if (at >= hi) break;
            const auto& L = C(t.v, t.u, uj);
            const size_t len = L.size();
            if (base + len > at) {
                const size_t end = std::min(hi, base + len);
                for (size_t p = at - base; base + p < end; ++p) fn((uint32_t)i, t, uj, L[p]);
                at = end;
            }
            base += len;
        }
    }
}

// calig.cpp:410-475 delAndCheck (one round; `del` becomes the next round).
void CaLiGIndex::del_and_check(std::vector<Task>& del) {
    dedupe(del, del.size() >= par_min_ / 8 ? threads_ : 1u);
    std::vector<size_t> first;
    const size_t total = item_offsets(del, first);
    const uint32_t T = total >= par_min_ ? threads_ : 1u;
    struct Item { uint64_t list; uint32_t vi, vj, ui, uj; };
    std::vector<std::vector<Item>> items((size_t)T * T);  // [slice * T + owner]
    run_threads(T, [&](uint32_t s) {
        scan_items(del, first, total * s / T, total * (s + 1) / T,
                   [&](uint32_t, const Task& t, uint32_t uj, uint32_t vj) {
                       if (lit(vj, uj))
                           items[(size_t)s * T + owner(vj, T)].push_back({list_index(vj, uj, t.u), t.v, vj, t.u, uj});
                   });
    });
    struct Chk { uint32_t u, v; int group; };
    std::vector<std::vector<Task>> next(T);
    std::vector<std::vector<DeltaOp>> erased(T);
    run_threads(T, [&](uint32_t k) {
        std::vector<Item> it;
        for (uint32_t s = 0; s < T; ++s) {
            auto& b = items[(size_t)s * T + k];
            it.insert(it.end(), b.begin(), b.end());
            std::vector<Item>().swap(b);
        }
        // erase each list's values in one pass; a list that ends empty turns
        // its (uj, vj) off (the sequential round sees it empty at its last
        // item; earlier items' group checks of a vertex that ends off change
        // nothing)
        // Group the items by list.  Within a list they arrive in ascending
        // vi (the queue is sorted by vertex and the slices keep its order),
        // so (list, item) keys, packed into one word when they fit, order
        // every group by value as erase_run needs.
        std::vector<uint32_t> ord(it.size());
        const int ib = std::max(1, 64 - __builtin_clzll((unsigned long long)it.size() | 1ull));
        if (lists_.size() < (1ull << (64 - ib))) {
            std::vector<uint64_t> key(it.size());
            for (size_t i = 0; i < it.size(); ++i) key[i] = it[i].list << ib | i;
            radix_sort(key, ib + (64 - __builtin_clzll((unsigned long long)lists_.size() | 1ull)));
            for (size_t i = 0; i < it.size(); ++i) ord[i] = (uint32_t)(key[i] & ((1ull << ib) - 1));
        } else {
            std::iota(ord.begin(), ord.end(), 0u);
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return it[a].list < it[b].list; });
        }
        std::vector<uint8_t> ends_empty(it.size()), hit;
        std::vector<uint32_t> vals;
        // group starts, so that the lists a few groups ahead are prefetched
        // (header 8 groups ahead, then its words 4 ahead)
        std::vector<uint32_t> gs;
        for (size_t q = 0; q < ord.size(); ++q)
            if (q == 0 || it[ord[q]].list != it[ord[q - 1]].list) gs.push_back((uint32_t)q);
        gs.push_back((uint32_t)ord.size());
        const size_t ngr = gs.size() - 1;
        for (size_t g = 0; g < ngr; ++g) {
            if (g + 8 < ngr) __builtin_prefetch(&lists_[it[ord[gs[g + 8]]].list]);
            if (g + 4 < ngr) {
                const auto& Lp = lists_[it[ord[gs[g + 4]]].list];
                if (!Lp.empty()) __builtin_prefetch(Lp.data() + Lp.size() / 2);
            }
            const size_t g0 = gs[g], g1 = gs[g + 1];
            vals.clear();
            for (size_t q = g0; q < g1; ++q) vals.push_back(it[ord[q]].vi);
            hit.assign(vals.size(), 0);
            auto& L = lists_[it[ord[g0]].list];
            erase_run(L, vals.data(), vals.size(), hit.data());
            for (size_t q = g0; q < g1; ++q) {
                const Item& e = it[ord[q]];
                if (hit[q - g0]) erased[k].push_back({e.vj, e.vi, e.uj, e.ui});
                ends_empty[ord[q]] = L.empty();
            }
        }
        std::vector<Chk> chk;
        for (size_t i = 0; i < it.size(); ++i) {
            const Item& e = it[i];
            if (ends_empty[i]) {
                unlight(e.vj, e.uj);
                next[k].push_back({e.uj, e.vj});
            } else {
                const int g = rep_of_label_[e.uj][label_slot_[qlabel_[e.ui]]];
                if (g >= 0) {
                    chk.push_back({e.uj, e.vj, g});
                    checked_[e.vj] &= ~(1u << e.uj);
                }
            }
        }
        for (auto& c : chk) {
            if ((checked_[c.v] >> c.u) & 1u) continue;
            checked_[c.v] |= 1u << c.u;
            std::vector<uint32_t> used;
            if (!try_nei(c.v, c.u, rep_[c.u][c.group], 0, used)) {
                unlight(c.v, c.u);
                next[k].push_back({c.u, c.v});
            }
        }
    });
    concat(delta_del, erased);
    del.clear();
    concat(del, next);
}

// calig.cpp:536-638 addAndCheck (one round; `add` becomes the next round).
//
// Each item of a task (ui, vi) inserts vi into (vj, uj -> ui)'s list for
// every vj in vi's (ui -> uj) list.  `settled` holds tasks whose (ui, vi)
// was lit before the batch: their inserts all find vi present, so only
// their unlit neighbours are collected.  Why: call vj in C(vi, ui, uj) with
// vi missing from C(vj, uj, ui) an asymmetry of (ui, vi).  The lists start
// symmetric (both hold the data edge); new edges insert both orientations;
// an insert of vj into C(vi, ui, uj) by a task (uj, vj) comes from vi in
// C(vj, uj, ui); erasing vj from vi's lists removes entries only.  The one
// step that creates an asymmetry of (ui, vi) is the erasure of vi by its
// own deletion, which turns (ui, vi) off; it comes back on only by an
// activation, whose task re-inserts vi into every list its own lists name.
// So a pair that stayed lit has none.  Tasks in `add` (activations) are
// looked up item by item, and the misses are inserted; a (list, value) pair
// occurs once per round (tasks are distinct), so each is inserted once.
void CaLiGIndex::add_and_check(std::vector<Task>& add, std::vector<Task>& settled,
                               std::vector<Task>& add_del, std::vector<Task>& activated) {
    dedupe(add, add.size() >= par_min_ / 8 ? threads_ : 1u);
    dedupe(settled, settled.size() >= par_min_ / 8 ? threads_ : 1u);
    // one queue: activations first, then the settled tasks
    const size_t nfresh = add.size();
    add.insert(add.end(), settled.begin(), settled.end());
    settled.clear();
    std::vector<size_t> first;
    const size_t total = item_offsets(add, first);
    const uint32_t T = total >= par_min_ ? threads_ : 1u;
    struct Ins { uint64_t list; uint32_t vi, vj, ui, uj; };
    std::vector<std::vector<Ins>> ins((size_t)T * T);     // [slice * T + owner]
    std::vector<std::vector<Task>> check((size_t)T * T);
    run_threads(T, [&](uint32_t s) {
        scan_items(add, first, total * s / T, total * (s + 1) / T,
                   [&](uint32_t i, const Task& t, uint32_t uj, uint32_t vj) {
                       const size_t b = (size_t)s * T + owner(vj, T);
                       if (i < nfresh) ins[b].push_back({list_index(vj, uj, t.u), t.v, vj, t.u, uj});
                       if (!lit(vj, uj)) check[b].push_back({uj, vj});
                   });
    });
    std::vector<std::vector<Task>> next(T), act(T), drop(T);
    std::vector<std::vector<DeltaOp>> added(T);
    run_threads(T, [&](uint32_t k) {
        // Lookups: dependent cache misses (list header, then list words), run
        // in groups whose next lines are prefetched for the whole group.
        std::vector<Ins> miss;
        constexpr size_t kGroup = 16;
        for (uint32_t s = 0; s < T; ++s) {
            const auto& b = ins[(size_t)s * T + k];
            for (size_t g0 = 0; g0 < b.size(); g0 += kGroup) {
                const size_t g1 = std::min(b.size(), g0 + kGroup);
                for (size_t i = g0; i < g1; ++i) __builtin_prefetch(&lists_[b[i].list]);
                for (size_t i = g0; i < g1; ++i) {
                    const auto& L = lists_[b[i].list];
                    if (!L.empty()) __builtin_prefetch(L.data() + L.size() / 2);
                }
                for (size_t i = g0; i < g1; ++i)
                    if (!sorted_has(lists_[b[i].list], b[i].vi)) miss.push_back(b[i]);
            }
        }
        std::sort(miss.begin(), miss.end(), [](const Ins& a, const Ins& b) {
            return a.list != b.list ? a.list < b.list : a.vi < b.vi;
        });
        std::vector<uint32_t> vals;
        for (size_t g0 = 0; g0 < miss.size();) {
            size_t g1 = g0 + 1;
            while (g1 < miss.size() && miss[g1].list == miss[g0].list) ++g1;
            vals.clear();
            for (size_t q = g0; q < g1; ++q) {
                vals.push_back(miss[q].vi);
                added[k].push_back({miss[q].vj, miss[q].vi, miss[q].uj, miss[q].ui});
            }
            insert_run(lists_[miss[g0].list], vals.data(), vals.size());
            g0 = g1;
        }
        // checks: clear the round's checked bits, then test each (u, v) once;
        // check_nei(v, u) reads v's own lists only, all final for this round
        for (uint32_t s = 0; s < T; ++s)
            for (auto& c : check[(size_t)s * T + k]) checked_[c.v] &= ~(1u << c.u);
        for (uint32_t s = 0; s < T; ++s)
            for (auto& c : check[(size_t)s * T + k]) {
                if ((checked_[c.v] >> c.u) & 1u) continue;
                checked_[c.v] |= 1u << c.u;
                if (check_nei(c.v, c.u)) {
                    light(c.v, c.u);
                    next[k].push_back(c);
                    act[k].push_back(c);
                } else {
                    drop[k].push_back(c);
                }
            }
    });
    concat(delta_ins, added);
    concat(activated, act);
    concat(add_del, drop);
    add.clear();
    concat(add, next);
}

// calig.cpp:950-1069 for an insertion batch.  Deletions (negative ids) are
// not processed: the reference loses their candidate-erasure tasks
// (turnOffCond takes its task list by value, calig.h:152) and indexes G with
// the negative ids in ConstructUpdate; they are skipped here.
void CaLiGIndex::update_index(uint32_t start, uint32_t count) {
    delta_ins.clear();
    delta_del.clear();
    delta_update.clear();
    const uint32_t end = std::min<uint32_t>(start + count, (uint32_t)update_.size());
    const uint32_t n = (uint32_t)glabel_.size();
    const uint32_t npairs = end > start ? (end - start) / 2 : 0;
    const uint32_t T = npairs >= par_min_ ? threads_ : 1u;
    // turnOnCond (calig.cpp:640-655) on slices of the batch, against the
    // adjacency before the batch (a pair listed twice is new both times)
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> ups(T);
    std::vector<std::vector<Tmp>> tmp((size_t)T * T);  // [slice * T + owner of the first vertex]
    run_threads(T, [&](uint32_t s) {
        for (uint32_t p = (uint32_t)((uint64_t)npairs * s / T); p < (uint32_t)((uint64_t)npairs * (s + 1) / T); ++p) {
            const int a = update_[start + 2 * p], b = update_[start + 2 * p + 1];
            if (a < 0 || b < 0 || (uint32_t)a >= n || (uint32_t)b >= n) continue;
            const uint32_t v1 = (uint32_t)a, v2 = (uint32_t)b;
            if (glabel_[v1] < 0 || glabel_[v2] < 0) continue;
            if (edges_.has(v1, v2)) continue;  // edge exists before this batch
            ups[s].emplace_back(v1, v2);
            for (int o = 0; o < 2; ++o) {
                const uint32_t x = o ? v2 : v1, y = o ? v1 : v2;
                for (uint32_t ui : qlist_[glabel_[x]])
                    for (uint32_t uj : qnei_[ui])
                        if (label_slot_[qlabel_[uj]] == glabel_[y])
                            tmp[(size_t)s * T + owner(x, T)].push_back({ui, uj, x, y});
            }
        }
    });
    // The batch's edges join the edge set (all pairs of slice k on thread k);
    // candidate-list inserts, then turnOnCheck (calig.cpp:657-693), by owner
    // of the first vertex: its lists, LI and checked bits.
    std::vector<std::vector<Task>> addp(T), setp(T), actp(T);
    size_t nup = 0;
    for (auto& part : ups) nup += part.size();
    edges_.reserve(nup);
    run_threads(T, [&](uint32_t k) {
        for (auto& [x, y] : ups[k]) edges_.insert(x, y);
        std::vector<std::pair<uint64_t, uint32_t>> ins;
        std::vector<uint32_t> vals;
        auto apply = [&](auto&& list_of) {
            // group by list, values ascending: packed list << 27 | value keys
            // (vertex ids < 2^27) radix-sorted when the list index fits
            const int lb = 64 - __builtin_clzll((unsigned long long)lists_.size() | 1ull);
            if (lb <= 37) {
                std::vector<uint64_t> key(ins.size());
                for (size_t i = 0; i < ins.size(); ++i) key[i] = ins[i].first << 27 | ins[i].second;
                radix_sort(key, lb + 27);
                for (size_t i = 0; i < ins.size(); ++i) ins[i] = {key[i] >> 27, (uint32_t)(key[i] & ((1u << 27) - 1u))};
            } else {
                std::sort(ins.begin(), ins.end());
            }
            for (size_t g0 = 0; g0 < ins.size();) {
                size_t g1 = g0 + 1;
                while (g1 < ins.size() && ins[g1].first == ins[g0].first) ++g1;
                vals.clear();
                for (size_t q = g0; q < g1; ++q) vals.push_back(ins[q].second);
                insert_run(list_of(ins[g0].first), vals.data(), vals.size());
                g0 = g1;
            }
        };
        std::vector<Task> check;
        for (uint32_t sl = 0; sl < T; ++sl)
            for (auto& t : tmp[(size_t)sl * T + k]) {
                ins.emplace_back(list_index(t.vi, t.ui, t.uj), t.vj);
                if (lit(t.vi, t.ui)) setp[k].push_back({t.ui, t.vi});
                else {
                    check.push_back({t.ui, t.vi});
                    checked_[t.vi] &= ~(1u << t.ui);
                }
            }
        apply([&](uint64_t l) -> std::vector<uint32_t>& { return lists_[l]; });
        for (auto& c : check) {
            if ((checked_[c.v] >> c.u) & 1u) continue;
            checked_[c.v] |= 1u << c.u;
            if (lit(c.v, c.u)) continue;
            if (check_nei(c.v, c.u)) {
                light(c.v, c.u);
                addp[k].push_back(c);
                actp[k].push_back(c);
            }
        }
    });
    std::vector<Task> add, settled, activated, add_del;
    concat(add, addp);
    concat(settled, setp);
    concat(activated, actp);
    // addAndCheck to the fix-point, then addAndCheckDelete (calig.cpp:695-703)
    while (!add.empty() || !settled.empty()) add_and_check(add, settled, add_del, activated);
    std::vector<Task> del;
    for (auto& c : add_del)
        if (!lit(c.v, c.u)) del.push_back(c);
    while (!del.empty()) del_and_check(del);
    // newly lit vertices contribute their whole candidate lists (calig.cpp:1048-1068)
    const uint32_t TA = activated.size() >= par_min_ ? threads_ : 1u;
    std::vector<std::vector<DeltaOp>> whole(TA);
    run_threads(TA, [&](uint32_t s) {
        for (size_t i = activated.size() * s / TA; i < activated.size() * (s + 1) / TA; ++i) {
            const Task& a = activated[i];
            if (!lit(a.v, a.u)) continue;
            for (uint32_t uj : qnei_[a.u])
                for (uint32_t vj : C(a.v, a.u, uj)) whole[s].push_back({a.v, vj, a.u, uj});
        }
    });
    concat(delta_ins, whole);
}

// calig.cpp:776-804: for every pair of the batch (as listed), each lit u1 of
// v1 whose (u1 -> u2) list holds v2 yields the delta edge in both directions,
// which is also scheduled for removal from the old index.  Read-only: slices
// of the batch on threads, concatenated in batch order.
void CaLiGIndex::construct_update(uint32_t start, uint32_t count) {
    const uint32_t end = std::min<uint32_t>(start + count, (uint32_t)update_.size());
    const uint32_t n = (uint32_t)glabel_.size();
    const uint32_t npairs = end > start ? (end - start) / 2 : 0;
    const uint32_t T = npairs >= par_min_ ? threads_ : 1u;
    std::vector<std::vector<DeltaOp>> upd(T);
    run_threads(T, [&](uint32_t s) {
        // lookups in groups of 16 whose list headers, then list words, are
        // prefetched together (each is a dependent cache miss); results are
        // emitted in the pairs' order
        constexpr size_t kGroup = 16;
        struct Look { const std::vector<uint32_t>* L; uint32_t v1, v2, u1, u2; };
        Look grp[kGroup];
        size_t ng = 0;
        auto flush = [&]() {
            for (size_t i = 0; i < ng; ++i)
                if (!grp[i].L->empty()) __builtin_prefetch(grp[i].L->data() + grp[i].L->size() / 2);
            for (size_t i = 0; i < ng; ++i) {
                const Look& q = grp[i];
                if (!sorted_has(*q.L, q.v2)) continue;
                upd[s].push_back({q.v1, q.v2, q.u1, q.u2});
                upd[s].push_back({q.v2, q.v1, q.u2, q.u1});
            }
            ng = 0;
        };
        for (uint32_t p = (uint32_t)((uint64_t)npairs * s / T); p < (uint32_t)((uint64_t)npairs * (s + 1) / T); ++p) {
            const int a = update_[start + 2 * p], b = update_[start + 2 * p + 1];
            if (a < 0 || b < 0 || (uint32_t)a >= n || (uint32_t)b >= n) continue;
            const uint32_t v1 = (uint32_t)a, v2 = (uint32_t)b;
            if (glabel_[v1] < 0) continue;
            for (uint32_t u1 : qlist_[glabel_[v1]]) {
                if (!lit(v1, u1)) continue;
                for (uint32_t u2 : qnei_[u1]) {
                    const std::vector<uint32_t>* L = &C(v1, u1, u2);
                    __builtin_prefetch(L);
                    grp[ng++] = {L, v1, v2, u1, u2};
                    if (ng == kGroup) flush();
                }
            }
        }
        flush();
    });
    concat(delta_update, upd);
    concat(delta_del, upd);
}

}  // namespace cgb
