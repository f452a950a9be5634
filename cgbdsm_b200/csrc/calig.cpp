#include "calig.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>
#include <thread>
#include <unordered_map>

namespace cgb {

namespace {

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
// Runs fn(0..n-1), each on its own thread (inline when n == 1).
template <class Fn>
void run_threads(uint32_t n, Fn fn) {
    if (n <= 1) { fn(0u); return; }
    std::vector<std::thread> pool;
    pool.reserve(n);
    for (uint32_t k = 0; k < n; ++k) pool.emplace_back(fn, k);
    for (auto& t : pool) t.join();
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

// Sorts and deduplicates a task queue.  Repeated tasks in the reference's
// queues only redo inserts that fail and checks guarded by the checked bit, so
// processing each distinct task once yields the same index and deltas.
template <typename T>
void dedupe(std::vector<T>& q) {
    std::sort(q.begin(), q.end(), [](const T& a, const T& b) { return a.v != b.v ? a.v < b.v : a.u < b.u; });
    q.erase(std::unique(q.begin(), q.end(), [](const T& a, const T& b) { return a.v == b.v && a.u == b.u; }),
            q.end());
}

}  // namespace

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
}

// calig.cpp:325-356 constructCand, then 705-717 staticFilter.
void CaLiGIndex::construct() {
    const uint32_t n = (uint32_t)glabel_.size();
    cbase_.assign(n + 1, 0);
    uint64_t total = 0;
    for (uint32_t v = 0; v < n; ++v) {
        cbase_[v] = total;
        if (glabel_[v] >= 0) total += block_size_[glabel_[v]];
    }
    cbase_[n] = total;
    lists_.assign(total, {});
    for (uint32_t v = 0; v < n; ++v) {
        li_[v] = 0;
        checked_[v] = 0;
        const int s = glabel_[v];
        if (s < 0) continue;
        for (uint32_t ui : qlist_[s]) {
            for (uint32_t vj : nei_[v]) {
                const int lj = glabel_[vj];
                if (lj < 0) continue;
                for (uint32_t uj : qnei_[ui])
                    if (label_slot_[qlabel_[uj]] == lj) C(v, ui, uj).push_back(vj);  // nei_ sorted -> lists sorted
            }
            li_[v] |= 1u << ui;
        }
    }
    // staticFilter: turnOff every lit (v, ui) failing checkNei, then delAndCheck to the fix-point
    std::vector<Task> del;
    for (uint32_t v = 0; v < n; ++v) {
        const int s = glabel_[v];
        if (s < 0) continue;
        for (uint32_t ui : qlist_[s]) {
            if (!lit(v, ui)) continue;
            if (!check_nei(v, ui)) {
                li_[v] &= ~(1u << ui);
                del.push_back({ui, v});
            }
        }
    }
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

// calig.cpp:410-475 delAndCheck (one round; `del` becomes the next round).
void CaLiGIndex::del_and_check(std::vector<Task>& del) {
    dedupe(del);
    std::vector<Tmp> tmp;
    for (auto& t : del)
        for (uint32_t uj : qnei_[t.u])
            for (uint32_t vj : C(t.v, t.u, uj))
                if (lit(vj, uj)) tmp.push_back({t.u, uj, t.v, vj});
    std::vector<Task> next;
    struct Chk { uint32_t u, v; int group; };
    std::vector<Chk> chk;
    for (auto& t : tmp) {
        auto& L = C(t.vj, t.uj, t.ui);
        if (sorted_erase(L, t.vi)) delta_del.push_back({t.vj, t.vi, t.uj, t.ui});
        if (L.empty()) {
            li_[t.vj] &= ~(1u << t.uj);
            next.push_back({t.uj, t.vj});
        } else {
            const int g = rep_of_label_[t.uj][label_slot_[qlabel_[t.ui]]];
            if (g >= 0) {
                chk.push_back({t.uj, t.vj, g});
                checked_[t.vj] &= ~(1u << t.uj);
            }
        }
    }
    for (auto& c : chk) {
        if ((checked_[c.v] >> c.u) & 1u) continue;
        checked_[c.v] |= 1u << c.u;
        std::vector<uint32_t> used;
        if (!try_nei(c.v, c.u, rep_[c.u][c.group], 0, used)) {
            li_[c.v] &= ~(1u << c.u);
            next.push_back({c.u, c.v});
        }
    }
    del.swap(next);
}

// calig.cpp:536-638 addAndCheck (one round; `add` becomes the next round).
void CaLiGIndex::add_and_check(std::vector<Task>& add, std::vector<Task>& add_del,
                               std::vector<Task>& activated) {
    dedupe(add);
    std::vector<Tmp> tmp;
    std::vector<Task> check;
    // The work list, in add order: slices of `add` on threads, concatenated
    // in slice order (checked_ bits are cleared atomically: clearing commutes).
    const uint32_t TB = add.size() >= 4096 ? threads_ : 1u;
    std::vector<std::vector<Tmp>> ptmp(TB);
    std::vector<std::vector<Task>> pchk(TB);
    run_threads(TB, [&](uint32_t k) {
        const size_t a0 = add.size() * k / TB, a1 = add.size() * (k + 1) / TB;
        auto& lt = TB == 1 ? tmp : ptmp[k];
        auto& lc = TB == 1 ? check : pchk[k];
        for (size_t i = a0; i < a1; ++i) {
            const Task& t = add[i];
            for (uint32_t uj : qnei_[t.u])
                for (uint32_t vj : C(t.v, t.u, uj)) {
                    lt.push_back({t.u, uj, t.v, vj});
                    if (!lit(vj, uj)) {
                        lc.push_back({uj, vj});
                        __atomic_fetch_and(&checked_[vj], ~(1u << uj), __ATOMIC_RELAXED);
                    }
                }
        }
    });
    if (TB > 1)
        for (uint32_t k = 0; k < TB; ++k) {
            tmp.insert(tmp.end(), ptmp[k].begin(), ptmp[k].end());
            check.insert(check.end(), pchk[k].begin(), pchk[k].end());
        }
    // Insert each vi into its candidate list.  Most of these inserts find the
    // value present already, and each is a cache-missing search in a long
    // list, so large rounds run on threads_ threads, each owning the lists
    // with index % threads_ == its id: every list still sees its inserts in
    // tmp order, and the inserted (new) entries are the same multiset.
    const uint32_t T = tmp.size() >= (1u << 16) ? threads_ : 1u;
    if (T <= 1) {
        for (auto& t : tmp)
            if (sorted_insert(C(t.vj, t.uj, t.ui), t.vi)) delta_ins.push_back({t.vj, t.vi, t.uj, t.ui});
    } else {
        // counting sort of the items by owner (list % T), stable, then one
        // thread per owner
        const size_t n = tmp.size();
        std::vector<uint64_t> L(n);
        std::vector<size_t> off((size_t)T * T, 0);  // [chunk][owner]
        run_threads(T, [&](uint32_t c) {
            for (size_t i = n * c / T; i < n * (c + 1) / T; ++i) {
                L[i] = list_index(tmp[i].vj, tmp[i].uj, tmp[i].ui);
                ++off[(size_t)c * T + L[i] % T];
            }
        });
        std::vector<size_t> start(T + 1, 0);
        size_t acc = 0;
        for (uint32_t k = 0; k < T; ++k) {
            start[k] = acc;
            for (uint32_t c = 0; c < T; ++c) {
                const size_t x = off[(size_t)c * T + k];
                off[(size_t)c * T + k] = acc;
                acc += x;
            }
        }
        start[T] = acc;
        std::vector<uint32_t> order(n);
        run_threads(T, [&](uint32_t c) {
            for (size_t i = n * c / T; i < n * (c + 1) / T; ++i) order[off[(size_t)c * T + L[i] % T]++] = (uint32_t)i;
        });
        std::vector<std::vector<DeltaOp>> part(T);
        run_threads(T, [&](uint32_t k) {
            for (size_t q = start[k]; q < start[k + 1]; ++q) {
                const Tmp& t = tmp[order[q]];
                if (sorted_insert(lists_[L[order[q]]], t.vi)) part[k].push_back({t.vj, t.vi, t.uj, t.ui});
            }
        });
        for (auto& q : part) delta_ins.insert(delta_ins.end(), q.begin(), q.end());
    }
    std::vector<Task> next;
    for (auto& c : check) {
        if ((checked_[c.v] >> c.u) & 1u) continue;
        checked_[c.v] |= 1u << c.u;
        if (check_nei(c.v, c.u)) {
            li_[c.v] |= 1u << c.u;
            next.push_back(c);
            activated.push_back(c);
        } else {
            add_del.push_back(c);
        }
    }
    add.swap(next);
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
    std::vector<std::pair<uint32_t, uint32_t>> ups;
    std::vector<Tmp> tmp;
    for (uint32_t t = start; t + 1 < end; t += 2) {
        const int a = update_[t], b = update_[t + 1];
        if (a < 0 || b < 0 || (uint32_t)a >= n || (uint32_t)b >= n) continue;
        const uint32_t v1 = (uint32_t)a, v2 = (uint32_t)b;
        if (glabel_[v1] < 0 || glabel_[v2] < 0) continue;
        if (sorted_has(nei_[v1], v2)) continue;  // edge exists before this batch
        ups.emplace_back(v1, v2);
        // turnOnCond (calig.cpp:640-655), both orientations
        for (int o = 0; o < 2; ++o) {
            const uint32_t x = o ? v2 : v1, y = o ? v1 : v2;
            for (uint32_t ui : qlist_[glabel_[x]])
                for (uint32_t uj : qnei_[ui])
                    if (label_slot_[qlabel_[uj]] == glabel_[y]) tmp.push_back({ui, uj, x, y});
        }
    }
    for (auto& [x, y] : ups) {
        sorted_insert(nei_[x], y);
        sorted_insert(nei_[y], x);
    }
    // turnOnCheck (calig.cpp:657-693)
    std::vector<Task> add, check, activated, add_del;
    for (auto& t : tmp) {
        sorted_insert(C(t.vi, t.ui, t.uj), t.vj);
        if (lit(t.vi, t.ui)) add.push_back({t.ui, t.vi});
        else {
            check.push_back({t.ui, t.vi});
            checked_[t.vi] &= ~(1u << t.ui);
        }
    }
    for (auto& c : check) {
        if ((checked_[c.v] >> c.u) & 1u) continue;
        checked_[c.v] |= 1u << c.u;
        if (lit(c.v, c.u)) continue;
        if (check_nei(c.v, c.u)) {
            li_[c.v] |= 1u << c.u;
            add.push_back(c);
            activated.push_back(c);
        }
    }
    // addAndCheck to the fix-point, then addAndCheckDelete (calig.cpp:695-703)
    while (!add.empty()) add_and_check(add, add_del, activated);
    std::vector<Task> del;
    for (auto& c : add_del)
        if (!lit(c.v, c.u)) del.push_back(c);
    while (!del.empty()) del_and_check(del);
    // newly lit vertices contribute their whole candidate lists (calig.cpp:1048-1068)
    for (auto& a : activated) {
        if (!lit(a.v, a.u)) continue;
        for (uint32_t uj : qnei_[a.u])
            for (uint32_t vj : C(a.v, a.u, uj)) delta_ins.push_back({a.v, vj, a.u, uj});
    }
}

// calig.cpp:776-804: for every pair of the batch (as listed), each lit u1 of
// v1 whose (u1 -> u2) list holds v2 yields the delta edge in both directions,
// which is also scheduled for removal from the old index.
void CaLiGIndex::construct_update(uint32_t start, uint32_t count) {
    const uint32_t end = std::min<uint32_t>(start + count, (uint32_t)update_.size());
    const uint32_t n = (uint32_t)glabel_.size();
    for (uint32_t t = start; t + 1 < end; t += 2) {
        const int a = update_[t], b = update_[t + 1];
        if (a < 0 || b < 0 || (uint32_t)a >= n || (uint32_t)b >= n) continue;
        const uint32_t v1 = (uint32_t)a, v2 = (uint32_t)b;
        if (glabel_[v1] < 0) continue;
        for (uint32_t u1 : qlist_[glabel_[v1]]) {
            if (!lit(v1, u1)) continue;
            for (uint32_t u2 : qnei_[u1]) {
                if (!sorted_has(C(v1, u1, u2), v2)) continue;
                delta_update.push_back({v1, v2, u1, u2});
                delta_del.push_back({v1, v2, u1, u2});
                delta_update.push_back({v2, v1, u2, u1});
                delta_del.push_back({v2, v1, u2, u1});
            }
        }
    }
}

}  // namespace cgb
