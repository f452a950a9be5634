// Seeded synthetic workloads in the reference's text formats.
//
// The reference measures on public graphs (LiveJournal, Orkut, ...) that are
// not available here; these generators produce graphs, update streams and
// query patterns with the shapes, sizes and distributions of the workloads the
// engine is measured on:
//   * data graph  "v <id> <label>" for every id, then "e <a> <b> 0"
//                 (format: reference README.md:151-166, read by calig.cpp:166-216)
//   * update file "e <a> <b> 0" per insertion (calig.cpp:719-733)
//   * query       "v <i> <label>" then "e <a> <b> 0" (calig.cpp:111-164, graph.cpp:43-121)
// Query shapes follow the reference sampler's definitions
// (sampler/graph_sampler.h:150-272): dense = BFS-sampled vertex set with all
// induced edges and average degree >= 3; sparse = BFS tree plus random induced
// edges up to 1.5n-1 edges; tree = random-DFS tree of depth >= max(2,(n+2)/3)
// (the reference grows trees by pushing every neighbour of the stack top,
// which yields stars on graphs whose degree exceeds the pattern size).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <queue>
#include <random>
#include <set>
#include <stack>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

struct Workload {
    uint32_t n = 0;
    std::vector<uint64_t> edges;  // (min<<32)|max, generation order, distinct
    std::vector<uint32_t> labels;
};

inline uint64_t pack(uint32_t a, uint32_t b) {
    if (a > b) std::swap(a, b);
    return ((uint64_t)a << 32) | b;
}

// Keep the first occurrence of every key, preserving order.
void stable_unique(std::vector<uint64_t>& v) {
    std::vector<uint32_t> idx(v.size());
    for (uint32_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return v[a] < v[b]; });
    std::vector<uint8_t> keep(v.size(), 0);
    for (size_t i = 0; i < idx.size(); ++i)
        if (i == 0 || v[idx[i]] != v[idx[i - 1]]) keep[idx[i]] = 1;
    size_t w = 0;
    for (size_t i = 0; i < v.size(); ++i)
        if (keep[i]) v[w++] = v[i];
    v.resize(w);
}

void gen_edges(Workload& W, uint32_t n, uint64_t m, int rmat, double a, double b, double c,
               uint64_t seed) {
    W.n = n;
    std::mt19937_64 rng(seed);
    uint32_t scale = 0;
    while ((1ull << scale) < n) ++scale;
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::uniform_int_distribution<uint32_t> UV(0, n - 1);
    std::vector<uint64_t> acc;
    acc.reserve(m + m / 8);
    while (acc.size() < m) {
        uint64_t need = m - acc.size();
        uint64_t batch = need + need / 8 + 1024;
        for (uint64_t i = 0; i < batch; ++i) {
            uint32_t x, y;
            if (rmat) {
                x = 0; y = 0;
                for (uint32_t l = 0; l < scale; ++l) {
                    double r = U(rng);
                    uint32_t bx = 0, by = 0;
                    if (r < a) { }
                    else if (r < a + b) { by = 1; }
                    else if (r < a + b + c) { bx = 1; }
                    else { bx = 1; by = 1; }
                    x = (x << 1) | bx;
                    y = (y << 1) | by;
                }
            } else {
                x = UV(rng);
                y = UV(rng);
            }
            if (x >= n || y >= n || x == y) continue;
            acc.push_back(pack(x, y));
        }
        stable_unique(acc);
    }
    acc.resize(m);
    W.edges.swap(acc);
}

void gen_labels(Workload& W, uint32_t L, double zipf_s, uint64_t seed) {
    std::mt19937_64 rng(seed);
    W.labels.resize(W.n);
    if (zipf_s <= 0.0) {
        std::uniform_int_distribution<uint32_t> d(0, L - 1);
        for (auto& l : W.labels) l = d(rng);
        return;
    }
    std::vector<double> w(L);
    for (uint32_t k = 0; k < L; ++k) w[k] = std::pow((double)(k + 1), -zipf_s);
    std::discrete_distribution<uint32_t> d(w.begin(), w.end());
    for (auto& l : W.labels) l = d(rng);
}

struct Adj {
    std::vector<uint64_t> off;
    std::vector<uint32_t> nbr;
};

Adj build_adj(uint32_t n, const std::vector<uint64_t>& edges) {
    Adj A;
    A.off.assign(n + 1, 0);
    for (uint64_t e : edges) { A.off[(e >> 32) + 1]++; A.off[(uint32_t)e + 1]++; }
    for (uint32_t i = 0; i < n; ++i) A.off[i + 1] += A.off[i];
    A.nbr.resize(A.off[n]);
    std::vector<uint64_t> pos(A.off.begin(), A.off.end() - 1);
    for (uint64_t e : edges) {
        uint32_t x = (uint32_t)(e >> 32), y = (uint32_t)e;
        A.nbr[pos[x]++] = y;
        A.nbr[pos[y]++] = x;
    }
    for (uint32_t i = 0; i < n; ++i) std::sort(A.nbr.begin() + A.off[i], A.nbr.begin() + A.off[i + 1]);
    return A;
}

bool adjacent(const Adj& A, uint32_t x, uint32_t y) {
    return std::binary_search(A.nbr.begin() + A.off[x], A.nbr.begin() + A.off[x + 1], y);
}

// Returns vertices (order of discovery) and tree edges.  BFS growth attaches
// every unvisited neighbour of the dequeued vertex (shuffled) until k vertices
// are reached; tree (dfs) growth is a random depth-first walk that attaches one
// unvisited neighbour of the stack top at a time, backtracking when there is
// none, so trees come out deep rather than star-shaped.
void grow(const Adj& A, uint32_t start, uint32_t k, bool dfs, std::mt19937_64& rng,
          std::vector<uint32_t>& vs, std::vector<std::pair<uint32_t, uint32_t>>& tree) {
    vs.assign(1, start);
    tree.clear();
    std::unordered_set<uint32_t> seen{start};
    if (dfs) {
        std::vector<uint32_t> stack{start};
        while (!stack.empty() && vs.size() < k) {
            uint32_t v = stack.back();
            std::vector<uint32_t> nb;
            for (uint64_t p = A.off[v]; p < A.off[v + 1]; ++p)
                if (!seen.count(A.nbr[p])) nb.push_back(A.nbr[p]);
            if (nb.empty()) { stack.pop_back(); continue; }
            uint32_t u = nb[std::uniform_int_distribution<size_t>(0, nb.size() - 1)(rng)];
            seen.insert(u);
            vs.push_back(u);
            tree.emplace_back(v, u);
            // occasionally branch from an earlier vertex instead of going deeper
            if (stack.size() > 1 && (rng() & 3) == 0) stack.pop_back();
            stack.push_back(u);
        }
        return;
    }
    std::deque<uint32_t> frontier{start};
    while (!frontier.empty() && vs.size() < k) {
        uint32_t v = frontier.front();
        frontier.pop_front();
        std::vector<uint32_t> nb(A.nbr.begin() + A.off[v], A.nbr.begin() + A.off[v + 1]);
        std::shuffle(nb.begin(), nb.end(), rng);
        for (uint32_t u : nb) {
            if (vs.size() >= k) break;
            if (seen.insert(u).second) {
                vs.push_back(u);
                tree.emplace_back(v, u);
                frontier.push_back(u);
            }
        }
    }
}

int tree_depth(uint32_t root, const std::vector<std::pair<uint32_t, uint32_t>>& tree) {
    std::vector<std::pair<uint32_t, int>> q{{root, 0}};
    std::unordered_set<uint32_t> seen{root};
    int best = 0;
    for (size_t h = 0; h < q.size(); ++h) {
        auto [v, d] = q[h];
        best = std::max(best, d);
        for (auto& [a, b] : tree) {
            uint32_t o = a == v ? b : (b == v ? a : UINT32_MAX);
            if (o != UINT32_MAX && seen.insert(o).second) q.push_back({o, d + 1});
        }
    }
    return best;
}

int write_graph(const char* path, const Workload& W, const std::vector<uint64_t>& edges) {
    FILE* f = std::fopen(path, "w");
    if (!f) return -1;
    std::vector<char> buf(1 << 22);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    for (uint32_t v = 0; v < W.n; ++v) std::fprintf(f, "v %u %u\n", v, W.labels[v]);
    for (uint64_t e : edges) std::fprintf(f, "e %u %u 0\n", (uint32_t)(e >> 32), (uint32_t)e);
    std::fclose(f);
    return 0;
}

// Graph, labels and the held-out stream of one workload (the stream in its
// shuffled order with the orientation the update file is written in).
struct Generated {
    Workload W;
    std::vector<uint64_t> initial;  // (min << 32) | max
    std::vector<std::pair<uint32_t, uint32_t>> stream;
    Adj final_adj;                  // initial + stream, for query sampling
};

void generate(Generated& G, int kind, uint32_t n, uint64_t m, double a, double b, double c, uint32_t num_labels,
              double zipf_s, uint64_t holdout, uint64_t seed_graph, uint64_t seed_labels, uint64_t seed_holdout,
              bool want_adj) {
    Workload& W = G.W;
    gen_edges(W, n, m, kind, a, b, c, seed_graph);
    gen_labels(W, num_labels, zipf_s, seed_labels);
    // holdout: random subset, re-inserted in shuffled order
    std::vector<uint32_t> perm(W.edges.size());
    for (uint32_t i = 0; i < perm.size(); ++i) perm[i] = i;
    std::mt19937_64 hr(seed_holdout);
    std::shuffle(perm.begin(), perm.end(), hr);
    if (holdout > W.edges.size()) holdout = W.edges.size();
    std::vector<uint8_t> held(W.edges.size(), 0);
    std::vector<uint64_t> stream;
    stream.reserve(holdout);
    for (uint64_t i = 0; i < holdout; ++i) { held[perm[i]] = 1; stream.push_back(W.edges[perm[i]]); }
    G.initial.clear();
    G.initial.reserve(W.edges.size() - holdout);
    for (size_t i = 0; i < W.edges.size(); ++i)
        if (!held[i]) G.initial.push_back(W.edges[i]);
    std::mt19937_64 dr(seed_holdout ^ 0x5bd1e995ull);
    G.stream.clear();
    G.stream.reserve(stream.size());
    for (uint64_t e : stream) {
        uint32_t x = (uint32_t)(e >> 32), y = (uint32_t)e;
        if (dr() & 1) std::swap(x, y);  // random orientation, as an edge stream would have
        G.stream.emplace_back(x, y);
    }
    if (want_adj) G.final_adj = build_adj(W.n, W.edges);
}

// Samples one query pattern from the final graph (see cgbgen_workload for the
// shape rules).  Returns 0 and the pattern's vertices' data ids / local edges,
// or < 0.
int sample_query(const Generated& G, int qshape, uint32_t qsize, uint32_t max_qedges, uint64_t seed_query,
                 std::vector<uint32_t>& out_vs, std::vector<std::pair<uint32_t, uint32_t>>& out_qe) {
    const Workload& W = G.W;
    const Adj& A = G.final_adj;
    std::mt19937_64 qr(seed_query);
    std::uniform_int_distribution<uint32_t> pick(0, W.n - 1);
    std::vector<uint32_t> vs;
    std::vector<std::pair<uint32_t, uint32_t>> tree;
    // Dense patterns need average degree >= 3; sparse graphs (e.g. ER with
    // average degree 10) almost never yield one, so the densest induced sample
    // seen within the attempt budget is used instead (deterministic fallback).
    std::vector<uint32_t> best_vs;
    std::vector<std::pair<uint32_t, uint32_t>> best_qe;
    const int budget = 20000;
    auto emit = [&](const std::vector<uint32_t>& V, std::vector<std::pair<uint32_t, uint32_t>> qe) {
        std::sort(qe.begin(), qe.end());
        out_vs = V;
        out_qe = qe;
        return 0;
    };
    for (int attempt = 0; attempt < budget; ++attempt) {
        uint32_t s = pick(qr);
        if (A.off[s + 1] == A.off[s]) continue;
        grow(A, s, qsize, qshape == 2, qr, vs, tree);
        if (vs.size() < qsize) continue;
        std::vector<std::pair<uint32_t, uint32_t>> qe;  // local ids
        std::vector<std::pair<uint32_t, uint32_t>> induced;
        for (uint32_t i = 0; i < vs.size(); ++i)
            for (uint32_t j = i + 1; j < vs.size(); ++j)
                if (adjacent(A, vs[i], vs[j])) induced.emplace_back(i, j);
        auto local = [&](uint32_t v) { return (uint32_t)(std::find(vs.begin(), vs.end(), v) - vs.begin()); };
        if (qshape == 0) {
            if (induced.size() > max_qedges) continue;
            if (induced.size() > best_qe.size()) { best_qe = induced; best_vs = vs; }
            if (2.0 * induced.size() / vs.size() < 3.0) continue;
            qe = induced;
        } else if (qshape == 2) {
            int min_depth = std::max(2, (int)(qsize + 2) / 3);
            if (tree_depth(s, tree) < min_depth) continue;
            for (auto& [x, y] : tree) qe.emplace_back(std::min(local(x), local(y)), std::max(local(x), local(y)));
        } else {
            std::set<std::pair<uint32_t, uint32_t>> ts;
            for (auto& [x, y] : tree) ts.insert({std::min(local(x), local(y)), std::max(local(x), local(y))});
            qe.assign(ts.begin(), ts.end());
            std::vector<std::pair<uint32_t, uint32_t>> extra;
            for (auto& p : induced) if (!ts.count(p)) extra.push_back(p);
            std::shuffle(extra.begin(), extra.end(), qr);
            uint32_t max_e = (3 * qsize) / 2 - 1;
            for (auto& p : extra) { if (qe.size() >= max_e) break; qe.push_back(p); }
            if (qe.size() == ts.size()) continue;  // must not be a tree
        }
        if (qe.size() > max_qedges) continue;
        return emit(vs, qe);
    }
    if (qshape == 0 && !best_vs.empty()) return emit(best_vs, best_qe);
    return -4;
}

}  // namespace

extern "C" {

// Generates a data graph + insertion stream + one query.
//   kind: 0 = Erdos-Renyi (uniform pairs), 1 = R-MAT(a, b, c, 1-a-b-c)
//   zipf_s <= 0: uniform labels, else P(k) ~ (k+1)^-zipf_s over num_labels
//   holdout edges are chosen uniformly (seed_holdout) and written in shuffled order
//   qshape: 0 = dense, 1 = sparse, 2 = tree; qsize vertices; queries sampled from
//   the final graph; resampled until the query has <= max_qedges edges.
// Returns 0 on success, <0 on failure; *out_qedges receives the query edge count.
int cgbgen_workload(const char* graph_path, const char* update_path, const char* query_path,
                    int kind, uint32_t n, uint64_t m, double a, double b, double c,
                    uint32_t num_labels, double zipf_s, uint64_t holdout,
                    uint64_t seed_graph, uint64_t seed_labels, uint64_t seed_holdout,
                    int qshape, uint32_t qsize, uint32_t max_qedges, uint64_t seed_query,
                    uint32_t* out_qedges) {
    const bool query_only = graph_path == nullptr;  // graph/stream already written
    Generated G;
    generate(G, kind, n, m, a, b, c, num_labels, zipf_s, holdout, seed_graph, seed_labels, seed_holdout, true);
    if (!query_only && write_graph(graph_path, G.W, G.initial) != 0) return -1;
    if (!query_only) {
        FILE* f = std::fopen(update_path, "w");
        if (!f) return -2;
        std::vector<char> buf(1 << 22);
        std::setvbuf(f, buf.data(), _IOFBF, buf.size());
        for (auto& [x, y] : G.stream) std::fprintf(f, "e %u %u 0\n", x, y);
        std::fclose(f);
    }
    std::vector<uint32_t> vs;
    std::vector<std::pair<uint32_t, uint32_t>> qe;
    const int rc = sample_query(G, qshape, qsize, max_qedges, seed_query, vs, qe);
    if (rc != 0) return rc;
    FILE* f = std::fopen(query_path, "w");
    if (!f) return -3;
    for (uint32_t i = 0; i < vs.size(); ++i) std::fprintf(f, "v %u %u\n", i, G.W.labels[vs[i]]);
    for (auto& [x, y] : qe) std::fprintf(f, "e %u %u 0\n", x, y);
    std::fclose(f);
    if (out_qedges) *out_qedges = (uint32_t)qe.size();
    return 0;
}

// In-memory form of the same workloads: the graph, labels and stream as
// arrays, and any number of query patterns sampled from one generated graph
// (query seed s gives the same pattern as cgbgen_workload with seed_query s).
void* cgbgen_open(int kind, uint32_t n, uint64_t m, double a, double b, double c, uint32_t num_labels,
                  double zipf_s, uint64_t holdout, uint64_t seed_graph, uint64_t seed_labels,
                  uint64_t seed_holdout) {
    Generated* G = new Generated();
    generate(*G, kind, n, m, a, b, c, num_labels, zipf_s, holdout, seed_graph, seed_labels, seed_holdout, true);
    return G;
}

void cgbgen_close(void* h) { delete (Generated*)h; }

// Sizes: out3[0] = vertices, out3[1] = initial edges, out3[2] = stream edges.
void cgbgen_sizes(void* h, uint64_t* out3) {
    const Generated* G = (const Generated*)h;
    out3[0] = G->W.n;
    out3[1] = G->initial.size();
    out3[2] = G->stream.size();
}

// labels[n]; initial[2 * initial edges] as (min, max) pairs in generation
// order; stream[2 * stream edges] as written to the update file.
void cgbgen_copy(void* h, uint32_t* labels, uint32_t* initial, uint32_t* stream) {
    const Generated* G = (const Generated*)h;
    if (labels) std::memcpy(labels, G->W.labels.data(), G->W.labels.size() * 4);
    if (initial)
        for (size_t i = 0; i < G->initial.size(); ++i) {
            initial[2 * i] = (uint32_t)(G->initial[i] >> 32);
            initial[2 * i + 1] = (uint32_t)G->initial[i];
        }
    if (stream)
        for (size_t i = 0; i < G->stream.size(); ++i) {
            stream[2 * i] = G->stream[i].first;
            stream[2 * i + 1] = G->stream[i].second;
        }
}

// One query: labels_out[<= 12], edges_out[2 * <= 66]; *qv, *qe set.
int cgbgen_query(void* h, int qshape, uint32_t qsize, uint32_t max_qedges, uint64_t seed_query,
                 uint32_t* labels_out, uint32_t* edges_out, uint32_t* qv, uint32_t* qe) {
    const Generated* G = (const Generated*)h;
    std::vector<uint32_t> vs;
    std::vector<std::pair<uint32_t, uint32_t>> e;
    const int rc = sample_query(*G, qshape, qsize, max_qedges, seed_query, vs, e);
    if (rc != 0) return rc;
    for (uint32_t i = 0; i < vs.size(); ++i) labels_out[i] = G->W.labels[vs[i]];
    for (size_t i = 0; i < e.size(); ++i) {
        edges_out[2 * i] = e[i].first;
        edges_out[2 * i + 1] = e[i].second;
    }
    *qv = (uint32_t)vs.size();
    *qe = (uint32_t)e.size();
    return 0;
}

}  // extern "C"
