#include "query.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <sstream>

namespace cgb {

std::string parse_query_file(const std::string& path, std::vector<uint32_t>& labels,
                             std::vector<uint32_t>& edges, uint32_t& qv) {
    // Text format of graph.cpp:57-114 / calig.cpp:111-164: 't' lines are
    // skipped, "v id label", "e a b label".
    std::ifstream in(path);
    if (!in) return "cannot open query file " + path;
    labels.clear();
    edges.clear();
    qv = 0;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        char t;
        if (!(ss >> t)) continue;
        if (t == 'v') {
            uint32_t id, lb;
            if (!(ss >> id >> lb)) return "bad vertex line: " + line;
            if (id >= labels.size()) labels.resize(id + 1, 0);
            labels[id] = lb;
            qv = std::max(qv, id + 1);
        } else if (t == 'e') {
            uint32_t a, b;
            if (!(ss >> a >> b)) return "bad edge line: " + line;
            edges.push_back(a);
            edges.push_back(b);
        }
    }
    return "";
}

std::string build_query_meta(uint32_t qv, uint32_t qe, const uint32_t* edges, const uint32_t* labels,
                             QueryMeta& q) {
    if (qv < 2 || qv > (uint32_t)kMaxQV) return "query must have 2..12 vertices";
    if (qe == 0 || 2 * qe > (uint32_t)kMaxDir) return "query must have 1..16 edges (5-bit directed index)";
    q = QueryMeta();
    q.qv = qv;
    if (labels) q.labels.assign(labels, labels + qv);
    q.nbrs.assign(qv, {});
    for (uint32_t i = 0; i < qe; ++i) {
        uint32_t a = edges[2 * i], b = edges[2 * i + 1];
        if (a >= qv || b >= qv || a == b) return "bad query edge";
        auto& na = q.nbrs[a];
        if (std::find(na.begin(), na.end(), b) != na.end()) return "duplicate query edge";
        na.push_back(b);
        q.nbrs[b].push_back(a);
    }
    for (auto& n : q.nbrs) std::sort(n.begin(), n.end());
    std::memset(q.eidx, 255, sizeof(q.eidx));
    uint32_t pos = 0;
    for (uint32_t u = 0; u < qv; ++u)
        for (uint32_t w : q.nbrs[u]) {
            q.eidx[u * kMaxQV + w] = (uint8_t)pos;
            q.dir_src[pos] = (uint8_t)u;
            q.dir_dst[pos] = (uint8_t)w;
            ++pos;
        }
    q.nd = pos;
    uint32_t e = 0;
    for (uint32_t u = 0; u < qv; ++u)
        for (uint32_t w : q.nbrs[u]) {
            if (u > w) continue;
            q.qe_u[e] = (uint8_t)u;
            q.qe_v[e] = (uint8_t)w;
            q.qe_dir[e][0] = q.eidx[u * kMaxQV + w];
            q.qe_dir[e][1] = q.eidx[w * kMaxQV + u];
            q.dir_to_edge[q.qe_dir[e][0]] = (uint8_t)e;
            q.dir_to_edge[q.qe_dir[e][1]] = (uint8_t)e;
            ++e;
        }
    q.qe = e;
    // connected patterns only: every vertex after the first edge needs a
    // backward neighbour to draw candidates from
    std::vector<int> seen(qv, 0);
    std::vector<uint32_t> st{0};
    seen[0] = 1;
    while (!st.empty()) {
        uint32_t u = st.back();
        st.pop_back();
        for (uint32_t w : q.nbrs[u])
            if (!seen[w]) { seen[w] = 1; st.push_back(w); }
    }
    for (uint32_t u = 0; u < qv; ++u)
        if (!seen[u]) return "query pattern must be connected";
    return "";
}

// Per-edge vertex order: ei's endpoints first (the delta edge is the seed),
// then greedily the unvisited core vertex with the most visited neighbours,
// ties broken by the smallest estimated candidate count (min avg run length
// over its backward edges), then by vertex id.  The tie-breaking criteria
// restate the reference's global-order rules 1 and 4 (plan.cpp:595-708); the
// start is the delta edge instead of a global edge because matching is seeded
// from the delta lists.
//
// Tail: a maximal set of mutually non-adjacent vertices (other than ei's
// endpoints) whose removal leaves the core connected, chosen by ascending
// query degree.  All neighbours of a tail vertex are core vertices, so once
// the core is matched each tail vertex's candidates are one intersection of
// resolved lists, independent of the other tail vertices except for
// injectivity: the tail is counted, not enumerated.  This is the reference's
// Cartesian-product tail (plan.cpp:899-952, enumerated there by
// cartesian_product.cu:304-427).  Tail vertices are grouped by label (only
// same-label vertices can collide); groups are limited to 3 members, extra
// members go back to the core.
void plan_edges(const QueryMeta& q, const float* avg_deg, EdgePlan* plans, bool analytic_tail, bool pick_last) {
    for (uint32_t ei = 0; ei < q.qe; ++ei) {
        EdgePlan& p = plans[ei];
        std::memset(&p, 0, sizeof(p));
        p.n = (uint8_t)q.qv;
        uint32_t a = q.qe_u[ei], b = q.qe_v[ei];
        p.vs[0] = (uint8_t)a;
        p.vs[1] = (uint8_t)b;
        p.seed_dir = q.eidx[a * kMaxQV + b];
        std::vector<int> pos(q.qv, -1);
        pos[a] = 0;
        pos[b] = 1;
        auto lab = [&](uint32_t u) { return q.labels.empty() ? 0u : q.labels[u]; };
        std::vector<uint32_t> tail;
        if (analytic_tail && q.qv > 2) {
            std::vector<char> in_t(q.qv, 0);
            std::vector<uint32_t> cand;
            for (uint32_t u = 0; u < q.qv; ++u)
                if (u != a && u != b) cand.push_back(u);
            std::stable_sort(cand.begin(), cand.end(),
                             [&](uint32_t x, uint32_t y) { return q.nbrs[x].size() < q.nbrs[y].size(); });
            auto core_connected = [&]() {
                std::vector<char> seen(q.qv, 0);
                std::vector<uint32_t> st{a};
                seen[a] = 1;
                uint32_t reached = 1, need = 0;
                for (uint32_t u = 0; u < q.qv; ++u) need += in_t[u] ? 0 : 1;
                while (!st.empty()) {
                    uint32_t u = st.back();
                    st.pop_back();
                    for (uint32_t w : q.nbrs[u])
                        if (!in_t[w] && !seen[w]) { seen[w] = 1; ++reached; st.push_back(w); }
                }
                return reached == need;
            };
            for (uint32_t u : cand) {
                bool adj = false;
                for (uint32_t w : q.nbrs[u]) adj |= in_t[w] != 0;
                if (adj) continue;
                in_t[u] = 1;
                if (!core_connected()) in_t[u] = 0;
            }
            for (uint32_t u : cand)
                if (in_t[u]) tail.push_back(u);
            std::stable_sort(tail.begin(), tail.end(), [&](uint32_t x, uint32_t y) { return lab(x) < lab(y); });
            std::vector<uint32_t> kept;
            for (size_t i = 0; i < tail.size();) {
                size_t j = i;
                while (j < tail.size() && lab(tail[j]) == lab(tail[i])) ++j;
                for (size_t k = i; k < j && k < i + 3; ++k) kept.push_back(tail[k]);
                i = j;
            }
            tail.swap(kept);
        }
        std::vector<char> is_tail(q.qv, 0);
        for (uint32_t u : tail) is_tail[u] = 1;
        const uint32_t n_core = q.qv - (uint32_t)tail.size();
        // last core vertex: the one with the fewest tail neighbours (its
        // tail lists must be re-scanned per candidate), among those whose
        // removal keeps the rest of the core connected
        int last = -1;
        if (pick_last && n_core > 2) {
            int best_t = 1 << 30, best_c = -1;
            for (uint32_t u = 0; u < q.qv; ++u) {
                if (is_tail[u] || u == a || u == b) continue;
                std::vector<char> seen(q.qv, 0);
                std::vector<uint32_t> st{a};
                seen[a] = 1;
                uint32_t reached = 1;
                while (!st.empty()) {
                    uint32_t x = st.back();
                    st.pop_back();
                    for (uint32_t w : q.nbrs[x])
                        if (!is_tail[w] && w != u && !seen[w]) { seen[w] = 1; ++reached; st.push_back(w); }
                }
                if (reached != n_core - 1) continue;
                int nt = 0, ncn = 0;
                for (uint32_t w : q.nbrs[u]) { nt += is_tail[w] ? 1 : 0; ncn += is_tail[w] ? 0 : 1; }
                if (nt < best_t || (nt == best_t && ncn > best_c)) { best_t = nt; best_c = ncn; last = (int)u; }
            }
        }
        for (uint32_t j = 2; j < n_core; ++j) {
            if (last >= 0 && j == n_core - 1) {
                pos[last] = (int)j;
                p.vs[j] = (uint8_t)last;
                break;
            }
            int best = -1, best_bn = -1;
            float best_est = 0.f;
            for (uint32_t u = 0; u < q.qv; ++u) {
                if (pos[u] >= 0 || is_tail[u] || (int)u == last) continue;
                int nbn = 0;
                float est = 3.4e38f;
                for (uint32_t w : q.nbrs[u])
                    if (pos[w] >= 0) {
                        ++nbn;
                        est = std::min(est, avg_deg[q.eidx[w * kMaxQV + u]]);
                    }
                if (nbn == 0) continue;
                if (nbn > best_bn || (nbn == best_bn && est < best_est)) {
                    best = (int)u;
                    best_bn = nbn;
                    best_est = est;
                }
            }
            if (best < 0) {  // cannot happen for a connected core; fall back to any remaining vertex
                for (uint32_t u = 0; u < q.qv; ++u)
                    if (pos[u] < 0 && !is_tail[u] && (int)u != last) { best = (int)u; break; }
            }
            pos[best] = (int)j;  // the core minus `last` is connected, so some vertex is adjacent
            p.vs[j] = (uint8_t)best;
        }
        p.n_core = (uint8_t)n_core;
        std::memset(p.tail_gid, 255, sizeof(p.tail_gid));
        uint8_t gid = 0;
        for (size_t i = 0; i < tail.size(); ++i) {
            const uint32_t j = n_core + (uint32_t)i;
            p.vs[j] = (uint8_t)tail[i];
            pos[tail[i]] = (int)j;
            if (i > 0 && lab(tail[i]) != lab(tail[i - 1])) ++gid;
            p.tail_gid[j] = gid;
        }
        uint32_t k = 0;
        for (uint32_t j = 0; j < q.qv; ++j) {
            p.bn_off[j] = (uint8_t)k;
            if (j < 2) continue;
            uint32_t u = p.vs[j];
            for (uint32_t t = 0; t < j; ++t) {
                uint32_t w = p.vs[t];
                uint8_t d = q.eidx[w * kMaxQV + u];
                if (d == 255) continue;
                p.bn_pos[k] = (uint8_t)t;
                p.bn_dir[k] = d;
                p.bn_dvis[k] = q.dir_to_edge[d] < ei ? 1 : 0;
                ++k;
            }
        }
        p.bn_off[q.qv] = (uint8_t)k;
    }
}

}  // namespace cgb
