#include "query.h"

#include <limits>

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
                             QueryMeta& q, uint32_t max_qe) {
    if (qv < 2 || qv > (uint32_t)kMaxQV) return "query must have 2..12 vertices";
    if (max_qe > (uint32_t)kMaxQE) max_qe = kMaxQE;
    if (qe == 0 || qe > max_qe)
        return max_qe == (uint32_t)kMaxQEKeyed ? "query must have 1..16 edges (5-bit directed index)"
                                               : "query must have 1..32 edges";
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
void plan_edges(const QueryMeta& q, const float* avg_deg, EdgePlan* plans, bool analytic_tail, bool pick_last,
                bool group_pendant, bool lane_tail, bool level_sum, bool dense_sums) {
    for (uint32_t ei = 0; ei < q.qe; ++ei) {
        EdgePlan& p = plans[ei];
        std::memset(&p, 0, sizeof(p));
        p.n = (uint8_t)q.qv;
        uint32_t a = q.qe_u[ei], b = q.qe_v[ei];
        // a pendant endpoint goes to position 1: seeds then arrive sorted by
        // the other endpoint, one contiguous run per grouped DFS
        if (q.nbrs[a].size() == 1 && q.nbrs[b].size() > 1) std::swap(a, b);
        const bool pendant = group_pendant && !q.labels.empty() && q.qv > 2 && q.nbrs[b].size() == 1;
        p.vs[0] = (uint8_t)a;
        p.vs[1] = (uint8_t)b;
        p.seed_dir = q.eidx[a * kMaxQV + b];
        std::vector<int> pos(q.qv, -1);
        pos[a] = 0;
        pos[b] = 1;
        auto lab = [&](uint32_t u) { return q.labels.empty() ? 0u : q.labels[u]; };
        // A tail vertex with several lists that hangs off the last core
        // vertex would be counted by one intersection per last-level
        // candidate, and would keep the rest of the tail from being constant
        // per prefix; enumerated as a core vertex its intersection runs
        // chunked and narrowed.  Such vertices move to the core (`forced`)
        // and the tail and last vertex are chosen again.
        std::vector<char> forced(q.qv, 0), is_tail;
        if (pendant)  // a tail vertex of the pendant's label would need per-member weights
            for (uint32_t u = 0; u < q.qv; ++u)
                if (u != a && u != b && q.labels[u] == q.labels[b]) forced[u] = 1;
        std::vector<uint32_t> tail;
        uint32_t n_core = q.qv;
        int last = -1;
        for (;;) {
            tail.clear();
            if (analytic_tail && q.qv > 2) {
                std::vector<char> in_t(q.qv, 0);
                std::vector<uint32_t> cand;
                for (uint32_t u = 0; u < q.qv; ++u)
                    if (u != a && u != b && !forced[u]) cand.push_back(u);
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
            is_tail.assign(q.qv, 0);
            for (uint32_t u : tail) is_tail[u] = 1;
            n_core = q.qv - (uint32_t)tail.size();
            // last core vertex: the one with the fewest tail neighbours (its
            // tail lists must be re-scanned per candidate), among those whose
            // removal keeps the rest of the core connected
            last = -1;
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
            int move = -1;
            if (last >= 0)
                for (uint32_t t : tail)
                    if (q.nbrs[t].size() >= 2 && q.eidx[(uint32_t)last * kMaxQV + t] != 255) { move = (int)t; break; }
            if (move < 0) break;
            forced[move] = 1;
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
        const bool known = !q.labels.empty();
        for (uint32_t t = n_core; t < q.qv; ++t)
            for (uint32_t c = 0; c < n_core; ++c)
                if (!known || lab(p.vs[c]) == lab(p.vs[t])) p.excl[t] |= (uint16_t)(1u << c);
        if (known && n_core > 2 && n_core < q.qv) {
            bool cst = true;
            const uint32_t jl = n_core - 1;
            for (uint32_t t = n_core; t < q.qv; ++t) {
                cst &= lab(p.vs[t]) != lab(p.vs[jl]);
                for (uint32_t b = p.bn_off[t]; b < p.bn_off[t + 1]; ++b) cst &= p.bn_pos[b] != jl;
            }
            p.tail_const = cst ? 1 : 0;
        }
        for (uint32_t t = n_core; t < q.qv; ++t) {
            for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2)
                if (p.bn_pos[b2] + 1u < n_core) p.tail_dep = std::max<uint8_t>(p.tail_dep, p.bn_pos[b2]);
            for (uint32_t c = 0; c + 1 < n_core; ++c)
                if ((p.excl[t] >> c) & 1u) p.tail_dep = std::max<uint8_t>(p.tail_dep, (uint8_t)c);
        }
        if (lane_tail && n_core >= 2 && n_core < q.qv && !p.tail_const) {
            // tail vertices hanging off the last core vertex: lane-countable
            // when each has one list and a label group of its own
            bool off_last = false, single = true;
            for (uint32_t t = n_core; t < q.qv; ++t) {
                bool t_off = false;
                for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2) t_off |= p.bn_pos[b2] + 1u == n_core;
                if (!t_off) continue;
                off_last = true;
                const bool alone = (t == n_core || p.tail_gid[t - 1] != p.tail_gid[t]) &&
                                   (t + 1 == q.qv || p.tail_gid[t + 1] != p.tail_gid[t]);
                single &= alone && p.bn_off[t + 1] - p.bn_off[t] == 1;
            }
            p.tail_lane = !off_last ? 1 : (single ? 2 : 0);
        }
        if (pendant) {
            p.grouped = 1;
            for (uint32_t j = 2; j < n_core; ++j)
                if (lab(p.vs[j]) == lab(b)) p.hit_mask |= (uint16_t)(1u << j);
        }
        if (level_sum && analytic_tail && n_core >= 3 && (n_core == q.qv || p.tail_lane || p.tail_const)) {
            // one position: the last core position j
            const uint32_t j = n_core - 1;
            if (p.bn_off[j + 1] - p.bn_off[j] == 1 && !(p.grouped && ((p.hit_mask >> j) & 1u))) {
                bool ok = true;
                uint16_t tails = 0;
                for (uint32_t t = n_core; t < q.qv; ++t) {
                    bool off = false;
                    for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2) off |= p.bn_pos[b2] == j;
                    if (off) {
                        tails |= (uint16_t)(1u << t);
                        ok &= (p.excl[t] & ((1u << j) - 1u)) == 0;
                    } else {
                        ok &= ((p.excl[t] >> j) & 1u) == 0;
                    }
                }
                if (ok) {
                    p.sum_from = (uint8_t)j;
                    p.sum_tails = tails;
                    for (uint32_t t = 0; t < j; ++t)
                        if (!known || lab(p.vs[t]) == lab(p.vs[j])) p.sum_same |= (uint16_t)(1u << t);
                }
            }
        }
        if (level_sum && dense_sums && analytic_tail && known && n_core >= 4) {
            // several positions [s, n_core) with labels of their own: the
            // smallest s >= 2 whose positions each have one backward list and
            // whose pendant tails are single-list groups with labels of their own
            std::vector<uint32_t> lcount(64, 0);
            for (uint32_t u = 0; u < q.qv; ++u)
                if (q.labels[u] < lcount.size()) ++lcount[q.labels[u]];
            auto unique = [&](uint32_t u) { return q.labels[u] < lcount.size() && lcount[q.labels[u]] == 1; };
            auto pos_ok = [&](uint32_t k, uint16_t& tails) {
                if (p.bn_off[k + 1] - p.bn_off[k] != 1 || !unique(p.vs[k])) return false;
                uint32_t nt = 0, nch = 0;
                for (uint32_t t = n_core; t < q.qv; ++t) {
                    bool off = false;
                    for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2) off |= p.bn_pos[b2] == k;
                    if (!off) continue;
                    const bool alone = (t == n_core || p.tail_gid[t - 1] != p.tail_gid[t]) &&
                                       (t + 1 == q.qv || p.tail_gid[t + 1] != p.tail_gid[t]);
                    if (p.bn_off[t + 1] - p.bn_off[t] != 1 || !alone || !unique(p.vs[t])) return false;
                    tails |= (uint16_t)(1u << t);
                    ++nt;
                }
                for (uint32_t l = k + 1; l < n_core; ++l) nch += p.bn_pos[p.bn_off[l]] == k ? 1u : 0u;
                return nt <= kMaxSumTails && nch <= kMaxSumChildren;
            };
            uint32_t best = n_core;
            uint16_t best_tails = 0;
            for (uint32_t s0 = n_core - 1; s0 >= 2; --s0) {
                uint16_t tails = 0;
                bool ok = true;
                for (uint32_t k = s0; k < n_core && ok; ++k) ok = pos_ok(k, tails);
                if (ok) { best = s0; best_tails = tails; }
                else break;  // a position that fails stays inside every larger range
            }
            if (best + 1 < n_core) {
                p.sum_from = (uint8_t)best;
                p.sum_dense = 1;
                p.sum_tails = best_tails;
                p.sum_same = 0;  // labels of their own: no prefix vertex can lie in a G_k
            }
        }
        if (level_sum && analytic_tail && n_core >= 4) {
            // pair counting at the last core position
            const uint32_t j = n_core - 1;
            if (p.bn_off[j + 1] - p.bn_off[j] == 2) {
                const uint32_t b0 = p.bn_off[j], b1 = b0 + 1;
                const bool first_prev = p.bn_pos[b0] == j - 1;
                const uint32_t bb = first_prev ? b0 : b1, ba = first_prev ? b1 : b0;
                bool ok = p.bn_pos[bb] == j - 1 && p.bn_pos[ba] < j - 1;
                for (uint32_t t = n_core; t < q.qv && ok; ++t) {
                    for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2) ok &= p.bn_pos[b2] + 1u < j;
                    ok &= ((p.excl[t] >> (j - 1)) & 3u) == 0;
                }
                if (p.grouped) ok &= ((p.hit_mask >> (j - 1)) & 3u) == 0;
                if (ok) {
                    p.pair_last = 1;
                    p.pair_a = (uint8_t)ba;
                    p.pair_b = (uint8_t)bb;
                    for (uint32_t t = 0; t + 1 < j; ++t)
                        if (!known || lab(p.vs[t]) == lab(p.vs[j])) p.pair_excl |= (uint16_t)(1u << t);
                }
            }
        }
        if (level_sum && known && analytic_tail && n_core >= 4) {
            // subtree memo: the first split [s, n_core), with the latest prefix
            // position p < s that works (not a seed-group position), such that
            // every backward list of the range and every tail list hangs off p
            // or the range
            auto in_range = [&](uint32_t pos, uint32_t s0, uint32_t p0) { return pos == p0 || pos >= s0; };
            for (uint32_t s0 = 2; s0 + 2 <= n_core && !p.memo_from; ++s0) {
                for (int pp = (int)s0 - 1; pp >= 0 && !p.memo_from; --pp) {
                    const uint32_t p0 = (uint32_t)pp;
                    if (p.grouped && p0 < 2) continue;  // one unit per first vertex: no reuse
                    bool ok = true;
                    for (uint32_t k = s0; k < n_core && ok; ++k)
                        for (uint32_t b2 = p.bn_off[k]; b2 < p.bn_off[k + 1]; ++b2)
                            ok &= in_range(p.bn_pos[b2], s0, p0);
                    for (uint32_t t = n_core; t < q.qv && ok; ++t) {
                        for (uint32_t b2 = p.bn_off[t]; b2 < p.bn_off[t + 1]; ++b2)
                            ok &= in_range(p.bn_pos[b2], s0, p0);
                        for (uint32_t c = 0; c < s0; ++c)
                            if (c != p0) ok &= ((p.excl[t] >> c) & 1u) == 0;
                    }
                    for (uint32_t k = s0; k < n_core && ok; ++k)
                        for (uint32_t c = 0; c < s0; ++c)
                            if (c != p0) ok &= lab(p.vs[k]) != lab(p.vs[c]);
                    if (p.grouped) ok &= (p.hit_mask >> s0) == 0;
                    // dense sums that already cover the range leave nothing to reuse
                    if (p.sum_dense && p.sum_from <= s0) ok = false;
                    if (ok) {
                        p.memo_from = (uint8_t)s0;
                        p.memo_pos = (uint8_t)p0;
                    }
                }
            }
        }
    }
}

void select_starting_edge(const QueryMeta& q, const uint64_t* card, const float* avg, uint32_t out[2]) {
    std::vector<uint32_t> sel, nxt;
    // 1. largest endpoint degree sum
    size_t best = 0;
    for (uint32_t e = 0; e < q.qe; ++e) {
        const size_t sd = q.nbrs[q.qe_u[e]].size() + q.nbrs[q.qe_v[e]].size();
        if (sd > best) { best = sd; sel.assign(1, e); }
        else if (sd == best) sel.push_back(e);
    }
    // 2. most triangles
    if (sel.size() > 1) {
        uint32_t bt = 0;
        nxt.clear();
        for (uint32_t e : sel) {
            const uint32_t a = q.qe_u[e], b = q.qe_v[e];
            uint32_t t = 0;
            for (uint32_t x = 0; x < q.qv; ++x)
                t += (q.eidx[x * kMaxQV + a] != 255 && q.eidx[x * kMaxQV + b] != 255) ? 1u : 0u;
            if (t > bt) { bt = t; nxt.assign(1, e); }
            else if (t == bt) nxt.push_back(e);
        }
        sel.swap(nxt);
    }
    // 3. fewest index entries on (a -> b)
    if (sel.size() > 1) {
        uint64_t bc = UINT32_MAX;
        nxt.clear();
        for (uint32_t e : sel) {
            const uint64_t c = card[q.eidx[q.qe_u[e] * kMaxQV + q.qe_v[e]]];
            if (c < bc) { bc = c; nxt.assign(1, e); }
            else if (c == bc) nxt.push_back(e);
        }
        sel.swap(nxt);
    }
    // 4. smallest sum of the other incident directions' mean list lengths
    //    (float, summed in neighbour order as the reference does)
    if (sel.size() > 1) {
        float bs = std::numeric_limits<float>::max();
        nxt.clear();
        for (uint32_t e : sel) {
            const uint32_t a = q.qe_u[e], b = q.qe_v[e];
            float sum = 0.0f;
            for (uint32_t w : q.nbrs[a])
                if (w != b) sum += avg[q.eidx[a * kMaxQV + w]];
            for (uint32_t w : q.nbrs[b])
                if (w != a) sum += avg[q.eidx[b * kMaxQV + w]];
            if (sum < bs) { bs = sum; nxt.assign(1, e); }
            else if (sum == bs) nxt.push_back(e);
        }
        sel.swap(nxt);
    }
    out[0] = q.qe_u[sel[0]];
    out[1] = q.qe_v[sel[0]];
}

std::string plan_valid_bits(const QueryMeta& q, const uint32_t start[2], VbPlan* plans) {
    const uint32_t qv = q.qv;
    auto adj = [&](uint32_t a, uint32_t b) { return q.eidx[a * kMaxQV + b] != 255; };
    for (uint32_t ei = 0; ei < q.qe; ++ei) {
        VbPlan& P = plans[ei];
        std::memset(&P, 0, sizeof(P));
        const uint32_t u0 = q.qe_u[ei], u1 = q.qe_v[ei];
        // indexing order: BFS by levels, neighbours ascending
        std::vector<uint32_t> order{u0, u1};
        std::vector<char> vis(qv, 0);
        vis[u0] = vis[u1] = 1;
        for (size_t lo = 0; lo < order.size();) {
            const size_t hi = order.size();
            for (size_t i = lo; i < hi; ++i)
                for (uint32_t w : q.nbrs[order[i]])
                    if (!vis[w]) { vis[w] = 1; order.push_back(w); }
            lo = hi;
        }
        if (order.size() != qv) return "query is not connected";
        uint32_t k = 0;
        for (uint32_t j = 0; j < qv; ++j) {
            P.vs[j] = (uint8_t)order[j];
            P.off[j] = (uint8_t)k;
            for (uint32_t t = 0; t < j; ++t)
                if (adj(order[j], order[t])) {
                    const uint8_t d = q.eidx[order[j] * kMaxQV + order[t]];
                    P.bpos[k] = (uint8_t)t;
                    P.bdir[k] = d;
                    P.bvis[k] = q.dir_to_edge[d] <= ei ? 1 : 0;
                    ++k;
                }
        }
        P.off[qv] = (uint8_t)k;
        P.d01 = q.eidx[u0 * kMaxQV + u1];
        P.d10 = q.eidx[u1 * kMaxQV + u0];
        // rebuild edges: every simple path from a starting vertex to u0 or u1
        std::vector<char> f((size_t)qv * qv, 0);
        f[u0 * qv + u1] = f[u1 * qv + u0] = 1;
        for (int si = 0; si < 2; ++si) {
            std::vector<uint32_t> path(qv + 1, 0), ci(qv + 1, 0);
            std::vector<char> on(qv, 0);
            on[start[si]] = 1;
            path[0] = start[si];
            uint32_t depth = 1;
            for (;;) {
                const auto& nb = q.nbrs[path[depth - 1]];
                bool pushed = false;
                while (ci[depth] < nb.size()) {
                    const uint32_t nv = nb[ci[depth]];
                    if (on[nv]) { ++ci[depth]; continue; }
                    if (nv == u0 || nv == u1) {
                        path[depth] = nv;
                        for (uint32_t i = 0; i < depth; ++i)
                            f[path[i] * qv + path[i + 1]] = f[path[i + 1] * qv + path[i]] = 1;
                        ++ci[depth];
                        continue;
                    }
                    on[nv] = 1;
                    path[depth] = nv;
                    ++depth;
                    pushed = true;
                    break;
                }
                if (pushed) continue;
                ci[depth] = 0;
                if (--depth == 0) break;
                on[path[depth]] = 0;
                ++ci[depth];
            }
        }
        // rebuilt vertices: all or none of a vertex's backward edges rebuilt
        for (uint32_t i = 0; i < qv; ++i) {
            const uint32_t u = P.vs[i];
            if (i == 0) { P.rebuild |= (uint16_t)(1u << u); continue; }
            uint32_t sum = 0;
            for (uint32_t b = P.off[i]; b < P.off[i + 1]; ++b) sum += f[P.vs[P.bpos[b]] * qv + u] ? 1u : 0u;
            if (sum == P.off[i + 1] - P.off[i]) P.rebuild |= (uint16_t)(1u << u);
            else if (sum != 0) return "rebuild flags are inconsistent for this pattern (plan.cpp:1361-1366)";
        }
    }
    return "";
}

}  // namespace cgb
