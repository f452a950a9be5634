// Query pattern metadata and per-edge matching plans (host side).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cgb {

constexpr int kMaxQV = 12;   // utils/config.h:5 (MAX_VCOUNT)
// Query edges of a pattern.  The single-query engine's keys carry the directed
// query-edge index in 5 bits (calig_helper_gamma.cu:228), so it takes at most
// kMaxQEKeyed edges; the multi-query engine keys its index by data-vertex
// label instead and takes up to kMaxQE (dense 11- and 12-vertex patterns).
constexpr int kMaxQE = 32;
constexpr int kMaxQEKeyed = 16;
constexpr int kMaxDir = 2 * kMaxQE;
constexpr int kMaxBN = 48;

// Query graph metadata, numbered exactly as the reference numbers it:
//   dir index  graph.cpp:137-148  (vertex ascending, neighbour ascending)
//   edge order graph.cpp:184-199  ((u, uu) with u < uu, u ascending then uu)
struct QueryMeta {
    uint32_t qv = 0, qe = 0, nd = 0;
    std::vector<uint32_t> labels;                  // query labels; empty = unknown (all leaves may collide)
    std::vector<std::vector<uint32_t>> nbrs;       // sorted neighbour lists
    uint8_t eidx[kMaxQV * kMaxQV];                 // 255 = no edge
    uint8_t qe_u[kMaxQE], qe_v[kMaxQE];            // undirected edges
    uint8_t qe_dir[kMaxQE][2];                     // eidx(u,v), eidx(v,u)
    uint8_t dir_to_edge[kMaxDir];
    uint8_t dir_src[kMaxDir], dir_dst[kMaxDir];
};

// Matching plan of one query edge ei: vertex order starting at ei's endpoints,
// and for every later position the backward neighbours (BN) whose lists
// constrain it.  bn_dvis marks BN directions whose delta part is visible to
// ei (dir_to_edge < ei; enumeration.cu:937, cpu_dfs.cpp:76-77).
//
// Positions [n_core, n) form the tail: mutually non-adjacent vertices whose
// neighbours are all core vertices (so every neighbour is a backward
// neighbour).  Their count is computed instead of enumerated: per label group
// (tail_gid, contiguous) of k <= 3 vertices, the number of injective
// assignments of the group to its candidate sets (intersections of resolved
// lists) minus the matched core vertices, by inclusion-exclusion.  Vertices of
// different labels have disjoint candidate sets, so groups multiply.
struct EdgePlan {
    uint8_t n;
    uint8_t n_core;
    uint8_t seed_dir;
    uint8_t vs[kMaxQV];
    uint8_t bn_off[kMaxQV + 1];
    uint8_t bn_pos[kMaxBN];
    uint8_t bn_dir[kMaxBN];
    uint8_t bn_dvis[kMaxBN];
    uint8_t tail_gid[kMaxQV];
    // tail_const: the last core vertex has no tail neighbour and its label
    // differs from every tail label, so the tail count is the same for every
    // candidate of the last core position (labels must be known).
    uint8_t tail_const;
    // grouped: vs[1] is a pendant (query degree 1, only neighbour vs[0]) and
    // no tail vertex shares its label.  Then the count of a seed (x, y)
    // depends on x only through injectivity, so one DFS per y serves every
    // seed edge at y: with X = y's delta list towards vs[1] (sorted, the
    // seeds' x values with multiplicity), each embedding of the other
    // vertices counts |X| minus the multiplicity in X of the vertices it
    // places at hit_mask positions (core positions with vs[1]'s label).
    uint8_t grouped;
    // excl[t] (tail position t): core positions whose matched vertex can lie
    // in t's candidate sets (same label; every core position when labels are
    // unknown); only those are excluded from t's counts.
    uint16_t excl[kMaxQV];
    uint16_t hit_mask;
    // Level sums: core positions [sum_from, n_core) are counted, not
    // enumerated.  Each such position k has one backward list G_k owned by a
    // position p_k < k, and the tail vertices with a list at k are pendants
    // of k (one list, a label group of their own), collected in sum_tails.
    // With W_k(x) = sum over c in G_k(x) of the lengths of c's lists towards
    // its pendants times W_l(c) for every position l owned by k, a prefix
    // m[0..sum_from) contributes the product of W_r(m[p_r]) over the
    // positions r with p_r < sum_from, times the prefix-only tail count.
    //   sum_from = n_core - 1 (sum_dense 0): one position j; no prefix
    //     position shares a label with its pendants, no prefix-only tail
    //     group shares the label of vs[j], and the matched prefix vertices at
    //     positions sum_same (same label as vs[j]) that lie in G are
    //     subtracted per prefix; W is computed on demand per (plan, vertex)
    //     and launch, shared through a table.
    //   sum_from < n_core - 1 (sum_dense 1): every position in the range and
    //     every pendant of one has a label no other query vertex has, so no
    //     two of them can coincide; W_k is precomputed for every vertex
    //     before the launch (children first) into array wslot + k - sum_from.
    uint16_t sum_tails;
    uint16_t sum_same;  // positions < j whose vertex can lie in G (same label)
    // tail_lane: each lane evaluates its own candidate's tail count at the
    // last core position.  1: no tail list hangs off the last core vertex,
    // so a candidate changes the tail count only by lying in prefix-only
    // lists (same label).  2: as 1, except for tail vertices whose only list
    // hangs off the last core vertex and whose label group they form alone:
    // such a count is the length of the candidate's list minus the excluded
    // prefix vertices in it.  0: the warp counts one embedding at a time.
    uint8_t tail_lane;
    // tail_dep: the deepest core position below n_core - 1 that a tail count
    // reads (a list's owner or an excluded vertex); a prefix change at a
    // deeper position leaves every prefix-only tail count as it was.
    uint8_t tail_dep;
    uint8_t sum_from;   // 0: no level sums
    uint8_t sum_dense;
    uint8_t wslot;
    // kPlan* bits: per-plan schedule choices (the multi-query autotuner's)
    uint8_t flags;
    // Subtree memo: every backward list of positions [memo_from, n_core) and
    // every list of the tail sits at position memo_pos or inside that range,
    // the range's core vertices share no label with prefix positions other
    // than memo_pos, no tail excludes such a position, and (grouped plans) no
    // position of the range is a hit position.  The count below depth
    // memo_from is then a function of m[memo_pos] alone: the normal DFS
    // counts it (unweighted, weighted once when complete) and, when none of
    // it went to other warps, shares it through the level-sum table, once per
    // (plan, vertex) and launch.  0: none.
    uint8_t memo_from;
    uint8_t memo_pos;
    // Pair counting at the last core position j = n_core - 1: its two lists
    // are bn[pair_a] (owned by a position < j - 1) and bn[pair_b] (owned by
    // j - 1), and no tail list or tail exclusion involves j - 1 or j.  Each
    // lane then counts its own depth-(j - 1) candidate's last level as the
    // intersection size of the two lists, less the matched prefix vertices
    // at positions pair_excl (same label as vs[j]) lying in both, times the
    // prefix-only tail count, instead of the warp descending into it.
    uint8_t pair_last;
    uint8_t pair_a, pair_b;
    uint8_t pad_;
    uint16_t pair_excl;
    uint16_t pad2_;
};
constexpr uint8_t kPlanNoTailCache = 0x1;  // recount every tail subset per core embedding
constexpr uint32_t kMaxSumTails = 4;     // pendant tails per dense level-sum position
constexpr uint32_t kMaxSumChildren = 4;  // level-sum positions owned by one dense level-sum position

// Valid-bit plan of one query edge ei (the reference's 1-bit support masks,
// BuildLocalIndexBitAll, graph_gpu.cu:803-869): its indexing order (BFS from
// ei's endpoints, plan.cpp:1180-1230), each position's backward neighbours
// with the direction vs[d] -> neighbour and whether that direction's delta
// part is visible while building (dir_to_edge <= ei, indexing.cu:2345), and
// the rebuilt vertices (plan.cpp:1277-1370); other vertices' masks are all
// ones.
struct VbPlan {
    uint8_t vs[kMaxQV];
    uint8_t off[kMaxQV + 1];
    uint8_t bpos[kMaxBN];
    uint8_t bdir[kMaxBN];
    uint8_t bvis[kMaxBN];
    uint16_t rebuild;
    uint8_t d01, d10;  // directions vs[0] -> vs[1] and back
};

// SelectStartingEdge (plan.cpp:428-533): the first two vertices of the
// reference's global order from the query and the initial index's
// per-direction entry counts and mean list lengths.
void select_starting_edge(const QueryMeta& q, const uint64_t* card, const float* avg, uint32_t out[2]);
// Valid-bit plans for every query edge; "" or the reference's order error
// (plan.cpp:1361-1366).
std::string plan_valid_bits(const QueryMeta& q, const uint32_t start[2], VbPlan* plans);

// Returns "" on success, else an error message; at most max_qe edges.
std::string build_query_meta(uint32_t qv, uint32_t qe, const uint32_t* edges, const uint32_t* labels,
                             QueryMeta& q, uint32_t max_qe = kMaxQEKeyed);
std::string parse_query_file(const std::string& path, std::vector<uint32_t>& labels,
                             std::vector<uint32_t>& edges, uint32_t& qv);
// avg_deg[dir]: mean run length of direction dir in the initial index.
// analytic_tail = false keeps every vertex in the enumerated core.
// pick_last = true puts the core vertex with the fewest tail neighbours last.
// group_pendant = true groups the seeds of edges with a pendant endpoint
// (EdgePlan::grouped; needs labels).  lane_tail = false leaves tail_lane 0;
// level_sum = false leaves sum_from 0; dense_sums = false allows only the
// one-position (table) level sums.  wslot is left 0 (the engine assigns it).
void plan_edges(const QueryMeta& q, const float* avg_deg, EdgePlan* plans, bool analytic_tail = true,
                bool pick_last = true, bool group_pendant = true, bool lane_tail = true, bool level_sum = true,
                bool dense_sums = false);

}  // namespace cgb
