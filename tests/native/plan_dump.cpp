// Prints the matching plans cgb::plan_edges makes for a query file (one line
// per query edge, space-separated fields and '|'-separated arrays), with the
// single-query engine's options (dense level sums on) or, with a second
// argument "mq", the multi-query engine's (one-position level sums only).
// Mean list lengths are taken as 1 for every direction.
#include <cstdio>
#include <string>
#include <vector>

#include "query.h"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::vector<uint32_t> labels, edges;
    uint32_t qv = 0;
    std::string err = cgb::parse_query_file(argv[1], labels, edges, qv);
    if (!err.empty()) { std::printf("error %s\n", err.c_str()); return 1; }
    const bool mq = argc > 2 && std::string(argv[2]) == "mq";
    cgb::QueryMeta q;
    err = cgb::build_query_meta(qv, (uint32_t)(edges.size() / 2), edges.data(), labels.data(), q,
                                mq ? cgb::kMaxQE : cgb::kMaxQEKeyed);
    if (!err.empty()) { std::printf("error %s\n", err.c_str()); return 1; }
    float avg[cgb::kMaxDir];
    for (float& x : avg) x = 1.f;
    std::vector<cgb::EdgePlan> plans(cgb::kMaxQE);
    cgb::plan_edges(q, avg, plans.data(), true, true, true, true, true, !mq);
    for (uint32_t ei = 0; ei < q.qe; ++ei) {
        const cgb::EdgePlan& p = plans[ei];
        std::printf("%u %u %u %u %u %u %u %u %u %u %u %u %u %u %u %u |", ei, p.n, p.n_core, p.sum_from, p.sum_dense,
                    p.sum_tails, p.sum_same, p.memo_from, p.memo_pos, p.grouped, p.hit_mask, p.tail_lane, p.pair_last,
                    p.pair_a, p.pair_b, p.pair_excl);
        for (uint32_t j = 0; j < p.n; ++j) std::printf(" %u", p.vs[j]);
        std::printf(" |");
        for (uint32_t j = 0; j <= p.n; ++j) std::printf(" %u", p.bn_off[j]);
        std::printf(" |");
        for (uint32_t b = 0; b < p.bn_off[p.n]; ++b) std::printf(" %u", p.bn_pos[b]);
        std::printf(" |");
        for (uint32_t j = 0; j < p.n; ++j) std::printf(" %u", p.excl[j]);
        std::printf(" |");
        for (uint32_t j = 0; j < p.n; ++j) std::printf(" %u", p.tail_gid[j]);
        std::printf("\n");
    }
    return 0;
}
