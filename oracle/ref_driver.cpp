// Oracle driver for the REFERENCE CPU path (test infrastructure only).
//
// Linked against the reference's own, unmodified CPU sources compiled where
// they lie (index/calig.cpp, graph/graph.cpp, graph/plan.cpp,
// index/cpu_index_mirror.cpp, index/cpu_dfs.cpp, utils/constants.cpp) by
// oracle/Makefile into oracle/_ref/libcgbref.so.  Only tests/, the smoke check
// and bench.py's reference/cpu_baseline legs load that library; the product
// never does.
//
// The reference keeps its host-side staging inside a CUDA translation unit
// (index/calig_helper_gamma.cu), which cannot run without a GPU, so this file
// restates those host-only steps, each citing the reference lines it follows:
//   * compressed vertex ids      calig_helper_gamma.cu:77-105, 132-181
//   * initial key generation     calig_helper_gamma.cu:238-277, 304-311
//   * PrepareUpdateAll           calig_helper_gamma.cu:363-401
//   * PrepareUpdateIndex         calig_helper_gamma.cu:403-445
//   * per-batch S2 order         main_calig.cpp:281-384 and
//                                calig_helper_gamma.cu:485-517, 539-597
//   * mask-free host seed        enumeration.cu:727-809 (writeInitialResultsAllBit
//                                without the support-mask prune, which the
//                                reference documents as count-preserving,
//                                cpu_dfs.h:21-29)
// and then calls the reference's CPUIndexMirror and cpuExtendBFSAllBitCount.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "tbb/parallel_for.h"
#include "utils/config.h"
#include "utils/constants.h"
#include "graph/graph.h"
#include "graph/plan.h"
#include "index/calig.h"
#include "index/cpu_dfs.h"
#include "index/cpu_index_mirror.h"

namespace {

using Clock = std::chrono::high_resolution_clock;
inline double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}
inline uint64_t enc(uint32_t e, uint32_t u, uint32_t v) {
    return ((uint64_t)e << 59) | ((uint64_t)u << 32) | (uint64_t)v;
}

struct RefPipeline {
    std::string qpath, dpath, upath;
    uint32_t batch_size = UINT32_MAX;
    uint32_t num_updates = 0, num_batches = 0, next_batch = 0;
    bool quiet = true;

    CaLiG* calig = nullptr;
    QueryGraph query;
    Plan* plan = nullptr;
    CPUIndexMirror* mirror = nullptr;
    uint32_t num_dir = 0;

    // compressed ids (calig_helper_gamma.cu:35-37)
    ska::flat_hash_map<uint32_t, uint32_t> vid2new;
    std::vector<uint32_t> dense_map;  // original -> compressed (UINT32_MAX = unmapped)
    std::vector<uint32_t> new2old;    // compressed -> original
    uint32_t dv_count = 0;

    uint32_t cardinalities[MAX_ECOUNT * 2] = {0};
    float avg_degrees[MAX_ECOUNT * 2] = {0};
    std::vector<uint64_t> init_keys;

    // last batch
    std::vector<uint64_t> ins_keys, del_keys, delta_keys;
    std::vector<uint8_t> edge_ok;
    uint64_t last_count = 0;
    uint64_t last_seed_rows = 0;
    bool last_matched = false;
    double t_s1_ms = 0, t_stage_ms = 0, t_mirror_ms = 0, t_match_ms = 0;
    uint64_t total_count = 0;
    int dfs_parallel = 0;
    int do_count = 1;
    // bounded sampling of the count (bench baseline): stop after budget_ms
    double sample_budget_ms = 0;
    uint64_t sample_rows_done = 0, sample_rows_total = 0;
    double sample_ms = 0;
    // optional progress block (shared with a supervising process):
    // [0] rows done, [1] rows total, [2] S1 us, [3] staging us, [4] mirror us,
    // [5] count us so far, [6] phase (1 = S1 done, 2 = counting, 3 = finished)
    volatile uint64_t* progress = nullptr;

    // calig_helper_gamma.cu:77-105 (UpdateVertexMappingCPU) and :132-154
    // (buildGlobalVertexMapping): every vertex with any LI bit gets the next
    // compressed id, append-only.  The reference walks a hash set whose order
    // depends on thread scheduling; ids are compared in original-id space, so
    // ascending original-id order is used here.
    void update_mapping() {
        const uint32_t n = (uint32_t)calig->G.size();
        for (uint32_t v = 0; v < n; v++) {
            if (calig->G_Li[v] == 0) continue;
            if (dense_map[v] != UINT32_MAX) continue;
            uint32_t id = (uint32_t)vid2new.size();
            vid2new[v] = id;
            dense_map[v] = id;
            new2old.push_back(v);
        }
        dv_count = (uint32_t)vid2new.size();
    }
    inline uint32_t nid(uint32_t v) const {
        return v < dense_map.size() ? dense_map[v] : UINT32_MAX;
    }
    inline uint32_t eidx(uint32_t ui, uint32_t uj) const {
        return query.eidx_[ui * query.vcount_ + uj];
    }

    void open() {
        calig = new CaLiG();
        calig->inputQ(qpath);
        if (dpath.size() >= 6 && dpath.compare(dpath.size() - 6, 6, ".graph") == 0) {
            calig->inputG(dpath);
            calig->inputUpdate(upath, 0);
        } else {
            calig->inputGBin(dpath);
        }
        num_updates = calig->getUpdateSize();
        num_batches = (batch_size >= num_updates) ? 1 : (num_updates + batch_size - 1) / batch_size;
        calig->constructCand(num_batches);
        calig->staticFilter();

        plan = new Plan(query);
        CPUGraphLoader cpu_loader(qpath, query);
        cpu_loader.SetQueryMeta();
        plan->GenerateIndexingOrders_v2();
        num_dir = 0;
        for (uint32_t u = 0; u < calig->Q.size(); ++u) num_dir += (uint32_t)calig->Q[u].nei.size();
        mirror = new CPUIndexMirror(plan->query_, *plan, num_dir);

        dense_map.assign(calig->G.size(), UINT32_MAX);
        update_mapping();
        DV_COUNT = dv_count;

        // calig_helper_gamma.cu:248-277: keys of every lit (u_q) candidate list,
        // restricted to mapped targets; cardinalities / avg degrees :304-311.
        uint32_t nodes[MAX_ECOUNT * 2] = {0};
        init_keys.clear();
        for (uint32_t new_u = 0; new_u < dv_count; ++new_u) {
            uint32_t u_data = new2old[new_u];
            if (calig->G_Li[u_data] == 0) continue;
            for (auto const& kv : calig->G[u_data].cand) {
                uint32_t u_q = (uint32_t)kv.first;
                if (!(calig->G_Li[u_data] & (1u << u_q))) continue;
                for (auto const& kv2 : kv.second) {
                    uint32_t v_q = (uint32_t)kv2.first;
                    uint32_t e = eidx(u_q, v_q);
                    uint32_t sz = 0;
                    for (auto v_data : kv2.second) {
                        uint32_t new_v = nid((uint32_t)v_data);
                        if (new_v == UINT32_MAX) continue;
                        cardinalities[e]++;
                        sz++;
                        init_keys.push_back(enc(e, new_u, new_v));
                    }
                    nodes[e] += (sz != 0);
                }
            }
        }
        std::sort(init_keys.begin(), init_keys.end());
        for (uint32_t e = 0; e < num_dir; ++e)
            avg_degrees[e] = nodes[e] > 0 ? (float)cardinalities[e] / nodes[e] : 0.0f;
        mirror->ResizeForDVCount(dv_count);
        mirror->InitFromSortedEdges(init_keys);
        plan->GenerateMatchingOrders_v2(cardinalities, avg_degrees);
    }

    // One batch: S1 (main_calig.cpp:220-251) then S2 (main_calig.cpp:281-384)
    // against the host mirror, with the mask-free seed + reference DFS count.
    int step() {
        if (next_batch >= num_batches) return -1;
        const uint32_t b = next_batch++;
        const uint32_t start = b * batch_size;
        const uint32_t count = std::min(batch_size, calig->getUpdateSize() - start);

        auto t0 = Clock::now();
        calig->updateIndex(start, count, b);
        calig->ConstructUpdate(start, count);
        calig->mergeDeltas(b);
        t_s1_ms = ms_since(t0);
        if (progress) { progress[2] = (uint64_t)(t_s1_ms * 1e3); progress[6] = 1; }

        t0 = Clock::now();
        // PrepareUpdateAll (calig_helper_gamma.cu:363-401)
        update_mapping();
        ins_keys.clear();
        for (auto const& d : calig->getInsDeltas(b)) {
            if (!(calig->G_Li[d.vi] & (1u << d.ui))) continue;
            uint32_t nu = nid(d.vi), nv = nid(d.vj);
            if (nu == UINT32_MAX || nv == UINT32_MAX) continue;
            ins_keys.push_back(enc(eidx(d.ui, d.uj), nu, nv));
        }
        del_keys.clear();
        for (auto const& d : calig->getDelDeltas(b)) {
            uint32_t nu = nid(d.vi), nv = nid(d.vj);
            if (nu == UINT32_MAX || nv == UINT32_MAX) continue;
            del_keys.push_back(enc(eidx(d.ui, d.uj), nu, nv));
        }
        // PrepareUpdateIndex (calig_helper_gamma.cu:403-445)
        delta_keys.clear();
        std::vector<uint32_t> dir_count(num_dir, 0);
        for (auto const& d : calig->getUpdateDeltas(b)) {
            uint32_t e = eidx(d.ui, d.uj);
            uint32_t nu = nid(d.vi), nv = nid(d.vj);
            if (nu == UINT32_MAX || nv == UINT32_MAX) continue;
            delta_keys.push_back(enc(e, nu, nv));
            dir_count[e]++;
        }
        edge_ok.assign(QE_COUNT, 0);
        for (uint32_t e = 0; e < QE_COUNT; ++e)
            edge_ok[e] = dir_count[query.qe_eidx_[e].first] && dir_count[query.qe_eidx_[e].second];
        t_stage_ms = ms_since(t0);

        // TransferUpdateAll (calig_helper_gamma.cu:485-517) on the mirror
        t0 = Clock::now();
        DV_COUNT = dv_count;
        mirror->ResizeForDVCount(dv_count);
        mirror->MergeInsert(ins_keys);
        mirror->MergeRemove(del_keys);
        t_mirror_ms = ms_since(t0);
        if (progress) { progress[3] = (uint64_t)(t_stage_ms * 1e3); progress[4] = (uint64_t)(t_mirror_ms * 1e3); }

        last_count = 0;
        last_seed_rows = 0;
        last_matched = false;
        t_match_ms = 0;
        // TransferUpdateIndex returns false on an empty delta: main_calig.cpp:301-302
        // then skips matching and BatchUpdateGlobalIndex for this batch.
        if (delta_keys.empty()) return (int)b;
        last_matched = true;
        t0 = Clock::now();
        mirror->RebuildUpdate(delta_keys);
        last_count = do_count ? count_matches() : 0;
        t_match_ms = ms_since(t0);
        total_count += last_count;

        // BatchUpdateGlobalIndex (calig_helper_gamma.cu:539-567): merge delta back.
        t0 = Clock::now();
        mirror->MergeInsert(delta_keys);
        t_mirror_ms += ms_since(t0);
        return (int)b;
    }

    // enumeration.cu:727-809 without masks, then cpu_dfs.cpp:137-170.
    // With sample_budget_ms > 0 the rows are counted in chunks until the budget
    // is spent; rows_done / rows_total are recorded for extrapolation.
    uint64_t count_matches() {
        auto t_begin = Clock::now();
        sample_rows_done = sample_rows_total = 0;
        const OrderPerEdge& go = plan->global_order_;
        const uint32_t qv0 = go.vs_[0], qv1 = go.vs_[1];
        const uint32_t idx = eidx(qv0, qv1);
        const uint8_t d2e = mirror->DirToEdge(idx);
        std::vector<uint32_t> rows;
        uint64_t total = 0;
        if (progress) {
            // total seed rows first, so a supervisor can extrapolate from rows done
            uint64_t all = 0;
            for (uint32_t ei = 0; ei < QE_COUNT; ++ei) {
                if (!edge_ok[ei]) continue;
                const auto& io = plan->indexing_orders_[ei];
                const uint32_t sa = eidx(io.vs_[0], io.vs_[1]), sb = eidx(io.vs_[1], io.vs_[0]);
                const bool upd = (idx == sa || idx == sb);
                for (uint32_t v = 0; v < dv_count; ++v) {
                    uint32_t bl = 0, al = 0;
                    if (upd) mirror->UpdateList(idx, v, bl); else mirror->MainList(idx, v, bl);
                    if (d2e < ei) mirror->UpdateList(idx, v, al);
                    all += bl + al;
                }
            }
            progress[1] = all;
            progress[0] = 0;
            progress[6] = 2;
        }
        for (uint32_t ei = 0; ei < QE_COUNT; ++ei) {
            if (!edge_ok[ei]) continue;
            const auto& io = plan->indexing_orders_[ei];
            const uint32_t sa = eidx(io.vs_[0], io.vs_[1]), sb = eidx(io.vs_[1], io.vs_[0]);
            const bool seed_is_update = (idx == sa || idx == sb);
            rows.clear();
            for (uint32_t v = 0; v < dv_count; ++v) {
                uint32_t bl = 0, al = 0;
                const uint32_t* base = seed_is_update ? mirror->UpdateList(idx, v, bl)
                                                      : mirror->MainList(idx, v, bl);
                const uint32_t* app = (d2e < ei) ? mirror->UpdateList(idx, v, al) : nullptr;
                for (uint32_t k = 0; k < bl; ++k) { rows.push_back((ei << 27) | v); rows.push_back(base[k]); }
                for (uint32_t k = 0; k < al; ++k) { rows.push_back((ei << 27) | v); rows.push_back(app[k]); }
            }
            const uint64_t n = rows.size() / 2;
            last_seed_rows += n;
            sample_rows_total += n;
            if (n == 0) continue;
            if (progress) {
                // supervised sample: every row on its own across all host threads,
                // with per-row progress (a supervisor stops the process at its deadline)
                std::atomic<uint64_t> acc{0};
                tbb::parallel_for((uint64_t)0, n, [&](uint64_t r) {
                    acc += cpuExtendBFSAllBitCount(rows.data() + 2 * r, 1, 2, *mirror, query, *plan);
                    __atomic_fetch_add((uint64_t*)&progress[0], 1ull, __ATOMIC_RELAXED);
                    progress[5] = (uint64_t)(ms_since(t_begin) * 1e3);
                });
                total += acc.load();
                sample_rows_done += n;
                continue;
            }
            const uint64_t chunk = sample_budget_ms > 0 ? 4096 : n;
            for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
                if (sample_budget_ms > 0 && ms_since(t_begin) > sample_budget_ms) break;
                const uint64_t k = std::min(chunk, n - r0);
                if (dfs_parallel) {
                    tbb::task_arena arena;
                    total += cpuExtendBFSAllBitCountParallel(rows.data() + 2 * r0, k, 2, *mirror, query, *plan, arena);
                } else {
                    total += cpuExtendBFSAllBitCount(rows.data() + 2 * r0, k, 2, *mirror, query, *plan);
                }
                sample_rows_done += k;
            }
        }
        sample_ms = ms_since(t_begin);
        if (progress) progress[6] = 3;
        return total;
    }

    // Main index as canonical keys in ORIGINAL vertex ids, sorted.
    void dump_main(std::vector<uint64_t>& out) const {
        out.clear();
        for (uint32_t d = 0; d < num_dir; ++d)
            for (uint32_t u = 0; u < dv_count; ++u) {
                uint32_t len = 0;
                const uint32_t* p = mirror->MainList(d, u, len);
                for (uint32_t k = 0; k < len; ++k)
                    out.push_back(((uint64_t)d << 59) | ((uint64_t)new2old[u] << 32) | new2old[p[k]]);
            }
        std::sort(out.begin(), out.end());
    }
};

std::string g_err;

}  // namespace

extern "C" {

void* cgbref_open(const char* q, const char* d, const char* u, uint32_t batch_size_ints, int quiet) {
    auto* p = new RefPipeline();
    p->qpath = q; p->dpath = d; p->upath = u ? u : "";
    p->batch_size = batch_size_ints;
    p->quiet = quiet != 0;
    std::streambuf* old = nullptr;
    std::ostringstream sink;
    if (p->quiet) old = std::cout.rdbuf(sink.rdbuf());
    p->open();
    if (old) std::cout.rdbuf(old);
    return p;
}
void cgbref_close(void* h) { delete (RefPipeline*)h; }
void cgbref_set_parallel_dfs(void* h, int on) { ((RefPipeline*)h)->dfs_parallel = on; }
// 0 = skip the match count (S1/staging/mirror only).
void cgbref_set_count(void* h, int on) { ((RefPipeline*)h)->do_count = on; }
// Bounded count: stop after budget_ms (0 = complete count).
void cgbref_set_sample_budget(void* h, double ms) { ((RefPipeline*)h)->sample_budget_ms = ms; }
// Progress block written while stepping (see RefPipeline::progress).
void cgbref_set_progress(void* h, uint64_t* p) { ((RefPipeline*)h)->progress = p; }
// Rows counted / rows total / ms spent in the last batch's count.
void cgbref_last_sample(void* h, uint64_t* done, uint64_t* total, double* ms) {
    auto* p = (RefPipeline*)h;
    *done = p->sample_rows_done; *total = p->sample_rows_total; *ms = p->sample_ms;
}
uint32_t cgbref_num_batches(void* h) { return ((RefPipeline*)h)->num_batches; }
uint32_t cgbref_num_updates(void* h) { return ((RefPipeline*)h)->num_updates; }
uint32_t cgbref_num_dir(void* h) { return ((RefPipeline*)h)->num_dir; }
uint32_t cgbref_qv(void* h) { return ((RefPipeline*)h)->query.vcount_; }
uint32_t cgbref_qe(void* h) { return ((RefPipeline*)h)->query.ecount_; }
uint32_t cgbref_dv_count(void* h) { return ((RefPipeline*)h)->dv_count; }
const uint32_t* cgbref_new2old(void* h) { return ((RefPipeline*)h)->new2old.data(); }
uint64_t cgbref_init_keys(void* h, const uint64_t** out) {
    auto* p = (RefPipeline*)h; *out = p->init_keys.data(); return p->init_keys.size();
}
void cgbref_free_init(void* h) { auto* p = (RefPipeline*)h; std::vector<uint64_t>().swap(p->init_keys); }
const uint32_t* cgbref_cardinalities(void* h) { return ((RefPipeline*)h)->cardinalities; }
const float* cgbref_avg_degrees(void* h) { return ((RefPipeline*)h)->avg_degrees; }
// Global matching order chosen by the reference planner (plan.cpp:535-745).
void cgbref_global_order(void* h, uint8_t* vs) {
    auto* p = (RefPipeline*)h;
    for (uint32_t i = 0; i < p->query.vcount_; ++i) vs[i] = p->plan->global_order_.vs_[i];
}
// Indexing order of query edge ei (plan.cpp:1180-1230): vertices, backward
// neighbour offsets and positions; returns the number of bni_ entries.
uint32_t cgbref_indexing_order(void* h, uint32_t ei, uint8_t* vs, uint8_t* offs, uint8_t* bni) {
    auto* p = (RefPipeline*)h;
    const auto& io = p->plan->indexing_orders_[ei];
    const uint32_t qv = p->query.vcount_;
    for (uint32_t i = 0; i < qv; ++i) vs[i] = io.vs_[i];
    for (uint32_t i = 0; i <= qv; ++i) offs[i] = io.bni_offs_[i];
    const uint32_t n = io.bni_offs_[qv];
    for (uint32_t i = 0; i < n; ++i) bni[i] = io.bni_[i];
    return n;
}
// Rebuild vertex flags of query edge ei (plan.cpp:1334-1370) as a bit mask.
uint32_t cgbref_rebuild_vertices(void* h, uint32_t ei) {
    auto* p = (RefPipeline*)h;
    uint32_t m = 0;
    for (uint32_t u = 0; u < p->query.vcount_; ++u)
        if (p->plan->rebuild_v_flags_[ei][u]) m |= 1u << u;
    return m;
}
int cgbref_step(void* h) {
    auto* p = (RefPipeline*)h;
    std::streambuf* old = nullptr;
    std::ostringstream sink;
    if (p->quiet) old = std::cout.rdbuf(sink.rdbuf());
    int r = p->step();
    if (old) std::cout.rdbuf(old);
    return r;
}
uint64_t cgbref_last_count(void* h) { return ((RefPipeline*)h)->last_count; }
int cgbref_last_matched(void* h) { return ((RefPipeline*)h)->last_matched ? 1 : 0; }
uint64_t cgbref_last_seed_rows(void* h) { return ((RefPipeline*)h)->last_seed_rows; }
uint64_t cgbref_total_count(void* h) { return ((RefPipeline*)h)->total_count; }
uint64_t cgbref_last_keys(void* h, int which, const uint64_t** out) {
    auto* p = (RefPipeline*)h;
    const std::vector<uint64_t>& v = which == 0 ? p->ins_keys : which == 1 ? p->del_keys : p->delta_keys;
    *out = v.data();
    return v.size();
}
const uint8_t* cgbref_last_edge_ok(void* h) { return ((RefPipeline*)h)->edge_ok.data(); }
void cgbref_last_times(void* h, double* t4) {
    auto* p = (RefPipeline*)h;
    t4[0] = p->t_s1_ms; t4[1] = p->t_stage_ms; t4[2] = p->t_mirror_ms; t4[3] = p->t_match_ms;
}
// Sorted main-index keys in original ids; returns count, fills up to cap.
uint64_t cgbref_dump_main(void* h, uint64_t* out, uint64_t cap) {
    auto* p = (RefPipeline*)h;
    std::vector<uint64_t> v;
    p->dump_main(v);
    if (out) std::memcpy(out, v.data(), sizeof(uint64_t) * std::min<uint64_t>(cap, v.size()));
    return v.size();
}
// LI bitmask per original vertex (calig.h:82).
uint64_t cgbref_li(void* h, uint32_t* out, uint64_t cap) {
    auto* p = (RefPipeline*)h;
    uint64_t n = p->calig->G_Li.size();
    if (out) std::memcpy(out, p->calig->G_Li.data(), sizeof(uint32_t) * std::min<uint64_t>(cap, n));
    return n;
}

}  // extern "C"
