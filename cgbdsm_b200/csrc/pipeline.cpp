// Stage-1 producer: CaLiG index + host staging -> per-batch keys (C ABI in cgbdsm.h).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "calig.h"
#include "cgbdsm.h"

namespace {

using Clock = std::chrono::high_resolution_clock;
inline double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}
inline uint64_t enc(uint32_t e, uint32_t u, uint32_t v) {
    return ((uint64_t)e << 59) | ((uint64_t)u << 32) | (uint64_t)v;
}

}  // namespace

struct cgb_producer {
    cgb::CaLiGIndex idx;
    std::string err;
    uint32_t batch_size = UINT32_MAX;
    uint32_t num_batches = 0, next_batch = 0;
    // query numbering (graph.cpp:137-148, 184-199)
    uint32_t qv = 0, qe = 0;
    std::vector<uint8_t> eidx;      // qv*qv
    std::vector<uint8_t> qe_dir;    // qe*2
    // compressed ids (calig_helper_gamma.cu:77-105)
    std::vector<uint32_t> dense;    // original -> compressed
    std::vector<uint32_t> new2old;
    std::vector<uint64_t> init_keys;
    std::vector<uint64_t> ins, del, delta;
    std::vector<uint8_t> edge_ok;

    inline uint32_t nid(uint32_t v) const { return v < dense.size() ? dense[v] : UINT32_MAX; }
    inline uint32_t dir(uint32_t ui, uint32_t uj) const { return eidx[ui * qv + uj]; }

    // New compressed ids go to lit, unmapped vertices in ascending id order:
    // slices of the id range are scanned on threads and numbered in order.
    void update_mapping() {
        const auto& li = idx.li();
        const uint32_t n = (uint32_t)li.size();
        const uint32_t T = n >= (1u << 16) ? idx.threads() : 1u;
        std::vector<std::vector<uint32_t>> fresh(T);
        cgb::run_threads(T, [&](uint32_t s) {
            for (uint32_t v = (uint32_t)((uint64_t)n * s / T); v < (uint32_t)((uint64_t)n * (s + 1) / T); ++v)
                if (li[v] && dense[v] == UINT32_MAX) fresh[s].push_back(v);
        });
        for (auto& f : fresh)
            for (uint32_t v : f) {
                dense[v] = (uint32_t)new2old.size();
                new2old.push_back(v);
            }
    }

    // Keys of the delta ops that `keep` accepts and whose ends are mapped, in
    // the ops' order (slices on threads, concatenated); per_dir counts them.
    template <class Keep>
    void encode(const std::vector<cgb::DeltaOp>& ops, Keep keep, std::vector<uint64_t>& out,
                std::vector<uint32_t>* per_dir) {
        const size_t n = ops.size();
        const uint32_t T = n >= (1u << 14) ? idx.threads() : 1u;
        std::vector<std::vector<uint64_t>> part(T);
        std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(32, 0));
        cgb::run_threads(T, [&](uint32_t s) {
            for (size_t i = n * s / T; i < n * (s + 1) / T; ++i) {
                const cgb::DeltaOp& d = ops[i];
                if (!keep(d)) continue;
                const uint32_t nu = nid(d.vi), nv = nid(d.vj);
                if (nu == UINT32_MAX || nv == UINT32_MAX) continue;
                const uint32_t dd = dir(d.ui, d.uj);
                part[s].push_back(enc(dd, nu, nv));
                cnt[s][dd]++;
            }
        });
        out.clear();
        for (auto& q : part) out.insert(out.end(), q.begin(), q.end());
        if (per_dir)
            for (auto& c : cnt)
                for (uint32_t dd = 0; dd < 32; ++dd) (*per_dir)[dd] += c[dd];
    }
};

extern "C" {

cgb_status cgb_producer_open(const char* query_path, const char* data_path, const char* update_path,
                             uint32_t batch_size_ints, uint32_t threads, cgb_producer** out) {
    if (!out || !query_path || !data_path) return CGB_ERR_ARG;
    auto* p = new cgb_producer();
    *out = p;
    p->idx.set_threads(threads);
    p->batch_size = batch_size_ints ? batch_size_ints : UINT32_MAX;
    std::string e = p->idx.load_query(query_path);
    // main_calig.cpp:93-101: a data path ending in ".graph" is text and takes
    // the update file; anything else is a binary CSR prefix whose update
    // stream is derived from the graph (the update path is ignored)
    const std::string dp = data_path;
    const bool text = dp.size() >= 6 && dp.compare(dp.size() - 6, 6, ".graph") == 0;
    if (e.empty()) e = text ? p->idx.load_graph(data_path) : p->idx.load_graph_bin(dp);
    if (e.empty() && text && update_path) e = p->idx.load_updates(update_path);
    if (!e.empty()) {
        p->err = e;
        return CGB_ERR_IO;
    }
    // directed numbering of query edges (graph.cpp:137-148)
    const auto& qn = p->idx.query_nbrs();
    p->qv = p->idx.query_size();
    if (p->qv > 12) { p->err = "query has more than 12 vertices (utils/config.h:5)"; return CGB_ERR_LIMIT; }
    p->eidx.assign((size_t)p->qv * p->qv, 255);
    uint32_t pos = 0;
    for (uint32_t u = 0; u < p->qv; ++u)
        for (uint32_t w : qn[u]) p->eidx[u * p->qv + w] = (uint8_t)pos++;
    if (pos > 32) { p->err = "query has more than 16 edges (5-bit directed index)"; return CGB_ERR_LIMIT; }
    for (uint32_t u = 0; u < p->qv; ++u)
        for (uint32_t w : qn[u])
            if (u < w) {
                p->qe_dir.push_back(p->eidx[u * p->qv + w]);
                p->qe_dir.push_back(p->eidx[w * p->qv + u]);
            }
    p->qe = (uint32_t)p->qe_dir.size() / 2;
    const uint32_t nu = p->idx.num_update_ints();
    p->num_batches = (p->batch_size >= nu) ? 1 : (uint32_t)(((uint64_t)nu + p->batch_size - 1) / p->batch_size);
    if (nu == 0) p->num_batches = 0;
    p->idx.construct();
    // ConvertGlobalIndex key generation (calig_helper_gamma.cu:248-277)
    p->dense.assign(p->idx.num_vertices(), UINT32_MAX);
    p->update_mapping();
    const auto& li = p->idx.li();
    for (uint32_t nu2 = 0; nu2 < (uint32_t)p->new2old.size(); ++nu2) {
        const uint32_t v = p->new2old[nu2];
        for (uint32_t ui = 0; ui < p->qv; ++ui) {
            if (!((li[v] >> ui) & 1u)) continue;
            for (uint32_t uj : qn[ui]) {
                const auto* L = p->idx.cand(v, ui, uj);
                if (!L) continue;
                const uint32_t d = p->dir(ui, uj);
                for (uint32_t vj : *L) {
                    const uint32_t nv = p->nid(vj);
                    if (nv != UINT32_MAX) p->init_keys.push_back(enc(d, nu2, nv));
                }
            }
        }
    }
    return CGB_OK;
}

void cgb_producer_close(cgb_producer* p) { delete p; }

const char* cgb_producer_last_error(const cgb_producer* p) { return p ? p->err.c_str() : "null producer"; }

uint32_t cgb_producer_num_batches(const cgb_producer* p) { return p ? p->num_batches : 0; }

cgb_status cgb_producer_initial(cgb_producer* p, const uint64_t** keys, uint64_t* n, uint32_t* dv_count) {
    if (!p || !keys || !n || !dv_count) return CGB_ERR_ARG;
    *keys = p->init_keys.data();
    *n = p->init_keys.size();
    *dv_count = (uint32_t)p->new2old.size();
    return CGB_OK;
}

cgb_status cgb_producer_vertex_map(const cgb_producer* p, const uint32_t** new2old, uint32_t* n) {
    if (!p || !new2old || !n) return CGB_ERR_ARG;
    *new2old = p->new2old.data();
    *n = (uint32_t)p->new2old.size();
    return CGB_OK;
}

cgb_status cgb_producer_next(cgb_producer* p, cgb_batch_keys* out) {
    if (!p || !out) return CGB_ERR_ARG;
    if (p->next_batch >= p->num_batches) {
        p->err = "no more batches";
        return CGB_ERR_STATE;
    }
    const uint32_t b = p->next_batch++;
    const uint32_t start = b * p->batch_size;
    const uint32_t count = std::min(p->batch_size, p->idx.num_update_ints() - start);
    auto t0 = Clock::now();
    p->idx.update_index(start, count);
    const double t_ui = ms_since(t0);
    t0 = Clock::now();
    p->idx.construct_update(start, count);
    const double t_cu = ms_since(t0);
    t0 = Clock::now();
    // PrepareUpdateAll (calig_helper_gamma.cu:363-401): mapping first, then
    // LI-filtered insert keys and delete keys, both restricted to mapped ids
    p->update_mapping();
    const auto& li = p->idx.li();
    p->encode(p->idx.delta_ins, [&](const cgb::DeltaOp& d) { return ((li[d.vi] >> d.ui) & 1u) != 0; }, p->ins,
              nullptr);
    p->encode(p->idx.delta_del, [](const cgb::DeltaOp&) { return true; }, p->del, nullptr);
    // PrepareUpdateIndex (calig_helper_gamma.cu:403-445)
    std::vector<uint32_t> per_dir(32, 0);
    p->encode(p->idx.delta_update, [](const cgb::DeltaOp&) { return true; }, p->delta, &per_dir);
    p->edge_ok.assign(p->qe, 0);
    for (uint32_t e = 0; e < p->qe; ++e)
        p->edge_ok[e] = per_dir[p->qe_dir[2 * e]] && per_dir[p->qe_dir[2 * e + 1]];
    const double t_pr = ms_since(t0);
    std::memset(out, 0, sizeof(*out));
    out->ins = p->ins.data();
    out->n_ins = p->ins.size();
    out->del = p->del.data();
    out->n_del = p->del.size();
    out->delta = p->delta.data();
    out->n_delta = p->delta.size();
    out->edge_ok = p->edge_ok.data();
    out->qe = p->qe;
    out->dv_count = (uint32_t)p->new2old.size();
    out->batch = b;
    out->num_edges = count / 2;
    out->ms_update_index = t_ui;
    out->ms_construct_update = t_cu;
    out->ms_prepare = t_pr;
    return CGB_OK;
}

}  // extern "C"
