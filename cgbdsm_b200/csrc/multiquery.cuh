// Multi-query engine: one device-resident data-graph index shared by many
// registered query patterns, every pattern matched per batch in one
// persistent launch.  Included by engine.cu (same translation unit: it reuses
// the index pool, the fused merge, the run bit sets and the warp DFS).
//
// The reference runs one query per process: a CaLiG candidate index per
// query (index/calig.cpp), GAMMA staging per query
// (index/calig_helper_gamma.cu:363-597) and one MatchingBitAll per batch
// (graph/graph_gpu.cu:1261-1480; main_calig.cpp:203-384).  Here the index is
// the data graph itself, keyed by target-vertex label: the list of (label L,
// vertex x) holds x's neighbours of label L, sorted.  A query edge (a -> b)
// at x reads the list (label(b), x), which holds every vertex the CaLiG list
// of (a -> b) at x can hold (CaLiG's lists are these lists pruned by the
// local-candidacy filter, calig.cpp:358-408, which every embedding passes).
// A batch's count per query is the number of embeddings that map some query
// edge to an inserted data edge, counted once at its largest such edge with
// the reference's visibility rule (enumeration.cu:768, 797, 937): the same
// number the CaLiG pipeline produces, |Emb(G after)| - |Emb(G before)|, and
// the tests check it batch by batch against the reference's CPU path and the
// single-query engine.
//
// Per batch:
//   1. the previous batch's inserted edges are merged into the index;
//   2. deletions (if any): the deleted edges present in the index are removed,
//      then matched as the delta against the index without them: the
//      embeddings the deletions destroy (negative matches);
//   3. insertions: the inserted edges not yet in the index (deduplicated)
//      become the delta, are matched, and are merged at the next batch.
// Delta keys are packed as ((label(y) << lb | label(x)) << 2B) | x << B | y,
// so the seeds of a query edge (a, b) are the contiguous range with
// (label(b), label(a)), and the delta list of (label L, vertex x) is one run.

namespace {

constexpr uint32_t kMqMaxQueries = CGB_MQ_MAX_QUERIES;
constexpr uint32_t kMqMaxLabels = CGB_MQ_MAX_LABELS;
constexpr uint32_t kMqSeedThreads = 1024;

// Directed index keys of data edges: (label(y) << 59 | x << 32 | y) and its
// mirror; invalid edges (ids out of range, self-loops) become the all-ones
// padding key and raise error bit 1.
__global__ void k_mq_edge_keys(const uint32_t* __restrict__ pairs, uint64_t m, const uint8_t* __restrict__ lab,
                               uint32_t n, uint64_t* __restrict__ out, unsigned int* err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = pairs[2 * i], y = pairs[2 * i + 1];
        if (x >= n || y >= n || x == y) {
            out[2 * i] = out[2 * i + 1] = ~0ull;
            atomicOr(err, 1u);
            continue;
        }
        out[2 * i] = ((uint64_t)lab[y] << 59) | ((uint64_t)x << 32) | y;
        out[2 * i + 1] = ((uint64_t)lab[x] << 59) | ((uint64_t)y << 32) | x;
    }
}

// Packed delta keys of data edges, both orientations (see the file comment).
__global__ void k_mq_pack(const uint32_t* __restrict__ pairs, uint64_t m, const uint8_t* __restrict__ lab,
                          uint32_t n, uint32_t B, uint32_t lb, uint64_t* __restrict__ out, unsigned int* err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = pairs[2 * i], y = pairs[2 * i + 1];
        if (x >= n || y >= n || x == y) {
            out[2 * i] = out[2 * i + 1] = ~0ull;
            atomicOr(err, 1u);
            continue;
        }
        const uint64_t lx = lab[x], ly = lab[y];
        out[2 * i] = (((ly << lb) | lx) << (2 * B)) | ((uint64_t)x << B) | y;
        out[2 * i + 1] = (((lx << lb) | ly) << (2 * B)) | ((uint64_t)y << B) | x;
    }
}

// keep[i] for the sorted packed keys: the first of equal keys, and (want
// present) an edge the index holds, or (!want present) one it does not.
__global__ void k_mq_mark(const uint64_t* __restrict__ P, uint64_t n, const uint4* __restrict__ rec, uint32_t dvcap,
                          const uint32_t* __restrict__ pool, uint32_t B, uint32_t lb, int want_present,
                          uint8_t* __restrict__ keep) {
    const uint64_t vmask = (1ull << B) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = P[i];
        uint8_t ok = 0;
        if (k != ~0ull && (i == 0 || P[i - 1] != k)) {
            const uint32_t d = (uint32_t)(k >> (2 * B + lb)), u = (uint32_t)((k >> B) & vmask),
                           v = (uint32_t)(k & vmask);
            const uint4 r = rec[(size_t)d * dvcap + u];
            uint32_t lo = 0, hi = r.y;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (pool[r.x + mid] < v) lo = mid + 1; else hi = mid;
            }
            const bool present = lo < r.y && pool[r.x + lo] == v;
            ok = (present == (want_present != 0)) ? 1 : 0;
        }
        keep[i] = ok;
    }
}

// Run key (label(y) << B | x) of every packed delta key (all ones for
// padding): the delta runs are the runs of equal keys, since the source label
// between them is a function of x.
__global__ void k_mq_extract_du(const uint64_t* __restrict__ P, uint64_t n, uint32_t B, uint32_t lb,
                                uint32_t* __restrict__ du) {
    const uint64_t vmask = (1ull << B) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = P[i];
        du[i] = k == ~0ull ? 0xffffffffu : (uint32_t)(((k >> (2 * B + lb)) << B) | ((k >> B) & vmask));
    }
}

// Entries [*nsel, n) of the selected keys become padding (all ones, sorted last).
__global__ void k_mq_pad(uint64_t* P, uint64_t n, const int* nsel) {
    for (uint64_t i = (uint64_t)*nsel + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        P[i] = ~0ull;
}

// Index keys (dir << 59 | u << 32 | v) of packed delta keys; padding stays all ones.
__global__ void k_mq_unpack(const uint64_t* __restrict__ P, uint64_t n, uint32_t B, uint32_t lb,
                            uint64_t* __restrict__ ext) {
    const uint64_t vmask = (1ull << B) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = P[i];
        ext[i] = k == ~0ull ? ~0ull
                            : ((k >> (2 * B + lb)) << 59) | (((k >> B) & vmask) << 32) | (k & vmask);
    }
}

// Seeds of every plan: plan g takes the delta keys whose label prefix is
// pair[g] = label(vs1) << lb | label(vs0) (a contiguous range of the sorted,
// padded keys; *nsel real ones).  seed_pre = exclusive prefix of the range
// sizes (seed_pre[G] = all seeds).  One block.
__global__ void __launch_bounds__(kMqSeedThreads) k_mq_seed_ranges(const uint64_t* __restrict__ P, const int* nsel,
                                                                  uint32_t B, const uint16_t* __restrict__ pair,
                                                                  uint32_t G, uint32_t* seed_lo, uint32_t* seed_pre) {
    using Scan = cub::BlockScan<uint32_t, kMqSeedThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t carry;
    const uint64_t n = (uint64_t)*nsel;
    auto lower = [&](uint64_t key) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (P[mid] < key) lo = mid + 1; else hi = mid;
        }
        return (uint32_t)lo;
    };
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < G; base += kMqSeedThreads) {
        const uint32_t g = base + threadIdx.x;
        uint32_t cnt = 0;
        if (g < G) {
            const uint64_t pfx = (uint64_t)pair[g];
            const uint32_t lo = lower(pfx << (2 * B)), hi = lower((pfx + 1) << (2 * B));
            seed_lo[g] = lo;
            cnt = hi - lo;
        }
        uint32_t before = 0, all = 0;
        Scan(tmp).ExclusiveSum(cnt, before, all);
        if (g < G) seed_pre[g] = carry + before;
        __syncthreads();
        if (threadIdx.x == 0) carry += all;
        __syncthreads();
    }
    if (threadIdx.x == 0) seed_pre[G] = carry;
}

__global__ void k_mq_label_stats(const uint32_t* __restrict__ pairs, uint64_t m, const uint8_t* __restrict__ lab,
                                 uint32_t L, unsigned long long* cnt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t lx = lab[pairs[2 * i]], ly = lab[pairs[2 * i + 1]];
        atomicAdd(cnt + lx * L + ly, 1ull);
        atomicAdd(cnt + ly * L + lx, 1ull);
    }
}

// Vertices x of label a with at least one neighbour of label b, over the
// built index (run lengths of (b, x)).
__global__ void k_mq_label_nodes(const uint4* __restrict__ rec, uint32_t dvcap, uint32_t n,
                                 const uint8_t* __restrict__ lab, uint32_t L, unsigned long long* nodes) {
    const uint64_t total = (uint64_t)L * n;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = (uint32_t)(i / n), x = (uint32_t)(i % n);
        if (rec[(size_t)b * dvcap + x].y) atomicAdd(nodes + lab[x] * L + b, 1ull);
    }
}

}  // namespace

// ===========================================================================
// host side
// ===========================================================================
struct cgb_mq {
    cgb_mq_config cfg{};
    cgb_handle* h = nullptr;  // label-keyed engine holding the index
    std::string err;
    uint32_t n = 0, L = 0;
    std::vector<uint32_t> vlabel;
    std::vector<float> avg;   // [a * L + b]: mean number of label-b neighbours of a label-a vertex with any
    uint64_t launches = 0;

    struct Query {
        bool live = false;
        cgb::QueryMeta q;
        EdgePlan plans[kMaxQE];
        uint16_t pair[kMaxQE];
        uint32_t variant = 0;  // autotuned plan variant (kVariants)
        bool tuned = false;
        float tuned_ms = -1.f;
    };
    std::vector<Query> queries;  // by id
    std::vector<uint32_t> plan_query;   // plan -> query id
    std::vector<uint32_t> plan_edge;    // plan -> query edge index
    uint32_t G = 0;
    bool plans_dirty = true;
    EdgePlan* d_plans = nullptr;
    uint16_t* d_pair = nullptr;
    uint32_t* d_seed = nullptr;              // [0, cap) lo, [cap, 2 cap + 1) pre
    unsigned long long* d_counts = nullptr;  // per plan
    unsigned long long* h_counts = nullptr;  // pinned
    size_t plan_cap = 0;
    // trial plans of the autotuner (one query's variant)
    EdgePlan* d_tplans = nullptr;
    uint16_t* d_tpair = nullptr;

    // delta preparation
    uint32_t* d_pairs = nullptr; size_t pairs_cap = 0;  // uploaded edge pairs (host-buffer entry point)
    uint64_t* d_sel = nullptr; size_t sel_cap = 0;      // selected, padded delta keys (the DFS reads these)
    uint8_t* d_keep = nullptr; size_t keep_cap = 0;
    int* d_nsel = nullptr;

    // schedule (autotuned)
    bool tuned_global = false;
    bool tuned_now = false;  // the current batch ran the autotuner
    uint32_t tuned_plans = 0;  // plan count when the grid was last tuned
    int bps = 0;        // DFS blocks per SM
    bool steal = true;

    // CUDA graph of the matching step, replayed while its arguments are unchanged
    cudaGraphExec_t gexec = nullptr;
    unsigned char gkey[512];
    size_t gkey_len = 0;

    float last_t[4] = {0, 0, 0, 0};
    cudaEvent_t ev[6] = {};
    uint64_t last_stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

namespace {

cgb_status mq_fail(cgb_mq* m, cgb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (m) m->err = buf;
    return s;
}

// Runs an engine-internal step and carries its error text over.
#define MQ_TRY(call)                                          \
    do {                                                      \
        cgb_status s_ = (call);                               \
        if (s_ != CGB_OK) {                                   \
            m->err = m->h->err;                               \
            return s_;                                        \
        }                                                     \
    } while (0)

#define MCK(call)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return mq_fail(m, e_ == cudaErrorMemoryAllocation ? CGB_ERR_OOM : CGB_ERR_CUDA,     \
                           "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// Plan variants the autotuner times per query (bit mask over the planner's options).
enum : uint32_t { kVarPlainCore = 1, kVarNoTailCache = 2, kVarNoSeedGroups = 4 };
constexpr uint32_t kVariants[] = {0, kVarPlainCore, kVarNoTailCache, kVarNoSeedGroups};

// Plans of one query under a variant, remapped to the label-keyed index: a
// backward list (w -> u) is the list of label(u); the seed direction is
// label(vs1); the seed range prefix is label(vs1) << lb | label(vs0).
void mq_plan(const cgb_mq* m, cgb_mq::Query& Q, uint32_t variant) {
    const cgb::QueryMeta& q = Q.q;
    float avg[kMaxDir];
    for (uint32_t d = 0; d < q.nd; ++d) avg[d] = m->avg[q.labels[q.dir_src[d]] * m->L + q.labels[q.dir_dst[d]]];
    cgb::plan_edges(q, avg, Q.plans, true, !(variant & kVarPlainCore), !(variant & kVarNoSeedGroups));
    for (uint32_t ei = 0; ei < q.qe; ++ei) {
        EdgePlan& P = Q.plans[ei];
        for (uint32_t j = 2; j < P.n; ++j)
            for (uint32_t k = P.bn_off[j]; k < P.bn_off[j + 1]; ++k) P.bn_dir[k] = (uint8_t)q.labels[P.vs[j]];
        P.seed_dir = (uint8_t)q.labels[P.vs[1]];
        P.flags = (variant & kVarNoTailCache) ? cgb::kPlanNoTailCache : 0;
        Q.pair[ei] = (uint16_t)((q.labels[P.vs[1]] << m->h->lb) | q.labels[P.vs[0]]);
    }
    Q.variant = variant;
}

cgb_status mq_grow_plans(cgb_mq* m, size_t need) {
    if (need <= m->plan_cap && m->d_plans) return CGB_OK;
    size_t nc = std::max<size_t>(need, 256);
    void* olds[] = {m->d_plans, m->d_pair, m->d_seed, m->d_counts, m->d_tplans, m->d_tpair};
    for (void* p : olds) if (p) MCK(cudaFree(p));
    if (m->h_counts) MCK(cudaFreeHost(m->h_counts));
    MCK(cudaMalloc(&m->d_plans, nc * sizeof(EdgePlan)));
    MCK(cudaMalloc(&m->d_pair, nc * sizeof(uint16_t)));
    MCK(cudaMalloc(&m->d_seed, (2 * nc + 2) * sizeof(uint32_t)));
    MCK(cudaMalloc(&m->d_counts, nc * sizeof(unsigned long long)));
    MCK(cudaMallocHost(&m->h_counts, nc * sizeof(unsigned long long)));
    MCK(cudaMalloc(&m->d_tplans, kMaxQE * sizeof(EdgePlan)));
    MCK(cudaMalloc(&m->d_tpair, kMaxQE * sizeof(uint16_t)));
    m->plan_cap = nc;
    return CGB_OK;
}

// Uploads the plans of every live query, heaviest (tuned) first, so that the
// warps take the long seeds early.
cgb_status mq_upload_plans(cgb_mq* m) {
    if (!m->plans_dirty) return CGB_OK;
    std::vector<uint32_t> ids;
    for (uint32_t i = 0; i < m->queries.size(); ++i)
        if (m->queries[i].live) ids.push_back(i);
    std::stable_sort(ids.begin(), ids.end(),
                     [&](uint32_t a, uint32_t b) { return m->queries[a].tuned_ms > m->queries[b].tuned_ms; });
    std::vector<EdgePlan> plans;
    std::vector<uint16_t> pair;
    m->plan_query.clear();
    m->plan_edge.clear();
    for (uint32_t id : ids) {
        const cgb_mq::Query& Q = m->queries[id];
        for (uint32_t e = 0; e < Q.q.qe; ++e) {
            plans.push_back(Q.plans[e]);
            pair.push_back(Q.pair[e]);
            m->plan_query.push_back(id);
            m->plan_edge.push_back(e);
        }
    }
    cgb_status s;
    if ((s = mq_grow_plans(m, std::max<size_t>(plans.size(), 1))) != CGB_OK) return s;
    if (!plans.empty()) {
        MCK(cudaMemcpy(m->d_plans, plans.data(), plans.size() * sizeof(EdgePlan), cudaMemcpyHostToDevice));
        MCK(cudaMemcpy(m->d_pair, pair.data(), pair.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    }
    m->G = (uint32_t)plans.size();
    m->plans_dirty = false;
    return CGB_OK;
}

// Delta keys of `mpairs` data edges (device pairs) in m->d_sel: packed,
// sorted, deduplicated, kept when present / absent in the index as asked,
// padded with all-ones keys up to 2 * mpairs; delta values, delta runs and
// the records' delta fields set.  Returns the padded length in *n2.
cgb_status mq_prepare_delta(cgb_mq* m, const uint32_t* pairs, uint64_t mpairs, bool want_present, uint64_t* n2) {
    cgb_handle* h = m->h;
    const uint64_t n = 2 * mpairs;
    *n2 = n;
    const uint32_t B = bits_for(h->dv);
    unsigned int* d_err = (unsigned int*)(h->d_scal + 2);
    MQ_TRY(ensure_delta_buffers(h, n));
    if (n > m->sel_cap || !m->d_sel) {
        if (m->d_sel) MCK(cudaFree(m->d_sel));
        if (m->d_keep) MCK(cudaFree(m->d_keep));
        m->sel_cap = std::max<size_t>(n + n / 2, 1 << 16);
        MCK(cudaMalloc(&m->d_sel, m->sel_cap * sizeof(uint64_t)));
        MCK(cudaMalloc(&m->d_keep, m->sel_cap));
    }
    k_mq_pack<<<grid_for(h, mpairs), 256, 0, h->stream>>>(pairs, mpairs, h->d_vlabel, h->dv, B, h->lb, h->d_dkeys,
                                                          d_err);
    LAUNCHED();
    MQ_TRY(radix_sort(h, h->d_dkeys, h->d_dkeys_alt, n, 2 * (int)B + 5 + (int)h->lb));
    k_mq_mark<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_dkeys, n, h->rec, h->dvcap, h->pool, B, h->lb,
                                                     want_present ? 1 : 0, m->d_keep);
    LAUNCHED();
    size_t tb = 0;
    MCK(cub::DeviceSelect::Flagged(nullptr, tb, h->d_dkeys, m->d_keep, m->d_sel, m->d_nsel, (int64_t)n, h->stream));
    MQ_TRY(grow_temp(h, tb));
    MCK(cub::DeviceSelect::Flagged(h->d_temp, tb, h->d_dkeys, m->d_keep, m->d_sel, m->d_nsel, (int64_t)n,
                                   h->stream));
    LAUNCHED();
    k_mq_pad<<<grid_for(h, n), 256, 0, h->stream>>>(m->d_sel, n, m->d_nsel);
    LAUNCHED();
    k_delta_values<<<grid_for(h, n), 256, 0, h->stream>>>(m->d_sel, n, (1ull << B) - 1, h->d_dval);
    LAUNCHED();
    k_mq_extract_du<<<grid_for(h, n), 256, 0, h->stream>>>(m->d_sel, n, B, h->lb, h->d_ddu);
    LAUNCHED();
    MQ_TRY(segment(h, h->d_ddu, n, h->d_drun_du, h->d_drun_len, h->d_drun_off, h->d_num_runs + 1));
    k_delta_recs<<<grid_for(h, n), 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                        h->d_drun_off, h->d_num_runs + 1, B, 0);
    LAUNCHED();
    MCK(cudaGetLastError());
    return CGB_OK;
}

DfsArgs mq_dfs_args(cgb_mq* m, const EdgePlan* plans, uint32_t G, uint64_t budget_ms, bool steal) {
    cgb_handle* h = m->h;
    DfsArgs da;
    std::memset(&da, 0, sizeof(da));
    da.rec = h->rec;
    da.dvcap = h->dvcap;
    da.pool = h->pool;
    da.dval = h->d_dval;
    da.dkeys = m->d_sel;
    da.B = bits_for(h->dv);
    da.qe = G;
    da.seed_lo = m->d_seed;
    da.seed_pre = m->d_seed + m->plan_cap;
    da.counts = m->d_counts;
    da.work_next = (unsigned int*)(h->d_scal + 3);
    da.err = (unsigned int*)(h->d_scal + 2);
    da.stats = h->d_stats;
    da.tasks = h->d_tasks;
    da.task_cap = kTaskCap;
    da.qctr = h->d_qctr;
    da.epoch = 0;
    da.epoch_ptr = h->d_epoch;
    da.force_split = 0;
    da.num_shards = 1;
    da.shard = 0;
    da.steal = steal ? 1u : 0u;
    da.tail_cache = 1;
    da.self_seen = h->d_self;
    da.vb = nullptr;
    da.vb_stride = 0;
    da.qv = 0;
    const bool rb_on = !(h->cfg.flags & CGB_FLAG_NO_RUN_BITS) && h->rb_valid;
    da.rb_slot = rb_on ? h->d_rb_slot : nullptr;
    da.rb_bits = h->d_rb_bits;
    da.rb_words = h->rb_words;
    da.plans = plans;
    da.touched = nullptr;
    da.budget_ns = budget_ms * 1000000ull;
    lsum_bind(h, true, da);
    da.wsum = nullptr;  // one-position (table) level sums only
    da.pair_lane_max = h->pair_lane_max;
    return da;
}

// The matching step on the prepared delta (m->d_sel, padded length n2):
// seed ranges of G plans, the persistent DFS, and (clear) the records' delta
// fields cleared afterwards.  Autotuner trials keep them for the next trial.
// Counts land in m->d_counts[0, G).
cgb_status mq_match_enqueue(cgb_mq* m, const EdgePlan* plans, const uint16_t* pair, uint32_t G, uint64_t n2,
                            int bps, bool steal, uint64_t budget_ms, bool clear = true) {
    cgb_handle* h = m->h;
    const uint32_t B = bits_for(h->dv);
    MCK(cudaMemsetAsync(h->d_scal + 3, 0, sizeof(unsigned long long), h->stream));
    MCK(cudaMemsetAsync(m->d_counts, 0, std::max<uint32_t>(G, 1) * sizeof(unsigned long long), h->stream));
    MCK(cudaMemsetAsync(h->d_qctr, 0, 8 * sizeof(unsigned int), h->stream));
    k_mq_seed_ranges<<<1, kMqSeedThreads, 0, h->stream>>>(m->d_sel, m->d_nsel, B, pair, G, m->d_seed,
                                                          m->d_seed + m->plan_cap);
    LAUNCHED();
    k_epoch_bump<<<1, 1, 0, h->stream>>>(h->d_epoch);
    LAUNCHED();
    DfsArgs da = mq_dfs_args(m, plans, G, budget_ms, steal);
    if (lsum_clear(h, da) != CGB_OK) return mq_fail(m, CGB_ERR_CUDA, "%s", h->err.c_str());
    k_dfs_count<true><<<h->num_sms * bps, kDfsWarps * 32, 0, h->stream>>>(da);
    LAUNCHED();
    // fixed grid (grid-stride over the runs counted on the device): the step's
    // launch arguments do not depend on the batch size
    if (clear) {
        k_delta_recs<<<h->num_sms * 8, 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                            h->d_drun_off, h->d_num_runs + 1, B, 1);
        LAUNCHED();
    }
    MCK(cudaGetLastError());
    (void)n2;
    return CGB_OK;
}

int mq_occupancy(cgb_mq* m) {
    cgb_handle* h = m->h;
    if (h->dfs_occupancy == 0) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_dfs_count<true>, kDfsWarps * 32, 0) != cudaSuccess)
            occ = 1;
        h->dfs_occupancy = std::max(occ, 1);
    }
    return h->dfs_occupancy;
}

// Matching of all live plans, through a CUDA graph of the step when its
// arguments are those it was captured with (recaptured otherwise).
cgb_status mq_match_all(cgb_mq* m, uint64_t n2) {
    cgb_handle* h = m->h;
    const uint64_t budget = m->cfg.dfs_budget_ms ? m->cfg.dfs_budget_ms : 600000ull;
    if (m->cfg.flags & CGB_MQ_FLAG_NO_GRAPH)
        return mq_match_enqueue(m, m->d_plans, m->d_pair, m->G, n2, m->bps, m->steal, budget);
    // the graph is valid while every argument of its launches is unchanged
    DfsArgs da = mq_dfs_args(m, m->d_plans, m->G, budget, m->steal);
    unsigned char key[sizeof(DfsArgs) + 64];
    size_t kl = 0;
    auto put = [&](const void* p, size_t s) { std::memcpy(key + kl, p, s); kl += s; };
    put(&da, sizeof(da));
    const int bps = m->bps;
    put(&bps, sizeof(bps));
    put(&h->d_drun_du, sizeof(void*));
    put(&m->d_pair, sizeof(void*));
    if (m->gexec && kl == m->gkey_len && std::memcmp(key, m->gkey, kl) == 0) {
        MCK(cudaGraphLaunch(m->gexec, h->stream));
        h->launches += 4;  // seed ranges, epoch, DFS, delta clear
        return CGB_OK;
    }
    if (m->gexec) {
        MCK(cudaGraphExecDestroy(m->gexec));
        m->gexec = nullptr;
    }
    cudaGraph_t g = nullptr;
    MCK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cgb_status s = mq_match_enqueue(m, m->d_plans, m->d_pair, m->G, n2, m->bps, m->steal, budget);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (s != CGB_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    MCK(e);
    e = cudaGraphInstantiate(&m->gexec, g, 0);
    cudaGraphDestroy(g);
    MCK(e);
    std::memcpy(m->gkey, key, kl);
    m->gkey_len = kl;
    MCK(cudaGraphLaunch(m->gexec, h->stream));
    return CGB_OK;
}

// Reads the error word and stats of the last step (synchronizes).
cgb_status mq_sync(cgb_mq* m) {
    cgb_handle* h = m->h;
    MQ_TRY(sync_scalars(h));
    for (int i = 0; i < 8; ++i) m->last_stats[i] = h->h_scal[4 + kMaxQE + i];
    return CGB_OK;
}

// Autotuner, run on the first matched batch after the query set changed:
// every new query alone under each plan variant (counts must agree; the
// fastest variant is kept), then (first time, and whenever the plan count
// has doubled since) the whole set under a few DFS grid sizes and with work
// stealing on and off.  Trials run on the batch's prepared delta;
// the DFS does not modify the index, so every trial sees the same input.
cgb_status mq_autotune(cgb_mq* m, uint64_t n2) {
    cgb_handle* h = m->h;
    const int occ = mq_occupancy(m);
    if (m->bps == 0) m->bps = m->cfg.dfs_blocks_per_sm ? std::min<int>(occ, m->cfg.dfs_blocks_per_sm) : occ;
    float ms = 0;
    bool any_new = false;
    for (uint32_t id = 0; id < m->queries.size(); ++id) {
        cgb_mq::Query& Q = m->queries[id];
        if (!Q.live || Q.tuned) continue;
        any_new = true;
        float best = 3.4e38f;
        uint32_t best_v = 0;
        std::vector<unsigned long long> ref;
        for (uint32_t v : kVariants) {
            cgb_mq::Query T = Q;
            mq_plan(m, T, v);
            MCK(cudaMemcpyAsync(m->d_tplans, T.plans, Q.q.qe * sizeof(EdgePlan), cudaMemcpyHostToDevice, h->stream));
            MCK(cudaMemcpyAsync(m->d_tpair, T.pair, Q.q.qe * sizeof(uint16_t), cudaMemcpyHostToDevice, h->stream));
            MCK(cudaMemsetAsync(h->d_scal + 2, 0, sizeof(unsigned long long), h->stream));
            // later variants stop once they are clearly slower than the best so far
            const uint64_t budget = best < 3e38f ? (uint64_t)std::max(2.0f * best + 20.0f, 50.0f)
                                                 : (m->cfg.dfs_budget_ms ? m->cfg.dfs_budget_ms : 600000ull);
            MCK(cudaEventRecord(m->ev[4], h->stream));
            cgb_status s = mq_match_enqueue(m, m->d_tplans, m->d_tpair, Q.q.qe, n2, m->bps, m->steal, budget, false);
            if (s != CGB_OK) return s;
            MCK(cudaEventRecord(m->ev[5], h->stream));
            MQ_TRY(sync_scalars(h));
            MCK(cudaEventElapsedTime(&ms, m->ev[4], m->ev[5]));
            if (h->h_scal[2] & 8u) continue;  // over budget
            if (h->h_scal[2]) return mq_fail(m, CGB_ERR_ARG, "autotune: error bits %llu", h->h_scal[2]);
            std::vector<unsigned long long> c(Q.q.qe);
            MCK(cudaMemcpy(c.data(), m->d_counts, Q.q.qe * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
            unsigned long long tot = 0, rtot = 0;
            for (auto x : c) tot += x;
            for (auto x : ref) rtot += x;
            if (!ref.empty() && tot != rtot)
                return mq_fail(m, CGB_ERR_STATE, "autotune: query %u variant %u counts %llu, variant 0 %llu", id, v,
                               tot, rtot);
            if (ref.empty()) ref = c;
            if (ms < best) { best = ms; best_v = v; }
        }
        if (best >= 3e38f) return mq_fail(m, CGB_ERR_TIMEOUT, "autotune: query %u exceeded the matching budget", id);
        mq_plan(m, Q, best_v);
        Q.tuned = true;
        Q.tuned_ms = best;
        m->plans_dirty = true;
    }
    MQ_TRY(mq_upload_plans(m));
    // the grid is timed again only once the plan count has doubled since
    // its last tuning (a registration alone does not pay for four launches
    // of the whole set)
    if (m->tuned_global && (!any_new || m->G < 2 * m->tuned_plans)) return CGB_OK;
    // grid size and stealing for the whole set
    struct Cfg { int bps; bool steal; };
    std::vector<Cfg> cfgs;
    if (m->cfg.dfs_blocks_per_sm) cfgs.push_back({m->bps, true});
    else
        for (int b = occ; b >= std::max(1, occ - 2); --b) cfgs.push_back({b, true});
    cfgs.push_back({cfgs.front().bps, false});
    float best = 3.4e38f;
    Cfg best_c = cfgs.front();
    for (const Cfg& c : cfgs) {
        MCK(cudaMemsetAsync(h->d_scal + 2, 0, sizeof(unsigned long long), h->stream));
        const uint64_t budget = best < 3e38f ? (uint64_t)std::max(2.0f * best + 20.0f, 50.0f)
                                             : (m->cfg.dfs_budget_ms ? m->cfg.dfs_budget_ms : 600000ull);
        MCK(cudaEventRecord(m->ev[4], h->stream));
        cgb_status s = mq_match_enqueue(m, m->d_plans, m->d_pair, m->G, n2, c.bps, c.steal, budget, false);
        if (s != CGB_OK) return s;
        MCK(cudaEventRecord(m->ev[5], h->stream));
        MQ_TRY(sync_scalars(h));
        MCK(cudaEventElapsedTime(&ms, m->ev[4], m->ev[5]));
        if (h->h_scal[2] & 8u) continue;
        if (h->h_scal[2]) return mq_fail(m, CGB_ERR_ARG, "autotune: error bits %llu", h->h_scal[2]);
        if (ms < best) { best = ms; best_c = c; }
    }
    m->bps = best_c.bps;
    m->steal = best_c.steal;
    m->tuned_global = true;
    m->tuned_plans = m->G;
    MCK(cudaMemsetAsync(h->d_scal + 2, 0, sizeof(unsigned long long), h->stream));
    MCK(cudaMemsetAsync(h->d_stats, 0, 8 * sizeof(unsigned long long), h->stream));
    return CGB_OK;
}

// Adds the counts of the last matching step (plans) into out[query id].
cgb_status mq_collect(cgb_mq* m, uint64_t* out, uint32_t cap) {
    if (m->G) {
        MCK(cudaMemcpyAsync(m->h_counts, m->d_counts, m->G * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            m->h->stream));
        MCK(cudaStreamSynchronize(m->h->stream));
    }
    for (uint32_t g = 0; g < m->G; ++g)
        if (out && m->plan_query[g] < cap) out[m->plan_query[g]] += m->h_counts[g];
    return CGB_OK;
}

cgb_status mq_check_err(cgb_mq* m) {
    cgb_handle* h = m->h;
    if (h->h_scal[2]) {
        const unsigned long long e = h->h_scal[2];
        h->rb_valid = false;
        cgb_status st = (e & 24u) ? CGB_ERR_TIMEOUT : (e & 4u) ? CGB_ERR_OOM : CGB_ERR_ARG;
        return mq_fail(m, st,
                       "batch rejected: error bits %llu (1 = edge out of range or self-loop, 4 = pool exhausted, "
                       "8 = matching exceeded its time budget)", e);
    }
    return CGB_OK;
}

}  // namespace

extern "C" {

void cgb_mq_default_config(cgb_mq_config* cfg) {
    if (cfg) std::memset(cfg, 0, sizeof(*cfg));
}

cgb_status cgb_mq_create(const cgb_mq_config* cfg, cgb_mq** out) {
    if (!out) return CGB_ERR_ARG;
    *out = nullptr;
    cgb_mq* m = new cgb_mq();
    if (cfg) m->cfg = *cfg;
    *out = m;
    cgb_config ec;
    cgb_default_config(&ec);
    ec.device = m->cfg.device;
    ec.pool_words = m->cfg.pool_words;
    ec.dfs_budget_ms = m->cfg.dfs_budget_ms;
    ec.flags = (m->cfg.flags & CGB_MQ_FLAG_NO_RUN_BITS) ? CGB_FLAG_NO_RUN_BITS : 0u;
    cgb_status s = cgb_create(&ec, &m->h);
    if (s != CGB_OK) {
        m->err = m->h ? m->h->err : "engine creation failed";
        return s;
    }
    m->h->mq = true;
    MCK(cudaMalloc(&m->d_nsel, sizeof(int)));
    MCK(cudaMalloc(&m->h->d_epoch, sizeof(unsigned int)));
    MCK(cudaMemset(m->h->d_epoch, 0, sizeof(unsigned int)));
    for (auto& e : m->ev) MCK(cudaEventCreate(&e));
    return CGB_OK;
}

void cgb_mq_destroy(cgb_mq* m) {
    if (!m) return;
    if (m->h) cudaSetDevice(m->h->device);
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    void* ptrs[] = {m->d_plans, m->d_pair, m->d_seed, m->d_counts, m->d_tplans, m->d_tpair, m->d_pairs, m->d_sel,
                    m->d_keep, m->d_nsel};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (m->h_counts) cudaFreeHost(m->h_counts);
    for (auto& e : m->ev)
        if (e) cudaEventDestroy(e);
    if (m->h) {
        if (m->h->d_vlabel) cudaFree(m->h->d_vlabel);
        if (m->h->d_epoch) cudaFree(m->h->d_epoch);
        m->h->d_vlabel = nullptr;
        m->h->d_epoch = nullptr;
        cgb_destroy(m->h);
    }
    delete m;
}

const char* cgb_mq_last_error(const cgb_mq* m) { return m ? m->err.c_str() : "null handle"; }

cgb_status cgb_mq_load_graph(cgb_mq* m, uint32_t n, const uint32_t* labels, uint64_t num_edges,
                             const uint32_t* edges) {
    if (!m || !labels || (num_edges && !edges)) return CGB_ERR_ARG;
    cgb_handle* h = m->h;
    if (h->have_index) return mq_fail(m, CGB_ERR_STATE, "graph already loaded");
    if (n == 0 || n > CGB_MAX_VID) return mq_fail(m, CGB_ERR_LIMIT, "vertex count must be 1..2^27-1");
    if (num_edges > kMaxBatchKeys / 2) return mq_fail(m, CGB_ERR_LIMIT, "too many edges");
    uint32_t L = 0;
    for (uint32_t v = 0; v < n; ++v) L = std::max(L, labels[v] + 1);
    if (L > kMqMaxLabels) return mq_fail(m, CGB_ERR_LIMIT, "labels must be < %u", kMqMaxLabels);
    MCK(cudaSetDevice(h->device));
    m->n = n;
    m->L = L;
    m->vlabel.assign(labels, labels + n);
    std::vector<uint8_t> lab8(n);
    for (uint32_t v = 0; v < n; ++v) lab8[v] = (uint8_t)labels[v];
    h->nd = L;
    h->lb = 1;
    while ((1u << h->lb) < L) ++h->lb;
    h->have_query = true;
    // query-independent plan for the engine's own structures: none (plans per query)
    h->dv = n;
    MQ_TRY(ensure_dvcap(h, n));
    MCK(cudaMalloc(&h->d_vlabel, std::max<uint32_t>(n, 1)));
    MCK(cudaMemcpy(h->d_vlabel, lab8.data(), n, cudaMemcpyHostToDevice));
    // index keys of every edge, both directions
    const uint64_t nk = 2 * num_edges;
    unsigned long long cap = m->cfg.pool_words;
    if (cap == 0) cap = std::max<unsigned long long>(nk + nk / 2 + (128ull << 20), 192ull << 20);
    MCK(cudaMalloc(&h->pool, cap * sizeof(uint32_t)));
    h->pool_cap = cap;
    h->h_pool_top = 0;
    h->h_live = 0;
    MCK(cudaMemsetAsync(h->d_scal, 0, 4 * sizeof(unsigned long long), h->stream));
    uint32_t* d_edges = nullptr;
    MCK(cudaMalloc(&d_edges, std::max<uint64_t>(num_edges, 1) * 2 * sizeof(uint32_t)));
    if (num_edges) MCK(cudaMemcpyAsync(d_edges, edges, num_edges * 8, cudaMemcpyHostToDevice, h->stream));
    cgb_status s = CGB_OK;
    if ((s = grow(h, h->d_keys_in, h->keys_in_cap, std::max<uint64_t>(nk, 1))) == CGB_OK) {
        if (num_edges) {
            k_mq_edge_keys<<<grid_for(h, num_edges), 256, 0, h->stream>>>(d_edges, num_edges, h->d_vlabel, n,
                                                                           h->d_keys_in,
                                                                           (unsigned int*)(h->d_scal + 2));
            LAUNCHED();
        }
        s = apply_edits(h, h->d_keys_in, nk, nullptr, 0, nullptr, 0);
    }
    // planner statistics: directed edges and vertices with such an edge per label pair
    unsigned long long* d_st = nullptr;
    std::vector<unsigned long long> cnt((size_t)L * L), nodes((size_t)L * L);
    if (s == CGB_OK) {
        MCK(cudaMalloc(&d_st, 2 * (size_t)L * L * sizeof(unsigned long long)));
        MCK(cudaMemsetAsync(d_st, 0, 2 * (size_t)L * L * sizeof(unsigned long long), h->stream));
        if (num_edges) {
            k_mq_label_stats<<<grid_for(h, num_edges), 256, 0, h->stream>>>(d_edges, num_edges, h->d_vlabel, L, d_st);
            LAUNCHED();
        }
        k_mq_label_nodes<<<grid_for(h, (uint64_t)L * n), 256, 0, h->stream>>>(h->rec, h->dvcap, n, h->d_vlabel, L,
                                                                               d_st + (size_t)L * L);
        LAUNCHED();
        MCK(cudaMemcpyAsync(cnt.data(), d_st, cnt.size() * 8, cudaMemcpyDeviceToHost, h->stream));
        MCK(cudaMemcpyAsync(nodes.data(), d_st + (size_t)L * L, nodes.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(d_edges);
    if (d_st) cudaFree(d_st);
    if (s != CGB_OK) {
        m->err = h->err;
        return s;
    }
    MQ_TRY(sync_scalars(h));
    if (h->h_scal[2]) return mq_fail(m, CGB_ERR_ARG, "edges out of range or self-loops (error bits %llu)",
                                     h->h_scal[2]);
    m->avg.assign((size_t)L * L, 0.f);
    for (size_t i = 0; i < cnt.size(); ++i) m->avg[i] = nodes[i] ? (float)cnt[i] / (float)nodes[i] : 0.f;
    h->have_index = true;
    return CGB_OK;
}

cgb_status cgb_mq_register_query(cgb_mq* m, uint32_t qv, const uint32_t* labels, uint32_t qe, const uint32_t* edges,
                                 uint32_t* query_id) {
    if (!m || !labels || !edges || !query_id) return CGB_ERR_ARG;
    if (!m->h->have_index) return mq_fail(m, CGB_ERR_STATE, "load the graph first");
    cgb_mq::Query Q;
    std::string e = cgb::build_query_meta(qv, qe, edges, labels, Q.q, kMaxQE);
    if (!e.empty()) return mq_fail(m, CGB_ERR_ARG, "%s", e.c_str());
    for (uint32_t i = 0; i < qv; ++i)
        if (labels[i] >= kMqMaxLabels) return mq_fail(m, CGB_ERR_ARG, "query label %u out of range", labels[i]);
    uint32_t id = 0;
    while (id < m->queries.size() && m->queries[id].live) ++id;
    if (id >= kMqMaxQueries) return mq_fail(m, CGB_ERR_LIMIT, "at most %u queries", kMqMaxQueries);
    Q.live = true;
    mq_plan(m, Q, 0);
    if (m->cfg.flags & CGB_MQ_FLAG_NO_AUTOTUNE) Q.tuned = true;
    if (id == m->queries.size()) m->queries.push_back(Q);
    else m->queries[id] = Q;
    m->plans_dirty = true;
    *query_id = id;
    return CGB_OK;
}

cgb_status cgb_mq_unregister_query(cgb_mq* m, uint32_t query_id) {
    if (!m) return CGB_ERR_ARG;
    if (query_id >= m->queries.size() || !m->queries[query_id].live)
        return mq_fail(m, CGB_ERR_ARG, "no query %u", query_id);
    m->queries[query_id].live = false;
    m->plans_dirty = true;
    return CGB_OK;
}

cgb_status cgb_mq_apply_batch_device(cgb_mq* m, const uint32_t* ins_device, uint64_t n_ins,
                                     const uint32_t* del_device, uint64_t n_del, void* stream, uint64_t* pos_counts,
                                     uint64_t* neg_counts, uint32_t cap) {
    if (!m) return CGB_ERR_ARG;
    cgb_handle* h = m->h;
    if (!h->have_index) return mq_fail(m, CGB_ERR_STATE, "load the graph first");
    if ((n_ins && !ins_device) || (n_del && !del_device)) return CGB_ERR_ARG;
    if (n_ins > kMaxBatchKeys / 2 || n_del > kMaxBatchKeys / 2) return mq_fail(m, CGB_ERR_LIMIT, "batch too large");
    if (2 * n_ins > 0xffffffffull || 2 * n_del > 0xffffffffull)
        return mq_fail(m, CGB_ERR_LIMIT, "at most 2^31 - 1 edges per batch");
    if (pos_counts) std::memset(pos_counts, 0, cap * sizeof(uint64_t));
    if (neg_counts) std::memset(neg_counts, 0, cap * sizeof(uint64_t));
    MCK(cudaSetDevice(h->device));
    cudaStream_t user = (cudaStream_t)stream;
    if (user && user != h->stream) {
        MCK(cudaEventRecord(h->ev[4], user));
        MCK(cudaStreamWaitEvent(h->stream, h->ev[4], 0));
    }
    cgb_status s;
    if ((s = mq_upload_plans(m)) != CGB_OK) return s;
    MCK(cudaMemsetAsync(h->d_scal + 2, 0, 2 * sizeof(unsigned long long), h->stream));
    MCK(cudaMemsetAsync(h->d_stats, 0, 8 * sizeof(unsigned long long), h->stream));
    MCK(cudaEventRecord(m->ev[0], h->stream));
    // 1. the previous batch's insertions join the index
    MQ_TRY(apply_edits(h, h->d_pending, h->n_pending, nullptr, 0, nullptr, 0));
    h->n_pending = 0;
    const bool rb_on = !(h->cfg.flags & CGB_FLAG_NO_RUN_BITS);
    if (rb_on && !h->rb_valid) MQ_TRY(rebuild_run_bits(h));
    MCK(cudaEventRecord(m->ev[1], h->stream));
    float t_delta = 0, t_match = 0;
    float ms = 0;
    // 2. deletions: remove the present ones, then count what they destroyed
    if (n_del) {
        uint64_t n2 = 0;
        MCK(cudaEventRecord(m->ev[2], h->stream));
        if ((s = mq_prepare_delta(m, del_device, n_del, true, &n2)) != CGB_OK) return s;
        MQ_TRY(grow(h, h->d_keys_in, h->keys_in_cap, n2));
        k_mq_unpack<<<grid_for(h, n2), 256, 0, h->stream>>>(m->d_sel, n2, bits_for(h->dv), h->lb, h->d_keys_in);
        LAUNCHED();
        MQ_TRY(apply_edits(h, nullptr, 0, nullptr, 0, h->d_keys_in, n2));
        MCK(cudaEventRecord(m->ev[3], h->stream));
        if (m->G) {
            if ((s = mq_match_enqueue(m, m->d_plans, m->d_pair, m->G, n2, m->bps ? m->bps : mq_occupancy(m),
                                      m->steal, m->cfg.dfs_budget_ms ? m->cfg.dfs_budget_ms : 600000ull)) != CGB_OK)
                return s;
        } else {
            k_delta_recs<<<grid_for(h, n2), 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                                 h->d_drun_off, h->d_num_runs + 1,
                                                                 bits_for(h->dv), 1);
            LAUNCHED();
        }
        MCK(cudaEventRecord(m->ev[4], h->stream));
        MQ_TRY(mq_sync(m));
        if ((s = mq_check_err(m)) != CGB_OK) return s;
        if ((s = mq_collect(m, neg_counts, cap)) != CGB_OK) return s;
        MCK(cudaEventElapsedTime(&ms, m->ev[2], m->ev[3]));
        t_delta += ms;
        MCK(cudaEventElapsedTime(&ms, m->ev[3], m->ev[4]));
        t_match += ms;
    }
    // 3. insertions: the new edges are the delta; merged at the next batch
    if (n_ins) {
        uint64_t n2 = 0;
        MCK(cudaEventRecord(m->ev[2], h->stream));
        if ((s = mq_prepare_delta(m, ins_device, n_ins, false, &n2)) != CGB_OK) return s;
        MCK(cudaEventRecord(m->ev[3], h->stream));
        if (m->G) {
            const bool need_tune = !(m->cfg.flags & CGB_MQ_FLAG_NO_AUTOTUNE) &&
                                   (!m->tuned_global || std::any_of(m->queries.begin(), m->queries.end(),
                                                                    [](const cgb_mq::Query& q) { return q.live && !q.tuned; }));
            if (need_tune) {
                if ((s = mq_autotune(m, n2)) != CGB_OK) return s;
                m->tuned_now = true;
                MCK(cudaEventRecord(m->ev[3], h->stream));  // the step's time excludes the trials
            } else if (m->bps == 0) {
                m->bps = m->cfg.dfs_blocks_per_sm ? std::min<int>(mq_occupancy(m), m->cfg.dfs_blocks_per_sm)
                                                  : mq_occupancy(m);
            }
            if ((s = mq_match_all(m, n2)) != CGB_OK) return s;
        } else {
            k_delta_recs<<<grid_for(h, n2), 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                                 h->d_drun_off, h->d_num_runs + 1,
                                                                 bits_for(h->dv), 1);
            LAUNCHED();
        }
        MCK(cudaEventRecord(m->ev[4], h->stream));
        // this batch's new edges, as index keys, are merged at the next batch
        MQ_TRY(grow(h, h->d_pending, h->pending_cap, n2));
        k_mq_unpack<<<grid_for(h, n2), 256, 0, h->stream>>>(m->d_sel, n2, bits_for(h->dv), h->lb, h->d_pending);
        LAUNCHED();
        h->n_pending = n2;
        MQ_TRY(mq_sync(m));
        if ((s = mq_check_err(m)) != CGB_OK) {
            h->n_pending = 0;
            return s;
        }
        if ((s = mq_collect(m, pos_counts, cap)) != CGB_OK) return s;
        MCK(cudaEventElapsedTime(&ms, m->ev[2], m->ev[3]));
        t_delta += ms;
        MCK(cudaEventElapsedTime(&ms, m->ev[3], m->ev[4]));
        t_match += ms;
    } else {
        MQ_TRY(mq_sync(m));
        if ((s = mq_check_err(m)) != CGB_OK) return s;
    }
    MCK(cudaEventRecord(m->ev[5], h->stream));
    MCK(cudaEventSynchronize(m->ev[5]));
    float t_upd = 0, t_all = 0;
    MCK(cudaEventElapsedTime(&t_upd, m->ev[0], m->ev[1]));
    MCK(cudaEventElapsedTime(&t_all, m->ev[0], m->ev[5]));
    m->last_t[0] = t_upd;
    m->last_t[1] = t_delta;
    m->last_t[2] = t_match;
    // the whole batch without the autotuner's trials (they run on the first
    // batch after the query set changes)
    m->last_t[3] = m->tuned_now ? t_upd + t_delta + t_match : t_all;
    m->tuned_now = false;
    return CGB_OK;
}

cgb_status cgb_mq_apply_batch(cgb_mq* m, const uint32_t* ins, uint64_t n_ins, const uint32_t* del, uint64_t n_del,
                              uint64_t* pos_counts, uint64_t* neg_counts, uint32_t cap) {
    if (!m) return CGB_ERR_ARG;
    if ((n_ins && !ins) || (n_del && !del)) return CGB_ERR_ARG;
    if (n_ins > kMaxBatchKeys / 2 || n_del > kMaxBatchKeys / 2) return mq_fail(m, CGB_ERR_LIMIT, "batch too large");
    cgb_handle* h = m->h;
    MCK(cudaSetDevice(h->device));
    const uint64_t n = n_ins + n_del;
    if (2 * n > m->pairs_cap || !m->d_pairs) {
        if (m->d_pairs) MCK(cudaFree(m->d_pairs));
        m->pairs_cap = std::max<uint64_t>(2 * n + n, 1 << 16);
        MCK(cudaMalloc(&m->d_pairs, m->pairs_cap * sizeof(uint32_t)));
    }
    if (n_ins) MCK(cudaMemcpyAsync(m->d_pairs, ins, n_ins * 8, cudaMemcpyHostToDevice, h->stream));
    if (n_del) MCK(cudaMemcpyAsync(m->d_pairs + 2 * n_ins, del, n_del * 8, cudaMemcpyHostToDevice, h->stream));
    return cgb_mq_apply_batch_device(m, m->d_pairs, n_ins, m->d_pairs + 2 * n_ins, n_del, nullptr, pos_counts,
                                     neg_counts, cap);
}

cgb_status cgb_mq_last_timings(const cgb_mq* m, float* t4) {
    if (!m || !t4) return CGB_ERR_ARG;
    for (int i = 0; i < 4; ++i) t4[i] = m->last_t[i];
    return CGB_OK;
}

cgb_status cgb_mq_last_stats(const cgb_mq* m, uint64_t* out8) {
    if (!m || !out8) return CGB_ERR_ARG;
    for (int i = 0; i < 8; ++i) out8[i] = m->last_stats[i];
    return CGB_OK;
}

cgb_status cgb_mq_query_info(const cgb_mq* m, uint32_t query_id, uint32_t* variant, float* tuned_ms) {
    if (!m) return CGB_ERR_ARG;
    if (query_id >= m->queries.size() || !m->queries[query_id].live) return CGB_ERR_ARG;
    if (variant) *variant = m->queries[query_id].variant;
    if (tuned_ms) *tuned_ms = m->queries[query_id].tuned_ms;
    return CGB_OK;
}

cgb_status cgb_mq_schedule(const cgb_mq* m, uint32_t* blocks_per_sm, uint32_t* steal) {
    if (!m) return CGB_ERR_ARG;
    if (blocks_per_sm) *blocks_per_sm = (uint32_t)m->bps;
    if (steal) *steal = m->steal ? 1u : 0u;
    return CGB_OK;
}

uint64_t cgb_mq_kernel_launches(const cgb_mq* m) { return m && m->h ? m->h->launches : 0; }

void* cgb_mq_stream(const cgb_mq* m) { return m && m->h ? (void*)m->h->stream : nullptr; }

}  // extern "C"
