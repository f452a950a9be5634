// CaLiG candidate index (Stage 1 producer of the per-batch keys).
//
// Restates the reference's CaLiG maintenance (index/calig.{h,cpp}) with flat
// storage: per data vertex v and query vertex ui of v's label, one sorted
// candidate list per query neighbour uj of ui (the reference's
// G[v].cand[ui][uj] hash sets, calig.h:28-33), plus the LI bitmask G_Li
// (calig.h:82) and the per-(v,ui) "checked" bit (calig.h:32).  The update
// algorithm keeps the reference's phase structure so the emitted delta
// multisets are identical:
//   updateIndex     calig.cpp:950-1069
//   ConstructUpdate calig.cpp:776-804
//   mergeDeltas     calig.cpp:1071-1088 (deltas are returned per batch)
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace cgb {

// Process-wide worker threads for the producer's parallel phases.  A phase
// costs a wake-up instead of thread creation (~250 us for 8 threads, ~480
// for 16, and a batch runs ~40 phases).  Jobs from different callers are
// serialised; a job started from inside a job runs inline.
void pool_run(uint32_t n, const std::function<void(uint32_t)>& fn);

// Runs fn(0..n-1), task k on its own worker (inline when n == 1).
template <class Fn>
void run_threads(uint32_t n, Fn fn) {
    if (n <= 1) { fn(0u); return; }
    pool_run(n, std::function<void(uint32_t)>(fn));
}

struct DeltaOp {  // calig.h:35
    uint32_t vi, vj, ui, uj;
};

// Set of undirected data edges, for updateIndex's test whether a batch pair
// is an edge already (calig.cpp:972-975): open addressing with linear
// probing over keys min << 32 | max, sized when built for every edge the
// update stream can add (load <= 2/3, no growth); inserts are lock-free (a
// compare-and-swap on the empty slot), so batch pairs go in from all threads.
class EdgeSet {
public:
    void reset(size_t max_edges);
    // room for `more` inserts at load <= 3/4 (rehashes; single-threaded)
    void reserve(size_t more);
    bool has(uint32_t a, uint32_t b) const;
    void insert(uint32_t a, uint32_t b);

private:
    static constexpr uint64_t kEmpty = ~0ull;  // no key: vertex ids are < 2^32 - 1
    std::vector<uint64_t> slots_;
    int bits_ = 10;
    size_t count_ = 0;  // keys held (updated atomically by insert)
    static uint64_t key(uint32_t a, uint32_t b) { return a < b ? (uint64_t)a << 32 | b : (uint64_t)b << 32 | a; }
    size_t slot(uint64_t k) const { return (size_t)((k * 0x9E3779B97F4A7C15ull) >> (64 - bits_)); }
};

class CaLiGIndex {
public:
    // Loading (reference text formats, calig.cpp:111-216, 719-733).
    std::string load_query(const std::string& path);
    std::string load_graph(const std::string& path);
    std::string load_updates(const std::string& path);
    // Binary CSR prefix (calig.cpp:218-323): <prefix>.meta.txt, .vertex.bin
    // (u64 row pointers), .edge.bin (u32 neighbours).  Labels are drawn with
    // the C library's rand() sequence from its default seed, the update stream
    // is the hash-selected 10% of the edges, shuffled with mt19937(42).
    std::string load_graph_bin(const std::string& prefix);

    // constructCand + staticFilter (calig.cpp:325-356, 705-717)
    void construct();

    uint32_t threads() const { return threads_; }
    // Host threads for the list-parallel phases (0 = all hardware threads);
    // also reads CGB_PRODUCER_MIN_PARALLEL (smallest phase run on threads).
    void set_threads(uint32_t n);

    // One batch over update[start, start+count) (ints; two per edge).
    void update_index(uint32_t start, uint32_t count);
    void construct_update(uint32_t start, uint32_t count);

    uint32_t num_update_ints() const { return (uint32_t)update_.size(); }
    uint32_t num_vertices() const { return (uint32_t)glabel_.size(); }
    uint32_t query_size() const { return qn_; }
    const std::vector<uint32_t>& li() const { return li_; }
    const std::vector<std::vector<uint32_t>>& query_nbrs() const { return qnei_; }
    const std::vector<int>& query_labels() const { return qlabel_; }

    // candidate list of (v, ui -> uj); nullptr if v has no slot for ui
    const std::vector<uint32_t>* cand(uint32_t v, uint32_t ui, uint32_t uj) const;

    // deltas of the last batch
    std::vector<DeltaOp> delta_ins, delta_del, delta_update;

private:
    // query
    uint32_t qn_ = 0;
    std::vector<int> qlabel_;
    std::vector<std::vector<uint32_t>> qnei_;
    std::vector<std::vector<std::vector<uint32_t>>> rep_;  // per ui: groups of same-label neighbours (size > 1)
    std::vector<std::vector<int>> rep_of_label_;            // per ui, per label slot -> group index or -1
    std::vector<int> label_slot_;                           // raw label -> dense label index or -1
    std::vector<std::vector<uint32_t>> qlist_;              // dense label -> query vertices ascending
    std::vector<uint32_t> block_off_;                       // per ui: offset of its lists in a vertex block
    std::vector<uint32_t> block_size_;                      // per dense label
    std::vector<int> npos_;                                 // ui*qn + uj -> position in qnei_[ui]

    // data
    std::vector<int> glabel_;        // dense label index or -1 (pruned)
    std::vector<std::vector<uint32_t>> nei_;  // adjacency while loading and constructing; freed after
    EdgeSet edges_;                           // the data edges from construct() on
    std::vector<uint64_t> cbase_;    // per vertex: first list index
    std::vector<std::vector<uint32_t>> lists_;
    std::vector<uint32_t> li_, checked_;
    // LI transposed: bit v of row u (row = words_ 64-bit words) is bit u of
    // li_[v].  The scans test one (v, u) per item; a row is n / 8 bytes and
    // stays in a core's L2 where li_ (4 n bytes) does not.  Rows are shared
    // by vertices of different owners: updates are atomic.
    std::vector<uint64_t> litbits_;
    size_t words_ = 0;
    std::vector<int> update_;
    uint32_t threads_ = 1;
    uint64_t par_min_ = 4096;

    inline uint64_t list_index(uint32_t v, uint32_t ui, uint32_t uj) const {
        return cbase_[v] + block_off_[ui] + (uint32_t)npos_[ui * qn_ + uj];
    }
    inline std::vector<uint32_t>& C(uint32_t v, uint32_t ui, uint32_t uj) { return lists_[list_index(v, ui, uj)]; }
    inline bool lit(uint32_t v, uint32_t u) const {
        return (__atomic_load_n(&litbits_[u * words_ + (v >> 6)], __ATOMIC_RELAXED) >> (v & 63)) & 1u;
    }
    // set / clear bit u of li_[v] (the owner of v only)
    inline void light(uint32_t v, uint32_t u) {
        li_[v] |= 1u << u;
        __atomic_fetch_or(&litbits_[u * words_ + (v >> 6)], 1ull << (v & 63), __ATOMIC_RELAXED);
    }
    inline void unlight(uint32_t v, uint32_t u) {
        li_[v] &= ~(1u << u);
        __atomic_fetch_and(&litbits_[u * words_ + (v >> 6)], ~(1ull << (v & 63)), __ATOMIC_RELAXED);
    }
    bool has_slot(uint32_t v, uint32_t u) const {
        return glabel_[v] >= 0 && glabel_[v] == label_slot_[qlabel_[u]];
    }
    bool check_nei(uint32_t v, uint32_t u);
    bool try_nei(uint32_t v, uint32_t u, const std::vector<uint32_t>& group, size_t th,
                 std::vector<uint32_t>& used);

    struct Task { uint32_t u, v; };
    struct Tmp { uint32_t ui, uj, vi, vj; };
    void add_and_check(std::vector<Task>& add, std::vector<Task>& settled, std::vector<Task>& add_del,
                       std::vector<Task>& activated);
    void del_and_check(std::vector<Task>& del);
    size_t item_offsets(const std::vector<Task>& q, std::vector<size_t>& first);
    template <class Fn>
    void scan_items(const std::vector<Task>& q, const std::vector<size_t>& first, size_t lo, size_t hi, Fn&& fn);
};

}  // namespace cgb
