/*
 * cgbdsm.h — C ABI of the B200 continuous-subgraph-matching engine.
 *
 * The engine owns, on one CUDA device, the per-batch GPU half of the
 * reference's pipeline ("Stage 2", main_calig.cpp:281-384):
 *
 *   index update     TransferUpdateAll        calig_helper_gamma.cu:485-517
 *   delta lists      TransferUpdateIndex      calig_helper_gamma.cu:569-597
 *   matching         MatchingBitAll           graph_gpu.cu:1261-1480
 *   delta merge-back BatchUpdateGlobalIndex   calig_helper_gamma.cu:539-567
 *
 * Inputs are the reference's 64-bit keys
 *     key = (dir << 59) | (u << 32) | v
 * with dir the directed query-edge index (graph.cpp:137-148, < 32), u and v
 * compressed data-vertex ids (< 2^27, calig_helper_gamma.cu:77-105, 228-229).
 *
 * Conventions: every call returns a cgb_status; nothing calls exit().  A handle
 * is used by one host thread at a time; distinct handles are independent.
 * Host pointers are plain host memory unless a name says "device".
 */
#ifndef CGBDSM_H
#define CGBDSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CGB_OK = 0,
    CGB_ERR_ARG = 1,      /* invalid argument (sizes, ids, key fields)          */
    CGB_ERR_CUDA = 2,     /* CUDA runtime error; cgb_last_error() has the text   */
    CGB_ERR_OOM = 3,      /* device allocation failed                            */
    CGB_ERR_LIMIT = 4,    /* a documented limit was exceeded                     */
    CGB_ERR_STATE = 5,    /* call out of order (e.g. batch before index build)   */
    CGB_ERR_TIMEOUT = 6,  /* a bounded device wait ran out                       */
    CGB_ERR_IO = 7        /* file could not be read                              */
} cgb_status;

typedef struct cgb_handle cgb_handle;

typedef struct {
    int device;              /* CUDA device ordinal (reference: argv[4], main_calig.cpp:64) */
    uint64_t pool_words;     /* neighbour-run pool capacity in u32 words; 0 = automatic     */
    uint32_t dfs_blocks_per_sm; /* persistent DFS blocks per SM; 0 = automatic              */
    uint32_t flags;          /* CGB_FLAG_* below                                           */
    uint32_t dfs_budget_ms;  /* wall-clock budget of one matching launch; past it the batch
                                fails with CGB_ERR_TIMEOUT (count incomplete); 0 = 600 s   */
    uint32_t shard_index;    /* multi-GPU: this engine matches the seed groups whose key      */
    uint32_t num_shards;     /* (query edge ei, vertex x at the edge plan's first position)  */
                             /* hashes to shard_index (splitmix64 finaliser of ei << 32 | x,  */
                             /* modulo num_shards); 0 or 1 = all seeds.  Every shard applies   */
                             /* every batch to its own full index replica; the batch count is */
                             /* the sum of the shards' counts modulo 2^64.                    */
} cgb_config;

#define CGB_FLAG_NO_MERGE_BACK_DEFER 0x1u /* apply the delta merge-back eagerly after matching */
#define CGB_FLAG_ENUMERATE_TAIL 0x2u      /* enumerate the independent tail instead of counting it */
#define CGB_FLAG_FORCE_SPLIT 0x4u         /* share every long shallow DFS range through the work queue */
#define CGB_FLAG_NO_STEAL 0x8u            /* never share DFS ranges (one warp per seed)                 */
#define CGB_FLAG_NO_TAIL_CACHE 0x10u      /* recount every tail subset for every core embedding        */
#define CGB_FLAG_PLAIN_CORE_ORDER 0x20u   /* greedy core order only (no choice of the last core vertex) */
#define CGB_FLAG_VALID_BITS 0x40u         /* compute the reference's valid bits every matched batch     */
#define CGB_FLAG_MASK_PRUNE 0x80u         /* valid bits, and skip core candidates whose bit is clear    */
#define CGB_FLAG_NO_SEED_GROUPS 0x100u    /* one DFS per seed even where a pendant endpoint allows one per group */
#define CGB_FLAG_NO_RUN_BITS 0x200u       /* binary-search long runs instead of testing their per-batch bit sets */
#define CGB_FLAG_FOOTPRINT 0x400u         /* measure the matching footprint (cgb_last_stats[4]); slower   */
#define CGB_FLAG_WARP_TAIL 0x800u         /* count last-level tails one embedding at a time per warp,
                                             never one candidate per lane                                */
#define CGB_FLAG_NO_LEVEL_SUM 0x1000u     /* enumerate every core level: no level sums (one-position or
                                             dense), no subtree memos, no per-lane pair counting          */

/* Limits (reference: utils/config.h:5-6; key layout calig_helper_gamma.cu:228-229). */
#define CGB_MAX_QV 12
#define CGB_MAX_DIR 32
#define CGB_MAX_VID ((1u << 27) - 1u)

/* Fills *cfg with defaults (device 0, automatic sizes). */
void cgb_default_config(cgb_config* cfg);

/* Creates an engine on cfg->device.  Replaces GPUGraphLoader's constructor
 * (graph_gpu.cu:58-102) and CaLiGHelperGamma's (calig_helper_gamma.cu:19-49). */
cgb_status cgb_create(const cgb_config* cfg, cgb_handle** out);
void cgb_destroy(cgb_handle* h);
/* Text of the last error on this handle ("" if none).  Valid until the next call. */
const char* cgb_last_error(const cgb_handle* h);

/* Loads the query pattern: qv vertices (<= 12, connected), their labels
 * (NULL = unknown), qe undirected edges given as (a, b) pairs, a != b.
 * Directed indices follow graph.cpp:137-148 (CSR order: vertex ascending,
 * neighbour ascending); undirected edge order graph.cpp:184-199.  Labels let
 * the matcher count degree-1 tail vertices of different labels independently;
 * they must be the labels the producer used (lists of a direction (a -> b)
 * hold only vertices of b's label).  Replaces CPUGraphLoader::SetQueryMeta +
 * GPUGraphLoader::LoadQuery (graph.cpp:123-209, graph_gpu.cu:156-172).
 * 2*qe must be <= 32. */
cgb_status cgb_load_query(cgb_handle* h, uint32_t qv, const uint32_t* labels, uint32_t qe,
                          const uint32_t* edges);
/* Same, from a query file in the reference text format (graph.cpp:43-121). */
cgb_status cgb_load_query_file(cgb_handle* h, const char* path);
/* Directed index of query edge (a -> b), or 255 if not an edge. */
uint32_t cgb_query_dir(const cgb_handle* h, uint32_t a, uint32_t b);

/* Builds the initial device index from keys (any order, no duplicates) over
 * dv_count compressed vertices, and plans the matching orders from the index's
 * per-direction cardinalities.  Replaces ConvertGlobalIndex
 * (calig_helper_gamma.cu:238-360) + Plan::GenerateMatchingOrders_v2 + LoadPlan
 * + AllocOnline (plan.cpp:31-54, graph_gpu.cu:174-209). */
cgb_status cgb_build_index(cgb_handle* h, const uint64_t* keys, uint64_t n, uint32_t dv_count);

/* One batch, host buffers (copied to the device inside the call):
 *   ins    keys inserted into the index (LI-filtered by the producer);
 *          duplicates allowed, deduplicated (calig_helper_gamma.cu:254-256)
 *   del    keys removed from the index (calig_helper_gamma.cu:260-265)
 *   delta  this batch's delta keys: matched with the delta visibility rule,
 *          then merged into the index (calig_helper_gamma.cu:569-597, 539-567)
 *   dv_count  compressed-vertex count after this batch's mapping update
 *          (non-decreasing; calig_helper_gamma.cu:107-130)
 *   edge_ok   optional (NULL = derived): per undirected query edge, non-zero if
 *          both of its directions have delta keys (calig_helper_gamma.cu:436-444)
 *   *out_count  positive matches of this batch (graph_gpu.cu:1261-1480):
 *          sum over query edges ei with edge_ok of the embeddings that map ei to
 *          a delta edge, edges e < ei to old-or-delta edges, edges e > ei to old
 *          edges only (enumeration.cu:768, 797, 937).
 * Order of effects, as in the reference: index := (index + ins) - del; match;
 * index := index + delta.  An empty delta skips matching and the merge-back
 * (main_calig.cpp:301-302) and yields *out_count = 0. */
cgb_status cgb_apply_batch(cgb_handle* h, uint32_t dv_count,
                           const uint64_t* ins, uint64_t n_ins,
                           const uint64_t* del, uint64_t n_del,
                           const uint64_t* delta, uint64_t n_delta,
                           const uint8_t* edge_ok, uint64_t* out_count);

/* Same batch with the three key arrays already in device memory (HBM) and the
 * work enqueued on `stream` (a cudaStream_t; NULL = the handle's stream).
 * The count is written to *out_count after the call returns (it synchronizes
 * the stream once at the end). */
cgb_status cgb_apply_batch_device(cgb_handle* h, uint32_t dv_count,
                                  const uint64_t* ins_device, uint64_t n_ins,
                                  const uint64_t* del_device, uint64_t n_del,
                                  const uint64_t* delta_device, uint64_t n_delta,
                                  const uint8_t* edge_ok, void* stream,
                                  uint64_t* out_count);

/* Per-query-edge counts of the last batch (qe entries). */
cgb_status cgb_last_edge_counts(const cgb_handle* h, uint64_t* out, uint32_t cap);

/* The current index (after any pending delta merge-back) as sorted keys.
 * With out == NULL only *n is set.  Replaces reading RelationsGPU
 * (graph_gpu.h:41-49) for parity checks. */
cgb_status cgb_read_index(cgb_handle* h, uint64_t* out, uint64_t cap, uint64_t* n);

/* Timing of the last batch on the device (CUDA events, milliseconds):
 * t[0] index update, t[1] delta lists, t[2] matching, t[3] the whole batch
 * (first to last device operation, before the final count read-back). */
cgb_status cgb_last_timings(const cgb_handle* h, float* t4);

/* Number of kernels this engine has launched so far. */
uint64_t cgb_kernel_launches(const cgb_handle* h);

/* Work counters of the last batch (8 entries): [0] seeds (delta edges
 * expanded), [1] 32-candidate chunks evaluated, [2] candidates tested,
 * [3] tail counts, [4] matching bytes: with CGB_FLAG_FOOTPRINT the footprint
 * (16 B per distinct record resolved plus 4 B per entry of its old and delta
 * lists, each record counted once), else a probe estimate (seed keys 8 B,
 * list records 16 B, candidate words 4 B, one 32 B sector per binary-search
 * step),
 * [5] index-update algorithmic bytes (edits 8 B, old and new run words 4 B,
 * record 32 B per touched run), [6] touched runs, [7] reserved. */
cgb_status cgb_last_stats(const cgb_handle* h, uint64_t* out8);

/* The engine's CUDA stream (a cudaStream_t) on which all its work runs. */
void* cgb_stream(const cgb_handle* h);

/* Query vertex at the first position of query edge ei's matching plan (one of
 * ei's endpoints): the vertex whose data vertex keys the seed shard.  The
 * reference plans one global order instead (plan.cpp:535-745).  Available
 * after cgb_build_index. */
cgb_status cgb_plan_anchor(const cgb_handle* h, uint32_t ei, uint32_t* qvertex);

/* How query edge ei's plan counts (after cgb_build_index), for tests and
 * tuning: out4[0] = core positions (the others are counted as the tail),
 * out4[1] = first position counted by level sums (0 = none), out4[2] = 1
 * when those sums are precomputed for every vertex (several positions),
 * out4[3] = per-lane tail mode at the last core position (0, 1 or 2) in bits
 * 0-7, the first position of a memoized subtree (0 = none) in bits 8-15 and
 * the position whose vertex keys it in bits 16-23. */
cgb_status cgb_plan_info(const cgb_handle* h, uint32_t ei, uint32_t* out4);

/* Index symmetry check (after any pending delta merge-back): *n_asym = number
 * of index entries y in the list of (a -> b) at x whose mirror entry (x in
 * the list of (b -> a) at y) is missing.  The matcher's per-edge seeding gives
 * the reference's global-order counts when this is 0 (the reference builds
 * both directions from one data edge, calig_helper_gamma.cu:248-277 and
 * calig.cpp:776-804). */
cgb_status cgb_check_symmetry(cgb_handle* h, uint64_t* n_asym);

/* ------------------------------------------------------------------------
 * Stage-1 producer: the CaLiG candidate index on the host and the host
 * staging that turns its deltas into the keys above.  Replaces, per batch,
 * CaLiG::updateIndex / ConstructUpdate / mergeDeltas (calig.cpp:950-1088)
 * and CaLiGHelperGamma::PrepareUpdateAll / PrepareUpdateIndex
 * (calig_helper_gamma.cu:363-445); at open, CaLiG::inputQ/inputG/inputUpdate,
 * constructCand, staticFilter and ConvertGlobalIndex's key generation
 * (calig.cpp:111-216, 325-356, 705-733; calig_helper_gamma.cu:238-311).
 * Compressed ids are assigned append-only to vertices with any LI bit, in
 * ascending original-id order per batch.
 * ------------------------------------------------------------------------ */
typedef struct cgb_producer cgb_producer;

typedef struct {
    const uint64_t* ins;   uint64_t n_ins;
    const uint64_t* del;   uint64_t n_del;
    const uint64_t* delta; uint64_t n_delta;
    const uint8_t* edge_ok;  /* qe entries */
    uint32_t qe;
    uint32_t dv_count;
    uint32_t batch;
    uint32_t num_edges;      /* insertions listed in this batch */
    double ms_update_index;  /* reference timer [S1] updateIndex (main_calig.cpp:224-226) */
    double ms_construct_update;
    double ms_prepare;       /* [S1] PrepareUpdateAll + PrepareUpdateIndex */
} cgb_batch_keys;

/* batch_size_ints counts ints, two per edge, as the reference CLI does
 * (main_calig.cpp:65-69, 103-104); UINT32_MAX = one batch.  A data_path
 * ending in ".graph" is a text graph and update_path its update stream;
 * any other data_path is a binary CSR prefix (.meta.txt, .vertex.bin,
 * .edge.bin; calig.cpp:218-323) whose update stream is derived from the
 * graph, and update_path is ignored (main_calig.cpp:93-101).  threads: host
 * threads for Stage 1's list-parallel phases (0 = all hardware threads; the
 * emitted key multisets do not depend on it).  Phases smaller than
 * $CGB_PRODUCER_MIN_PARALLEL items (default 4096) run on the calling thread. */
cgb_status cgb_producer_open(const char* query_path, const char* data_path, const char* update_path,
                             uint32_t batch_size_ints, uint32_t threads, cgb_producer** out);
void cgb_producer_close(cgb_producer* p);
const char* cgb_producer_last_error(const cgb_producer* p);
uint32_t cgb_producer_num_batches(const cgb_producer* p);
/* Initial index keys (pointer valid until close) and compressed-vertex count. */
cgb_status cgb_producer_initial(cgb_producer* p, const uint64_t** keys, uint64_t* n, uint32_t* dv_count);
/* Runs Stage 1 for the next batch; arrays valid until the next call. */
cgb_status cgb_producer_next(cgb_producer* p, cgb_batch_keys* out);
/* Compressed id -> original vertex id (valid until the next producer call). */
cgb_status cgb_producer_vertex_map(const cgb_producer* p, const uint32_t** new2old, uint32_t* n);


/* ------------------------------------------------------------------------
 * Index update without device allocation.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: code running while a CUDA
 * graph is captured (cudaMalloc cannot be captured), hosts whose own
 * allocator owns all device memory or caps it per tenant, plugins that may
 * not grow a process's footprint after start-up.  Applies one batch of edits
 * to an index given as one flat, sorted, duplicate-free key array:
 *     out = (old U ins) \ del        (set semantics, as cgb_apply_batch)
 * Inputs and outputs are device pointers the caller owns: old keys (sorted,
 * u and v < dv_count), ins and del keys (any order, duplicates allowed),
 * out (capacity >= n_old + n_ins), out_n (one u64: the output length, or
 * UINT64_MAX if an edit key has u or v >= dv_count).  Work is enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream); nothing is
 * synchronized.  All temporaries live in one static device array of 11.5 MiB
 * that every GPU loading this library holds until the process exits; calls
 * keep their contents in it, so calls whose work overlaps on one GPU race and
 * must be ordered by the caller.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current,
 * and looks it up again after that device's context was reset: make the
 * first call before any stream capture.  Rejects more than
 * CGB_NOALLOC_MAX_EDITS edits (n_ins + n_del), or more than
 * CGB_NOALLOC_MAX_KEYS keys in all (n_old + n_ins + n_del), with
 * CGB_ERR_LIMIT; every limit is checked before any work is enqueued.  An
 * error already pending on the calling thread (cudaPeekAtLastError) makes the
 * call return CGB_ERR_CUDA without enqueuing anything and without clearing
 * it.  Never calls cudaMalloc or cudaFree.
 * ------------------------------------------------------------------------ */
#define CGB_NOALLOC_MAX_EDITS (1u << 18)
#define CGB_NOALLOC_MAX_KEYS (1ull << 27)
cgb_status cgb_merge_keys_noalloc(const uint64_t* old_keys_device, uint64_t n_old,
                                  const uint64_t* ins_device, uint64_t n_ins,
                                  const uint64_t* del_device, uint64_t n_del, uint32_t dv_count,
                                  uint64_t* out_device, uint64_t* out_n_device, void* stream);

/* ---- Packed-memory-array index layout (the reference's GPMA: Multi_GPMA
 * gpma/gpma.cuh:36-111, CGCSM_GPMA index/gpma_wrapper.cuh:10-40) ----
 * One PMA per query direction over the same 64-bit keys, batch-updated with
 * the engine's set semantics (index + ins) - del, rebalanced within windows
 * chosen by the reference's density bounds (0.92 at the leaves to 0.84 at
 * the root, gpma.cuh:55-58), without device-side launches.  All key arrays
 * are device pointers. */
typedef struct cgb_gpma cgb_gpma;
/* CGCSM_GPMA::Init (gpma_wrapper.cu:20-25). */
cgb_status cgb_gpma_create(int device, uint32_t num_dirs, cgb_gpma** out);
void cgb_gpma_destroy(cgb_gpma* g);
const char* cgb_gpma_last_error(const cgb_gpma* g);
/* CGCSM_GPMA::BulkLoad (gpma_wrapper.cu:27-58): any order, duplicates allowed;
 * replaces the contents. */
cgb_status cgb_gpma_bulk_load(cgb_gpma* g, const uint64_t* keys_device, uint64_t n);
/* CGCSM_GPMA::BatchUpdate (gpma_wrapper.cu:60-116). */
cgb_status cgb_gpma_batch_update(cgb_gpma* g, const uint64_t* ins_device, uint64_t n_ins,
                                 const uint64_t* del_device, uint64_t n_del);
/* CGCSM_GPMA::ExtractEdges (gpma_wrapper.cuh:35-37): the keys of direction
 * dir, ascending, as (u << 32 | v); out_device NULL = count only. */
cgb_status cgb_gpma_extract(cgb_gpma* g, uint32_t dir, uint64_t* out_device, uint64_t cap, uint64_t* n_out);
/* Last batch update: [0] slots, [1] windows rewritten, [2] keys rewritten,
 * [3] 1 if it rebuilt the structure, [4] device microseconds, [5] keys held. */
cgb_status cgb_gpma_stats(const cgb_gpma* g, uint64_t* out6);

/* Valid bits (the reference's 1-bit support masks, BuildLocalIndexBitAll,
 * graph_gpu.cu:803-869; indexing.cu:2295-2379), computed for every matched
 * batch when CGB_FLAG_VALID_BITS or CGB_FLAG_MASK_PRUNE is set, after the
 * delta lists and before matching.  Layout: words [ei][u][(dv_count+31)/32],
 * bit (x & 31) of word x >> 5 set when vertex x may take query vertex u in
 * an embedding that maps query edge ei to a delta edge.  Orders, rebuilt
 * vertices and the starting edge follow plan.cpp:428-533, 1180-1370; a
 * pattern whose rebuild flags are inconsistent (the reference exits,
 * plan.cpp:1361-1366) makes cgb_build_index fail with CGB_ERR_ARG when the
 * flag is set.  Pass out = NULL to get *n_words only; *ms (optional) gets
 * the pass's device time.  CGB_ERR_STATE if no batch has computed them. */
cgb_status cgb_valid_bits(cgb_handle* h, uint32_t* out, uint64_t cap, uint64_t* n_words, float* ms);
/* The starting edge (SelectStartingEdge, plan.cpp:428-533) the valid bits
 * use: out2[0], out2[1] = the first two vertices of the reference's global
 * order.  Available after cgb_build_index. */
cgb_status cgb_starting_edge(const cgb_handle* h, uint32_t* out2);

/* ------------------------------------------------------------------------
 * Multi-query engine.  No single counterpart in the reference, which runs one
 * query per process (main_calig.cpp:44-450: a CaLiG index, GAMMA staging
 * and one MatchingBitAll per batch, graph_gpu.cu:1261-1480); this engine
 * replaces N such processes on one device.
 *
 * One device-resident data-graph index, keyed by target-vertex label (the
 * list of (label L, vertex x) = x's neighbours of label L, sorted), is shared
 * by every registered query; all queries are matched per batch in one
 * persistent launch (replayed as a CUDA graph while its arguments are
 * unchanged), with the reference's count semantics per query: the
 * embeddings that map some query edge to a batch edge, counted once at
 * their largest such edge, edges before it matched to old-or-batch edges and
 * after it to old edges (enumeration.cu:768, 797, 937).  For insertions this
 * equals the CaLiG pipeline's positive matches (CaLiG's lists are these
 * lists pruned by a filter every embedding passes, calig.cpp:358-408);
 * deletions count the embeddings they destroy (negative matches), matched
 * against the graph without the deleted edges, before any insertion.
 * Queries: <= 12 vertices, <= 32 edges, labels < 32; registered or removed
 * between batches.  An autotuner times, on the first batch a query sees,
 * its plan variants (core order, tail counting cache, seed grouping) and
 * the DFS grid size and work stealing for the whole set, and keeps the
 * fastest (counts are identical across variants).
 * ------------------------------------------------------------------------ */
typedef struct cgb_mq cgb_mq;

typedef struct {
    int device;
    uint32_t flags;             /* CGB_MQ_FLAG_* */
    uint32_t dfs_budget_ms;     /* wall-clock budget of one matching launch; 0 = 600 s */
    uint32_t dfs_blocks_per_sm; /* 0 = autotuned */
    uint64_t pool_words;        /* neighbour-run pool capacity in u32 words; 0 = automatic */
} cgb_mq_config;

#define CGB_MQ_FLAG_NO_AUTOTUNE 0x1u  /* default plans and grid, no trials        */
#define CGB_MQ_FLAG_NO_GRAPH 0x2u     /* launch the matching step directly         */
#define CGB_MQ_FLAG_NO_RUN_BITS 0x4u  /* binary-search long runs (no bit sets)     */
#define CGB_MQ_MAX_QUERIES 256
#define CGB_MQ_MAX_LABELS 32

void cgb_mq_default_config(cgb_mq_config* cfg);
cgb_status cgb_mq_create(const cgb_mq_config* cfg, cgb_mq** out);
void cgb_mq_destroy(cgb_mq* m);
const char* cgb_mq_last_error(const cgb_mq* m);
/* The data graph: n vertices with labels[n] (< 32), num_edges undirected
 * edges as (x, y) pairs (no self-loops, no duplicates).  Host arrays. */
cgb_status cgb_mq_load_graph(cgb_mq* m, uint32_t n, const uint32_t* labels, uint64_t num_edges,
                             const uint32_t* edges);
/* Registers a query (qv vertices with labels, qe edges as (a, b) pairs);
 * *query_id indexes the count arrays.  Takes effect at the next batch. */
cgb_status cgb_mq_register_query(cgb_mq* m, uint32_t qv, const uint32_t* labels, uint32_t qe,
                                 const uint32_t* edges, uint32_t* query_id);
cgb_status cgb_mq_unregister_query(cgb_mq* m, uint32_t query_id);
/* One batch: n_del deleted and n_ins inserted undirected edges as (x, y)
 * pairs (host arrays; edges absent from / already in the graph, and repeats,
 * are ignored).  pos_counts[id] / neg_counts[id] (cap entries, optional)
 * receive each registered query's positive / negative matches, modulo 2^64.
 * Order: deletions (matched against the graph without them), then
 * insertions (matched, joining the graph before the next batch). */
cgb_status cgb_mq_apply_batch(cgb_mq* m, const uint32_t* ins_edges, uint64_t n_ins, const uint32_t* del_edges,
                              uint64_t n_del, uint64_t* pos_counts, uint64_t* neg_counts, uint32_t cap);
/* Same with the edge pairs in device memory; work enqueued after the
 * caller's prior work on `stream` (NULL = none); returns with counts read. */
cgb_status cgb_mq_apply_batch_device(cgb_mq* m, const uint32_t* ins_device, uint64_t n_ins,
                                     const uint32_t* del_device, uint64_t n_del, void* stream,
                                     uint64_t* pos_counts, uint64_t* neg_counts, uint32_t cap);
/* Last batch, device milliseconds: t[0] index merge, t[1] delta preparation,
 * t[2] matching (autotuner trials excluded), t[3] whole batch. */
cgb_status cgb_mq_last_timings(const cgb_mq* m, float* t4);
/* Work counters of the last batch (as cgb_last_stats). */
cgb_status cgb_mq_last_stats(const cgb_mq* m, uint64_t* out8);
/* Autotuned plan variant of a query (bit 0 plain core order, bit 1 no tail
 * cache, bit 2 no seed groups) and its matching time alone on the tuning
 * batch (ms; < 0 if not tuned). */
cgb_status cgb_mq_query_info(const cgb_mq* m, uint32_t query_id, uint32_t* variant, float* tuned_ms);
/* The DFS schedule in use: blocks per SM and whether work stealing is on. */
cgb_status cgb_mq_schedule(const cgb_mq* m, uint32_t* blocks_per_sm, uint32_t* steal);
uint64_t cgb_mq_kernel_launches(const cgb_mq* m);
void* cgb_mq_stream(const cgb_mq* m);

/* ------------------------------------------------------------------------
 * Serving loop over the multi-query engine.  No counterpart in the
 * reference (one query and one update file per process, main_calig.cpp).
 * The graph, its index and every registered query stay on the device while
 * requests arrive from any thread: update batches (result: every registered
 * query's positive / negative matches for that batch), query registrations
 * (joining the running query set at the next batch boundary; result: the
 * query id) and removals.  Requests take effect in submission order.
 * Admission by HBM budget: an update batch's edge pairs must fit a device
 * staging ring (they are copied as soon as space frees, on a copy stream, so
 * the copies of waiting batches overlap the running batch), and its working
 * set must fit the budget (else its result is CGB_ERR_LIMIT).
 * ------------------------------------------------------------------------ */
typedef struct cgb_server cgb_server;

typedef struct {
    cgb_mq_config mq;
    uint64_t hbm_budget_bytes;  /* device memory the server may add after loading the graph; 0 = 90% of free */
    uint64_t staging_bytes;     /* staging ring for edge pairs; 0 = 64 MiB                                 */
    uint32_t max_pending;       /* requests queued at once; 0 = 4096                                      */
} cgb_server_config;

#define CGB_SERVER_BATCH 0u
#define CGB_SERVER_REGISTER 1u
#define CGB_SERVER_UNREGISTER 2u

typedef struct {
    uint64_t ticket;
    uint32_t kind;          /* CGB_SERVER_* */
    int32_t status;         /* cgb_status of the request */
    uint32_t query_id;      /* registrations */
    uint32_t live_queries;  /* batches: queries registered when it ran */
    double t_submit_ms, t_staged_ms, t_start_ms, t_done_ms;  /* since the server started */
    float device_ms;        /* batches: device time of the batch */
} cgb_server_result;

void cgb_server_default_config(cgb_server_config* cfg);
/* Loads the graph (as cgb_mq_load_graph) and starts the server's threads. */
cgb_status cgb_server_create(const cgb_server_config* cfg, uint32_t n, const uint32_t* labels, uint64_t num_edges,
                             const uint32_t* edges, cgb_server** out);
/* Stops the threads (queued requests are dropped) and frees everything. */
void cgb_server_destroy(cgb_server* s);
const char* cgb_server_last_error(const cgb_server* s);
/* Requests (host arrays, copied before returning); *ticket identifies the result. */
cgb_status cgb_server_submit_batch(cgb_server* s, const uint32_t* ins, uint64_t n_ins, const uint32_t* del,
                                   uint64_t n_del, uint64_t* ticket);
cgb_status cgb_server_submit_register(cgb_server* s, uint32_t qv, const uint32_t* labels, uint32_t qe,
                                      const uint32_t* edges, uint64_t* ticket);
cgb_status cgb_server_submit_unregister(cgb_server* s, uint32_t query_id, uint64_t* ticket);
/* Waits up to timeout_ms for a request; fills *res and, for batches, the
 * counts per query id (cap entries).  A ticket is collected once.
 * CGB_ERR_TIMEOUT if it has not completed. */
cgb_status cgb_server_wait(cgb_server* s, uint64_t ticket, uint32_t timeout_ms, cgb_server_result* res,
                           uint64_t* pos, uint64_t* neg, uint32_t cap);
/* [0] batches done, [1] edges done, [2] rejected, [3] live queries, [4] queued,
 * [5] staging ring bytes, [6] HBM budget bytes, [7] device busy microseconds. */
cgb_status cgb_server_stats(const cgb_server* s, uint64_t* out8);

#ifdef __cplusplus
}
#endif
#endif /* CGBDSM_H */
