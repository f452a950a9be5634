/*
 * oracle.c — CPU restatement of the reference's per-batch GPU path.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's
 * cpu_baseline leg use it as the checker.  The product never links it.
 *
 * Parity pin: tests/test_oracle_pin.py runs this restatement and the
 * reference's own CPU path (oracle/_ref/libcgbref.so, built from the
 * reference's unmodified calig.cpp / cpu_index_mirror.cpp / cpu_dfs.cpp) on
 * the same seeded inputs and requires identical counts and index contents;
 * tests/golden/ holds the vectors that pin it without the reference tree.
 *
 * What it restates (reference file:line):
 *   index set semantics   cpu_index_mirror.cpp:132-229 (MergeInsert = sort,
 *                         unique, set_union; MergeRemove = sort,
 *                         set_difference), InitFromSortedEdges :98-130
 *   delta lists           cpu_index_mirror.cpp:231-269 (RebuildUpdate: sorted,
 *                         not deduplicated)
 *   batch order           main_calig.cpp:294-349: ins, del, [match], delta
 *                         merge-back; an empty delta skips both
 *                         (main_calig.cpp:301-302)
 *   query numbering       graph.cpp:137-148 (directed), :184-199 (undirected)
 *   matching semantics    cpu_dfs.cpp:64-132: for edge ei, lists of ei's own
 *                         directions are the delta lists only; other
 *                         directions are the main list plus the delta list
 *                         when dir_to_edge < ei; candidates from the first
 *                         backward neighbour, membership in the others,
 *                         injectivity against all matched vertices.
 *   seeding               enumeration.cu:727-809 without masks: every vertex
 *                         dv, every entry of the resolved list of the order's
 *                         first edge.
 * Two seeding modes are provided:
 *   ORC_GLOBAL  the reference's: one global vertex order for every ei, seeds
 *               over all dv (exactly cpu_dfs semantics given that order)
 *   ORC_PER_EDGE  per-edge orders starting at ei's endpoints, seeds = delta
 *               entries of ei; equal to ORC_GLOBAL whenever the index lists
 *               are symmetric ((a->b) contains y at x iff (b->a) contains x
 *               at y), which tests/ check as a property.
 *   ORC_TAIL  per-edge seeding with an independent tail counted instead of
 *             enumerated (see count_tail below): pins the engine's counted
 *             tails on workloads too large to enumerate.
 * Seeds may be restricted to one shard of the seed groups (orc_set_shard),
 * keyed like the engine's: a splitmix64 finaliser of (ei << 32 | x), x the
 * data vertex at a given query vertex of ei.
 * Plus an independent brute-force embedding counter for the incremental
 * identity  sum(batch counts) = |Emb(Q, G_after)| - |Emb(Q, G_before)|,
 * and the valid bits of BuildLocalIndexBitAll (graph_gpu.cu:803-869,
 * indexing.cu:2295-2379, orders and rebuild flags plan.cpp:428-533,
 * 1180-1370) with the starting edge of SelectStartingEdge.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXQV 12
#define ORC_MAXD 32
#define ORC_MAXQE 16

enum { ORC_GLOBAL = 0, ORC_PER_EDGE = 1, ORC_TAIL = 2 };

typedef struct {
    uint32_t* v;
    uint32_t n, cap;
} List;

typedef struct {
    uint32_t qv, qe, nd;
    uint8_t eidx[ORC_MAXQV * ORC_MAXQV];
    uint8_t qe_u[ORC_MAXQE], qe_v[ORC_MAXQE];
    uint8_t dir_to_edge[ORC_MAXD];
    uint32_t dv, dvcap;
    List* main;   /* [nd * dvcap] */
    List* delta;  /* [nd * dvcap] */
    uint64_t* pending;  /* delta keys of the last matched batch (merged before the next) */
    uint64_t n_pending;
    uint64_t last_edge_counts[ORC_MAXQE];
    /* seed shard: keep seeds whose (ei, data vertex at query vertex
     * shard_anchor[ei]) hashes to shard (num_shards <= 1: all seeds) */
    uint32_t shard, num_shards;
    uint8_t shard_anchor[ORC_MAXQE];
    /* valid bits (BuildLocalIndexBitAll) of the last matched batch */
    int vb_on;
    uint32_t vb_start[2];
    uint32_t* vb;        /* [qe][qv][stride] */
    uint64_t vb_words;
    int vb_error;        /* the reference's "Error in order generation" case */
} Orc;

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : x > y;
}
static void list_reserve(List* l, uint32_t n) {
    if (n <= l->cap) return;
    uint32_t c = l->cap ? l->cap : 4;
    while (c < n) c *= 2;
    l->v = (uint32_t*)realloc(l->v, (size_t)c * 4);
    l->cap = c;
}

static int list_has(const List* l, uint32_t x) {
    uint32_t lo = 0, hi = l->n;
    while (lo < hi) {
        uint32_t m = (lo + hi) >> 1;
        if (l->v[m] < x) lo = m + 1; else hi = m;
    }
    return lo < l->n && l->v[lo] == x;
}

static void grow_dv(Orc* o, uint32_t dv) {
    if (dv <= o->dvcap) { if (dv > o->dv) o->dv = dv; return; }
    uint32_t nc = o->dvcap ? o->dvcap : 64;
    while (nc < dv) nc *= 2;
    List* nm = (List*)calloc((size_t)o->nd * nc, sizeof(List));
    List* ndl = (List*)calloc((size_t)o->nd * nc, sizeof(List));
    for (uint32_t d = 0; d < o->nd; ++d)
        for (uint32_t u = 0; u < o->dvcap; ++u) {
            nm[(size_t)d * nc + u] = o->main[(size_t)d * o->dvcap + u];
            ndl[(size_t)d * nc + u] = o->delta[(size_t)d * o->dvcap + u];
        }
    free(o->main);
    free(o->delta);
    o->main = nm;
    o->delta = ndl;
    o->dvcap = nc;
    o->dv = dv;
}

#define KD(k) ((uint32_t)((k) >> 59))
#define KU(k) ((uint32_t)(((k) >> 32) & 0x07FFFFFFu))
#define KV(k) ((uint32_t)(k))

/* Applies sorted keys to main lists: set union (is_insert) or set difference. */
static void merge_sorted(Orc* o, const uint64_t* s, uint64_t n, int is_insert) {
    uint64_t i = 0;
    uint32_t* tmp = NULL;
    size_t tcap = 0;
    while (i < n) {
        uint32_t d = KD(s[i]), u = KU(s[i]);
        uint64_t j = i;
        while (j < n && KD(s[j]) == d && KU(s[j]) == u) ++j;
        List* l = &o->main[(size_t)d * o->dvcap + u];
        size_t need = (size_t)l->n + (j - i);
        if (need > tcap) { tcap = need * 2; tmp = (uint32_t*)realloc(tmp, tcap * 4); }
        uint32_t a = 0, c = 0;
        uint64_t b = i;
        while (a < l->n || b < j) {
            if (b >= j || (a < l->n && l->v[a] < KV(s[b]))) tmp[c++] = l->v[a++];
            else if (a >= l->n || KV(s[b]) < l->v[a]) { if (is_insert) tmp[c++] = KV(s[b]); ++b; }
            else { if (is_insert) tmp[c++] = l->v[a]; ++a; ++b; }
        }
        list_reserve(l, c);
        memcpy(l->v, tmp, (size_t)c * 4);
        l->n = c;
        i = j;
    }
    free(tmp);
}

static uint64_t* sorted_copy(const uint64_t* k, uint64_t n, int unique, uint64_t* out_n) {
    uint64_t* s = (uint64_t*)malloc((n ? n : 1) * 8);
    memcpy(s, k, n * 8);
    qsort(s, n, 8, cmp_u64);
    if (unique && n) {
        uint64_t w = 1;
        for (uint64_t i = 1; i < n; ++i) if (s[i] != s[w - 1]) s[w++] = s[i];
        n = w;
    }
    *out_n = n;
    return s;
}

/* ------------------------------------------------------------------ API */

void* orc_create(uint32_t qv, uint32_t qe, const uint32_t* edges) {
    if (qv < 2 || qv > ORC_MAXQV || qe == 0 || 2 * qe > ORC_MAXD) return NULL;
    Orc* o = (Orc*)calloc(1, sizeof(Orc));
    o->qv = qv;
    uint8_t adj[ORC_MAXQV][ORC_MAXQV];
    memset(adj, 0, sizeof(adj));
    for (uint32_t i = 0; i < qe; ++i) {
        uint32_t a = edges[2 * i], b = edges[2 * i + 1];
        if (a >= qv || b >= qv || a == b) { free(o); return NULL; }
        adj[a][b] = adj[b][a] = 1;
    }
    memset(o->eidx, 255, sizeof(o->eidx));
    uint32_t pos = 0;
    for (uint32_t u = 0; u < qv; ++u)           /* graph.cpp:137-148 */
        for (uint32_t w = 0; w < qv; ++w)
            if (adj[u][w]) o->eidx[u * ORC_MAXQV + w] = (uint8_t)pos++;
    o->nd = pos;
    uint32_t e = 0;
    for (uint32_t u = 0; u < qv; ++u)           /* graph.cpp:184-199 */
        for (uint32_t w = u + 1; w < qv; ++w)
            if (adj[u][w]) {
                o->qe_u[e] = (uint8_t)u;
                o->qe_v[e] = (uint8_t)w;
                o->dir_to_edge[o->eidx[u * ORC_MAXQV + w]] = (uint8_t)e;
                o->dir_to_edge[o->eidx[w * ORC_MAXQV + u]] = (uint8_t)e;
                ++e;
            }
    o->qe = e;
    return o;
}

void orc_destroy(void* h) {
    Orc* o = (Orc*)h;
    if (!o) return;
    for (size_t i = 0; i < (size_t)o->nd * o->dvcap; ++i) { free(o->main[i].v); free(o->delta[i].v); }
    free(o->main);
    free(o->delta);
    free(o->pending);
    free(o->vb);
    free(o);
}

uint32_t orc_num_dir(void* h) { return ((Orc*)h)->nd; }
uint32_t orc_num_edges(void* h) { return ((Orc*)h)->qe; }
uint32_t orc_dir(void* h, uint32_t a, uint32_t b) { return ((Orc*)h)->eidx[a * ORC_MAXQV + b]; }

/* InitFromSortedEdges (cpu_index_mirror.cpp:98-130). */
int orc_build(void* h, const uint64_t* keys, uint64_t n, uint32_t dv) {
    Orc* o = (Orc*)h;
    grow_dv(o, dv ? dv : 1);
    o->dv = dv;
    uint64_t m;
    uint64_t* s = sorted_copy(keys, n, 0, &m);
    for (uint64_t i = 0; i < m; ++i)
        if (KD(s[i]) >= o->nd || KU(s[i]) >= dv || KV(s[i]) >= dv) { free(s); return -1; }
    merge_sorted(o, s, m, 1);
    free(s);
    return 0;
}

static int test_bit(const uint32_t* m, uint32_t x) { return (m[x >> 5] >> (x & 31)) & 1u; }

/* ---- matching ---- */
typedef struct {
    const Orc* o;
    uint32_t ei;
    uint8_t vs[ORC_MAXQV];
    uint8_t bn_off[ORC_MAXQV + 1];
    uint8_t bn_pos[64], bn_dir[64];
    int seed_dirs[2];
    uint32_t m[ORC_MAXQV];
    uint32_t ncore;  /* ORC_TAIL: positions >= ncore are counted, not enumerated */
} Run;

/* cpu_dfs.cpp:67-78: (base, app) of directed edge d at vertex x under ei. */
static void resolve(const Run* r, uint32_t d, uint32_t x, const List** base, const List** app) {
    const Orc* o = r->o;
    size_t i = (size_t)d * o->dvcap + x;
    int seed = ((int)d == r->seed_dirs[0] || (int)d == r->seed_dirs[1]);
    *base = seed ? &o->delta[i] : &o->main[i];
    *app = (o->dir_to_edge[d] < r->ei) ? &o->delta[i] : NULL;
}

static uint64_t dfs(Run* r, uint32_t j) {
    const Orc* o = r->o;
    uint32_t b0 = r->bn_off[j], b1 = r->bn_off[j + 1];
    const List *gb, *ga;
    resolve(r, r->bn_dir[b0], r->m[r->bn_pos[b0]], &gb, &ga);
    uint64_t cnt = 0;
    for (int part = 0; part < 2; ++part) {
        const List* L = part ? ga : gb;
        if (!L) continue;
        for (uint32_t t = 0; t < L->n; ++t) {
            uint32_t c = L->v[t];
            int ok = 1;
            for (uint32_t k = 0; k < j && ok; ++k) ok = (r->m[k] != c);
            if (ok && o->vb_on == 2) {  /* prune by the valid bits (a sound superset) */
                const uint32_t stride = (o->dv + 31) / 32;
                ok = test_bit(o->vb + ((uint64_t)r->ei * o->qv + r->vs[j]) * stride, c);
            }
            for (uint32_t k = b0 + 1; k < b1 && ok; ++k) {
                const List *xb, *xa;
                resolve(r, r->bn_dir[k], r->m[r->bn_pos[k]], &xb, &xa);
                ok = list_has(xb, c) || (xa && list_has(xa, c));
            }
            if (!ok) continue;
            if (j + 1 == o->qv) ++cnt;
            else { r->m[j] = c; cnt += dfs(r, j + 1); }
        }
    }
    return cnt;
}

/* ---- counted tails (ORC_TAIL) ----
 * The tail positions T = [ncore, qv) hold pairwise non-adjacent query
 * vertices whose neighbours are all core vertices, so once the core is
 * matched each tail vertex p draws from a fixed candidate multiset: the
 * entries of its first backward list (base and, when visible, delta part)
 * that lie in every other backward list, weight w_p(c) = occurrences of c.
 * The enumeration would count, over injective assignments f of T avoiding
 * the core's vertices, the product of w_p(f(p)).  By Moebius inversion over
 * the lattice of set partitions of T (a partition's blocks are the tail
 * vertices that coincide), that is
 *     sum over partitions P of prod over blocks B of  mu(B) * W(B),
 *     mu(B) = (-1)^(|B|-1) (|B|-1)!,
 *     W(B)  = sum over c in (common candidates of B) minus the core's
 *             vertices of prod over p in B of w_p(c),
 * evaluated with the subset recursion F(S) = sum over blocks B of S that
 * contain S's lowest member of mu(B) W(B) F(S \ B), F(empty) = 1, in
 * arithmetic modulo 2^64 (the counters' own). */
typedef struct {
    uint32_t* v;  /* sorted distinct values */
    uint64_t* w;  /* product of the members' weights */
    uint32_t n;
} WSet;

static uint32_t* cand_tmp(uint32_t n) { return (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t)); }

/* Candidate multiset of tail position j as a weighted set. */
static void tail_candidates(Run* r, uint32_t j, WSet* out) {
    uint32_t b0 = r->bn_off[j], b1 = r->bn_off[j + 1];
    const List *gb, *ga;
    resolve(r, r->bn_dir[b0], r->m[r->bn_pos[b0]], &gb, &ga);
    uint32_t n = gb->n + (ga ? ga->n : 0);
    uint32_t* all = cand_tmp(n);
    uint32_t k = 0;
    for (int part = 0; part < 2; ++part) {
        const List* L = part ? ga : gb;
        if (!L) continue;
        for (uint32_t t = 0; t < L->n; ++t) {
            uint32_t c = L->v[t];
            int ok = 1;
            for (uint32_t q = b0 + 1; q < b1 && ok; ++q) {
                const List *xb, *xa;
                resolve(r, r->bn_dir[q], r->m[r->bn_pos[q]], &xb, &xa);
                ok = list_has(xb, c) || (xa && list_has(xa, c));
            }
            if (ok) all[k++] = c;
        }
    }
    /* sort (insertion sort is too slow for hubs: use qsort on u32) */
    uint64_t* tmp = (uint64_t*)malloc((k ? k : 1) * 8);
    for (uint32_t i = 0; i < k; ++i) tmp[i] = all[i];
    qsort(tmp, k, 8, cmp_u64);
    out->v = cand_tmp(k);
    out->w = (uint64_t*)malloc((k ? k : 1) * 8);
    out->n = 0;
    for (uint32_t i = 0; i < k;) {
        uint32_t e = i;
        while (e < k && tmp[e] == tmp[i]) ++e;
        out->v[out->n] = (uint32_t)tmp[i];
        out->w[out->n] = e - i;
        ++out->n;
        i = e;
    }
    free(tmp);
    free(all);
}

static void wset_intersect(const WSet* a, const WSet* b, WSet* out) {
    uint32_t cap = a->n < b->n ? a->n : b->n;
    out->v = cand_tmp(cap);
    out->w = (uint64_t*)malloc((cap ? cap : 1) * 8);
    out->n = 0;
    uint32_t i = 0, j = 0;
    while (i < a->n && j < b->n) {
        if (a->v[i] < b->v[j]) ++i;
        else if (b->v[j] < a->v[i]) ++j;
        else { out->v[out->n] = a->v[i]; out->w[out->n++] = a->w[i] * b->w[j]; ++i; ++j; }
    }
}

static uint64_t count_tail(Run* r) {
    const uint32_t nt = r->o->qv - r->ncore;
    const uint32_t ns = 1u << nt;
    WSet* sets = (WSet*)calloc(ns, sizeof(WSet));
    uint64_t* W = (uint64_t*)calloc(ns, 8);
    for (uint32_t p = 0; p < nt; ++p) tail_candidates(r, r->ncore + p, &sets[1u << p]);
    for (uint32_t S = 1; S < ns; ++S) {
        uint32_t top = 31 - __builtin_clz(S);
        if (S != (1u << top)) wset_intersect(&sets[S & ~(1u << top)], &sets[1u << top], &sets[S]);
        uint64_t sum = 0;
        for (uint32_t i = 0; i < sets[S].n; ++i) {
            int core = 0;
            for (uint32_t t = 0; t < r->ncore && !core; ++t) core = r->m[t] == sets[S].v[i];
            if (!core) sum += sets[S].w[i];
        }
        W[S] = sum;
    }
    uint64_t* F = (uint64_t*)calloc(ns, 8);
    F[0] = 1;
    for (uint32_t S = 1; S < ns; ++S) {
        const uint32_t low = S & (~S + 1u), rest = S & ~low;
        uint64_t f = 0;
        /* blocks B = low + any subset of rest */
        for (uint32_t sub = rest;; sub = (sub - 1) & rest) {
            const uint32_t B = low | sub;
            const uint32_t k = (uint32_t)__builtin_popcount(B);
            uint64_t mu = 1;
            for (uint32_t t = 2; t < k; ++t) mu *= t;     /* (k-1)! */
            if (k % 2 == 0) mu = (uint64_t)0 - mu;        /* (-1)^(k-1) */
            f += mu * W[B] * F[S & ~B];
            if (sub == 0) break;
        }
        F[S] = f;
    }
    uint64_t res = F[ns - 1];
    for (uint32_t S = 1; S < ns; ++S) { free(sets[S].v); free(sets[S].w); }
    free(sets);
    free(W);
    free(F);
    return res;
}

static uint64_t dfs_tail(Run* r, uint32_t j) {
    if (j == r->ncore) return count_tail(r);
    const Orc* o = r->o;
    uint32_t b0 = r->bn_off[j], b1 = r->bn_off[j + 1];
    const List *gb, *ga;
    resolve(r, r->bn_dir[b0], r->m[r->bn_pos[b0]], &gb, &ga);
    uint64_t cnt = 0;
    for (int part = 0; part < 2; ++part) {
        const List* L = part ? ga : gb;
        if (!L) continue;
        for (uint32_t t = 0; t < L->n; ++t) {
            uint32_t c = L->v[t];
            int ok = 1;
            for (uint32_t k = 0; k < j && ok; ++k) ok = (r->m[k] != c);
            for (uint32_t k = b0 + 1; k < b1 && ok; ++k) {
                const List *xb, *xa;
                resolve(r, r->bn_dir[k], r->m[r->bn_pos[k]], &xb, &xa);
                ok = list_has(xb, c) || (xa && list_has(xa, c));
            }
            if (!ok) continue;
            r->m[j] = c;
            cnt += dfs_tail(r, j + 1);
        }
    }
    (void)o;
    return cnt;
}

/* ORC_TAIL order: ei's endpoints; the tail = query vertices taken in id order
 * while not adjacent to the tail so far and leaving the other vertices
 * connected; the core in between by most visited neighbours. */
static uint32_t tail_order(const Orc* o, uint32_t ei, uint8_t* vs) {
    const uint32_t qv = o->qv, a = o->qe_u[ei], b = o->qe_v[ei];
    uint8_t tail[ORC_MAXQV] = {0};
    for (uint32_t u = 0; u < qv; ++u) {
        if (u == a || u == b) continue;
        int adjt = 0;
        for (uint32_t w = 0; w < qv; ++w) adjt |= tail[w] && o->eidx[u * ORC_MAXQV + w] != 255;
        if (adjt) continue;
        tail[u] = 1;
        /* the rest must stay connected */
        uint8_t seen[ORC_MAXQV] = {0}, st[ORC_MAXQV];
        uint32_t sp = 0, reached = 1, need = 0;
        for (uint32_t w = 0; w < qv; ++w) need += !tail[w];
        st[sp++] = (uint8_t)a;
        seen[a] = 1;
        while (sp) {
            uint32_t x = st[--sp];
            for (uint32_t w = 0; w < qv; ++w)
                if (!tail[w] && !seen[w] && o->eidx[x * ORC_MAXQV + w] != 255) { seen[w] = 1; ++reached; st[sp++] = (uint8_t)w; }
        }
        if (reached != need) tail[u] = 0;
    }
    uint8_t vis[ORC_MAXQV] = {0};
    uint32_t n = 0;
    vs[n++] = (uint8_t)a;
    vs[n++] = (uint8_t)b;
    vis[a] = vis[b] = 1;
    uint32_t ncore = 2;
    for (uint32_t u = 0; u < qv; ++u) ncore += !tail[u] && u != a && u != b;
    while (n < ncore) {
        int best = -1, bn = -1;
        for (uint32_t u = 0; u < qv; ++u) {
            if (vis[u] || tail[u]) continue;
            int c = 0;
            for (uint32_t w = 0; w < qv; ++w) if (vis[w] && o->eidx[u * ORC_MAXQV + w] != 255) ++c;
            if (c > bn) { bn = c; best = (int)u; }
        }
        vs[n++] = (uint8_t)best;
        vis[best] = 1;
    }
    for (uint32_t u = 0; u < qv; ++u)
        if (tail[u]) vs[n++] = (uint8_t)u;
    return ncore;
}

/* splitmix64 finaliser of (ei << 32 | x), modulo num_shards. */
static uint32_t seed_shard(uint32_t ei, uint32_t x, uint32_t num_shards) {
    uint64_t z = (((uint64_t)ei << 32) | x) + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (uint32_t)(z % num_shards);
}

static int seed_kept(const Orc* o, uint32_t ei, uint32_t xu, uint32_t xv) {
    if (o->num_shards <= 1) return 1;
    const uint32_t key = o->shard_anchor[ei] == o->qe_u[ei] ? xu : xv;
    return seed_shard(ei, key, o->num_shards) == o->shard;
}

void orc_set_shard(void* h, uint32_t shard, uint32_t num_shards, const uint8_t* anchor) {
    Orc* o = (Orc*)h;
    o->shard = shard;
    o->num_shards = num_shards;
    for (uint32_t e = 0; e < o->qe; ++e) o->shard_anchor[e] = anchor ? anchor[e] : o->qe_u[e];
}

static void make_run(const Orc* o, Run* r, uint32_t ei, const uint8_t* order) {
    memset(r, 0, sizeof(*r));
    r->o = o;
    r->ei = ei;
    memcpy(r->vs, order, o->qv);
    r->seed_dirs[0] = o->eidx[o->qe_u[ei] * ORC_MAXQV + o->qe_v[ei]];
    r->seed_dirs[1] = o->eidx[o->qe_v[ei] * ORC_MAXQV + o->qe_u[ei]];
    uint32_t k = 0;
    for (uint32_t j = 0; j < o->qv; ++j) {
        r->bn_off[j] = (uint8_t)k;
        if (j < 2) continue;
        /* backward neighbours: the first one generates candidates */
        for (uint32_t t = 0; t < j; ++t) {
            uint8_t d = o->eidx[r->vs[t] * ORC_MAXQV + r->vs[j]];
            if (d == 255) continue;
            r->bn_pos[k] = (uint8_t)t;
            r->bn_dir[k] = d;
            ++k;
        }
    }
    r->bn_off[o->qv] = (uint8_t)k;
}

/* Per-edge order: endpoints of ei, then BFS-like by most visited neighbours. */
static void per_edge_order(const Orc* o, uint32_t ei, uint8_t* vs) {
    uint8_t vis[ORC_MAXQV] = {0};
    vs[0] = o->qe_u[ei];
    vs[1] = o->qe_v[ei];
    vis[vs[0]] = vis[vs[1]] = 1;
    for (uint32_t j = 2; j < o->qv; ++j) {
        int best = -1, bn = -1;
        for (uint32_t u = 0; u < o->qv; ++u) {
            if (vis[u]) continue;
            int c = 0;
            for (uint32_t w = 0; w < o->qv; ++w) if (vis[w] && o->eidx[u * ORC_MAXQV + w] != 255) ++c;
            if (c > bn) { bn = c; best = (int)u; }
        }
        vs[j] = (uint8_t)best;
        vis[best] = 1;
    }
}

static uint64_t count_batch(Orc* o, const uint8_t* edge_ok, int mode, const uint8_t* global_order) {
    uint64_t total = 0;
    for (uint32_t ei = 0; ei < o->qe; ++ei) {
        o->last_edge_counts[ei] = 0;
        if (!edge_ok[ei]) continue;
        Run r;
        uint8_t vs[ORC_MAXQV];
        uint32_t ncore = o->qv;
        if (mode == ORC_GLOBAL) memcpy(vs, global_order, o->qv);
        else if (mode == ORC_TAIL) ncore = tail_order(o, ei, vs);
        else per_edge_order(o, ei, vs);
        make_run(o, &r, ei, vs);
        r.ncore = ncore;
        uint64_t c = 0;
        if (mode == ORC_GLOBAL) {
            /* enumeration.cu:727-809 without masks: every dv, resolved first-edge list */
            uint32_t d0 = o->eidx[vs[0] * ORC_MAXQV + vs[1]];
            for (uint32_t x = 0; x < o->dv; ++x) {
                const List *b, *a;
                resolve(&r, d0, x, &b, &a);
                for (int part = 0; part < 2; ++part) {
                    const List* L = part ? a : b;
                    if (!L) continue;
                    for (uint32_t t = 0; t < L->n; ++t) {
                        r.m[0] = x;
                        r.m[1] = L->v[t];
                        c += (o->qv == 2) ? 1 : dfs(&r, 2);
                    }
                }
            }
        } else {
            uint32_t d0 = r.seed_dirs[0];
            for (uint32_t x = 0; x < o->dv; ++x) {
                const List* L = &o->delta[(size_t)d0 * o->dvcap + x];
                for (uint32_t t = 0; t < L->n; ++t) {
                    if (!seed_kept(o, ei, x, L->v[t])) continue;
                    r.m[0] = x;
                    r.m[1] = L->v[t];
                    if (mode == ORC_TAIL) c += dfs_tail(&r, 2);
                    else c += (o->qv == 2) ? 1 : dfs(&r, 2);
                }
            }
        }
        o->last_edge_counts[ei] = c;
        total += c;
    }
    return total;
}

/* ---- valid bits: BuildLocalIndexBitAll with SUPPORT_MASK_WIDTH 1
 * (graph_gpu.cu:803-869; indexing.cu:2295-2379), orders and rebuild flags
 * from plan.cpp:1180-1370 ---- */
typedef struct {
    uint8_t vs[ORC_MAXQV];
    uint8_t off[ORC_MAXQV + 1];
    uint8_t bni[ORC_MAXQV * ORC_MAXQV];
} IdxOrder;

static int adj(const Orc* o, uint32_t a, uint32_t b) { return o->eidx[a * ORC_MAXQV + b] != 255; }

/* BuildIndexingOrder (plan.cpp:1180-1230): BFS from (u0, u1), neighbours in
 * ascending order; backward neighbours of position j = earlier positions
 * adjacent to vs[j], in position order. */
static void indexing_order(const Orc* o, uint32_t u0, uint32_t u1, IdxOrder* io) {
    uint8_t order[ORC_MAXQV], vis[ORC_MAXQV] = {0};
    uint32_t n = 0, lo = 0;
    order[n++] = (uint8_t)u0;
    order[n++] = (uint8_t)u1;
    vis[u0] = vis[u1] = 1;
    while (lo < n) {
        uint32_t hi = n;
        for (uint32_t i = lo; i < hi; ++i)
            for (uint32_t w = 0; w < o->qv; ++w)
                if (adj(o, order[i], w) && !vis[w]) { vis[w] = 1; order[n++] = (uint8_t)w; }
        lo = hi;
    }
    uint32_t k = 0;
    io->off[0] = 0;
    io->bni[k++] = 1; /* bni_[0] = 1 (plan.cpp:1213-1215); position 0 has none in use */
    io->off[1] = 1;
    io->vs[0] = order[0];
    for (uint32_t j = 1; j < o->qv; ++j) {
        io->vs[j] = order[j];
        for (uint32_t t = 0; t < j; ++t)
            if (adj(o, order[j], io->vs[t])) io->bni[k++] = (uint8_t)t;
        io->off[j + 1] = (uint8_t)k;
    }
}

/* GenerateRebuildFlagsWithOrder (plan.cpp:1277-1332): every edge on a simple
 * path from a starting vertex to u0 or u1 (stopping there), plus (u0,u1). */
static void rebuild_edges(const Orc* o, uint32_t u0, uint32_t u1, const uint32_t* starts, uint8_t* f) {
    const uint32_t qv = o->qv;
    memset(f, 0, ORC_MAXQV * ORC_MAXQV);
    f[u0 * ORC_MAXQV + u1] = f[u1 * ORC_MAXQV + u0] = 1;
    for (int s = 0; s < 2; ++s) {
        uint8_t path[ORC_MAXQV + 1], vis[ORC_MAXQV] = {0};
        uint32_t ci[ORC_MAXQV + 1] = {0};
        vis[starts[s]] = 1;
        path[0] = (uint8_t)starts[s];
        uint32_t depth = 1;
        for (;;) {
            /* next neighbour (ascending) of path[depth-1] from index ci[depth] */
            int advanced = 0;
            while (1) {
                uint32_t cnt = 0, nv = 255;
                for (uint32_t w = 0; w < qv; ++w)
                    if (adj(o, path[depth - 1], w)) {
                        if (cnt == ci[depth]) { nv = w; break; }
                        ++cnt;
                    }
                if (nv == 255) break;
                if (vis[nv]) { ci[depth]++; continue; }
                if (nv == u0 || nv == u1) {
                    path[depth] = (uint8_t)nv;
                    for (uint32_t i = 0; i < depth; ++i) {
                        f[path[i] * ORC_MAXQV + path[i + 1]] = 1;
                        f[path[i + 1] * ORC_MAXQV + path[i]] = 1;
                    }
                    ci[depth]++;
                    continue;
                }
                vis[nv] = 1;
                path[depth] = (uint8_t)nv;
                depth++;
                advanced = 1;
                break;
            }
            if (advanced) continue;
            ci[depth] = 0;
            depth--;
            if (depth == 0) break;
            vis[path[depth]] = 0;
            ci[depth]++;
        }
    }
}

/* GenerateRebuildVFlagsWithOrder (plan.cpp:1334-1370); -1 where the
 * reference stops with "Error in order generation!". */
static int rebuild_vertices(const Orc* o, const IdxOrder* io, const uint8_t* f, uint8_t* vf) {
    memset(vf, 0, ORC_MAXQV);
    for (uint32_t i = 0; i < o->qv; ++i) {
        uint32_t u = io->vs[i];
        if (i == 0) { vf[u] = 1; continue; }
        uint32_t sum = 0, nb = io->off[i + 1] - io->off[i];
        for (uint32_t b = io->off[i]; b < io->off[i + 1]; ++b) sum += f[io->vs[io->bni[b]] * ORC_MAXQV + u] ? 1 : 0;
        if (sum == 0) vf[u] = 0;
        else if (sum == nb) vf[u] = 1;
        else return -1;
    }
    return 0;
}

/* SelectStartingEdge (plan.cpp:428-533) from per-direction cardinalities and
 * average list lengths of the initial index. */
void orc_starting_edge(void* h, const uint32_t* card, const float* avg, uint32_t* out2) {
    Orc* o = (Orc*)h;
    uint32_t sel[ORC_MAXQE], ns = 0, nxt[ORC_MAXQE], nn;
    uint32_t deg[ORC_MAXQV] = {0};
    for (uint32_t u = 0; u < o->qv; ++u)
        for (uint32_t w = 0; w < o->qv; ++w) deg[u] += adj(o, u, w);
    uint32_t best = 0;
    for (uint32_t e = 0; e < o->qe; ++e) {
        uint32_t sd = deg[o->qe_u[e]] + deg[o->qe_v[e]];
        if (sd > best) { best = sd; ns = 0; sel[ns++] = e; }
        else if (sd == best) sel[ns++] = e;
    }
    if (ns > 1) {
        uint32_t bt = 0;
        nn = 0;
        for (uint32_t i = 0; i < ns; ++i) {
            uint32_t a = o->qe_u[sel[i]], b = o->qe_v[sel[i]], t = 0;
            for (uint32_t x = 0; x < o->qv; ++x) t += adj(o, x, a) && adj(o, x, b);
            if (t > bt) { bt = t; nn = 0; nxt[nn++] = sel[i]; }
            else if (t == bt) nxt[nn++] = sel[i];
        }
        memcpy(sel, nxt, sizeof(sel));
        ns = nn;
    }
    if (ns > 1) {
        uint32_t bc = UINT32_MAX;
        nn = 0;
        for (uint32_t i = 0; i < ns; ++i) {
            uint32_t c = card[o->eidx[o->qe_u[sel[i]] * ORC_MAXQV + o->qe_v[sel[i]]]];
            if (c < bc) { bc = c; nn = 0; nxt[nn++] = sel[i]; }
            else if (c == bc) nxt[nn++] = sel[i];
        }
        memcpy(sel, nxt, sizeof(sel));
        ns = nn;
    }
    if (ns > 1) {
        float bs = 3.402823466e+38f;
        nn = 0;
        for (uint32_t i = 0; i < ns; ++i) {
            uint32_t a = o->qe_u[sel[i]], b = o->qe_v[sel[i]];
            float sum = 0.0f;
            for (uint32_t w = 0; w < o->qv; ++w)
                if (adj(o, a, w) && w != b) sum += avg[o->eidx[a * ORC_MAXQV + w]];
            for (uint32_t w = 0; w < o->qv; ++w)
                if (adj(o, b, w) && w != a) sum += avg[o->eidx[b * ORC_MAXQV + w]];
            if (sum < bs) { bs = sum; nn = 0; nxt[nn++] = sel[i]; }
            else if (sum == bs) nxt[nn++] = sel[i];
        }
        memcpy(sel, nxt, sizeof(sel));
        ns = nn;
    }
    out2[0] = o->qe_u[sel[0]];
    out2[1] = o->qe_v[sel[0]];
}


static int list_hits(const List* l, const uint32_t* m) {
    for (uint32_t t = 0; t < l->n; ++t)
        if (test_bit(m, l->v[t])) return 1;
    return 0;
}

static void compute_valid_bits(Orc* o) {
    const uint32_t stride = (o->dv + 31) / 32, qv = o->qv;
    o->vb_words = (uint64_t)o->qe * qv * stride;
    o->vb = (uint32_t*)realloc(o->vb, (o->vb_words ? o->vb_words : 1) * 4);
    o->vb_error = 0;
    for (uint32_t ei = 0; ei < o->qe; ++ei) {
        IdxOrder io;
        uint8_t f[ORC_MAXQV * ORC_MAXQV], vf[ORC_MAXQV];
        indexing_order(o, o->qe_u[ei], o->qe_v[ei], &io);
        rebuild_edges(o, o->qe_u[ei], o->qe_v[ei], o->vb_start, f);
        if (rebuild_vertices(o, &io, f, vf) < 0) { o->vb_error = 1; return; }
        uint32_t* M = o->vb + (uint64_t)ei * qv * stride;
        for (uint32_t u = 0; u < qv; ++u) memset(M + (uint64_t)u * stride, vf[u] ? 0x00 : 0xFF, stride * 4);
        uint32_t a = io.vs[0], b = io.vs[1];
        uint32_t i01 = o->eidx[a * ORC_MAXQV + b], i10 = o->eidx[b * ORC_MAXQV + a];
        for (uint32_t x = 0; x < o->dv; ++x) {
            if (o->delta[(size_t)i01 * o->dvcap + x].n) M[(uint64_t)a * stride + (x >> 5)] |= 1u << (x & 31);
            if (o->delta[(size_t)i10 * o->dvcap + x].n) M[(uint64_t)b * stride + (x >> 5)] |= 1u << (x & 31);
        }
        for (uint32_t d = 2; d < qv; ++d) {
            uint32_t u = io.vs[d];
            if (!vf[u]) continue;
            uint32_t* out = M + (uint64_t)u * stride;
            memset(out, 0, stride * 4);
            for (uint32_t x = 0; x < o->dv; ++x) {
                int valid = 1;
                for (uint32_t bp = io.off[d]; bp < io.off[d + 1] && valid; ++bp) {
                    uint32_t u1 = io.vs[io.bni[bp]];
                    uint32_t bwd = o->eidx[u * ORC_MAXQV + u1];
                    const uint32_t* m1 = M + (uint64_t)u1 * stride;
                    int sat = list_hits(&o->main[(size_t)bwd * o->dvcap + x], m1);
                    if (!sat && o->dir_to_edge[bwd] <= ei) sat = list_hits(&o->delta[(size_t)bwd * o->dvcap + x], m1);
                    valid = sat;
                }
                if (valid) out[x >> 5] |= 1u << (x & 31);
            }
        }
    }
}

/* The indexing order and rebuild-vertex flags of query edge ei for the
 * starting edge (s0, s1), for pinning against the reference planner.
 * Returns the number of bni entries; *vflags = bit mask, or ~0u on the
 * reference's "Error in order generation" case. */
uint32_t orc_indexing_order(void* h, uint32_t ei, uint32_t s0, uint32_t s1, uint8_t* vs, uint8_t* offs,
                            uint8_t* bni, uint32_t* vflags) {
    Orc* o = (Orc*)h;
    IdxOrder io;
    uint8_t f[ORC_MAXQV * ORC_MAXQV], vf[ORC_MAXQV];
    uint32_t st[2] = {s0, s1};
    indexing_order(o, o->qe_u[ei], o->qe_v[ei], &io);
    rebuild_edges(o, o->qe_u[ei], o->qe_v[ei], st, f);
    *vflags = 0;
    if (rebuild_vertices(o, &io, f, vf) < 0) *vflags = ~0u;
    else
        for (uint32_t u = 0; u < o->qv; ++u) *vflags |= (uint32_t)vf[u] << u;
    memcpy(vs, io.vs, o->qv);
    memcpy(offs, io.off, o->qv + 1);
    memcpy(bni, io.bni, io.off[o->qv]);
    return io.off[o->qv];
}

/* Valid bits are computed for every later matched batch (after its delta
 * lists, before matching) from the starting edge (s0, s1); on = 0 stops,
 * on = 2 also prunes the count's candidates by them (soundness check). */
void orc_set_valid_bits(void* h, int on, uint32_t s0, uint32_t s1) {
    Orc* o = (Orc*)h;
    o->vb_on = on;
    o->vb_start[0] = s0;
    o->vb_start[1] = s1;
}

/* Copies the last batch's valid bits ([qe][qv][(dv+31)/32] words) and returns
 * the word count; UINT64_MAX if the reference would have stopped. */
uint64_t orc_valid_bits(void* h, uint32_t* out, uint64_t cap) {
    Orc* o = (Orc*)h;
    if (o->vb_error) return UINT64_MAX;
    if (out) memcpy(out, o->vb, (cap < o->vb_words ? cap : o->vb_words) * 4);
    return o->vb_words;
}

static void flush_pending(Orc* o) {
    if (!o->n_pending) return;
    uint64_t m;
    uint64_t* s = sorted_copy(o->pending, o->n_pending, 1, &m);
    merge_sorted(o, s, m, 1);
    free(s);
    o->n_pending = 0;
}

/* One batch.  edge_ok may be NULL (derived: both directions have delta keys,
 * calig_helper_gamma.cu:436-444).  Returns the count, or UINT64_MAX on bad keys. */
uint64_t orc_batch(void* h, uint32_t dv, const uint64_t* ins, uint64_t n_ins, const uint64_t* del,
                   uint64_t n_del, const uint64_t* delta, uint64_t n_delta, const uint8_t* edge_ok,
                   int mode, const uint8_t* global_order) {
    Orc* o = (Orc*)h;
    flush_pending(o);  /* BatchUpdateGlobalIndex of the previous batch */
    grow_dv(o, dv);
    o->dv = dv;
    const uint64_t* arrs[3] = {ins, del, delta};
    uint64_t ns[3] = {n_ins, n_del, n_delta};
    for (int a = 0; a < 3; ++a)
        for (uint64_t i = 0; i < ns[a]; ++i)
            if (KD(arrs[a][i]) >= o->nd || KU(arrs[a][i]) >= dv || KV(arrs[a][i]) >= dv) return UINT64_MAX;
    uint64_t m;
    uint64_t* s = sorted_copy(ins, n_ins, 1, &m);
    merge_sorted(o, s, m, 1);
    free(s);
    s = sorted_copy(del, n_del, 0, &m);
    merge_sorted(o, s, m, 0);
    free(s);
    memset(o->last_edge_counts, 0, sizeof(o->last_edge_counts));
    if (n_delta == 0) return 0;
    /* RebuildUpdate: sorted, not unique */
    for (size_t i = 0; i < (size_t)o->nd * o->dvcap; ++i) o->delta[i].n = 0;
    s = sorted_copy(delta, n_delta, 0, &m);
    uint32_t dcount[ORC_MAXD] = {0};
    for (uint64_t i = 0; i < m; ++i) {
        List* l = &o->delta[(size_t)KD(s[i]) * o->dvcap + KU(s[i])];
        list_reserve(l, l->n + 1);
        l->v[l->n++] = KV(s[i]);
        dcount[KD(s[i])]++;
    }
    free(s);
    uint8_t ok[ORC_MAXQE];
    for (uint32_t e = 0; e < o->qe; ++e) {
        if (edge_ok) ok[e] = edge_ok[e];
        else
            ok[e] = dcount[o->eidx[o->qe_u[e] * ORC_MAXQV + o->qe_v[e]]] &&
                    dcount[o->eidx[o->qe_v[e] * ORC_MAXQV + o->qe_u[e]]];
    }
    if (o->vb_on) compute_valid_bits(o);
    uint64_t c = count_batch(o, ok, mode, global_order);
    o->pending = (uint64_t*)realloc(o->pending, n_delta * 8);
    memcpy(o->pending, delta, n_delta * 8);
    o->n_pending = n_delta;
    return c;
}

void orc_edge_counts(void* h, uint64_t* out) {
    Orc* o = (Orc*)h;
    memcpy(out, o->last_edge_counts, o->qe * 8);
}

/* Sorted keys of the main index after any pending merge-back. */
uint64_t orc_dump(void* h, uint64_t* out, uint64_t cap) {
    Orc* o = (Orc*)h;
    flush_pending(o);
    uint64_t n = 0;
    for (uint32_t d = 0; d < o->nd; ++d)
        for (uint32_t u = 0; u < o->dv; ++u) {
            const List* l = &o->main[(size_t)d * o->dvcap + u];
            for (uint32_t t = 0; t < l->n; ++t) {
                if (out && n < cap) out[n] = ((uint64_t)d << 59) | ((uint64_t)u << 32) | l->v[t];
                ++n;
            }
        }
    return n;
}

/* Fraction check helper: number of main entries whose mirror entry is missing. */
uint64_t orc_asymmetry(void* h) {
    Orc* o = (Orc*)h;
    uint64_t bad = 0;
    for (uint32_t a = 0; a < o->qv; ++a)
        for (uint32_t b = 0; b < o->qv; ++b) {
            uint8_t d = o->eidx[a * ORC_MAXQV + b];
            if (d == 255) continue;
            uint8_t r = o->eidx[b * ORC_MAXQV + a];
            for (uint32_t u = 0; u < o->dv; ++u) {
                const List* l = &o->main[(size_t)d * o->dvcap + u];
                for (uint32_t t = 0; t < l->n; ++t)
                    if (!list_has(&o->main[(size_t)r * o->dvcap + l->v[t]], u)) ++bad;
            }
        }
    return bad;
}

/* ---- brute force: label-preserving injective embeddings of Q in G ----
 * G as sorted CSR (off[n+1], adj), vertex labels glab; Q as labels + edges. */
typedef struct {
    uint32_t n;
    const uint64_t* off;
    const uint32_t* adj;
    const uint32_t* glab;
    uint32_t qv;
    const uint32_t* qlab;
    uint8_t qadj[ORC_MAXQV][ORC_MAXQV];
    uint8_t order[ORC_MAXQV];
    uint32_t m[ORC_MAXQV];
} BF;

static int g_has(const BF* b, uint32_t x, uint32_t y) {
    uint64_t lo = b->off[x], hi = b->off[x + 1];
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (b->adj[mid] < y) lo = mid + 1; else hi = mid;
    }
    return lo < b->off[x + 1] && b->adj[lo] == y;
}

static uint64_t bf_rec(BF* b, uint32_t j) {
    if (j == b->qv) return 1;
    uint32_t u = b->order[j];
    /* parent: first earlier query neighbour (connected order) */
    int par = -1;
    for (uint32_t t = 0; t < j; ++t) if (b->qadj[b->order[t]][u]) { par = (int)t; break; }
    uint64_t c = 0;
    if (par < 0) {
        for (uint32_t x = 0; x < b->n; ++x) {
            if (b->glab[x] != b->qlab[u]) continue;
            int ok = 1;
            for (uint32_t t = 0; t < j && ok; ++t) ok = b->m[t] != x;
            if (!ok) continue;
            b->m[j] = x;
            c += bf_rec(b, j + 1);
        }
        return c;
    }
    uint32_t pv = b->m[par];
    for (uint64_t p = b->off[pv]; p < b->off[pv + 1]; ++p) {
        uint32_t x = b->adj[p];
        if (b->glab[x] != b->qlab[u]) continue;
        int ok = 1;
        for (uint32_t t = 0; t < j && ok; ++t) {
            if (b->m[t] == x) ok = 0;
            else if (b->qadj[b->order[t]][u] && !g_has(b, b->m[t], x)) ok = 0;
        }
        if (!ok) continue;
        b->m[j] = x;
        c += bf_rec(b, j + 1);
    }
    return c;
}

uint64_t orc_bruteforce(uint32_t n, const uint64_t* off, const uint32_t* adj, const uint32_t* glab,
                        uint32_t qv, const uint32_t* qlab, uint32_t qe, const uint32_t* qedges) {
    BF b;
    memset(&b, 0, sizeof(b));
    b.n = n; b.off = off; b.adj = adj; b.glab = glab; b.qv = qv; b.qlab = qlab;
    for (uint32_t i = 0; i < qe; ++i) {
        b.qadj[qedges[2 * i]][qedges[2 * i + 1]] = 1;
        b.qadj[qedges[2 * i + 1]][qedges[2 * i]] = 1;
    }
    /* BFS order from vertex 0 keeps every later vertex adjacent to an earlier one */
    uint8_t vis[ORC_MAXQV] = {0};
    uint32_t k = 0;
    for (uint32_t s = 0; s < qv; ++s) {
        if (vis[s]) continue;
        vis[s] = 1;
        b.order[k++] = (uint8_t)s;
        for (uint32_t h = k - 1; h < k; ++h)
            for (uint32_t w = 0; w < qv; ++w)
                if (!vis[w] && b.qadj[b.order[h]][w]) { vis[w] = 1; b.order[k++] = (uint8_t)w; }
    }
    return bf_rec(&b, 0);
}
