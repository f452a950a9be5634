// Packed-memory-array layout of the index (the reference's GPMA:
// Multi_GPMA gpma/gpma.cuh:36-111, CGCSM_GPMA index/gpma_wrapper.cu:26-116,
// rebalance gpma/gpma.cu:493-665), rebuilt for sm_100a without device-side
// launches (the reference's rebalance uses CDP1, which sm_90+ lacks).
//
// Layout: one PMA per query direction d, `cap_d = kSeg * 2^h_d` slots of
// full 64-bit keys (d << 59 | u << 32 | v) plus a valid byte per slot; the
// directions are packed back to back, so the whole slot array is
// non-decreasing.  A slot that holds no key keeps a copy of an earlier key
// value (order is all that matters for it), so a plain lower_bound over the
// slots finds the first slot whose value is >= x, and x is present iff that
// slot is valid and holds x.
//
// Batch update, set semantics (index + ins) - del (the same as the engine's
// k_merge_runs; the reference's GPMA is bulk-loaded once and never updated
// or read by its matcher, calig_helper_gpma.cu:284-296, 383-414, so its
// update semantics are not a parity target):
//   1. sort the edits (key, op), one effect per distinct key: a present key
//      that is deleted loses its valid flag in place; an absent key that is
//      inserted is queued for its leaf (the leaf of its lower_bound slot)
//   2. per leaf with queued inserts, the smallest enclosing tree node whose
//      density after the batch is within the upper bound of its level
//      (0.92 at the leaves to 0.84 at the root, gpma.cuh:55-58) is its
//      window; windows are tree nodes, so keeping only the maximal ones (sort
//      by start, prefix max of end) leaves disjoint windows
//   3. each window's valid keys and queued inserts are gathered, sorted
//      (segmented) and spread evenly over the window's slots
//   4. if a root would exceed its bound, the whole structure is rebuilt with
//      capacities at density <= 1/2 (amortised doubling)
// Lower density bounds are not enforced: deletions leave slots invalid until
// a window rewrites them (space is reclaimed by later windows and rebuilds).
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "cgbdsm.h"

namespace {

constexpr uint32_t kSeg = 32;               // slots per leaf
constexpr double kUpLeaf = 0.92, kUpRoot = 0.84;

struct GpmaDir {
    uint64_t off = 0;      // first slot
    uint64_t cap = 0;      // slots (kSeg << h)
    uint32_t h = 0;        // tree height (leaves = 2^h)
    uint64_t leaf0 = 0;    // first leaf (global leaf index)
};

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t* __restrict__ a, uint64_t lo, uint64_t hi,
                                                    uint64_t x) {
    uint64_t len = hi - lo;
    while (len > 0) {
        const uint64_t half = len >> 1;
        if (a[lo + half] < x) { lo += half + 1; len -= half + 1; }
        else len = half;
    }
    return lo;
}

// Per-direction tables on the device.
struct DirTab {
    const uint64_t* off;
    const uint64_t* cap;
    const uint32_t* h;
    const uint64_t* leaf0;
};

// One thread per sorted edit; the first of each run of equal keys applies
// the run's effect (any delete wins: (S + ins) - del).
__global__ void k_gp_effect(const uint64_t* __restrict__ key, const uint8_t* __restrict__ op, uint64_t n,
                            uint64_t* slots, uint8_t* valid, DirTab dt, uint32_t nd, uint64_t* ins_key,
                            uint64_t* ins_leaf, unsigned long long* n_ins, int* leaf_delta, uint32_t* leaf_ins,
                            unsigned int* err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        if (i > 0 && key[i - 1] == k) continue;
        bool del = false, ins = false;
        for (uint64_t t = i; t < n && key[t] == k; ++t) {
            del |= op[t] != 0;
            ins |= op[t] == 0;
        }
        const uint32_t d = (uint32_t)(k >> 59);
        if (d >= nd) { atomicOr(err, 1u); continue; }
        const uint64_t s0 = dt.off[d], s1 = s0 + dt.cap[d];
        const uint64_t p = lower_bound_u64(slots, s0, s1, k);
        const bool present = p < s1 && valid[p] && slots[p] == k;
        const uint64_t leaf = dt.leaf0[d] + min((p - s0) / kSeg, (dt.cap[d] / kSeg) - 1);
        if (del) {
            if (present) {
                valid[p] = 0;
                atomicAdd(leaf_delta + leaf, -1);
            }
        } else if (ins && !present) {
            const unsigned long long q = atomicAdd(n_ins, 1ull);
            ins_key[q] = k;
            ins_leaf[q] = leaf;
            atomicAdd(leaf_delta + leaf, 1);
            atomicAdd(leaf_ins + leaf, 1u);
        }
    }
}

// Valid keys per leaf (one warp per leaf).
__global__ void k_gp_leafcount(const uint8_t* __restrict__ valid, uint64_t n_leaves, uint32_t* cnt) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t l = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < n_leaves; l += nw) {
        const uint32_t b = __ballot_sync(0xffffffffu, valid[l * kSeg + lane] != 0);
        if (lane == 0) cnt[l] = __popc(b);
    }
}

__global__ void k_gp_newcount(const uint32_t* cnt, const int* delta, uint64_t n, uint64_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint64_t)((int64_t)cnt[i] + delta[i]);
}

// Window of each leaf with queued inserts: smallest node within its level's
// upper density bound; encoded (first leaf << 32 | ~end leaf) so that an
// ascending sort lists windows by start, larger first.  P = inclusive prefix
// sums of the new per-leaf counts (P[l] = sum over leaves <= l).
__global__ void k_gp_window(const uint32_t* __restrict__ leaf_ins, const uint64_t* __restrict__ P,
                            const uint32_t* __restrict__ leaf_dir, DirTab dt, uint64_t n_leaves, uint64_t* win,
                            unsigned long long* n_win, unsigned int* resize) {
    for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < n_leaves;
         l += (uint64_t)gridDim.x * blockDim.x) {
        if (!leaf_ins[l]) continue;
        const uint32_t d = leaf_dir[l];
        const uint64_t base = dt.leaf0[d], rel = l - base;
        const uint32_t h = dt.h[d];
        bool found = false;
        for (uint32_t lv = 0; lv <= h; ++lv) {
            const uint64_t a = base + ((rel >> lv) << lv), b = a + (1ull << lv);
            const uint64_t c = P[b - 1] - (a > 0 ? P[a - 1] : 0);
            const double up = h ? kUpLeaf - (kUpLeaf - kUpRoot) * (double)lv / (double)h : kUpRoot;
            if ((double)c <= up * (double)((uint64_t)kSeg << lv)) {
                const unsigned long long q = atomicAdd(n_win, 1ull);
                win[q] = (a << 32) | (0xffffffffull - b);
                found = true;
                break;
            }
        }
        if (!found) atomicOr(resize, 1u);
    }
}

// Windows are maximal when their end exceeds every end before them.
__global__ void k_gp_maximal(const uint64_t* __restrict__ win, const uint64_t* __restrict__ prefmax_end, uint64_t n,
                             uint8_t* flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = 0xffffffffull - (win[i] & 0xffffffffull);
        flag[i] = (i == 0 || b > prefmax_end[i - 1]) ? 1 : 0;
    }
}

__global__ void k_gp_end(const uint64_t* win, uint64_t n, uint64_t* end) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        end[i] = 0xffffffffull - (win[i] & 0xffffffffull);
}

// New key count of each window and the value before it (read before any rewrite).
__global__ void k_gp_wininfo(const uint64_t* __restrict__ win, uint64_t n, const uint64_t* __restrict__ P,
                             const uint64_t* __restrict__ slots, uint64_t* wcount, uint64_t* wpred) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t a = win[i] >> 32, b = 0xffffffffull - (win[i] & 0xffffffffull);
        wcount[i] = P[b - 1] - (a > 0 ? P[a - 1] : 0);
        wpred[i] = a > 0 ? slots[a * kSeg - 1] : 0ull;
    }
}

// Gather a window's valid keys (block per window, in slot order) to tmp[off..).
__global__ void k_gp_gather(const uint64_t* __restrict__ win, uint64_t n_win, const uint64_t* __restrict__ woff,
                            const uint64_t* __restrict__ wcount, const uint64_t* __restrict__ slots,
                            const uint8_t* __restrict__ valid, uint64_t* tmp, uint64_t* wfill, unsigned int* bad) {
    typedef cub::BlockScan<uint32_t, 256> Scan;
    __shared__ typename Scan::TempStorage ts;
    __shared__ uint64_t s_base;
    for (uint64_t w = blockIdx.x; w < n_win; w += gridDim.x) {
        const uint64_t a = win[w] >> 32, b = 0xffffffffull - (win[w] & 0xffffffffull);
        const uint64_t s0 = a * kSeg, s1 = b * kSeg;
        if (threadIdx.x == 0) s_base = 0;
        __syncthreads();
        for (uint64_t t = s0; t < s1; t += 256) {
            const uint64_t s = t + threadIdx.x;
            const uint32_t f = (s < s1 && valid[s]) ? 1u : 0u;
            uint32_t pos, tot;
            Scan(ts).ExclusiveSum(f, pos, tot);
            if (f && s_base + pos < wcount[w]) tmp[woff[w] + s_base + pos] = slots[s];
            __syncthreads();
            if (threadIdx.x == 0) s_base += tot;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (s_base > wcount[w]) atomicOr(bad, 1u);
            wfill[w] = min(s_base, wcount[w]);
        }
        __syncthreads();
    }
}

// Queued inserts join their window (the maximal window holding their leaf).
// Every such leaf lies in a window and every window's slots in tmp number
// its new count; a violation of either sets `bad` and writes nothing.
__global__ void k_gp_place_ins(const uint64_t* __restrict__ ins_key, const uint64_t* __restrict__ ins_leaf,
                               uint64_t n, const uint64_t* __restrict__ win, uint64_t n_win,
                               const uint64_t* __restrict__ woff, const uint64_t* __restrict__ wcount,
                               unsigned long long* wfill, uint64_t* tmp, unsigned int* bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t leaf = ins_leaf[i];
        // last window whose first leaf <= leaf
        uint64_t lo = 0, len = n_win;
        while (len > 0) {
            const uint64_t half = len >> 1;
            if ((win[lo + half] >> 32) <= leaf) { lo += half + 1; len -= half + 1; }
            else len = half;
        }
        if (lo == 0) { atomicOr(bad, 1u); continue; }
        const uint64_t w = lo - 1;
        if (leaf >= 0xffffffffull - (win[w] & 0xffffffffull)) { atomicOr(bad, 1u); continue; }
        const unsigned long long q = atomicAdd(wfill + w, 1ull);
        if (q >= wcount[w]) { atomicOr(bad, 1u); continue; }
        tmp[woff[w] + q] = ins_key[i];
    }
}

// Spread each window's sorted keys evenly: key i to slot s0 + floor(i W / n);
// every other slot copies the last key before it (or the value before the window).
__global__ void k_gp_scatter(const uint64_t* __restrict__ win, uint64_t n_win, const uint64_t* __restrict__ woff,
                             const uint64_t* __restrict__ wcount, const uint64_t* __restrict__ wpred,
                             const uint64_t* __restrict__ sorted, uint64_t* slots, uint8_t* valid) {
    for (uint64_t w = blockIdx.x; w < n_win; w += gridDim.x) {
        const uint64_t a = win[w] >> 32, b = 0xffffffffull - (win[w] & 0xffffffffull);
        const uint64_t s0 = a * kSeg, W = (b - a) * kSeg, n = wcount[w];
        const uint64_t* src = sorted + woff[w];
        for (uint64_t r = threadIdx.x; r < W; r += blockDim.x) {
            // last key index placed at or before slot r: ceil((r + 1) n / W) - 1
            const uint64_t im = n ? ((r + 1) * n + W - 1) / W : 0;
            if (im == 0) {
                slots[s0 + r] = wpred[w];
                valid[s0 + r] = 0;
            } else {
                const uint64_t i = im - 1;
                slots[s0 + r] = src[i];
                valid[s0 + r] = (i * W / n == r) ? 1 : 0;
            }
        }
    }
}

// Rebuild: sorted unique keys spread over fresh capacities (density <= 1/2).
__global__ void k_gp_spread(const uint64_t* __restrict__ keys, uint64_t n, const uint64_t* __restrict__ dir_start,
                            const uint64_t* __restrict__ dir_n, DirTab dt, uint32_t nd, uint64_t* slots,
                            uint8_t* valid, uint64_t total_slots) {
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < total_slots;
         s += (uint64_t)gridDim.x * blockDim.x) {
        // direction of slot s
        uint32_t lo = 0, len = nd;
        while (len > 0) {
            const uint32_t half = len >> 1;
            if (dt.off[lo + half] <= s) { lo += half + 1; len -= half + 1; }
            else len = half;
        }
        const uint32_t d = lo - 1;
        const uint64_t r = s - dt.off[d], W = dt.cap[d], m = dir_n[d], st = dir_start[d];
        const uint64_t im = m ? ((r + 1) * m + W - 1) / W : 0;
        if (im == 0) {
            slots[s] = st > 0 ? keys[st - 1] : 0ull;
            valid[s] = 0;
        } else {
            const uint64_t i = im - 1;
            slots[s] = keys[st + i];
            valid[s] = (i * W / m == r) ? 1 : 0;
        }
    }
}

__global__ void k_gp_dir_hist(const uint64_t* keys, uint64_t n, uint32_t nd, unsigned long long* hist,
                              unsigned int* err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = (uint32_t)(keys[i] >> 59);
        if (d < nd) atomicAdd(hist + d, 1ull);
        else atomicOr(err, 1u);
    }
}

__global__ void k_gp_leafdir(uint32_t* leaf_dir, const uint64_t* leaf0, uint32_t nd, uint64_t n_leaves) {
    for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < n_leaves;
         l += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, len = nd;
        while (len > 0) {
            const uint32_t half = len >> 1;
            if (leaf0[lo + half] <= l) { lo += half + 1; len -= half + 1; }
            else len = half;
        }
        leaf_dir[l] = lo - 1;
    }
}

__global__ void k_gp_valid_flags(const uint8_t* valid, uint64_t n, uint8_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = valid[i];
}

__global__ void k_gp_strip_dir(const uint64_t* in, uint64_t n, uint64_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[i] & ((1ull << 59) - 1ull);
}

struct MaxOp {
    __device__ __forceinline__ uint64_t operator()(uint64_t a, uint64_t b) const { return a > b ? a : b; }
};

}  // namespace

struct cgb_gpma {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t nd = 0;
    std::string err;
    std::vector<GpmaDir> dirs;
    uint64_t total_slots = 0, n_leaves = 0, n_keys = 0;
    uint64_t* slots = nullptr;
    uint8_t* valid = nullptr;
    uint32_t* leaf_cnt = nullptr;
    int* leaf_delta = nullptr;
    uint32_t* leaf_ins = nullptr;
    uint32_t* leaf_dir = nullptr;
    uint64_t* d_off = nullptr; uint64_t* d_cap = nullptr; uint32_t* d_h = nullptr; uint64_t* d_leaf0 = nullptr;
    unsigned long long* d_scal = nullptr;  // [0] n_ins, [1] n_win, [2] resize|err<<1 (u32 pair), [3..] hist
    void* temp = nullptr; size_t temp_cap = 0;
    std::vector<void*> bufs;  // per-batch buffers, freed on growth / destroy
    uint64_t stats[6] = {0, 0, 0, 0, 0, 0};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

namespace {

cgb_status gfail(cgb_gpma* g, cgb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (g) g->err = buf;
    return s;
}

#define GCK(x)                                                                                    \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) return gfail(g, e_ == cudaErrorMemoryAllocation ? CGB_ERR_OOM : CGB_ERR_CUDA, \
                                            "%s: %s", #x, cudaGetErrorString(e_));                \
    } while (0)

unsigned grid_of(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148ull * 16)); }

template <typename T>
cgb_status galloc(cgb_gpma* g, T*& p, uint64_t n) {
    void* q = nullptr;
    GCK(cudaMalloc(&q, std::max<uint64_t>(n, 1) * sizeof(T)));
    g->bufs.push_back(q);
    p = (T*)q;
    return CGB_OK;
}

cgb_status gtemp(cgb_gpma* g, size_t need) {
    if (need <= g->temp_cap) return CGB_OK;
    if (g->temp) cudaFree(g->temp);
    g->temp = nullptr;
    g->temp_cap = 0;
    GCK(cudaMalloc(&g->temp, need));
    g->temp_cap = need;
    return CGB_OK;
}

void free_structure(cgb_gpma* g) {
    for (void* p : {(void*)g->slots, (void*)g->valid, (void*)g->leaf_cnt, (void*)g->leaf_delta, (void*)g->leaf_ins,
                    (void*)g->leaf_dir})
        if (p) cudaFree(p);
    g->slots = nullptr; g->valid = nullptr; g->leaf_cnt = nullptr; g->leaf_delta = nullptr;
    g->leaf_ins = nullptr; g->leaf_dir = nullptr;
}

void free_bufs(cgb_gpma* g) {
    for (void* p : g->bufs) cudaFree(p);
    g->bufs.clear();
}

// Rebuilds the structure from n sorted unique keys (device).
cgb_status rebuild(cgb_gpma* g, const uint64_t* keys, uint64_t n) {
    unsigned int* d_err = (unsigned int*)(g->d_scal + 2);
    unsigned long long* hist = g->d_scal + 3;
    GCK(cudaMemsetAsync(g->d_scal + 2, 0, (1 + g->nd) * sizeof(unsigned long long), g->stream));
    if (n) k_gp_dir_hist<<<grid_of(n), 256, 0, g->stream>>>(keys, n, g->nd, hist, d_err);
    std::vector<unsigned long long> h(1 + g->nd);
    GCK(cudaMemcpyAsync(h.data(), g->d_scal + 2, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        g->stream));
    GCK(cudaStreamSynchronize(g->stream));
    if (h[0]) return gfail(g, CGB_ERR_ARG, "key direction out of range (>= %u)", g->nd);
    free_structure(g);
    g->dirs.assign(g->nd, {});
    uint64_t off = 0, leaf = 0;
    std::vector<uint64_t> start(g->nd), cnt(g->nd);
    uint64_t acc = 0;
    for (uint32_t d = 0; d < g->nd; ++d) {
        cnt[d] = h[1 + d];
        start[d] = acc;
        acc += cnt[d];
        uint32_t hh = 0;
        while (((uint64_t)kSeg << hh) < 2 * cnt[d]) ++hh;  // density <= 1/2
        g->dirs[d] = {off, (uint64_t)kSeg << hh, hh, leaf};
        off += (uint64_t)kSeg << hh;
        leaf += 1ull << hh;
    }
    g->total_slots = off;
    g->n_leaves = leaf;
    g->n_keys = n;
    GCK(cudaMalloc(&g->slots, off * sizeof(uint64_t)));
    GCK(cudaMalloc(&g->valid, off));
    GCK(cudaMalloc(&g->leaf_cnt, leaf * sizeof(uint32_t)));
    GCK(cudaMalloc(&g->leaf_delta, leaf * sizeof(int)));
    GCK(cudaMalloc(&g->leaf_ins, leaf * sizeof(uint32_t)));
    GCK(cudaMalloc(&g->leaf_dir, leaf * sizeof(uint32_t)));
    std::vector<uint64_t> o(g->nd), c(g->nd), l0(g->nd);
    std::vector<uint32_t> hh(g->nd);
    for (uint32_t d = 0; d < g->nd; ++d) { o[d] = g->dirs[d].off; c[d] = g->dirs[d].cap; hh[d] = g->dirs[d].h; l0[d] = g->dirs[d].leaf0; }
    GCK(cudaMemcpyAsync(g->d_off, o.data(), g->nd * 8, cudaMemcpyHostToDevice, g->stream));
    GCK(cudaMemcpyAsync(g->d_cap, c.data(), g->nd * 8, cudaMemcpyHostToDevice, g->stream));
    GCK(cudaMemcpyAsync(g->d_h, hh.data(), g->nd * 4, cudaMemcpyHostToDevice, g->stream));
    GCK(cudaMemcpyAsync(g->d_leaf0, l0.data(), g->nd * 8, cudaMemcpyHostToDevice, g->stream));
    uint64_t *d_start = nullptr, *d_cnt = nullptr;
    cgb_status s;
    if ((s = galloc(g, d_start, g->nd)) != CGB_OK) return s;
    if ((s = galloc(g, d_cnt, g->nd)) != CGB_OK) return s;
    GCK(cudaMemcpyAsync(d_start, start.data(), g->nd * 8, cudaMemcpyHostToDevice, g->stream));
    GCK(cudaMemcpyAsync(d_cnt, cnt.data(), g->nd * 8, cudaMemcpyHostToDevice, g->stream));
    DirTab dt{g->d_off, g->d_cap, g->d_h, g->d_leaf0};
    k_gp_spread<<<grid_of(off), 256, 0, g->stream>>>(keys, n, d_start, d_cnt, dt, g->nd, g->slots, g->valid, off);
    k_gp_leafcount<<<grid_of(leaf * 32), 256, 0, g->stream>>>(g->valid, leaf, g->leaf_cnt);
    k_gp_leafdir<<<grid_of(leaf), 256, 0, g->stream>>>(g->leaf_dir, g->d_leaf0, g->nd, leaf);
    GCK(cudaGetLastError());
    GCK(cudaStreamSynchronize(g->stream));
    free_bufs(g);
    return CGB_OK;
}

// Sorted unique copy of keys (device) into *out (allocated in bufs).
cgb_status sort_unique(cgb_gpma* g, const uint64_t* keys, uint64_t n, uint64_t*& out, uint64_t& m) {
    uint64_t *a = nullptr, *b = nullptr;
    cgb_status s;
    if ((s = galloc(g, a, n)) != CGB_OK) return s;
    if ((s = galloc(g, b, n)) != CGB_OK) return s;
    size_t bytes = 0;
    GCK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys, a, n, 0, 64, g->stream));
    if ((s = gtemp(g, bytes)) != CGB_OK) return s;
    GCK(cub::DeviceRadixSort::SortKeys(g->temp, bytes, keys, a, n, 0, 64, g->stream));
    unsigned long long* d_m = g->d_scal + 0;
    bytes = 0;
    GCK(cub::DeviceSelect::Unique(nullptr, bytes, a, b, d_m, n, g->stream));
    if ((s = gtemp(g, bytes)) != CGB_OK) return s;
    GCK(cub::DeviceSelect::Unique(g->temp, bytes, a, b, d_m, n, g->stream));
    unsigned long long hm = 0;
    GCK(cudaMemcpyAsync(&hm, d_m, 8, cudaMemcpyDeviceToHost, g->stream));
    GCK(cudaStreamSynchronize(g->stream));
    out = b;
    m = hm;
    return CGB_OK;
}

}  // namespace

extern "C" {

cgb_status cgb_gpma_create(int device, uint32_t num_dirs, cgb_gpma** out) {
    if (!out || num_dirs == 0 || num_dirs > CGB_MAX_DIR) return CGB_ERR_ARG;
    auto* g = new cgb_gpma();
    *out = g;
    g->device = device;
    g->nd = num_dirs;
    GCK(cudaSetDevice(device));
    GCK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    GCK(cudaMalloc(&g->d_off, num_dirs * 8));
    GCK(cudaMalloc(&g->d_cap, num_dirs * 8));
    GCK(cudaMalloc(&g->d_h, num_dirs * 4));
    GCK(cudaMalloc(&g->d_leaf0, num_dirs * 8));
    GCK(cudaMalloc(&g->d_scal, (3 + CGB_MAX_DIR) * sizeof(unsigned long long)));
    GCK(cudaEventCreate(&g->e0));
    GCK(cudaEventCreate(&g->e1));
    uint64_t none = 0;
    return rebuild(g, &none, 0);
}

void cgb_gpma_destroy(cgb_gpma* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    free_structure(g);
    free_bufs(g);
    for (void* p : {(void*)g->d_off, (void*)g->d_cap, (void*)g->d_h, (void*)g->d_leaf0, (void*)g->d_scal, g->temp})
        if (p) cudaFree(p);
    if (g->e0) cudaEventDestroy(g->e0);
    if (g->e1) cudaEventDestroy(g->e1);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

const char* cgb_gpma_last_error(const cgb_gpma* g) { return g ? g->err.c_str() : "null handle"; }

cgb_status cgb_gpma_bulk_load(cgb_gpma* g, const uint64_t* keys_device, uint64_t n) {
    if (!g || (n && !keys_device)) return CGB_ERR_ARG;
    GCK(cudaSetDevice(g->device));
    uint64_t* u = nullptr;
    uint64_t m = 0;
    cgb_status s;
    if (n) {
        if ((s = sort_unique(g, keys_device, n, u, m)) != CGB_OK) return s;
    }
    const uint64_t none = 0;
    s = rebuild(g, n ? u : &none, m);
    return s;
}

cgb_status cgb_gpma_batch_update(cgb_gpma* g, const uint64_t* ins_device, uint64_t n_ins,
                                 const uint64_t* del_device, uint64_t n_del) {
    if (!g || (n_ins && !ins_device) || (n_del && !del_device)) return CGB_ERR_ARG;
    // bounded before the sum below, which must not wrap (2^36 keys = 512 GiB, beyond any HBM)
    if (n_ins > (1ull << 36) || n_del > (1ull << 36)) return gfail(g, CGB_ERR_LIMIT, "edit batch too large");
    GCK(cudaSetDevice(g->device));
    for (auto& x : g->stats) x = 0;
    const uint64_t n = n_ins + n_del;
    if (n == 0) return CGB_OK;
    GCK(cudaEventRecord(g->e0, g->stream));
    cgb_status s;
    // 1. edits sorted by key with their op (0 insert, 1 delete)
    uint64_t *k_in = nullptr, *k_out = nullptr;
    uint8_t *o_in = nullptr, *o_out = nullptr;
    if ((s = galloc(g, k_in, n)) != CGB_OK) return s;
    if ((s = galloc(g, k_out, n)) != CGB_OK) return s;
    if ((s = galloc(g, o_in, n)) != CGB_OK) return s;
    if ((s = galloc(g, o_out, n)) != CGB_OK) return s;
    if (n_ins) GCK(cudaMemcpyAsync(k_in, ins_device, n_ins * 8, cudaMemcpyDeviceToDevice, g->stream));
    if (n_del) GCK(cudaMemcpyAsync(k_in + n_ins, del_device, n_del * 8, cudaMemcpyDeviceToDevice, g->stream));
    GCK(cudaMemsetAsync(o_in, 0, n_ins, g->stream));
    GCK(cudaMemsetAsync(o_in + n_ins, 1, n_del, g->stream));
    size_t bytes = 0;
    GCK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, k_in, k_out, o_in, o_out, n, 0, 64, g->stream));
    if ((s = gtemp(g, bytes)) != CGB_OK) return s;
    GCK(cub::DeviceRadixSort::SortPairs(g->temp, bytes, k_in, k_out, o_in, o_out, n, 0, 64, g->stream));
    // 2. effects: deletes in place, inserts queued per leaf
    uint64_t *ins_key = nullptr, *ins_leaf = nullptr;
    if ((s = galloc(g, ins_key, n)) != CGB_OK) return s;
    if ((s = galloc(g, ins_leaf, n)) != CGB_OK) return s;
    GCK(cudaMemsetAsync(g->d_scal, 0, 3 * sizeof(unsigned long long), g->stream));
    GCK(cudaMemsetAsync(g->leaf_delta, 0, g->n_leaves * sizeof(int), g->stream));
    GCK(cudaMemsetAsync(g->leaf_ins, 0, g->n_leaves * sizeof(uint32_t), g->stream));
    DirTab dt{g->d_off, g->d_cap, g->d_h, g->d_leaf0};
    unsigned int* d_flags = (unsigned int*)(g->d_scal + 2);  // [0] resize, [1] error
    k_gp_effect<<<grid_of(n), 256, 0, g->stream>>>(k_out, o_out, n, g->slots, g->valid, dt, g->nd, ins_key, ins_leaf,
                                                   g->d_scal + 0, g->leaf_delta, g->leaf_ins, d_flags + 1);
    // 3. windows
    uint64_t *newc = nullptr, *P = nullptr, *win = nullptr;
    if ((s = galloc(g, newc, g->n_leaves)) != CGB_OK) return s;
    if ((s = galloc(g, P, g->n_leaves)) != CGB_OK) return s;
    if ((s = galloc(g, win, n)) != CGB_OK) return s;
    k_gp_newcount<<<grid_of(g->n_leaves), 256, 0, g->stream>>>(g->leaf_cnt, g->leaf_delta, g->n_leaves, newc);
    bytes = 0;
    GCK(cub::DeviceScan::InclusiveSum(nullptr, bytes, newc, P, g->n_leaves, g->stream));
    if ((s = gtemp(g, bytes)) != CGB_OK) return s;
    GCK(cub::DeviceScan::InclusiveSum(g->temp, bytes, newc, P, g->n_leaves, g->stream));
    k_gp_window<<<grid_of(g->n_leaves), 256, 0, g->stream>>>(g->leaf_ins, P, g->leaf_dir, dt, g->n_leaves, win,
                                                             g->d_scal + 1, d_flags);
    unsigned long long h3[3];
    GCK(cudaMemcpyAsync(h3, g->d_scal, sizeof(h3), cudaMemcpyDeviceToHost, g->stream));
    GCK(cudaStreamSynchronize(g->stream));
    const uint64_t nins = h3[0], nwin_all = h3[1];
    const unsigned int resize = (unsigned int)(h3[2] & 0xffffffffull), kerr = (unsigned int)(h3[2] >> 32);
    if (kerr) return gfail(g, CGB_ERR_ARG, "key direction out of range (>= %u)", g->nd);
    if (resize) {
        // 4. a root is over its bound: rebuild from the valid keys plus the inserts
        uint64_t *all = nullptr;
        if ((s = galloc(g, all, g->total_slots + nins)) != CGB_OK) return s;
        uint8_t* flags = nullptr;
        if ((s = galloc(g, flags, g->total_slots)) != CGB_OK) return s;
        k_gp_valid_flags<<<grid_of(g->total_slots), 256, 0, g->stream>>>(g->valid, g->total_slots, flags);
        bytes = 0;
        GCK(cub::DeviceSelect::Flagged(nullptr, bytes, g->slots, flags, all, g->d_scal + 1, g->total_slots, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceSelect::Flagged(g->temp, bytes, g->slots, flags, all, g->d_scal + 1, g->total_slots,
                                       g->stream));
        unsigned long long nv = 0;
        GCK(cudaMemcpyAsync(&nv, g->d_scal + 1, 8, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaStreamSynchronize(g->stream));
        if (nins) GCK(cudaMemcpyAsync(all + nv, ins_key, nins * 8, cudaMemcpyDeviceToDevice, g->stream));
        uint64_t* u = nullptr;
        uint64_t m = 0;
        if ((s = sort_unique(g, all, nv + nins, u, m)) != CGB_OK) return s;
        g->stats[3] = 1;
        s = rebuild(g, u, m);
        GCK(cudaEventRecord(g->e1, g->stream));
        GCK(cudaEventSynchronize(g->e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, g->e0, g->e1);
        g->stats[0] = g->total_slots;
        g->stats[4] = (uint64_t)(ms * 1000.0f);
        g->stats[5] = g->n_keys;
        return s;
    }
    uint64_t nwin = 0;
    uint64_t *wsorted = nullptr, *wmax = nullptr, *wend = nullptr;
    if (nwin_all) {
        if ((s = galloc(g, wsorted, nwin_all)) != CGB_OK) return s;
        if ((s = galloc(g, wend, nwin_all)) != CGB_OK) return s;
        if ((s = galloc(g, wmax, nwin_all)) != CGB_OK) return s;
        bytes = 0;
        GCK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, win, wsorted, nwin_all, 0, 64, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceRadixSort::SortKeys(g->temp, bytes, win, wsorted, nwin_all, 0, 64, g->stream));
        k_gp_end<<<grid_of(nwin_all), 256, 0, g->stream>>>(wsorted, nwin_all, wend);
        bytes = 0;
        GCK(cub::DeviceScan::InclusiveScan(nullptr, bytes, wend, wmax, MaxOp(), nwin_all, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceScan::InclusiveScan(g->temp, bytes, wend, wmax, MaxOp(), nwin_all, g->stream));
        uint8_t* flag = nullptr;
        if ((s = galloc(g, flag, nwin_all)) != CGB_OK) return s;
        k_gp_maximal<<<grid_of(nwin_all), 256, 0, g->stream>>>(wsorted, wmax, nwin_all, flag);
        bytes = 0;
        GCK(cub::DeviceSelect::Flagged(nullptr, bytes, wsorted, flag, win, g->d_scal + 1, nwin_all, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceSelect::Flagged(g->temp, bytes, wsorted, flag, win, g->d_scal + 1, nwin_all, g->stream));
        unsigned long long hw = 0;
        GCK(cudaMemcpyAsync(&hw, g->d_scal + 1, 8, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaStreamSynchronize(g->stream));
        nwin = hw;
    }
    uint64_t rewritten = 0;
    if (nwin) {
        // 5. rewrite the windows: gather, sort, spread
        uint64_t *wcount = nullptr, *wpred = nullptr, *woff = nullptr, *wfill = nullptr;
        if ((s = galloc(g, wcount, nwin)) != CGB_OK) return s;
        if ((s = galloc(g, wpred, nwin)) != CGB_OK) return s;
        if ((s = galloc(g, woff, nwin + 1)) != CGB_OK) return s;
        if ((s = galloc(g, wfill, nwin)) != CGB_OK) return s;
        k_gp_wininfo<<<grid_of(nwin), 256, 0, g->stream>>>(win, nwin, P, g->slots, wcount, wpred);
        bytes = 0;
        GCK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, wcount, woff, nwin + 0, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceScan::ExclusiveSum(g->temp, bytes, wcount, woff, nwin, g->stream));
        unsigned long long tail[2];
        GCK(cudaMemcpyAsync(&tail[0], woff + nwin - 1, 8, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaMemcpyAsync(&tail[1], wcount + nwin - 1, 8, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaStreamSynchronize(g->stream));
        const uint64_t total = tail[0] + tail[1];
        uint64_t *tmp = nullptr, *srt = nullptr;
        if ((s = galloc(g, tmp, total)) != CGB_OK) return s;
        if ((s = galloc(g, srt, total)) != CGB_OK) return s;
        GCK(cudaMemcpyAsync(woff + nwin, &total, 8, cudaMemcpyHostToDevice, g->stream));
        unsigned int* d_bad = d_flags + 1;  // cleared at the start of the batch
        k_gp_gather<<<(unsigned)std::min<uint64_t>(nwin, 148ull * 8), 256, 0, g->stream>>>(
            win, nwin, woff, wcount, g->slots, g->valid, tmp, wfill, d_bad);
        if (nins)
            k_gp_place_ins<<<grid_of(nins), 256, 0, g->stream>>>(ins_key, ins_leaf, nins, win, nwin, woff, wcount,
                                                                 (unsigned long long*)wfill, tmp, d_bad);
        unsigned int hb = 0;
        GCK(cudaMemcpyAsync(&hb, d_bad, 4, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaStreamSynchronize(g->stream));
        if (hb) return gfail(g, CGB_ERR_STATE, "internal: window bookkeeping inconsistent (no key written out of place)");
        bytes = 0;
        GCK(cub::DeviceSegmentedSort::SortKeys(nullptr, bytes, tmp, srt, total, nwin, woff, woff + 1, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceSegmentedSort::SortKeys(g->temp, bytes, tmp, srt, total, nwin, woff, woff + 1, g->stream));
        k_gp_scatter<<<(unsigned)std::min<uint64_t>(nwin, 148ull * 8), 256, 0, g->stream>>>(win, nwin, woff, wcount,
                                                                                             wpred, srt, g->slots,
                                                                                             g->valid);
        rewritten = total;
    }
    k_gp_leafcount<<<grid_of(g->n_leaves * 32), 256, 0, g->stream>>>(g->valid, g->n_leaves, g->leaf_cnt);
    GCK(cudaGetLastError());
    GCK(cudaEventRecord(g->e1, g->stream));
    GCK(cudaEventSynchronize(g->e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, g->e0, g->e1);
    // key count: sum of leaf counts
    {
        uint64_t* tot = nullptr;
        if ((s = galloc(g, tot, 1)) != CGB_OK) return s;
        bytes = 0;
        GCK(cub::DeviceReduce::Sum(nullptr, bytes, g->leaf_cnt, tot, g->n_leaves, g->stream));
        if ((s = gtemp(g, bytes)) != CGB_OK) return s;
        GCK(cub::DeviceReduce::Sum(g->temp, bytes, g->leaf_cnt, tot, g->n_leaves, g->stream));
        uint64_t ht = 0;
        GCK(cudaMemcpyAsync(&ht, tot, 8, cudaMemcpyDeviceToHost, g->stream));
        GCK(cudaStreamSynchronize(g->stream));
        g->n_keys = ht;
    }
    g->stats[0] = g->total_slots;
    g->stats[1] = nwin;
    g->stats[2] = rewritten;
    g->stats[3] = 0;
    g->stats[4] = (uint64_t)(ms * 1000.0f);
    g->stats[5] = g->n_keys;
    free_bufs(g);
    return CGB_OK;
}

cgb_status cgb_gpma_extract(cgb_gpma* g, uint32_t dir, uint64_t* out_device, uint64_t cap, uint64_t* n_out) {
    if (!g || !n_out || dir >= g->nd) return CGB_ERR_ARG;
    GCK(cudaSetDevice(g->device));
    const GpmaDir& D = g->dirs[dir];
    cgb_status s;
    uint64_t* tmp = nullptr;
    if ((s = galloc(g, tmp, D.cap)) != CGB_OK) return s;
    size_t bytes = 0;
    GCK(cub::DeviceSelect::Flagged(nullptr, bytes, g->slots + D.off, g->valid + D.off, tmp, g->d_scal + 1, D.cap,
                                   g->stream));
    if ((s = gtemp(g, bytes)) != CGB_OK) return s;
    GCK(cub::DeviceSelect::Flagged(g->temp, bytes, g->slots + D.off, g->valid + D.off, tmp, g->d_scal + 1, D.cap,
                                   g->stream));
    unsigned long long m = 0;
    GCK(cudaMemcpyAsync(&m, g->d_scal + 1, 8, cudaMemcpyDeviceToHost, g->stream));
    GCK(cudaStreamSynchronize(g->stream));
    *n_out = m;
    if (out_device) {
        if (cap < m) { free_bufs(g); return gfail(g, CGB_ERR_ARG, "buffer holds %llu of %llu keys", (unsigned long long)cap, m); }
        if (m) k_gp_strip_dir<<<grid_of(m), 256, 0, g->stream>>>(tmp, m, out_device);
        GCK(cudaStreamSynchronize(g->stream));
    }
    free_bufs(g);
    return CGB_OK;
}

cgb_status cgb_gpma_stats(const cgb_gpma* g, uint64_t* out6) {
    if (!g || !out6) return CGB_ERR_ARG;
    for (int i = 0; i < 6; ++i) out6[i] = g->stats[i];
    return CGB_OK;
}

}  // extern "C"
