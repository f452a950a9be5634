// B200 engine for the per-batch GPU path of continuous subgraph matching.
//
// Device data layout (HBM):
//   pool   u32 words holding every sorted neighbour run; runs start on 16-byte
//          boundaries; allocation is a bump pointer, updated runs are written
//          out of place and dead space is reclaimed by compaction.
//   rec    uint4 per (direction d, compressed vertex u), row-major [d][dvcap]:
//          x = run offset (words), y = run length, z = delta offset, w = delta length.
//          One 16-byte load resolves both the old list and this batch's delta
//          list of (d, u) (the two halves the reference keeps in index_gpu and
//          update_index, graph_gpu.h:41-49).
//   dval   this batch's delta values, sorted by (d, u, v), not deduplicated
//          (calig_helper_gamma.cu:569-573).
//
// Per batch (calig_helper_gamma.cu:485-597 + graph_gpu.cu:1261-1480):
//   1. edits = previous delta (deferred merge-back) + ins (add) + del (remove),
//      packed to (d,u,v,op) and radix-sorted; one warp per touched (d,u) writes
//      (old run U adds) \ removes.  One pass over each touched run per batch,
//      where the reference makes three (merge ins, remove del, merge delta).
//   2. delta keys packed + sorted -> dval and rec.z/.w for touched (d,u).
//   3. persistent warp DFS seeded from the delta edges of every query edge
//      (all query edges in one launch; the edge index ei travels with the seed).
//   4. rec.z/.w of touched (d,u) cleared; this batch's delta becomes the
//      pending merge-back of the next batch.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "cgbdsm.h"
#include "query.h"

using cgb::EdgePlan;
using cgb::kMaxBN;
using cgb::kMaxDir;
using cgb::kMaxQE;
using cgb::kMaxQV;

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kDfsWarps = 8;  // warps per DFS block
constexpr uint32_t kTaskCap = 1u << 20;  // stolen-range ring capacity (64 MiB), a power of two
constexpr uint32_t kTaskSlack = 1u << 13; // tickets kept between the ring's tail and head
constexpr uint64_t kMaxBatchKeys = 1ull << 36;  // per key array of one batch: 512 GiB, beyond any HBM

// Plans belong to a handle (several handles may share a process and a
// device): they live in the handle's device memory, and the DFS copies them
// to shared memory as 32-bit words.
static_assert(sizeof(EdgePlan) % 4 == 0, "EdgePlan must be a whole number of words");

// ---------------------------------------------------------------------------
// key packing
// ---------------------------------------------------------------------------
struct PackInfo {
    uint32_t B;      // bits per vertex id
    uint32_t nd;     // directions
    uint32_t dv;     // compressed vertex count
    uint32_t pad_ok; // an all-ones key is padding (skipped), not an invalid key
};

__device__ __forceinline__ bool decode_ext(uint64_t k, const PackInfo& pi, uint32_t& d, uint32_t& u,
                                           uint32_t& v) {
    d = (uint32_t)(k >> 59);
    u = (uint32_t)((k >> 32) & 0x07FFFFFFu);
    v = (uint32_t)k;
    return d < pi.nd && u < pi.dv && v < pi.dv;
}

__device__ __forceinline__ uint64_t pack_duv(uint32_t d, uint32_t u, uint32_t v, uint32_t B) {
    return ((uint64_t)d << (2 * B)) | ((uint64_t)u << B) | (uint64_t)v;
}

// Edits: ((d,u,v) << 1) | op, op 0 = add, 1 = remove.  Keys whose direction
// or vertex ids are out of range raise error bit 1 and become the all-ones
// marker, which sorts last and is skipped by the merge.
// Added keys with u == v (a self-loop in the data graph) set the sticky
// self_seen flag: until one appears no vertex lies in its own lists, which
// lets the matcher skip those exclusion tests.
__global__ void k_pack_edits(const uint64_t* __restrict__ in, uint64_t n, uint32_t op, PackInfo pi,
                             uint64_t* __restrict__ out, unsigned int* err, unsigned int* self_seen) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint32_t d, u, v;
        if (pi.pad_ok && in[i] == ~0ull) {
            out[i] = ~0ull;
        } else if (decode_ext(in[i], pi, d, u, v)) {
            if (op == 0 && u == v) atomicOr(self_seen, 1u);
            out[i] = (pack_duv(d, u, v, pi.B) << 1) | op;
        } else {
            out[i] = ~0ull;
            atomicOr(err, 1u);
        }
    }
}

__global__ void k_pack_delta(const uint64_t* __restrict__ in, uint64_t n, PackInfo pi,
                             uint64_t* __restrict__ out, unsigned int* err, unsigned int* self_seen) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint32_t d, u, v;
        if (decode_ext(in[i], pi, d, u, v)) {
            if (u == v) atomicOr(self_seen, 1u);
            out[i] = pack_duv(d, u, v, pi.B);
        } else {
            out[i] = ~0ull;
            atomicOr(err, 2u);
        }
    }
}

// du = (d << B) | u of a sorted packed array (shift = B or B+1 for edits);
// invalid (all-ones) entries map to 0xffffffff.
__global__ void k_extract_du(const uint64_t* __restrict__ in, uint64_t n, uint32_t shift,
                             uint32_t* __restrict__ du) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint64_t k = in[i];
        du[i] = (k == ~0ull) ? 0xffffffffu : (uint32_t)(k >> shift);
    }
}

// ---------------------------------------------------------------------------
// fused edit merge of every touched (d, u): warp per run below kBigRun merged
// entries, CTA per longer (hub) run
// ---------------------------------------------------------------------------
constexpr uint32_t kTinyRun = 32;        // merged entries up to which one lane merges the run
constexpr uint32_t kBigRun = 4096;       // merged entries (old run + edits) from which a CTA merges the run
constexpr uint32_t kMergeWarps = 8;      // warps of a CTA merge
constexpr uint32_t kSegWindows = 8;      // 32-entry windows a CTA warp merges per round
constexpr uint32_t kNoVal = 0xffffffffu; // window padding: above every vertex id (< 2^27)

struct MergeArgs {
    uint4* rec;
    uint32_t dvcap;
    uint32_t* pool;
    unsigned long long* pool_top;
    unsigned long long pool_cap;
    long long* live_words;       // sum of round4(len) over runs
    const uint64_t* edits;       // sorted ((d,u,v)<<1|op)
    const uint32_t* run_du;
    const uint32_t* run_len;
    const uint32_t* run_off;
    const int* num_runs;
    uint32_t* small_runs;        // run ids merged by a warp / by a CTA / by a lane (k_merge_classify)
    uint32_t* big_runs;
    uint32_t* tiny_runs;
    unsigned int* list_ctr;      // [0] small, [1] big, [2] tiny
    uint32_t B;
    unsigned int* err;
    unsigned long long* stats;   // [5] merge bytes (edits 8 B, old run 4 B/word, new run 4 B/word, record 32 B), [6] runs
    // run bit sets: a run that reaches rb_min_len without a bit set claims one
    // (slot table [d][dvcap], slot owners, claim counter, new-slot list)
    uint32_t* rb_slot;           // nullptr: not maintained by this merge
    uint32_t* rb_sel;
    unsigned int* rb_ctr;        // [0] slots claimed, [1] new slots this merge
    uint32_t* rb_new;
    uint32_t rb_cap;
    uint32_t rb_min_len;
};

__device__ __forceinline__ uint32_t round4(uint32_t x) { return (x + 3u) & ~3u; }

// Number of entries of the ascending warp-held window w (lane k holds w[k],
// padded with kNoVal) that are < x (or <= x when le): binary lifting over
// shuffles, six steps.
__device__ __forceinline__ uint32_t win_rank(uint32_t w, uint32_t x, bool le) {
    uint32_t lo = 0;
#pragma unroll
    for (uint32_t step = 16; step >= 1; step >>= 1) {
        const uint32_t v = __shfl_sync(kFull, w, lo + step - 1);
        if (le ? v <= x : v < x) lo += step;
    }
    const uint32_t v = __shfl_sync(kFull, w, lo);
    return lo + ((le ? v <= x : v < x) ? 1u : 0u);
}

// Merge-path split of diagonal k of X (old run) and Y (edits): the number of
// X entries among the first k merged entries, X winning ties (so for equal
// values the old entry precedes an add, and an add precedes a remove).
__device__ __forceinline__ uint32_t merge_split(const uint32_t* X, uint32_t xl, const uint64_t* Y,
                                                uint32_t yl, uint32_t k, uint64_t vmask) {
    uint32_t lo = k > yl ? k - yl : 0;
    uint32_t hi = k < xl ? k : xl;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t yv = (uint32_t)((__ldg(Y + (k - 1 - mid)) >> 1) & vmask);
        if (__ldg(X + mid) <= yv) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// One window step of a warp merge: the next nout (<= 32) entries of the merge
// of X[i..) and Y[j..), from coalesced 32-entry windows of both.  Lane p
// gets entry p in *val and whether it is emitted: the last entry of its value
// group and not a remove, i.e. the set (X U adds) \ removes.  Advances i, j.
// sbuf: 32 words of this warp's shared memory.
__device__ __forceinline__ bool merge_window(const uint32_t* __restrict__ X, uint32_t xl,
                                             const uint64_t* __restrict__ Y, uint32_t yl, uint64_t vmask,
                                             uint32_t& i, uint32_t& j, uint32_t nout, uint32_t lane,
                                             uint32_t* sbuf, uint32_t& val) {
    const uint32_t xv = (i + lane < xl) ? __ldg(X + i + lane) : kNoVal;
    uint32_t yv = kNoVal, yop = 0;
    if (j + lane < yl) {
        const uint64_t e = __ldg(Y + j + lane);
        yv = (uint32_t)((e >> 1) & vmask);
        yop = (uint32_t)(e & 1ull);
    }
    // merged position: an old entry follows the edits strictly below it, an
    // edit follows the old entries up to and including its value
    const uint32_t px = lane + win_rank(yv, xv, false);
    const uint32_t py = lane + win_rank(xv, yv, true);
    if (px < nout) sbuf[px] = xv;
    if (py < nout) sbuf[py] = yv | (yop << 31);
    const uint32_t cx = __popc(__ballot_sync(kFull, px < nout));
    const uint32_t cy = nout - cx;
    // the entry after the window's last: first unconsumed entry of X or Y
    uint32_t nx = __shfl_sync(kFull, xv, cx & 31), ny = __shfl_sync(kFull, yv, cy & 31);
    if (cx == 32) nx = (i + 32 < xl) ? __ldg(X + i + 32) : kNoVal;
    if (cy == 32) ny = (j + 32 < yl) ? (uint32_t)((__ldg(Y + j + 32) >> 1) & vmask) : kNoVal;
    __syncwarp();
    bool emit = false;
    if (lane < nout) {
        const uint32_t e = sbuf[lane];
        val = e & 0x7fffffffu;
        const uint32_t nv = (lane + 1 < nout) ? (sbuf[lane + 1] & 0x7fffffffu) : min(nx, ny);
        emit = nv != val && !(e >> 31);
    }
    __syncwarp();
    i += cx;
    j += cy;
    return emit;
}

// Splits the runs into warp-merged and CTA-merged lists by merged length.
__global__ void k_merge_classify(MergeArgs a) {
    const int n = *a.num_runs;
    const uint32_t vmask = (1u << a.B) - 1u;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t du = a.run_du[r];
        if (du == 0xffffffffu) continue;  // invalid keys
        const uint32_t xl = a.rec[(size_t)(du >> a.B) * a.dvcap + (du & vmask)].y;
        const uint32_t total = xl + a.run_len[r];
        if (total >= kBigRun) a.big_runs[atomicAdd(a.list_ctr + 1, 1u)] = (uint32_t)r;
        else if (total > kTinyRun) a.small_runs[atomicAdd(a.list_ctr + 0, 1u)] = (uint32_t)r;
        else a.tiny_runs[atomicAdd(a.list_ctr + 2, 1u)] = (uint32_t)r;
    }
}

// Pool space for a merged run of at most `bound` entries (~0 when exhausted).
__device__ __forceinline__ unsigned long long pool_alloc(const MergeArgs& a, uint32_t bound) {
    unsigned long long off = atomicAdd(a.pool_top, (unsigned long long)round4(bound));
    if (off + round4(bound) > a.pool_cap) {
        atomicOr(a.err, 4u);
        off = ~0ull;
    }
    return off;
}

// Accounting of the runs one warp merged, added to the launch's counters
// once per warp (per-run atomics on these few words serialised the merge).
struct MergeAcc {
    unsigned long long bytes = 0, runs = 0;
    long long live = 0;
    __device__ __forceinline__ void add(uint32_t xl, uint32_t yl, uint32_t outn) {
        bytes += 8ull * yl + 4ull * xl + 4ull * outn + 32ull;
        runs += 1;
        live += (long long)round4(outn) - (long long)round4(xl);
    }
    // every lane of the warp calls it; lane sums are combined
    __device__ __forceinline__ void flush(const MergeArgs& a, uint32_t lane) {
        for (int o = 16; o > 0; o >>= 1) {
            bytes += __shfl_xor_sync(kFull, bytes, o);
            runs += __shfl_xor_sync(kFull, runs, o);
            live += __shfl_xor_sync(kFull, live, o);
        }
        if (lane == 0) {
            if (bytes) atomicAdd(a.stats + 5, bytes);
            if (runs) atomicAdd(a.stats + 6, runs);
            if (live) atomicAdd((unsigned long long*)a.live_words, (unsigned long long)live);
        }
    }
};

// Record update after a run was merged (one thread); a run that reached the
// bit-set length without a bit set claims one.  The unused tail of the
// allocation is dead space until compaction.
__device__ __forceinline__ void merge_record(const MergeArgs& a, uint4* recp, uint4 old, unsigned long long off,
                                             uint32_t outn, uint32_t d, uint32_t u) {
    *recp = make_uint4((uint32_t)off, outn, old.z, old.w);
    if (a.rb_slot && outn >= a.rb_min_len) {
        uint32_t* sp = a.rb_slot + (size_t)d * a.dvcap + u;
        if (*sp == kNoVal) {
            const unsigned int c = atomicAdd(a.rb_ctr, 1u);
            if (c < a.rb_cap) {
                *sp = c;
                a.rb_sel[c] = d << 27 | u;
                a.rb_new[atomicAdd(a.rb_ctr + 1, 1u)] = c;
            }
        }
    }
}

// Lane per run for runs of at most kTinyRun merged entries (most runs of a
// batch touch a handful of entries): a serial merge per lane, one pool
// allocation per warp step (a warp prefix over the lanes' bounds).
__global__ void k_merge_tiny(MergeArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t n = a.list_ctr[2];
    const uint32_t vmask = (1u << a.B) - 1u;
    const uint64_t emask = (1ull << a.B) - 1ull;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    MergeAcc acc;
    for (uint32_t base = gw * 32; base < n; base += nw * 32) {
        const uint32_t q = base + lane;
        const bool on = q < n;
        uint32_t r = 0, d = 0, u = 0, yl = 0;
        uint4 old = make_uint4(0, 0, 0, 0);
        uint4* recp = nullptr;
        if (on) {
            r = a.tiny_runs[q];
            const uint32_t du = a.run_du[r];
            d = du >> a.B;
            u = du & vmask;
            yl = a.run_len[r];
            recp = a.rec + (size_t)d * a.dvcap + u;
            old = *recp;
        }
        const uint32_t bound = on ? round4(old.y + yl) : 0u;
        uint32_t pre = bound;  // inclusive prefix over the lanes
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, pre, o);
            if (lane >= (uint32_t)o) pre += v;
        }
        const uint32_t total = __shfl_sync(kFull, pre, 31);
        unsigned long long wbase = 0;
        if (lane == 0 && total) {
            wbase = atomicAdd(a.pool_top, (unsigned long long)total);
            if (wbase + total > a.pool_cap) {
                atomicOr(a.err, 4u);
                wbase = ~0ull;
            }
        }
        wbase = __shfl_sync(kFull, wbase, 0);
        if (!on || wbase == ~0ull) continue;  // pool exhausted: runs left unchanged, error raised
        const unsigned long long off = wbase + pre - bound;
        const uint32_t* X = a.pool + old.x;
        const uint64_t* Y = a.edits + a.run_off[r];
        uint32_t* C = a.pool + off;
        uint32_t i = 0, j = 0, outn = 0;
        while (i < old.y || j < yl) {
            const uint32_t xv = i < old.y ? X[i] : kNoVal;
            const uint32_t yv = j < yl ? (uint32_t)((Y[j] >> 1) & emask) : kNoVal;
            const uint32_t v = min(xv, yv);
            bool present = false;
            if (xv == v) { present = true; ++i; }
            // the value's edits in order (adds before removes): the last decides
            while (j < yl && (uint32_t)((Y[j] >> 1) & emask) == v) { present = (Y[j] & 1ull) == 0; ++j; }
            if (present) C[outn++] = v;
        }
        merge_record(a, recp, old, off, outn, d, u);
        acc.add(old.y, yl, outn);
    }
    acc.flush(a, lane);
}

// Warp per run: 32 merged entries per step from two coalesced windows.
__global__ void k_merge_runs(MergeArgs a) {
    __shared__ uint32_t s_win[8][32];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nruns = a.list_ctr[0];
    const uint64_t vmask = (1ull << a.B) - 1ull;
    uint32_t* sbuf = s_win[(threadIdx.x >> 5) & 7];
    MergeAcc acc;
    for (uint32_t q = gw; q < nruns; q += nw) {
        const uint32_t r = a.small_runs[q];
        const uint32_t du = a.run_du[r];
        const uint32_t d = du >> a.B, u = du & (uint32_t)vmask;
        const uint64_t* Y = a.edits + a.run_off[r];
        const uint32_t yl = a.run_len[r];
        uint4* recp = a.rec + (size_t)d * a.dvcap + u;
        const uint4 old = *recp;
        const uint32_t* X = a.pool + old.x;
        const uint32_t xl = old.y;
        unsigned long long off = 0;
        if (lane == 0) off = pool_alloc(a, xl + yl);
        off = __shfl_sync(kFull, off, 0);
        if (off == ~0ull) continue;  // pool exhausted: run left unchanged, error raised
        uint32_t* C = a.pool + off;
        const uint32_t total = xl + yl;
        uint32_t outn = 0, i = 0, j = 0;
        for (uint32_t done = 0; done < total; done += 32) {
            const uint32_t nout = min(32u, total - done);
            uint32_t val = 0;
            const bool emit = merge_window(X, xl, Y, yl, vmask, i, j, nout, lane, sbuf, val);
            const uint32_t bal = __ballot_sync(kFull, emit);
            if (emit) C[outn + __popc(bal & ((1u << lane) - 1u))] = val;
            outn += __popc(bal);
        }
        if (lane == 0) {
            merge_record(a, recp, old, off, outn, d, u);
            acc.add(xl, yl, outn);
        }
    }
    acc.flush(a, lane);
}

// CTA per long run: each round, warp w merges the 256 entries from diagonal
// k0 + 256 w (one merge-path split per warp and round), stages what it emits
// in shared memory, and the CTA writes the round's output contiguously.
__global__ void __launch_bounds__(kMergeWarps * 32) k_merge_big(MergeArgs a) {
    constexpr uint32_t kSeg = 32 * kSegWindows;
    __shared__ uint32_t s_win[kMergeWarps][32];
    __shared__ uint32_t s_out[kMergeWarps][kSeg];
    __shared__ uint32_t s_cnt[kMergeWarps];
    __shared__ unsigned long long s_off;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t nruns = a.list_ctr[1];
    const uint64_t vmask = (1ull << a.B) - 1ull;
    MergeAcc acc;
    for (uint32_t q = blockIdx.x; q < nruns; q += gridDim.x) {
        const uint32_t r = a.big_runs[q];
        const uint32_t du = a.run_du[r];
        const uint32_t d = du >> a.B, u = du & (uint32_t)vmask;
        const uint64_t* Y = a.edits + a.run_off[r];
        const uint32_t yl = a.run_len[r];
        uint4* recp = a.rec + (size_t)d * a.dvcap + u;
        const uint4 old = *recp;
        const uint32_t* X = a.pool + old.x;
        const uint32_t xl = old.y;
        const uint32_t total = xl + yl;
        if (threadIdx.x == 0) s_off = pool_alloc(a, total);
        __syncthreads();
        const unsigned long long off = s_off;
        if (off == ~0ull) { __syncthreads(); continue; }
        uint32_t* C = a.pool + off;
        uint32_t outn = 0;
        for (uint32_t k0 = 0; k0 < total; k0 += kMergeWarps * kSeg) {
            const uint32_t ks = k0 + w * kSeg;
            uint32_t cnt = 0;
            if (ks < total) {
                const uint32_t ke = min(ks + kSeg, total);
                uint32_t i = 0;
                if (lane == 0) i = merge_split(X, xl, Y, yl, ks, vmask);
                i = __shfl_sync(kFull, i, 0);
                uint32_t j = ks - i;
                for (uint32_t k = ks; k < ke; k += 32) {
                    const uint32_t nout = min(32u, ke - k);
                    uint32_t val = 0;
                    const bool emit = merge_window(X, xl, Y, yl, vmask, i, j, nout, lane, s_win[w], val);
                    const uint32_t bal = __ballot_sync(kFull, emit);
                    if (emit) s_out[w][cnt + __popc(bal & ((1u << lane) - 1u))] = val;
                    cnt += __popc(bal);
                }
            }
            if (lane == 0) s_cnt[w] = cnt;
            __syncthreads();
            uint32_t before = 0, all = 0;
            for (uint32_t t = 0; t < kMergeWarps; ++t) {
                before += t < w ? s_cnt[t] : 0u;
                all += s_cnt[t];
            }
            for (uint32_t t = lane; t < cnt; t += 32) C[outn + before + t] = s_out[w][t];
            outn += all;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            merge_record(a, recp, old, off, outn, d, u);
            acc.add(xl, yl, outn);
        }
        __syncthreads();
    }
    if (threadIdx.x < 32) acc.flush(a, lane);
}

// ---------------------------------------------------------------------------
// delta lists
// ---------------------------------------------------------------------------
__global__ void k_delta_values(const uint64_t* __restrict__ keys, uint64_t n, uint64_t vmask,
                               uint32_t* __restrict__ dval) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) dval[i] = (uint32_t)(keys[i] & vmask);
}

// du = (d << lb | label bits) << B | u (lb = 0: no label bits).
__global__ void k_delta_recs(uint4* rec, uint32_t dvcap, const uint32_t* run_du, const uint32_t* run_len,
                             const uint32_t* run_off, const int* num_runs, uint32_t B, int clear, uint32_t lb = 0) {
    const int n = *num_runs;
    const uint32_t umask = (1u << B) - 1u;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        uint32_t du = run_du[r];
        if (du == 0xffffffffu) continue;
        uint4* p = rec + (size_t)(du >> (B + lb)) * dvcap + (du & umask);
        uint4 v = *p;
        if (clear) { v.z = 0; v.w = 0; }
        else { v.z = run_off[r]; v.w = run_len[r]; }
        *p = v;
    }
}

// Seed ranges: delta entries of direction seed_dir(ei) form one contiguous
// range of the sorted packed delta array.
__global__ void k_seed_ranges(const uint64_t* __restrict__ dkeys, uint64_t n, uint32_t B, uint32_t qe,
                              const EdgePlan* __restrict__ plans, const uint8_t* qe_dirs /*[qe][2]*/,
                              const uint8_t* edge_ok, int have_ok, uint32_t* seed_lo, uint32_t* seed_pre) {
    __shared__ uint32_t cnt[kMaxQE];
    const uint32_t t = threadIdx.x;
    auto lower = [&](uint64_t key) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (dkeys[mid] < key) lo = mid + 1; else hi = mid;
        }
        return (uint32_t)lo;
    };
    if (t < qe) {
        uint32_t s = plans[t].seed_dir;
        uint32_t lo = lower((uint64_t)s << (2 * B));
        uint32_t hi = lower((uint64_t)(s + 1) << (2 * B));
        uint32_t d0 = qe_dirs[2 * t], d1 = qe_dirs[2 * t + 1];
        uint32_t c0 = lower((uint64_t)(d0 + 1) << (2 * B)) - lower((uint64_t)d0 << (2 * B));
        uint32_t c1 = lower((uint64_t)(d1 + 1) << (2 * B)) - lower((uint64_t)d1 << (2 * B));
        bool ok = have_ok ? (edge_ok[t] != 0) : (c0 > 0 && c1 > 0);
        seed_lo[t] = lo;
        cnt[t] = ok ? hi - lo : 0;
    }
    __syncthreads();
    if (t == 0) {
        uint32_t acc = 0;
        for (uint32_t e = 0; e < qe; ++e) { seed_pre[e] = acc; acc += cnt[e]; }
        seed_pre[qe] = acc;
    }
}

// ---------------------------------------------------------------------------
// run bit sets: every old run of at least kRunBitsMinLen entries is also kept
// as a bit set over the compressed ids, rebuilt each batch after the index
// update, so that a membership test in a long (hub) run, in the DFS probes
// and in the tail counts, is one load instead of a binary search
// ---------------------------------------------------------------------------
constexpr uint32_t kNoSlot = 0xffffffffu;
constexpr uint32_t kRunBitsMinLen = 128;        // $CGB_RUN_BITS_MIN_LEN overrides (tests use 1)
constexpr size_t kRunBitsBytes = 512ull << 20;  // runs beyond this budget are searched

// Full rebuild: the slot of every (direction, vertex) of the table (all
// dvcap rows) whose run is long enough, in claim order while slots last
// (ctr[0] counts claims), else kNoSlot; sel[slot] = dir << 27 | vertex.
// Afterwards each merge keeps the sets current (k_rb_fill_new, k_rb_edits).
__global__ void k_rb_select(const uint4* __restrict__ rec, uint32_t dvcap, uint32_t nd, uint32_t min_len,
                            uint32_t cap, uint32_t* slot, uint32_t* sel, unsigned int* ctr) {
    const size_t n = (size_t)nd * dvcap;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t sl = kNoSlot;
        if (rec[i].y >= min_len) {
            const unsigned int c = atomicAdd(ctr, 1u);
            if (c < cap) {
                sl = c;
                sel[c] = (uint32_t)(i / dvcap) << 27 | (uint32_t)(i % dvcap);
            }
        }
        slot[i] = sl;
    }
}

__global__ void k_rb_zero(uint32_t* bits, uint32_t words, uint32_t cap, const unsigned int* ctr) {
    const size_t n = (size_t)min(*ctr, cap) * words;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        bits[i] = 0;
}

// one warp per selected run: the bits of its words, set with atomicOr
// (lanes can share a word)
__global__ void k_rb_fill(const uint4* __restrict__ rec, uint32_t dvcap, const uint32_t* __restrict__ pool,
                          const uint32_t* __restrict__ sel, uint32_t cap, const unsigned int* ctr, uint32_t* bits,
                          uint32_t words) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nsel = min(*ctr, cap);
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nsel; c += nw) {
        const uint32_t du = sel[c];
        const uint4 r = rec[(size_t)(du >> 27) * dvcap + (du & ((1u << 27) - 1u))];
        uint32_t* b = bits + (size_t)c * words;
        for (uint32_t t = lane; t < r.y; t += 32) {
            const uint32_t v = __ldg(pool + r.x + t);
            atomicOr(b + (v >> 5), 1u << (v & 31));
        }
    }
}

// Slots claimed by runs that grew past the length threshold in this merge
// (ctr[1] of them, listed in fresh): zeroed, then filled from the merged run.
__global__ void k_rb_fill_new(const uint4* __restrict__ rec, uint32_t dvcap, const uint32_t* __restrict__ pool,
                              const uint32_t* __restrict__ sel, const uint32_t* __restrict__ fresh,
                              const unsigned int* ctr, uint32_t* bits, uint32_t words) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t n = ctr[1];
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n; q += nw) {
        const uint32_t c = fresh[q];
        const uint32_t du = sel[c];
        const uint4 r = rec[(size_t)(du >> 27) * dvcap + (du & ((1u << 27) - 1u))];
        uint32_t* b = bits + (size_t)c * words;
        for (uint32_t t = lane; t < words; t += 32) b[t] = 0;
        __syncwarp();
        for (uint32_t t = lane; t < r.y; t += 32) {
            const uint32_t v = __ldg(pool + r.x + t);
            atomicOr(b + (v >> 5), 1u << (v & 31));
        }
    }
}

// Applies a merge's sorted edits ((d,u,v) << 1 | op) to the bit sets of
// runs that have one: the last edit of each (d,u,v) decides, as in the merge
// (an add sets the bit, a remove clears it).
__global__ void k_rb_edits(const uint64_t* __restrict__ edits, uint64_t n, uint32_t B, uint32_t dvcap,
                           const uint32_t* __restrict__ slot, uint32_t* bits, uint32_t words) {
    const uint64_t vmask = (1ull << B) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = edits[i];
        if (e == ~0ull) continue;
        if (i + 1 < n && (edits[i + 1] >> 1) == (e >> 1)) continue;  // not the last edit of its value
        const uint64_t p = e >> 1;
        const uint32_t v = (uint32_t)(p & vmask), u = (uint32_t)((p >> B) & vmask), d = (uint32_t)(p >> (2 * B));
        const uint32_t sl = slot[(size_t)d * dvcap + u];
        if (sl == kNoSlot) continue;
        uint32_t* w = bits + (size_t)sl * words + (v >> 5);
        if (e & 1ull) atomicAnd(w, ~(1u << (v & 31)));
        else atomicOr(w, 1u << (v & 31));
    }
}

// Index symmetry: number of entries y in run (d, x) whose mirror entry (x in
// run (rev[d], y)) is missing.  Warp per run.
__global__ void k_asymmetry(const uint4* __restrict__ rec, uint32_t dvcap, uint32_t dv, uint32_t nd,
                            const uint32_t* __restrict__ pool, const uint8_t* __restrict__ rev,
                            unsigned long long* bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t total = (uint64_t)nd * dv;
    unsigned long long miss = 0;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total;
         i += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint32_t d = (uint32_t)(i / dv), x = (uint32_t)(i % dv);
        const uint4 r = rec[(size_t)d * dvcap + x];
        const uint32_t rd = rev[d];
        for (uint32_t t = lane; t < r.y; t += 32) {
            const uint32_t y = pool[r.x + t];
            bool ok = false;
            if (y < dv && rd < nd) {
                const uint4 m = rec[(size_t)rd * dvcap + y];
                uint32_t lo = 0, hi = m.y;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (pool[m.x + mid] < x) lo = mid + 1; else hi = mid;
                }
                ok = lo < m.y && pool[m.x + lo] == x;
            }
            miss += ok ? 0 : 1;
        }
    }
    for (int o = 16; o > 0; o >>= 1) miss += __shfl_xor_sync(kFull, miss, o);
    if (lane == 0 && miss) atomicAdd(bad, miss);
}

// ---------------------------------------------------------------------------
// persistent warp DFS (count only)
// ---------------------------------------------------------------------------
struct DfsArgs {
    const uint4* rec;
    uint32_t dvcap;
    const uint32_t* pool;
    const uint32_t* dval;
    const uint64_t* dkeys;
    uint32_t B;
    uint32_t qe;
    const uint32_t* seed_lo;
    const uint32_t* seed_pre;
    unsigned long long* counts;  // [qe]
    unsigned int* work_next;
    unsigned int* err;
    unsigned long long* stats;   // [8]: seeds, chunks, tested, tails, algorithmic bytes read, .., .., stolen tasks
    unsigned long long budget_ns;  // per-launch wall-clock budget (0 = unlimited)
    uint32_t* tasks;             // stolen-range queue [task_cap][16 words]
    uint32_t task_cap;
    unsigned int* qctr;          // [8]: tasks reserved, tickets issued, -, completed, -, -, seeds issued
    uint32_t epoch;              // per-launch tag written as a task's ready flag (never 0)
    uint32_t force_split;        // publish unstarted work at every chunk, waited for or not (tests)
    uint32_t shard, num_shards;  // this engine expands the seed groups whose key hashes to shard (seed_shard)
    uint32_t steal;              // share long shallow ranges through the queue
    uint32_t tail_cache;         // count prefix-only tail subsets once per prefix
    const unsigned int* self_seen;  // sticky self-loop flag (see k_pack_edits)
    const uint32_t* vb;          // valid bits [qe][qv][vb_stride] or nullptr (no pruning)
    uint32_t vb_stride;
    uint32_t qv;
    const uint32_t* rb_slot;     // run bit sets: slot of (dir, vertex) [nd][dvcap] or nullptr (none)
    const uint32_t* rb_bits;     // [slot][rb_words]
    uint32_t rb_words;
    const EdgePlan* plans;       // [qe] (k_dfs_count<true>: every registered query's plans)
    const unsigned int* epoch_ptr;  // non-null: the launch tag is read here (k_epoch_bump)
    uint32_t* touched;           // footprint runs: bit per record resolved (nullptr: off)
    unsigned long long* lsum_tab;  // level-sum table [lsum_mask + 1][2], zeroed before the launch (nullptr: none)
    uint32_t lsum_mask;
    const unsigned long long* wsum;  // dense level sums [array][dvcap] (nullptr: none)
    uint32_t pair_lane_max;      // pair counting: longest shorter list a lane scans alone
};

// Footprint of a matching launch: the bytes of every distinct record it
// resolved (16 B) and of that record's whole old and delta lists (4 B per
// entry), each counted once.  Added to *out.
__global__ void k_footprint(const uint4* __restrict__ rec, uint64_t n, const uint32_t* __restrict__ touched,
                            unsigned long long* out) {
    unsigned long long b = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if ((touched[i >> 5] >> (i & 31)) & 1u) {
            const uint4 r = rec[i];
            b += 16ull + 4ull * ((unsigned long long)r.y + r.w);
        }
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(kFull, b, o);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(out, b);
}

// Next launch tag for a DFS launch that reads it from memory; the low 20
// bits (the tag's epoch field) are never 0.
__global__ void k_epoch_bump(unsigned int* e) {
    unsigned int v = *e + 1;
    if ((v & 0xfffffu) == 0) ++v;
    *e = v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Resolved candidate list of one (direction, vertex): the old run (pool) and,
// when visible, this batch's delta run (dval); the two are disjoint.
struct ListRef {
    const uint32_t* m;
    uint32_t ml;
    const uint32_t* d;
    uint32_t dl;
};

// Membership in the ascending p[0..n): halves the range with a select
// instead of a branch, so the trip count is ceil(log2 n) for every x.
// Invariant: if x is present it lies in [p, p + n).
__device__ __forceinline__ bool sorted_has_bl(const uint32_t* __restrict__ p, uint32_t n, uint32_t x) {
    if (n == 0) return false;
    while (n > 1) {
        const uint32_t half = n >> 1;
        p = (__ldg(p + half) <= x) ? p + half : p;
        n -= half;
    }
    return __ldg(p) == x;
}

__device__ __forceinline__ bool list_contains(const uint32_t* __restrict__ pool, const uint32_t* __restrict__ dval,
                                              const uint4& r, uint32_t x) {
    return sorted_has_bl(pool + r.x, r.y, x) || (r.w && sorted_has_bl(dval + r.z, r.w, x));
}

// Bit sets of the long old runs (rebuilt each batch): slot[(dir, vertex)]
// names a bit set over the compressed ids, or kNoSlot; a warp keeps the slot
// of every resolved record bn[k] in bslot[k].  slot == nullptr: none.
struct RunBits {
    const uint32_t* slot;
    const uint32_t* bits;
    uint32_t words;
    uint32_t* bslot;
    __device__ __forceinline__ void note(uint32_t k, size_t at) const {
        if (slot) bslot[k] = __ldg(slot + at);
    }
    // a lane's own record (not kept in bslot): nothing to note here
    __device__ __forceinline__ void touch(size_t) const {}
    __device__ __forceinline__ uint32_t slot_at(size_t at) const { return slot ? __ldg(slot + at) : kNoSlot; }
    // x in the list r whose old run has the bit set sl: one bit test for a long old run
    __device__ __forceinline__ bool has_slot(uint32_t sl, const uint4& r, const uint32_t* __restrict__ pool,
                                            const uint32_t* __restrict__ dval, uint32_t x) const {
        if (sl != kNoSlot) {
            if ((__ldg(bits + (size_t)sl * words + (x >> 5)) >> (x & 31)) & 1u) return true;
            return r.w && sorted_has_bl(dval + r.z, r.w, x);
        }
        return list_contains(pool, dval, r, x);
    }
    // x in the resolved list bn[k] = r
    __device__ __forceinline__ bool has(uint32_t k, const uint4& r, const uint32_t* __restrict__ pool,
                                       const uint32_t* __restrict__ dval, uint32_t x) const {
        return has_slot(slot ? bslot[k] : kNoSlot, r, pool, dval, x);
    }
};

// Footprint runs (a separate instantiation of the DFS, so that the timed
// kernel carries no trace of it): also sets the bit of every record resolved
// in touched (one bit per record).
struct RunBitsCount : RunBits {
    uint32_t* touched;
    __device__ __forceinline__ void note(uint32_t k, size_t at) const {
        RunBits::note(k, at);
        touch(at);
    }
    __device__ __forceinline__ void touch(size_t at) const { atomicOr(touched + (at >> 5), 1u << (at & 31)); }
};


// Number of x in the intersection of the resolved lists bn[ids[0..nl)] with x
// not among the matched core vertices m[t], t in the bit set excl (positions
// whose vertex can lie in these lists).  Warp-cooperative; the result is
// warp-uniform.  One list: its length minus the excluded vertices it holds.
// Several: the shortest list is scanned 32 elements at a time and each
// element probed in the others.
template <class RB>
__device__ unsigned long long isect_count(const uint4* bn, const uint8_t* ids, uint32_t nl, const uint32_t* m,
                                          uint32_t excl, const uint32_t* __restrict__ pool,
                                          const uint32_t* __restrict__ dval, uint32_t lane,
                                          unsigned long long& bytes, const RB& rb) {
    if (nl == 1) {
        const uint4 r = bn[ids[0]];
        bool in = false;
        if (lane < 16 && ((excl >> lane) & 1u)) {
            // a vertex held by two positions (a self-loop seed edge) is excluded once
            bool dup = false;
            for (uint32_t e = excl & ((1u << lane) - 1u); e; e &= e - 1) dup |= m[__ffs(e) - 1] == m[lane];
            if (!dup) in = rb.has(ids[0], r, pool, dval, m[lane]);
            bytes += 32u * (33u - __clz(r.y | 1u));
        }
        return (unsigned long long)(r.y + r.w) - __popc(__ballot_sync(kFull, in));
    }
    uint32_t g = 0, glen = 0xffffffffu;
    for (uint32_t i = 0; i < nl; ++i) {
        const uint4 r = bn[ids[i]];
        if (r.y + r.w < glen) { glen = r.y + r.w; g = i; }
    }
    const uint4 gr = bn[ids[g]];
    unsigned long long c = 0;
    for (uint32_t base = 0; base < glen; base += 32) {
        const uint32_t idx = base + lane;
        bool ok = idx < glen;
        if (ok) {
            const uint32_t x = idx < gr.y ? __ldg(pool + gr.x + idx) : __ldg(dval + gr.z + (idx - gr.y));
            bytes += 4;
            for (uint32_t e = excl; e; e &= e - 1) ok &= (x != m[__ffs(e) - 1]);
            for (uint32_t i = 0; i < nl && ok; ++i) {
                if (i == g) continue;
                const uint4 r = bn[ids[i]];
                bytes += 32u * (33u - __clz(r.y | 1u));
                ok = rb.has(ids[i], r, pool, dval, x);
            }
        }
        c += __popc(__ballot_sync(kFull, ok));
    }
    return c;
}

// Positions owning the lists bn[ids[0..nl)]: without self-loops a matched
// vertex never lies in its own lists, so excluding it needs no test.
__device__ __forceinline__ uint32_t owner_mask(const EdgePlan& P, const uint8_t* ids, uint32_t nl) {
    uint32_t o = 0;
    for (uint32_t i = 0; i < nl; ++i) o |= 1u << P.bn_pos[ids[i]];
    return o;
}

// Injective assignments of a label group of k <= 3 tail vertices from the
// sizes sc[mask] of the intersections of its members' candidate sets
// (inclusion-exclusion over coinciding members).
__device__ __forceinline__ unsigned long long group_count(const unsigned long long* sc, uint32_t k) {
    if (k == 1) return sc[1];
    if (k == 2) return sc[1] * sc[2] - sc[3];
    return sc[1] * sc[2] * sc[4] - sc[3] * sc[4] - sc[5] * sc[2] - sc[6] * sc[1] + 2 * sc[7];
}

// Number of injective assignments of the tail vertices given the matched core
// m[0..n_core): per label group, inclusion-exclusion over the sizes of the
// members' candidate sets and of their intersections (core vertices
// excluded); groups multiply.  Warp-cooperative, warp-uniform result.
template <class RB>
__device__ unsigned long long tail_count_warp(const EdgePlan& P, const uint32_t* m, uint4* bn, const uint4* rec,
                                              uint32_t dvcap, const uint32_t* __restrict__ pool,
                                              const uint32_t* __restrict__ dval, bool self_loops, uint32_t lane,
                                              unsigned long long& bytes, const RB& rb) {
    const uint32_t nc = P.n_core, n = P.n;
    // resolve every tail BN record once
    for (uint32_t k = P.bn_off[nc] + lane; k < P.bn_off[n]; k += 32) {
        const size_t at = (size_t)P.bn_dir[k] * dvcap + m[P.bn_pos[k]];
        uint4 r = rec[at];
        if (!P.bn_dvis[k]) r.w = 0;
        bn[k] = r;
        rb.note(k, at);
        bytes += 16;
    }
    __syncwarp();
    unsigned long long prod = 1;
    uint32_t t = nc;
    while (t < n && prod) {
        uint32_t e = t;
        while (e < n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        const uint32_t k = e - t;
        unsigned long long sc[8];
        for (uint32_t mask = 1; mask < (1u << k); ++mask) {
            uint8_t ids[kMaxBN];
            uint32_t nl = 0;
            for (uint32_t i = 0; i < k; ++i)
                if (mask & (1u << i))
                    for (uint32_t q = P.bn_off[t + i]; q < P.bn_off[t + i + 1]; ++q) ids[nl++] = (uint8_t)q;
            const uint32_t ex = P.excl[t] & ~(self_loops ? 0u : owner_mask(P, ids, nl));
            sc[mask] = isect_count(bn, ids, nl, m, ex, pool, dval, lane, bytes, rb);
        }
        prod *= group_count(sc, k);
        t = e;
    }
    return prod;
}

// At the last core depth j = n_core - 1 the prefix m[0..j) is fixed while all
// candidates of position j are scanned.  Subsets of a tail group whose lists
// hang only off prefix vertices have counts that do not depend on the
// candidate: tail_prepare computes them once per prefix (excluding the prefix
// vertices); tail_eval then only subtracts whether the candidate itself lies
// in the set, and intersects the subsets with lists at position j per
// candidate.
constexpr unsigned long long kDynamic = ~0ull;
constexpr uint32_t kPairLaneMax = 64;  // pair counting: longest shorter list a lane scans alone ($CGB_PAIR_LANE_MAX)
constexpr uint32_t kClean = 0xffu;  // tail cache up to date

// Recounts only the entries that depend on a position >= dirty (the shallowest
// position whose vertex changed since the last call): an entry's count
// depends on the positions of its lists' backward neighbours and of the
// excluded core vertices, so e.g. a subset hanging off positions 0 and 1
// is counted once per (m[0], m[1]), not once per prefix.  Positions >= j
// are not matched yet: subsets with a list there are left kDynamic.
template <class RB>
__device__ void tail_prepare(const EdgePlan& P, const uint32_t* m, uint4* bn, unsigned long long* cache,
                             uint32_t dirty, uint32_t j, const uint4* rec, uint32_t dvcap,
                             const uint32_t* __restrict__ pool, const uint32_t* __restrict__ dval, bool self_loops,
                             uint32_t lane, unsigned long long& bytes, const RB& rb) {
    const uint32_t nc = P.n_core, n = P.n;
    for (uint32_t k = P.bn_off[nc] + lane; k < P.bn_off[n]; k += 32) {
        if (P.bn_pos[k] >= j || P.bn_pos[k] < dirty) continue;  // records of unchanged owners are current
        const size_t at = (size_t)P.bn_dir[k] * dvcap + m[P.bn_pos[k]];
        uint4 r = rec[at];
        if (!P.bn_dvis[k]) r.w = 0;
        bn[k] = r;
        rb.note(k, at);
        bytes += 16;
    }
    __syncwarp();
    uint32_t t = nc;
    while (t < n) {
        uint32_t e = t;
        while (e < n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        const uint32_t k = e - t;
        for (uint32_t mask = 1; mask < (1u << k); ++mask) {
            uint8_t ids[kMaxBN];
            uint32_t nl = 0, dep = 0;
            bool dynamic = false;
            for (uint32_t i = 0; i < k; ++i)
                if (mask & (1u << i))
                    for (uint32_t q = P.bn_off[t + i]; q < P.bn_off[t + i + 1]; ++q) {
                        ids[nl++] = (uint8_t)q;
                        dynamic |= P.bn_pos[q] >= j;
                        dep = max(dep, (uint32_t)P.bn_pos[q]);
                    }
            const uint32_t ex = P.excl[t] & ((1u << j) - 1u) & ~(self_loops ? 0u : owner_mask(P, ids, nl));
            if (ex) dep = max(dep, 31u - __clz(ex));
            if (!dynamic && dep < dirty) continue;  // still valid
            const unsigned long long v = dynamic ? kDynamic : isect_count(bn, ids, nl, m, ex, pool, dval, lane, bytes, rb);
            if (lane == 0) cache[t * 8 + mask] = v;
        }
        t = e;
    }
    __syncwarp();
}

// Tail count for the core embedding m[0..n_core) (m[j] = the candidate).
template <class RB>
__device__ unsigned long long tail_eval(const EdgePlan& P, const uint32_t* m, uint4* bn,
                                        const unsigned long long* cache, const uint4* rec, uint32_t dvcap,
                                        const uint32_t* __restrict__ pool, const uint32_t* __restrict__ dval,
                                        bool self_loops, uint32_t lane, unsigned long long& bytes,
                                        const RB& rb) {
    const uint32_t nc = P.n_core, n = P.n, j = nc - 1;
    const uint32_t c = m[j];
    for (uint32_t k = P.bn_off[nc] + lane; k < P.bn_off[n]; k += 32) {
        if (P.bn_pos[k] != j) continue;
        const size_t at = (size_t)P.bn_dir[k] * dvcap + c;
        uint4 r = rec[at];
        if (!P.bn_dvis[k]) r.w = 0;
        bn[k] = r;
        rb.note(k, at);
        bytes += 16;
    }
    __syncwarp();
    unsigned long long prod = 1;
    uint32_t t = nc;
    while (t < n && prod) {
        uint32_t e = t;
        while (e < n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        const uint32_t k = e - t;
        unsigned long long sc[8];
        for (uint32_t mask = 1; mask < (1u << k); ++mask) {
            uint8_t ids[kMaxBN];
            uint32_t nl = 0;
            for (uint32_t i = 0; i < k; ++i)
                if (mask & (1u << i))
                    for (uint32_t q = P.bn_off[t + i]; q < P.bn_off[t + i + 1]; ++q) ids[nl++] = (uint8_t)q;
            const unsigned long long cv = cache[t * 8 + mask];
            if (cv != kDynamic && !((P.excl[t] >> j) & 1u)) {
                sc[mask] = cv;  // the candidate cannot lie in these lists (another label)
            } else if (cv != kDynamic) {
                bool in = true;
                if (lane < nl) {
                    const uint4 r = bn[ids[lane]];
                    in = rb.has(ids[lane], r, pool, dval, c);
                    bytes += 32u * (33u - __clz(r.y | 1u));
                }
                sc[mask] = cv - (__all_sync(kFull, in) ? 1ull : 0ull);
            } else {
                const uint32_t ex = P.excl[t] & ~(self_loops ? 0u : owner_mask(P, ids, nl));
                sc[mask] = isect_count(bn, ids, nl, m, ex, pool, dval, lane, bytes, rb);
            }
        }
        prod *= group_count(sc, k);
        t = e;
    }
    return prod;
}

// Tail count for the candidate c of the last core position, evaluated by
// one lane (plans with tail_lane): every cached subset count is prefix-only
// and c is removed from it when c lies in all of the subset's lists (only
// for groups sharing the last core vertex's label).  A group whose one list
// hangs off the last core position (tail_lane 2, cached as kDynamic) counts
// c's own list: its length minus the excluded prefix vertices it holds (c
// is not in its own list: no self-loops on this path).  Lanes diverge only
// in the loads and searches.
template <bool kLane2, class RB>
__device__ unsigned long long tail_eval_lane(const EdgePlan& P, const uint4* bn, const unsigned long long* cache,
                                             const uint4* __restrict__ rec, uint32_t dvcap, const uint32_t* m,
                                             const uint32_t* __restrict__ pool, const uint32_t* __restrict__ dval,
                                             uint32_t c, unsigned long long& bytes, const RB& rb) {
    const uint32_t nc = P.n_core, n = P.n, j = nc - 1;
    unsigned long long prod = 1;
    uint32_t t = nc;
    while (t < n && prod) {
        uint32_t e = t;
        while (e < n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        const uint32_t k = e - t;
        const bool same_label = (P.excl[t] >> j) & 1u;
        unsigned long long sc[8];
        for (uint32_t mask = 1; mask < (1u << k); ++mask) {
            unsigned long long cv = cache[t * 8 + mask];
            if (kLane2 && cv == kDynamic) {
                const uint32_t q = P.bn_off[t];
                const size_t at = (size_t)P.bn_dir[q] * dvcap + c;
                uint4 r = rec[at];
                if (!P.bn_dvis[q]) r.w = 0;
                rb.touch(at);
                bytes += 16;
                cv = (unsigned long long)r.y + r.w;
                const uint32_t ex = P.excl[t] & ((1u << j) - 1u);
                if (ex) {
                    const uint32_t sl = rb.slot_at(at);
                    for (uint32_t b = ex; b; b &= b - 1) {
                        bytes += 32u * (33u - __clz(r.y | 1u));
                        cv -= rb.has_slot(sl, r, pool, dval, m[__ffs(b) - 1]) ? 1ull : 0ull;
                    }
                }
            } else if (same_label) {
                bool in = true;
                for (uint32_t i = 0; i < k && in; ++i)
                    if (mask & (1u << i))
                        for (uint32_t q = P.bn_off[t + i]; q < P.bn_off[t + i + 1] && in; ++q) {
                            const uint4 r = bn[q];
                            bytes += 32u * (33u - __clz(r.y | 1u));
                            in = rb.has(q, r, pool, dval, c);
                        }
                cv -= in ? 1ull : 0ull;
            }
            sc[mask] = cv;
        }
        prod *= group_count(sc, k);
        t = e;
    }
    return prod;
}

// Tail count of a plan with tail_const: every subset is prefix-only and no
// candidate of the last core position can lie in a tail list, so the count
// is the product of the cached group counts.
__device__ unsigned long long tail_const_value(const EdgePlan& P, const unsigned long long* cache) {
    unsigned long long prod = 1;
    uint32_t t = P.n_core;
    while (t < P.n && prod) {
        uint32_t e = t;
        while (e < P.n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        prod *= group_count(cache + t * 8, e - t);
        t = e;
    }
    return prod;
}

// Level sums (plans with sum_from): the product of the lengths of c's own
// lists towards the tail vertices in sum_tails (1 when there are none).
template <class RB>
__device__ __forceinline__ unsigned long long sum_lens(const EdgePlan& P, const uint4* __restrict__ rec,
                                                       uint32_t dvcap, uint32_t c, const RB& rb) {
    unsigned long long v = 1;
    for (uint32_t b = P.sum_tails; b; b &= b - 1) {
        const uint32_t q = P.bn_off[__ffs(b) - 1];
        const size_t at = (size_t)P.bn_dir[q] * dvcap + c;
        uint4 r = rec[at];
        if (!P.bn_dvis[q]) r.w = 0;
        rb.touch(at);
        v *= (unsigned long long)r.y + r.w;
    }
    return v;
}

// Level-sum table: slots of {key, value}; key 0 = empty, K << 1 = claimed
// by a warp computing the value, K << 1 | 1 = value published, with
// K = (plan << 27 | vertex) + 1.  Zeroed before every launch, so values never
// outlive the index state they were computed on.  A lookup probes
// kLsumProbes slots; a warp that finds its key busy or every probe taken by
// other keys computes the value itself (nobody waits).
constexpr uint32_t kLsumProbes = 4;
constexpr uint32_t kLsumNone = 0xffffffffu;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One thread: the published value of K (hit = true), or the slot this
// thread claimed for K (to publish into), or kLsumNone.
__device__ __forceinline__ uint32_t lsum_find(unsigned long long* tab, uint32_t mask, unsigned long long K, bool& hit,
                                              unsigned long long& val) {
    uint32_t s = (uint32_t)((K * 0x9e3779b97f4a7c15ull) >> 32) & mask;
    for (uint32_t probe = 0; probe < kLsumProbes; ++probe, s = (s + 1) & mask) {
        unsigned long long* slot = tab + 2 * (size_t)s;
        unsigned long long k = ld_acquire_u64(slot);
        if (k == 0) {
            const unsigned long long prev = atomicCAS(slot, 0ull, K << 1);
            if (prev == 0) return s;
            k = prev;
            if (k & 1ull) k = ld_acquire_u64(slot);  // published meanwhile: read with acquire
        }
        if ((k >> 1) == K) {
            if (k & 1ull) {
                hit = true;
                val = *(volatile const unsigned long long*)(slot + 1);
            }
            return kLsumNone;  // published, or being computed by another warp
        }
    }
    return kLsumNone;
}

// Product of the cached prefix-only group counts (groups whose lists hang
// off the last core position are cached as kDynamic and left out).
__device__ unsigned long long tail_static_product(const EdgePlan& P, const unsigned long long* cache) {
    unsigned long long prod = 1;
    uint32_t t = P.n_core;
    while (t < P.n && prod) {
        uint32_t e = t;
        while (e < P.n && P.tail_gid[e] == P.tail_gid[t]) ++e;
        if (cache[t * 8 + 1] != kDynamic) prod *= group_count(cache + t * 8, e - t);
        t = e;
    }
    return prod;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

// Work units of the DFS: seeds (delta edges) from a counter, and stolen
// ranges from a ring of tasks.  A task is 16 words: w0 = ei | depth << 16 |
// generator << 24, w1/w2 = [lo, hi) of the generator list, w3 = ready tag,
// w4..15 = the matched prefix.  A warp without a seed takes one ticket
// (atomicAdd on the ticket counter) and waits for task number `ticket`;
// tasks are numbered by an atomicAdd in the same order, so every task has
// exactly one consumer and neither side contends on a CAS.  While tickets outnumber reserved
// tasks, a busy warp publishes all the work it has not started at its
// shallowest level (top of its stack), so the biggest remaining subtrees
// move first.  Termination: a warp leaves when completed == seeds + reserved
// (completed read first); a unit's reservations happen before its
// completion, so equality means no unit is active and none can be created
// (and every reserved task was consumed, so the waiting warp's ticket will
// never be filled).
// Device-scope acquire load / release increment (cheaper than full fences).
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void add_release(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr uint32_t kTaskWords = 16;
constexpr uint32_t kNoTicket = 0xffffffffu;
constexpr uint32_t kNoVertex = 0xffffffffu;  // m[1] of a grouped unit: matches no candidate

// First index of the ascending X[0..n) whose value is >= c (> c when upper),
// for a warp-uniform c: 32-ary search, each round one load per lane.
__device__ __forceinline__ uint32_t warp_bound(const uint32_t* __restrict__ X, uint32_t n, uint32_t c, bool upper,
                                               uint32_t lane) {
    uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi]
    while (hi - lo > 32) {
        const uint32_t span = hi - lo;
        bool below = false;  // lanes 0..30 test the pivots lo + floor(span * (lane + 1) / 32)
        if (lane < 31) {
            const uint32_t x = __ldg(X + lo + (uint32_t)(((uint64_t)span * (lane + 1)) >> 5));
            below = upper ? x <= c : x < c;
        }
        const uint32_t k = __popc(__ballot_sync(kFull, below));
        const uint32_t nlo = k ? lo + (uint32_t)(((uint64_t)span * k) >> 5) + 1u : lo;
        hi = k < 31 ? lo + (uint32_t)(((uint64_t)span * (k + 1)) >> 5) : hi;
        lo = nlo;
    }
    bool below = false;
    if (lo + lane < hi) {
        const uint32_t x = __ldg(X + lo + lane);
        below = upper ? x <= c : x < c;
    }
    return lo + __popc(__ballot_sync(kFull, below));
}

// Seed group of a grouped unit: X = the delta list of (seed_dir, m[0]), the
// x values of all seeds (x, m[0]) with multiplicity.  Up to 32 values live
// one per lane in xv.
struct SeedGroup {
    const uint32_t* x;
    uint32_t n;
    uint32_t xv;
    // multiplicity of the warp-uniform c in X
    __device__ __forceinline__ uint32_t mult(uint32_t c, uint32_t lane) const {
        if (n <= 32) return __popc(__ballot_sync(kFull, xv == c));
        return warp_bound(x, n, c, true, lane) - warp_bound(x, n, c, false, lane);
    }
    // sum over the lanes with `on` of the multiplicity of their own c: only
    // the values of X inside the chunk's range [cmin, cmax] are looked at
    __device__ __forceinline__ uint32_t mult_sum(uint32_t c, bool on, uint32_t lane) const {
        const uint32_t cmin = __reduce_min_sync(kFull, on ? c : 0xffffffffu);
        const uint32_t cmax = __reduce_max_sync(kFull, on ? c : 0u);
        if (cmin > cmax) return 0;
        uint32_t r = 0;
        if (n <= 32) {
            uint32_t bits = __ballot_sync(kFull, lane < n && xv >= cmin && xv <= cmax);
            while (bits) {
                const uint32_t i = __ffs(bits) - 1;
                bits &= bits - 1;
                r += (__shfl_sync(kFull, xv, i) == c) ? 1u : 0u;
            }
        } else {
            const uint32_t lo = warp_bound(x, n, cmin, false, lane), hi = warp_bound(x, n, cmax, true, lane);
            if (lo == hi) return 0;
            if (on) {
                uint32_t p = lo, len = hi - lo;
                while (len > 0) {
                    const uint32_t half = len >> 1;
                    if (__ldg(x + p + half) < c) { p += half + 1; len -= half + 1; }
                    else len = half;
                }
                for (; p < hi && __ldg(x + p) == c; ++p) ++r;
            }
        }
        r = on ? r : 0u;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(kFull, r, o);
        return r;
    }
};
// Ready tag of ticket t in launch `epoch`: the epoch's low 20 bits and the
// ring lap of t, so a slot reused in a later lap or launch never shows a
// stale tag to the consumer of t.
__device__ __forceinline__ uint32_t task_tag(uint32_t epoch, uint32_t t) {
    return ((epoch & 0xfffffu) << 12) | ((t / kTaskCap) & 0xfffu);
}
// Shard of the seed group (query edge ei, vertex x at the plan's first
// position): splitmix64's finaliser of (ei << 32 | x), modulo the shard
// count.  Seeds of one group (a grouped plan's run of equal first vertices)
// share the key, so a group is never split between shards.
__host__ __device__ __forceinline__ uint32_t seed_shard(uint32_t ei, uint32_t x, uint32_t num_shards) {
    uint64_t z = ((uint64_t)ei << 32 | x) + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (uint32_t)(z % num_shards);
}

// s_cand entries: vertex id (< 2^27) | offset of the candidate in the
// generator chunk it came from << 27
constexpr uint32_t kCandBits = 27;
constexpr uint32_t kCandMask = (1u << kCandBits) - 1u;

// kMulti = false: one query, its plans (a.plans, one per edge, at most
// kMaxQEKeyed) and seed table copied to shared memory by every block.
// kMulti = true: the plans of every registered query in global memory
// (a.plans, one per (query, edge); a.qe of them), seed table searched in
// global memory, each warp's current plan copied to shared memory when its
// unit changes plan.  kSums = false compiles the level sums and the
// per-lane pendant tails (tail_lane 2) out: the kernel is bound by
// instruction fetch, and their code doubled its fetch stalls on patterns
// whose plans never use them.
template <bool kMulti, bool kFoot = false, bool kSums = true>
__global__ void __launch_bounds__(kDfsWarps * 32, 4) k_dfs_count(DfsArgs a) {
    __shared__ uint32_t s_cand[kDfsWarps][kMaxQV][32];
    __shared__ uint4 s_bn[kDfsWarps][kMaxBN];
    __shared__ uint32_t s_rbs[kDfsWarps][kMaxBN];  // run bit-set slot of each resolved record
    __shared__ uint32_t s_m[kDfsWarps][kMaxQV];
    __shared__ unsigned long long s_tc[kDfsWarps][kMaxQV * 8];
    __shared__ uint32_t s_pre[kMulti ? 1 : kMaxQE + 1];
    __shared__ uint32_t s_lo[kMulti ? 1 : kMaxQE];
    __shared__ __align__(16) EdgePlan s_plan[kMulti ? kDfsWarps : cgb::kMaxQEKeyed];

    const uint32_t lane = threadIdx.x & 31;
    const uint32_t w = threadIdx.x >> 5;
    const bool self_loops = *(const volatile unsigned int*)a.self_seen != 0;
    // launch tag of the task ring: a kernel argument, or (in a replayed CUDA
    // graph, whose arguments are fixed) a device word bumped before the launch
    const uint32_t epoch = a.epoch_ptr ? *(const volatile unsigned int*)a.epoch_ptr : a.epoch;
    if (!kMulti) {
        if (threadIdx.x <= a.qe) s_pre[threadIdx.x] = a.seed_pre[threadIdx.x];
        if (threadIdx.x < a.qe) s_lo[threadIdx.x] = a.seed_lo[threadIdx.x];
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.plans);
        uint32_t* dst = reinterpret_cast<uint32_t*>(s_plan);
        for (uint32_t t = threadIdx.x; t < a.qe * (uint32_t)(sizeof(EdgePlan) / 4); t += blockDim.x)
            dst[t] = __ldg(src + t);
    }
    __syncthreads();
    auto pre_at = [&](uint32_t e) -> uint32_t { return kMulti ? __ldg(a.seed_pre + e) : s_pre[e]; };
    auto lo_at = [&](uint32_t e) -> uint32_t { return kMulti ? __ldg(a.seed_lo + e) : s_lo[e]; };
    auto grouped_at = [&](uint32_t e) -> bool { return kMulti ? a.plans[e].grouped != 0 : s_plan[e].grouped != 0; };
    int plan_in_smem = -1;  // kMulti: plan held in s_plan[w]
    // every engine walks all seeds; a sharded one skips the groups of other shards
    const uint32_t total = pre_at(a.qe);
    const uint64_t vmask = (1ull << a.B) - 1ull;
    uint32_t* m = s_m[w];
    uint4* bn = s_bn[w];
    using RB = typename std::conditional<kFoot, RunBitsCount, RunBits>::type;
    RB rb;
    rb.slot = a.rb_slot;
    rb.bits = a.rb_bits;
    rb.words = a.rb_words;
    rb.bslot = s_rbs[w];
    if constexpr (kFoot) rb.touched = a.touched;
    volatile unsigned int* vq = a.qctr;  // [0] tasks reserved, [1] tickets issued, [3] completed, [6] seeds

    // per-depth state held by lane == depth
    uint32_t st_ncand = 0, st_pos = 0, st_next = 0, st_len = 0, st_gen = 0;
    uint32_t st_hs = 0;  // grouped units: X multiplicity of the vertices at hit positions < depth
    unsigned long long cnt = 0;  // lane-local partial count of the current edge
    unsigned long long n_seeds = 0, n_chunks = 0, n_tested = 0, n_tail = 0, n_tasks = 0;
    unsigned long long n_bytes = 0;  // algorithmic bytes: seed keys, records, list words, probe sectors
    int cur_ei = -1;
    const unsigned long long t_start = global_ns();
    uint32_t steps = 0;
    bool out_of_time = false;
    uint32_t ticket = kNoTicket;  // lane 0: ticket of the task ring this warp waits on
    uint32_t dirty = 0;  // shallowest position changed since the tail cache was filled (kClean: none)
    unsigned long long lsum = 0;  // one-position level sum over G of the current m[p]
    bool mb = false;              // counting a subtree memo (EdgePlan::memo_from) to publish
    bool mb_split = false;        // part of that subtree went to other warps: count it, publish nothing
    uint32_t mb_slot = kLsumNone;
    unsigned long long mb_base = 0;  // lane-local count when the memo's subtree was entered
    uint32_t ls_dirty = 0;        // shallowest position changed since lsum was computed (kClean: none)
    unsigned long long tail_const = 0;  // tail count of the current prefix (plans with tail_const)
    uint32_t idle_spins = 0;

    for (;;) {
        // ---- acquire a unit: 1 = seed, 2 = task, 3 = all done, 0 = nothing yet
        uint32_t kind = 0, item = 0;
        if (lane == 0) {
            if (ticket == kNoTicket && vq[6] < total) {  // vq[6] mirrors work_next without incrementing it
                item = atomicAdd(a.work_next, 1u);
                if (item < total) kind = 1;
                else atomicMax((unsigned int*)&a.qctr[6], total);
            }
            if (!kind) {
                // no seed left: hold one ticket of the task ring and wait for its task
                if (ticket == kNoTicket) ticket = atomicAdd((unsigned int*)&a.qctr[1], 1u);
                const volatile uint32_t* tk = a.tasks + (size_t)(ticket & (a.task_cap - 1u)) * kTaskWords;
                if (tk[3] == task_tag(epoch, ticket)) {
                    kind = 2;
                    item = ticket;
                    ticket = kNoTicket;
                } else if ((idle_spins & 3u) == 3u) {
                    // completed is read with acquire before reserved (see termination above)
                    const unsigned int done = ld_acquire((const unsigned int*)&a.qctr[3]);
                    const unsigned int made = ld_acquire((const unsigned int*)&a.qctr[0]);
                    if (done == total + made && vq[6] >= total) kind = 3;
                }
            }
        }
        kind = __shfl_sync(kFull, kind, 0);
        item = __shfl_sync(kFull, item, 0);
        if (kind == 3) break;
        if (kind == 0) {
            __nanosleep(idle_spins < 64 ? 128u : 1024u);
            ++idle_spins;
            if ((idle_spins & 255u) == 0) {
                const bool late = a.budget_ns && (global_ns() - t_start) > a.budget_ns;
                if (__shfl_sync(kFull, late ? 1 : 0, 0)) { out_of_time = true; break; }
            }
            continue;
        }
        idle_spins = 0;

        int ei = 0;
        uint32_t jbase = 2, tgen = 0, tlo = 0, thi = 0;
        if (kind == 1) {
            if (kMulti) {
                // last plan whose seeds start at or before item (empty plans skipped)
                uint32_t lo = 0, hi = a.qe;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (pre_at(mid) <= item) lo = mid; else hi = mid;
                }
                ei = (int)lo;
            } else {
                while (ei + 1 < (int)a.qe && s_pre[ei + 1] <= item) ++ei;
            }
            const uint32_t e_pre = pre_at(ei), e_lo = lo_at(ei);
            const uint64_t key = a.dkeys[e_lo + (item - e_pre)];
            ++n_seeds;
            if (grouped_at(ei) && item > e_pre) {
                // a grouped edge runs one DFS per first vertex: only the first
                // seed of each run of equal first vertices starts one
                const uint64_t prev = a.dkeys[e_lo + (item - e_pre) - 1];
                if (((prev ^ key) >> a.B & vmask) == 0) {
                    if (lane == 0) add_release((unsigned int*)&a.qctr[3], 1u);
                    continue;
                }
            }
            if (a.num_shards > 1 && seed_shard((uint32_t)ei, (uint32_t)((key >> a.B) & vmask), a.num_shards) != a.shard) {
                if (lane == 0) add_release((unsigned int*)&a.qctr[3], 1u);
                continue;
            }
            if (lane == 0) {
                m[0] = (uint32_t)((key >> a.B) & vmask);
                m[1] = grouped_at(ei) ? kNoVertex : (uint32_t)(key & vmask);
                n_bytes += 8;
            }
        } else {
            // lane 0 saw the ticket's ready tag: the task's words are published
            volatile uint32_t* tk = a.tasks + (size_t)(item & (a.task_cap - 1u)) * kTaskWords;
            __threadfence();
            const uint32_t wv = lane < kTaskWords ? tk[lane] : 0;
            const uint32_t w0 = __shfl_sync(kFull, wv, 0);
            ei = (int)(w0 & 0xffffu);
            jbase = (w0 >> 16) & 0xffu;
            tgen = (w0 >> 24) & 0xffu;
            tlo = __shfl_sync(kFull, wv, 1);
            thi = __shfl_sync(kFull, wv, 2);
            if (lane >= 4 && lane < 4 + kMaxQV) m[lane - 4] = wv;
            ++n_tasks;
        }
        __syncwarp();
        if (ei != cur_ei) {
            const unsigned long long c = warp_sum(cnt);
            if (cur_ei >= 0 && lane == 0 && c) atomicAdd(a.counts + cur_ei, c);
            cnt = 0;
            cur_ei = ei;
        }
        if (kMulti && plan_in_smem != ei) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(a.plans + ei);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&s_plan[w]);
            for (uint32_t t = lane; t < sizeof(EdgePlan) / 4; t += 32) dst[t] = __ldg(src + t);
            __syncwarp();
            plan_in_smem = ei;
        }
        const EdgePlan& P = kMulti ? s_plan[w] : s_plan[ei];
        const bool tail_cache = a.tail_cache && !(P.flags & cgb::kPlanNoTailCache);
        const uint32_t nc = P.n_core;
        const bool has_tail = nc < P.n;
        SeedGroup X{nullptr, 0u, kNoVertex};
        // weight of a grouped embedding with hs hits (1 inside a memo's subtree,
        // whose count is weighted once when it is complete)
        auto gw = [&](uint32_t hs) -> unsigned long long { return mb ? 1ull : (unsigned long long)(X.n - hs); };
        if (P.grouped) {
            const size_t xat = (size_t)P.seed_dir * a.dvcap + m[0];
            const uint4 xr = a.rec[xat];
            if (kFoot && lane == 0) atomicOr(a.touched + (xat >> 5), 1u << (xat & 31));
            X.x = a.dval + xr.z;
            X.n = xr.w;
            if (X.n <= 32 && lane < X.n) X.xv = __ldg(X.x + lane);
            if (lane == 0) n_bytes += 16 + 4ull * min(X.n, 32u);
        }
        if (kind == 1 && nc == 2) {  // the seed edge alone is the core: only the tail remains
            const unsigned long long tc =
                (P.n == 2) ? 1ull : tail_count_warp(P, m, bn, a.rec, a.dvcap, a.pool, a.dval, self_loops, lane, n_bytes, rb);
            if (lane == 0) { cnt += P.grouped ? tc * X.n : tc; ++n_tail; }
            __syncwarp();
            if (lane == 0) add_release((unsigned int*)&a.qctr[3], 1u);
            continue;
        }

        // set up depth j: resolve BN records, choose the shortest list as generator
        auto setup = [&](uint32_t j) {
            const uint32_t o0 = P.bn_off[j], o1 = P.bn_off[j + 1];
            const uint32_t nb = o1 - o0;
            uint32_t len = 0xffffffffu;
            if (lane < nb) {
                const uint32_t k = o0 + lane;
                const size_t at = (size_t)P.bn_dir[k] * a.dvcap + m[P.bn_pos[k]];
                uint4 r = a.rec[at];
                if (!P.bn_dvis[k]) r.w = 0;
                bn[k] = r;
                rb.note(k, at);
                len = r.y + r.w;
                n_bytes += 16;
            }
            // shortest list, lowest lane on ties: one redux over (length << 5 | lane)
            // (lengths are below 2^27; a longer one is only a worse generator)
            const uint32_t key = len == 0xffffffffu ? 0xffffffffu : (min(len, (1u << 27) - 1u) << 5) | lane;
            const uint32_t kmin = __reduce_min_sync(kFull, key);
            const uint32_t best = kmin >> 5, bl = kmin & 31u;
            if (lane == j) { st_ncand = 0; st_pos = 0; st_next = 0; st_len = nb ? best : 0; st_gen = bl; }
            __syncwarp();
        };

        dirty = 0;  // new unit: every cached tail count is stale
        ls_dirty = 0;
        const bool level_sum = kSums && P.sum_from && !a.vb && !self_loops && (tail_cache || !has_tail);
        const bool memo_on = kSums && P.memo_from && a.lsum_tab && !a.vb && !self_loops;
        const bool pair_on = kSums && P.pair_last && !a.vb && !self_loops && (tail_cache || !has_tail);
        mb = false;
        setup(jbase);
        if (kind == 2 && lane == jbase) { st_gen = tgen; st_next = tlo; st_len = thi; }
        if (P.grouped) {
            uint32_t h = 0;
            for (uint32_t p = 2; p < jbase; ++p)
                if ((P.hit_mask >> p) & 1u) h += X.mult(m[p], lane);
            if (lane == jbase) st_hs = h;
        }
        __syncwarp();
        uint32_t j = jbase;
        while (j >= jbase) {
            if (a.budget_ns && ((++steps & 1023u) == 0)) {
                // bounded run: give up (and report) once the budget is spent
                unsigned long long now = global_ns();
                out_of_time = __shfl_sync(kFull, (now - t_start) > a.budget_ns ? 1 : 0, 0) != 0;
                if (out_of_time) break;
            }
            const uint32_t ncand = __shfl_sync(kFull, st_ncand, j);
            const uint32_t pos = __shfl_sync(kFull, st_pos, j);
            if (pos < ncand) {
                if (lane == j) st_pos = pos + 1;
                if (lane == 0) m[j] = s_cand[w][j][pos] & kCandMask;
                __syncwarp();
                dirty = min(dirty, j);
                ls_dirty = min(ls_dirty, j);
                if (P.grouped) {
                    uint32_t h = __shfl_sync(kFull, st_hs, j);
                    if ((P.hit_mask >> j) & 1u) h += X.mult(m[j], lane);
                    if (lane == j + 1) st_hs = h;
                }
                ++j;
                setup(j);
                continue;
            }
            const uint32_t gnext = __shfl_sync(kFull, st_next, j);
            uint32_t glen = __shfl_sync(kFull, st_len, j);
            if (memo_on && !mb && j == P.memo_from && gnext == 0 && glen > 0) {
                // the whole level below m[memo_pos]: its count from the table,
                // or counted here (unweighted) and published at the level's end
                const uint4 gr = bn[P.bn_off[j] + __shfl_sync(kFull, st_gen, j)];
                if (glen == gr.y + gr.w) {
                    const unsigned long long K =
                        ((1ull << 42) | ((unsigned long long)ei << 27) | m[P.memo_pos]) + 1ull;
                    uint32_t claim = kLsumNone;
                    bool hit = false;
                    unsigned long long hv = 0;
                    if (lane == 0) claim = lsum_find(a.lsum_tab, a.lsum_mask, K, hit, hv);
                    if (__shfl_sync(kFull, hit ? 1u : 0u, 0)) {
                        unsigned long long v = __shfl_sync(kFull, hv, 0);
                        if (P.grouped) v *= gw(__shfl_sync(kFull, st_hs, j));
                        if (lane == 0) { cnt += v; ++n_tail; }
                        if (lane == j) st_next = glen;
                        __syncwarp();
                        continue;
                    }
                    claim = __shfl_sync(kFull, claim, 0);
                    if (claim != kLsumNone) {
                        mb = true;
                        mb_split = false;
                        mb_slot = claim;
                        mb_base = cnt;
                    }
                }
            }
            if (level_sum && P.sum_dense && a.wsum && j == P.sum_from && gnext == 0 && glen > 0 &&
                glen == bn[P.bn_off[j]].y + bn[P.bn_off[j]].w) {
                // positions [j, n_core) counted at once: the product of the
                // precomputed sums of the positions owned by prefix positions
                unsigned long long v = 1;
                if (lane >= j && lane < nc) {
                    const uint32_t p = P.bn_pos[P.bn_off[lane]];
                    if (p < j) {
                        v = __ldg(a.wsum + (size_t)(P.wslot + lane - j) * a.dvcap + m[p]);
                        n_bytes += 8;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) v *= __shfl_xor_sync(kFull, v, o);
                if (has_tail) {
                    if (dirty <= P.tail_dep)
                        tail_prepare(P, m, bn, s_tc[w], dirty, j, a.rec, a.dvcap, a.pool, a.dval, self_loops, lane,
                                     n_bytes, rb);
                    dirty = kClean;
                    v *= tail_static_product(P, s_tc[w]);
                }
                if (P.grouped) v *= gw(__shfl_sync(kFull, st_hs, j));
                if (lane == 0) { cnt += v; ++n_tail; }
                if (lane == j) st_next = glen;
                __syncwarp();
                continue;
            }
            if (level_sum && !P.sum_dense && j == nc - 1 && gnext == 0 && glen > 0) {
                // the whole last level at once (not a stolen part of it): the
                // level sum over G, less the matched prefix vertices in G
                const uint32_t o0 = P.bn_off[j];
                const uint4 gr = bn[o0];
                if (glen == gr.y + gr.w) {
                    if (ls_dirty <= P.bn_pos[o0]) {
                        // the sum over G of the owner m[p]: from the table, or
                        // scanned (and published when this warp claimed its slot)
                        const unsigned long long K = (((unsigned long long)ei << 27) | m[P.bn_pos[o0]]) + 1ull;
                        uint32_t claim = kLsumNone;
                        bool hit = false;
                        unsigned long long hv = 0;
                        if (a.lsum_tab && lane == 0) claim = lsum_find(a.lsum_tab, a.lsum_mask, K, hit, hv);
                        if (__shfl_sync(kFull, hit ? 1u : 0u, 0)) {
                            lsum = __shfl_sync(kFull, hv, 0);
                        } else {
                            unsigned long long sv = 0;
                            for (uint32_t idx = lane; idx < glen; idx += 32) {
                                const uint32_t c =
                                    idx < gr.y ? __ldg(a.pool + gr.x + idx) : __ldg(a.dval + gr.z + (idx - gr.y));
                                sv += sum_lens(P, a.rec, a.dvcap, c, rb);
                                n_bytes += 4;
                            }
                            lsum = warp_sum(sv);
                            if (lane == 0 && claim != kLsumNone) {
                                a.lsum_tab[2 * (size_t)claim + 1] = lsum;
                                st_release_u64(a.lsum_tab + 2 * (size_t)claim, (K << 1) | 1ull);
                            }
                        }
                        ls_dirty = kClean;
                    }
                    unsigned long long corr = 0;
                    bool hit = false;
                    if (lane < j && ((P.sum_same >> lane) & 1u)) {
                        const uint32_t x = m[lane];
                        if (x != kNoVertex && rb.has(o0, gr, a.pool, a.dval, x)) {
                            hit = true;
                            corr = sum_lens(P, a.rec, a.dvcap, x, rb);
                        }
                    }
                    corr = warp_sum(corr);
                    const uint32_t nhit = __popc(__ballot_sync(kFull, hit));
                    unsigned long long v = lsum - corr;
                    if (has_tail) {
                        if (dirty <= P.tail_dep)
                            tail_prepare(P, m, bn, s_tc[w], dirty, nc - 1, a.rec, a.dvcap, a.pool, a.dval,
                                         self_loops, lane,
                                         n_bytes, rb);
                        dirty = kClean;
                        v *= tail_static_product(P, s_tc[w]);
                    }
                    if (P.grouped) v *= gw(__shfl_sync(kFull, st_hs, j));
                    if (lane == 0) { cnt += v; n_tail += glen - nhit; }
                    if (lane == j) st_next = glen;
                    __syncwarp();
                    continue;
                }
            }
            if (gnext < glen) {
                const uint32_t g = __shfl_sync(kFull, st_gen, j);
                // While warps wait for tasks, hand the work not yet started at the
                // shallowest level of this unit to the queue: at a depth d < j
                // the buffered survivors not yet descended plus the unscanned
                // generator range, at d = j the range after this chunk.  The
                // survivors are a contiguous stretch of the generator (their
                // offsets in their chunk ride in the top bits of s_cand), so
                // one range [lo, hi) of depth d's generator describes it all.
                if (a.steal) {  // checked at every chunk: a waiting warp is served within one chunk's time
                    uint32_t want = 0;  // some warp holds a ticket no task has been reserved for
                    if (lane == 0) want = (a.force_split || (int)(vq[1] - vq[0]) > 0) ? 1u : 0u;
                    if (__shfl_sync(kFull, want, 0)) {
                        bool has = false;
                        if (lane >= jbase && lane < j) has = st_next < st_len || st_pos < st_ncand;
                        // at a pair-counting depth a chunk's passing candidates were
                        // partly counted already: only its unscanned range is shared
                        if (pair_on && lane == nc - 2 && lane >= jbase && lane < j) has = st_next < st_len;
                        if (lane == j) has = glen > gnext + 32u;
                        const uint32_t hb = __ballot_sync(kFull, has);
                        uint32_t slot = 0xffffffffu;
                        if (hb && lane == 0) {
                            // reserve the next task number while tickets wait for one (always, under
                            // force_split).  atomicAdd never fails, so concurrent producers may
                            // overshoot the demand by a few tasks; those wait in the ring for the
                            // next idle warps, and the slack keeps the ring from lapping its head.
                            const unsigned int t = vq[0], hd = vq[1];
                            if ((a.force_split || (int)(hd - t) > 0) && (int)(t - hd) < (int)(a.task_cap - kTaskSlack))
                                slot = atomicAdd((unsigned int*)&a.qctr[0], 1u);
                        }
                        slot = __shfl_sync(kFull, slot, 0);
                        if (slot != 0xffffffffu) {
                            const uint32_t d = __ffs(hb) - 1;
                            if (mb && d >= P.memo_from) mb_split = true;  // the memo's count is no longer all here
                            uint32_t lo = 0, hi = 0;
                            if (lane == d) {
                                if (d == j) {
                                    lo = gnext + 32u;
                                    hi = glen;
                                } else if (pair_on && d == nc - 2) {
                                    lo = st_next;  // the buffered survivors stay with this warp
                                    hi = st_len;
                                } else {
                                    lo = st_pos < st_ncand ? st_next - 32u + (s_cand[w][d][st_pos] >> kCandBits)
                                                           : st_next;
                                    hi = st_len;
                                }
                            }
                            lo = __shfl_sync(kFull, lo, d);
                            hi = __shfl_sync(kFull, hi, d);
                            const uint32_t gd = __shfl_sync(kFull, st_gen, d);
                            uint32_t* tk = a.tasks + (size_t)(slot & (a.task_cap - 1u)) * kTaskWords;
                            uint32_t v = 0;
                            if (lane == 0) v = (uint32_t)ei | (d << 16) | (gd << 24);
                            else if (lane == 1) v = lo;
                            else if (lane == 2) v = hi;
                            else if (lane >= 4 && lane < 4 + kMaxQV) v = (lane - 4 < d) ? m[lane - 4] : 0u;
                            if (lane < kTaskWords && lane != 3) tk[lane] = v;
                            __threadfence();
                            __syncwarp();
                            if (lane == 0) *(volatile uint32_t*)(tk + 3) = task_tag(epoch, slot);
                            if (lane == d) {
                                if (d == j) st_len = gnext + 32u;
                                else if (pair_on && d == nc - 2) st_len = st_next;
                                else { st_len = st_next; st_ncand = st_pos; }
                            }
                            if (d == j) glen = gnext + 32u;
                        }
                    }
                }
                const uint32_t o0 = P.bn_off[j], o1 = P.bn_off[j + 1];
                const uint4 gr = bn[o0 + g];
                const uint32_t idx = gnext + lane;
                bool ok = idx < glen;
                uint32_t c = 0;
                if (ok) {
                    c = idx < gr.y ? __ldg(a.pool + gr.x + idx) : __ldg(a.dval + gr.z + (idx - gr.y));
                    n_bytes += 4;
                    for (uint32_t t = 0; t < j; ++t) ok &= (c != m[t]);
                    if (ok && a.vb)  // the valid bits are a sound superset: a clear bit cannot match
                        ok = (__ldg(a.vb + ((size_t)ei * a.qv + P.vs[j]) * a.vb_stride + (c >> 5)) >> (c & 31)) & 1u;
                }
                if (ok) {
                    // Each candidate is searched in every other backward list,
                    // stopping at the first miss.  All lanes search the same list
                    // with the same trip count, so the branch-free search keeps
                    // the warp converged, and the first steps of every lane hit
                    // the same words.
                    for (uint32_t k = o0; k < o1 && ok; ++k) {
                        if (k == o0 + g) continue;
                        const uint4 r = bn[k];
                        const uint32_t sl = rb.slot ? s_rbs[w][k] : kNoSlot;
                        if (sl != kNoSlot) {
                            n_bytes += 4;
                            ok = (__ldg(rb.bits + (size_t)sl * rb.words + (c >> 5)) >> (c & 31)) & 1u;
                        } else {
                            n_bytes += 32u * (33u - __clz(r.y | 1u));
                            ok = sorted_has_bl(a.pool + r.x, r.y, c);
                        }
                        if (!ok && r.w) {
                            n_bytes += 32u * (33u - __clz(r.w | 1u));
                            ok = sorted_has_bl(a.dval + r.z, r.w, c);
                        }
                    }
                    ++n_tested;
                }
                ++n_chunks;
                if (j == nc - 1) {
                    // grouped units weigh each embedding by |X| minus the X
                    // multiplicity of its hit-position vertices
                    const uint32_t hs = P.grouped ? __shfl_sync(kFull, st_hs, j) : 0u;
                    const bool hit_last = P.grouped && ((P.hit_mask >> j) & 1u);
                    if (has_tail && P.tail_const && tail_cache) {
                        // the tail count depends on the prefix only: one value per prefix
                        const uint32_t bal = __ballot_sync(kFull, ok);
                        if (bal) {
                            if (dirty <= P.tail_dep) {
                                tail_prepare(P, m, bn, s_tc[w], dirty, nc - 1, a.rec, a.dvcap, a.pool, a.dval,
                                             self_loops, lane, n_bytes, rb);
                                tail_const = tail_const_value(P, s_tc[w]);
                            }
                            dirty = kClean;
                            unsigned long long wsum = __popc(bal);
                            if (P.grouped) {
                                wsum *= gw(hs);
                                if (hit_last) wsum -= X.mult_sum(c, ok, lane);
                            }
                            if (lane == 0) { cnt += wsum * tail_const; n_tail += __popc(bal); }
                        }
                    } else if (has_tail && P.tail_lane && (P.tail_lane == 1 || (kSums && !self_loops)) &&
                               tail_cache && !hit_last) {
                        // the tail depends on the candidate only through prefix-only
                        // lists: every lane counts its own candidate's tail
                        const uint32_t bal = __ballot_sync(kFull, ok);
                        if (bal) {
                            if (dirty <= P.tail_dep)
                                tail_prepare(P, m, bn, s_tc[w], dirty, nc - 1, a.rec, a.dvcap, a.pool, a.dval,
                                             self_loops, lane, n_bytes, rb);
                            dirty = kClean;
                            if (ok) {
                                const unsigned long long tc =
                                    tail_eval_lane<kSums>(P, bn, s_tc[w], a.rec, a.dvcap, m, a.pool, a.dval, c, n_bytes,
                                                          rb);
                                cnt += P.grouped ? tc * gw(hs) : tc;
                            }
                            if (lane == 0) n_tail += __popc(bal);
                        }
                    } else if (has_tail) {
                        // every surviving candidate completes a core embedding: count its tail
                        uint32_t bal = __ballot_sync(kFull, ok);
                        while (bal) {
                            const int l = __ffs(bal) - 1;
                            bal &= bal - 1;
                            const uint32_t cl = __shfl_sync(kFull, c, l);
                            if (dirty <= P.tail_dep && tail_cache) {
                                // first embedding since the prefix changed: recount the stale prefix-only subsets
                                tail_prepare(P, m, bn, s_tc[w], dirty, nc - 1, a.rec, a.dvcap, a.pool, a.dval,
                                             self_loops, lane, n_bytes, rb);
                            }
                            dirty = kClean;
                            if (lane == 0) m[j] = cl;
                            __syncwarp();
                            const unsigned long long tc =
                                tail_cache
                                    ? tail_eval(P, m, bn, s_tc[w], a.rec, a.dvcap, a.pool, a.dval, self_loops, lane,
                                                n_bytes, rb)
                                    : tail_count_warp(P, m, bn, a.rec, a.dvcap, a.pool, a.dval, self_loops, lane,
                                                      n_bytes, rb);
                            unsigned long long wt = 1;
                            if (P.grouped) wt = gw(hs) - (hit_last ? X.mult(cl, lane) : 0u);
                            if (lane == 0) { cnt += tc * wt; ++n_tail; }
                            __syncwarp();
                        }
                    } else if (P.grouped) {
                        const uint32_t nok = __popc(__ballot_sync(kFull, ok));
                        unsigned long long wsum = (unsigned long long)nok * gw(hs);
                        if (hit_last) wsum -= X.mult_sum(c, ok, lane);
                        if (lane == 0) cnt += wsum;
                    } else {
                        cnt += ok ? 1ull : 0ull;
                    }
                } else {
                    bool desc = ok;  // survivors buffered for the descent
                    if (pair_on && j == nc - 2) {
                        // each lane counts its candidate's last level: |A ∩ B|,
                        // A = the prefix list of the last position, B = the
                        // candidate's own; candidates whose shorter list is long
                        // descend as usual
                        const uint32_t ka = P.pair_a, kb = P.pair_b;
                        if (lane == 0) {
                            const size_t at = (size_t)P.bn_dir[ka] * a.dvcap + m[P.bn_pos[ka]];
                            uint4 r = a.rec[at];
                            if (!P.bn_dvis[ka]) r.w = 0;
                            bn[ka] = r;
                            rb.note(ka, at);
                        }
                        __syncwarp();
                        const uint4 ra = bn[ka];
                        const uint32_t la = ra.y + ra.w;
                        unsigned long long pc = 0;
                        bool counted = false;
                        if (ok) {
                            const size_t atb = (size_t)P.bn_dir[kb] * a.dvcap + c;
                            uint4 rq = a.rec[atb];
                            if (!P.bn_dvis[kb]) rq.w = 0;
                            rb.touch(atb);
                            n_bytes += 16;
                            const uint32_t lq = rq.y + rq.w;
                            if (min(la, lq) <= a.pair_lane_max) {
                                counted = true;
                                const uint32_t slq = rb.slot_at(atb);
                                if (lq <= la) {
                                    for (uint32_t i = 0; i < lq; ++i) {
                                        const uint32_t x = i < rq.y ? __ldg(a.pool + rq.x + i) : __ldg(a.dval + rq.z + (i - rq.y));
                                        pc += rb.has(ka, ra, a.pool, a.dval, x) ? 1ull : 0ull;
                                    }
                                } else {
                                    for (uint32_t i = 0; i < la; ++i) {
                                        const uint32_t x = i < ra.y ? __ldg(a.pool + ra.x + i) : __ldg(a.dval + ra.z + (i - ra.y));
                                        pc += rb.has_slot(slq, rq, a.pool, a.dval, x) ? 1ull : 0ull;
                                    }
                                }
                                for (uint32_t e = P.pair_excl; e; e &= e - 1) {
                                    const uint32_t x = m[__ffs(e) - 1];
                                    if (x != kNoVertex && rb.has(ka, ra, a.pool, a.dval, x) &&
                                        rb.has_slot(slq, rq, a.pool, a.dval, x))
                                        --pc;
                                }
                            }
                        }
                        const uint32_t cb = __ballot_sync(kFull, counted);
                        if (cb) {
                            unsigned long long tc = 1;
                            if (has_tail) {
                                if (dirty <= P.tail_dep)
                                    tail_prepare(P, m, bn, s_tc[w], dirty, nc - 2, a.rec, a.dvcap, a.pool, a.dval,
                                                 self_loops, lane, n_bytes, rb);
                                dirty = kClean;
                                tc = tail_static_product(P, s_tc[w]);
                                // the cache is marked current: so must be the prefix's tail
                                // count that the descending candidates' last level reads
                                if (P.tail_const) tail_const = tc;
                            }
                            const unsigned long long wgt = P.grouped ? gw(__shfl_sync(kFull, st_hs, j)) : 1ull;
                            if (counted) cnt += pc * tc * wgt;
                            if (lane == 0) n_tail += __popc(cb);
                        }
                        desc = ok && !counted;
                    }
                    const uint32_t bal = __ballot_sync(kFull, desc);
                    if (desc) s_cand[w][j][__popc(bal & ((1u << lane) - 1u))] = c | (lane << kCandBits);
                    if (lane == j) { st_ncand = __popc(bal); st_pos = 0; }
                }
                if (lane == j) st_next = gnext + 32;
                __syncwarp();
                continue;
            }
            if (mb && j == P.memo_from) {
                // the memo's subtree is complete: publish its count, weight it once
                const unsigned long long S = warp_sum(cnt - mb_base);
                if (lane == 0 && !mb_split) {
                    const unsigned long long K =
                        ((1ull << 42) | ((unsigned long long)ei << 27) | m[P.memo_pos]) + 1ull;
                    a.lsum_tab[2 * (size_t)mb_slot + 1] = S;
                    st_release_u64(a.lsum_tab + 2 * (size_t)mb_slot, (K << 1) | 1ull);
                }
                const unsigned long long wv =
                    P.grouped ? (unsigned long long)(X.n - __shfl_sync(kFull, st_hs, j)) : 1ull;
                cnt = mb_base + (lane == 0 ? S * wv : 0ull);
                mb = false;
            }
            --j;
        }
        if (out_of_time) {
            if (lane == 0) atomicOr(a.err, 8u);
            break;
        }
        if (lane == 0) add_release((unsigned int*)&a.qctr[3], 1u);
    }
    if (out_of_time && lane == 0) atomicOr(a.err, 8u);
    const unsigned long long c = warp_sum(cnt);
    if (cur_ei >= 0 && lane == 0 && c) atomicAdd(a.counts + cur_ei, c);
    const unsigned long long tested = warp_sum(n_tested), tails = warp_sum(n_tail), bytes = warp_sum(n_bytes);
    if (lane == 0) {
        atomicAdd(a.stats + 0, n_seeds);
        atomicAdd(a.stats + 1, n_chunks);
        atomicAdd(a.stats + 2, tested);
        atomicAdd(a.stats + 3, tails);
        atomicAdd(a.stats + 4, bytes);
        atomicAdd(a.stats + 7, n_tasks);
    }
}

// ---------------------------------------------------------------------------
// dense level sums: W_k(x) for every vertex x of one level-sum position k of
// a plan (EdgePlan::sum_dense), computed children first before the DFS
// ---------------------------------------------------------------------------
struct WsumJob {
    uint32_t dir, dvis;  // G_k(x): the list of direction dir at x (delta part if dvis)
    uint32_t nt;         // pendant tails of k: lists of direction tdir at c (delta part if tvis)
    uint32_t tdir[cgb::kMaxSumTails], tvis[cgb::kMaxSumTails];
    uint32_t nch;        // positions owned by k: their sums at c
    const unsigned long long* child[cgb::kMaxSumChildren];
    unsigned long long* out;
};
constexpr uint32_t kWsumLane = 16;  // owners with lists up to this long are summed by one lane

// W(x) = sum over c in G(x) of (product of c's pendant list lengths) x
// (product of the children's W(c)), for every x < dv, for the job
// jobs[job0 + blockIdx.y] (the jobs of one launch are independent: their
// children are done).  Lane per owner for short lists (records read
// coalesced, 32 consecutive owners per warp), the whole warp for each longer
// one.
__global__ void k_wsum(const uint4* __restrict__ rec, uint32_t dvcap, const uint32_t* __restrict__ pool,
                       const uint32_t* __restrict__ dval, uint32_t dv, const WsumJob* __restrict__ jobs,
                       uint32_t job0) {
    __shared__ WsumJob sJ;
    static_assert(sizeof(WsumJob) % 4 == 0, "WsumJob is copied as words");
    for (uint32_t t = threadIdx.x; t < sizeof(WsumJob) / 4; t += blockDim.x)
        reinterpret_cast<uint32_t*>(&sJ)[t] = reinterpret_cast<const uint32_t*>(jobs + job0 + blockIdx.y)[t];
    __syncthreads();
    const WsumJob& J = sJ;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    auto term = [&](uint32_t c) -> unsigned long long {
        unsigned long long v = 1;
#pragma unroll
        for (uint32_t i = 0; i < cgb::kMaxSumTails; ++i)
            if (i < J.nt) {
                const uint4 t = rec[(size_t)J.tdir[i] * dvcap + c];
                v *= (unsigned long long)t.y + (J.tvis[i] ? t.w : 0u);
            }
#pragma unroll
        for (uint32_t i = 0; i < cgb::kMaxSumChildren; ++i)
            if (i < J.nch) v *= __ldg(J.child[i] + c);
        return v;
    };
    for (uint64_t base = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) << 5; base < dv;
         base += nwarps * 32) {
        const uint64_t x = base + lane;
        uint4 r = make_uint4(0, 0, 0, 0);
        if (x < dv) {
            r = rec[(size_t)J.dir * dvcap + x];
            if (!J.dvis) r.w = 0;
        }
        const uint32_t len = r.y + r.w;
        unsigned long long acc = 0;
        if (len <= kWsumLane)
            for (uint32_t i = 0; i < len; ++i)
                acc += term(i < r.y ? __ldg(pool + r.x + i) : __ldg(dval + r.z + (i - r.y)));
        uint32_t big = __ballot_sync(kFull, len > kWsumLane);
        while (big) {
            const uint32_t i = __ffs(big) - 1;
            big &= big - 1;
            const uint32_t rx = __shfl_sync(kFull, r.x, i), ry = __shfl_sync(kFull, r.y, i);
            const uint32_t rz = __shfl_sync(kFull, r.z, i), rw = __shfl_sync(kFull, r.w, i);
            unsigned long long sv = 0;
            for (uint32_t t = lane; t < ry + rw; t += 32)
                sv += term(t < ry ? __ldg(pool + rx + t) : __ldg(dval + rz + (t - ry)));
            for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(kFull, sv, o);
            if (lane == i) acc = sv;
        }
        if (x < dv) J.out[x] = acc;
    }
}

// ---------------------------------------------------------------------------
// valid bits (BuildLocalIndexBitAll with 1-bit masks, graph_gpu.cu:803-869,
// indexing.cu:2295-2379): vb[ei][u][w] holds bit (dv & 31) of word dv >> 5
// for query vertex u under query edge ei.  A sound superset of the vertices
// that some embedding mapping ei to a delta edge can place at u.
// ---------------------------------------------------------------------------
// Rebuilt (ei, u) start empty, the others all ones (graph_gpu.cu:818-828).
__global__ void k_vb_fill(const cgb::VbPlan* __restrict__ vbp, uint32_t* vb, uint32_t qe, uint32_t qv,
                          uint32_t stride) {
    const size_t n = (size_t)qe * qv * stride;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t ei = (uint32_t)(i / ((size_t)qv * stride));
        const uint32_t u = (uint32_t)((i / stride) % qv);
        vb[i] = ((vbp[ei].rebuild >> u) & 1u) ? 0u : 0xffffffffu;
    }
}

// Endpoints of ei: vertices with a delta list in ei's own direction
// (setInitialValidBitsAll1Bit, indexing.cu:2295-2317), set from the sorted
// packed delta keys (d << 2B | u << B | v): one bit per key, no full sweep.
__global__ void k_vb_seed(const cgb::VbPlan* __restrict__ vbp, const uint8_t* __restrict__ dir_edge,
                          const uint64_t* __restrict__ dkeys, uint64_t n, uint32_t B, uint32_t* vb, uint32_t qv,
                          uint32_t stride) {
    const uint64_t m = (1ull << B) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = dkeys[i];
        const uint32_t d = (uint32_t)(k >> (2 * B)), u = (uint32_t)((k >> B) & m);
        const uint32_t ei = dir_edge[d];
        const cgb::VbPlan& P = vbp[ei];
        const uint32_t qu = d == P.d01 ? P.vs[0] : P.vs[1];
        atomicOr(vb + ((size_t)ei * qv + qu) * stride + (u >> 5), 1u << (u & 31));
    }
}

// Position `depth` of every query edge's indexing order (grid.y = ei): a
// vertex is valid if, for every backward neighbour, its list towards that
// neighbour (old run, plus the delta run when visible) holds a vertex whose
// bit is set (checkAllConstraintsAndSetBitsAll1Bit, indexing.cu:2319-2377).
// One warp per mask word, one lane per vertex.
__global__ void k_vb_depth(const cgb::VbPlan* __restrict__ vbp, const uint4* __restrict__ rec, uint32_t dvcap,
                           const uint32_t* __restrict__ pool, const uint32_t* __restrict__ dval, uint32_t dv,
                           uint32_t* vb, uint32_t qv, uint32_t stride, uint32_t depth) {
    const uint32_t ei = blockIdx.y;
    const cgb::VbPlan& P = vbp[ei];
    const uint32_t u = P.vs[depth];
    if (!((P.rebuild >> u) & 1u)) return;
    uint32_t* out = vb + ((size_t)ei * qv + u) * stride;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wi < stride; wi += nw) {
        const uint32_t x = wi * 32u + lane;
        bool valid = x < dv;
        for (uint32_t b = P.off[depth]; b < P.off[depth + 1] && valid; ++b) {
            const uint32_t* m1 = vb + ((size_t)ei * qv + P.vs[P.bpos[b]]) * stride;
            const uint4 r = rec[(size_t)P.bdir[b] * dvcap + x];
            bool sat = false;
            for (uint32_t t = 0; t < r.y && !sat; ++t) {
                const uint32_t nb = __ldg(pool + r.x + t);
                sat = (m1[nb >> 5] >> (nb & 31)) & 1u;
            }
            if (P.bvis[b])
                for (uint32_t t = 0; t < r.w && !sat; ++t) {
                    const uint32_t nb = __ldg(dval + r.z + t);
                    sat = (m1[nb >> 5] >> (nb & 31)) & 1u;
                }
            valid = sat;
        }
        const uint32_t word = __ballot_sync(kFull, valid);
        if (lane == 0) out[wi] = word;
    }
}

// ---------------------------------------------------------------------------
// maintenance kernels
// ---------------------------------------------------------------------------
__global__ void k_rec_sizes(const uint4* rec, uint32_t dvcap, uint32_t dv, uint32_t nd, uint32_t* out_round4,
                            uint32_t* out_len) {
    uint64_t total = (uint64_t)nd * dv;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t d = (uint32_t)(i / dv), u = (uint32_t)(i % dv);
        uint32_t len = rec[(size_t)d * dvcap + u].y;
        if (out_round4) out_round4[i] = round4(len);
        if (out_len) out_len[i] = len;
    }
}

// Copies every run to its compacted offset (warp per (d,u)).
__global__ void k_compact(uint4* rec, uint32_t dvcap, uint32_t dv, uint32_t nd, const uint32_t* src,
                          uint32_t* dst, const unsigned long long* new_off) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t total = (uint64_t)nd * dv;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total;
         i += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        uint32_t d = (uint32_t)(i / dv), u = (uint32_t)(i % dv);
        uint4* p = rec + (size_t)d * dvcap + u;
        uint4 r = *p;
        uint64_t no = new_off[i];
        for (uint32_t k = lane; k < r.y; k += 32) dst[no + k] = src[r.x + k];
        if (lane == 0) { r.x = (uint32_t)no; *p = r; }
    }
}

__global__ void k_dump(const uint4* rec, uint32_t dvcap, uint32_t dv, uint32_t nd, const uint32_t* pool,
                       const unsigned long long* off, uint64_t* out) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t total = (uint64_t)nd * dv;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total;
         i += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        uint32_t d = (uint32_t)(i / dv), u = (uint32_t)(i % dv);
        uint4 r = rec[(size_t)d * dvcap + u];
        uint64_t o = off[i];
        for (uint32_t k = lane; k < r.y; k += 32)
            out[o + k] = ((uint64_t)d << 59) | ((uint64_t)u << 32) | pool[r.x + k];
    }
}

__global__ void k_copy_rows(const uint4* src, uint32_t src_cap, uint4* dst, uint32_t dst_cap, uint32_t nd,
                            uint32_t dv) {
    uint64_t total = (uint64_t)nd * dv;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t d = (uint32_t)(i / dv), u = (uint32_t)(i % dv);
        dst[(size_t)d * dst_cap + u] = src[(size_t)d * src_cap + u];
    }
}

__global__ void k_u32_to_u64(const uint32_t* in, unsigned long long* out, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

inline uint32_t bits_for(uint32_t dv) {
    uint32_t b = 1;
    while ((1ull << b) < (uint64_t)dv) ++b;
    return b;
}

}  // namespace

// ===========================================================================
// host side
// ===========================================================================
struct cgb_handle {
    cgb_config cfg{};
    int device = 0;
    int num_sms = 148;
    int dfs_occupancy = 0;  // resident DFS blocks per SM
    uint32_t dfs_epoch = 0; // launch counter used as the task ready tag
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    uint64_t launches = 0;

    // query
    bool have_query = false;
    cgb::QueryMeta q;
    EdgePlan plans[kMaxQE];
    EdgePlan* d_plans = nullptr;       // [kMaxQE] device copy of plans
    cgb::VbPlan* d_vbplans = nullptr;  // [kMaxQE] valid-bit plans
    uint8_t* d_dir_edge = nullptr;     // [kMaxDir] query edge of each direction
    uint8_t* d_qe_dirs = nullptr;  // [qe][2]
    uint8_t* d_edge_ok = nullptr;  // [kMaxQE]

    // index
    bool have_index = false;
    uint32_t nd = 0, dv = 0, dvcap = 0;
    uint4* rec = nullptr;
    uint32_t* pool = nullptr;
    uint32_t* pool_alt = nullptr;
    unsigned long long pool_cap = 0;
    // device scalars: [0] pool_top, [1] live_words, [2] err, [3] work_next
    unsigned long long* d_scal = nullptr;
    unsigned int* d_self = nullptr;  // sticky: some added key was a self-loop (u == v)
    unsigned long long* h_scal = nullptr;  // pinned mirror (4 scalars + counts)
    unsigned long long h_pool_top = 0;
    long long h_live = 0;

    // per-batch buffers (grown on demand)
    uint64_t* d_keys_in = nullptr; size_t keys_in_cap = 0;       // uploaded ext keys (ins|del|delta)
    uint64_t* d_pending = nullptr; size_t pending_cap = 0; uint64_t n_pending = 0;  // ext delta keys
    uint64_t* d_edits = nullptr; uint64_t* d_edits_alt = nullptr; size_t edits_cap = 0;
    uint32_t* d_du = nullptr; uint32_t* d_run_du = nullptr; uint32_t* d_run_len = nullptr;
    uint32_t* d_run_off = nullptr; size_t runs_cap = 0;
    uint32_t* d_small_runs = nullptr; uint32_t* d_big_runs = nullptr;  // merge lists (k_merge_classify)
    uint32_t* d_tiny_runs = nullptr;
    unsigned int* d_list_ctr = nullptr;  // [0] small, [1] big, [2] tiny
    int* d_num_runs = nullptr;
    uint64_t* d_dkeys = nullptr; uint64_t* d_dkeys_alt = nullptr; size_t dkeys_cap = 0;
    uint32_t* d_dval = nullptr;
    uint32_t* d_ddu = nullptr;
    uint32_t* d_drun_du = nullptr; uint32_t* d_drun_len = nullptr; uint32_t* d_drun_off = nullptr;
    size_t druns_cap = 0;
    uint32_t* d_seed = nullptr;  // [0..kMaxQE) lo, [kMaxQE..2kMaxQE+1) pre
    unsigned long long* d_counts = nullptr;  // [kMaxQE]
    unsigned long long* d_stats = nullptr;   // [8]
    uint32_t* d_tasks = nullptr;             // stolen-range queue
    unsigned int* d_qctr = nullptr;          // queue counters [8]
    unsigned long long last_stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    void* d_temp = nullptr; size_t temp_cap = 0;

    // run bit sets: built in full on the first matched batch (and after the
    // record table grows), then kept current by every merge
    uint32_t* d_rb_slot = nullptr; size_t rb_slot_cap = 0;  // [nd][dvcap]
    uint32_t* d_rb_sel = nullptr; size_t rb_sel_cap = 0;
    uint32_t* d_rb_bits = nullptr; size_t rb_bits_cap = 0;
    uint32_t* d_rb_new = nullptr; size_t rb_new_cap = 0;    // slots claimed by the last merge
    unsigned int* d_rb_ctr = nullptr;  // [0] slots claimed, [1] claimed by the last merge
    uint32_t rb_words = 0;             // words per bit set: (dvcap + 31) / 32
    uint32_t rb_cap = 0;               // bit sets the budget holds
    bool rb_valid = false;             // slot table and bit sets match the index
    uint32_t rb_min_len = kRunBitsMinLen;
    uint32_t pair_lane_max = kPairLaneMax;
    uint8_t* d_rev = nullptr;          // reverse direction of each direction
    uint32_t* d_touched = nullptr; size_t touched_cap = 0;  // footprint runs: record bit set
    unsigned long long* d_lsum = nullptr;  // level-sum table, sized with the record table
    uint32_t lsum_slots = 0;
    unsigned long long* d_wsum = nullptr; size_t wsum_cap = 0;  // dense level sums [n_wsum][dvcap]
    uint32_t n_wsum = 0;
    WsumJob* d_wjobs = nullptr;                 // [n_wsum] jobs, ordered by height (children first)
    std::vector<uint32_t> wjob_level;           // job offsets of each height (size = heights + 1)
    const void* wjobs_for = nullptr;            // d_wsum the jobs were built for

    // label-keyed mode (the multi-query engine's data-graph index): the
    // "direction" of a key is the label of its target vertex, the delta keys
    // carry the source vertex's label (lb bits) between direction and source
    bool mq = false;
    uint32_t lb = 0;
    uint8_t* d_vlabel = nullptr;       // [dv] vertex labels
    unsigned int* d_epoch = nullptr;   // DFS launch tag read by replayed graphs

    // valid bits
    uint32_t vb_start[2] = {0, 0};   // starting edge (SelectStartingEdge)
    std::string vb_plan_error;       // set when the pattern has no consistent rebuild flags
    uint32_t* d_vb = nullptr; size_t vb_cap = 0;
    uint32_t vb_stride = 0;          // words per (ei, u) of the last matched batch; 0 = none
    float last_vb_ms = 0;

    uint64_t last_counts[kMaxQE] = {0};
    float last_t[4] = {0, 0, 0, 0};
    cudaEvent_t ev[7] = {};  // phases 0-3, caller-stream order 4, end 5, valid bits 6
};

namespace {

cgb_status fail(cgb_handle* h, cgb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    return s;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            return fail(h, e_ == cudaErrorMemoryAllocation ? CGB_ERR_OOM : CGB_ERR_CUDA,         \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
        }                                                                                        \
    } while (0)

#define LAUNCHED() (h->launches++)

template <typename T>
cgb_status grow(cgb_handle* h, T*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return CGB_OK;
    size_t nc = std::max<size_t>(need + need / 2, 1024);
    if (p) CK(cudaFree(p));
    p = nullptr;
    CK(cudaMalloc(&p, nc * sizeof(T)));
    cap = nc;
    return CGB_OK;
}

cgb_status grow_temp(cgb_handle* h, size_t need) {
    if (need <= h->temp_cap && h->d_temp) return CGB_OK;
    size_t nc = std::max<size_t>(need + need / 2, 1 << 20);
    if (h->d_temp) CK(cudaFree(h->d_temp));
    h->d_temp = nullptr;
    CK(cudaMalloc(&h->d_temp, nc));
    h->temp_cap = nc;
    return CGB_OK;
}

inline int grid_for(const cgb_handle* h, uint64_t n, int block = 256) {
    uint64_t g = (n + block - 1) / block;
    uint64_t cap = (uint64_t)h->num_sms * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

cgb_status ensure_dvcap(cgb_handle* h, uint32_t dv) {
    if (dv <= h->dvcap && h->rec) return CGB_OK;
    uint32_t nc = std::max<uint32_t>(dv + dv / 4 + 1024, h->dvcap * 2);
    uint4* nr = nullptr;
    CK(cudaMalloc(&nr, (size_t)h->nd * nc * sizeof(uint4)));
    CK(cudaMemsetAsync(nr, 0, (size_t)h->nd * nc * sizeof(uint4), h->stream));
    if (h->rec) {
        k_copy_rows<<<grid_for(h, (uint64_t)h->nd * h->dv), 256, 0, h->stream>>>(h->rec, h->dvcap, nr, nc, h->nd,
                                                                                   h->dv);
        LAUNCHED();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaFree(h->rec));
    }
    h->rec = nr;
    h->dvcap = nc;
    h->rb_valid = false;  // the slot table and the bit sets follow the record layout
    // level-sum table: about two slots per vertex, 2^12 to 2^24 slots (16 B each)
    uint32_t slots = 1u << 12;
    while (slots < (1u << 24) && slots < 2ull * nc) slots <<= 1;
    if (slots > h->lsum_slots) {
        if (h->d_lsum) CK(cudaFree(h->d_lsum));
        h->d_lsum = nullptr;
        h->lsum_slots = 0;
        CK(cudaMalloc(&h->d_lsum, (size_t)slots * 2 * sizeof(unsigned long long)));
        h->lsum_slots = slots;
    }
    return CGB_OK;
}

// Dense level sums of every plan with sum_dense, children before parents
// (a position's children sit at higher positions), on the stream.
// The jobs are built (and uploaded) when the arrays move; one launch per
// height runs every job of that height of every plan.
cgb_status dense_level_sums(cgb_handle* h) {
    cgb_status s;
    if ((s = grow(h, h->d_wsum, h->wsum_cap, (size_t)h->n_wsum * h->dvcap)) != CGB_OK) return s;
    if (h->wjobs_for != h->d_wsum) {
        std::vector<std::vector<WsumJob>> by_height;
        for (uint32_t e = 0; e < h->q.qe; ++e) {
            const EdgePlan& P = h->plans[e];
            if (!P.sum_dense) continue;
            const uint32_t s0 = P.sum_from, nc = P.n_core;
            auto arr = [&](uint32_t k) { return h->d_wsum + (size_t)(P.wslot + k - s0) * h->dvcap; };
            uint32_t height[cgb::kMaxQV] = {0};
            for (uint32_t k = nc; k-- > s0;) {  // children sit at higher positions
                WsumJob J;
                std::memset(&J, 0, sizeof(J));
                J.dir = P.bn_dir[P.bn_off[k]];
                J.dvis = P.bn_dvis[P.bn_off[k]];
                for (uint32_t t = nc; t < P.n; ++t)
                    if (((P.sum_tails >> t) & 1u) && P.bn_pos[P.bn_off[t]] == k) {
                        J.tdir[J.nt] = P.bn_dir[P.bn_off[t]];
                        J.tvis[J.nt] = P.bn_dvis[P.bn_off[t]];
                        ++J.nt;
                    }
                for (uint32_t l = k + 1; l < nc; ++l)
                    if (P.bn_pos[P.bn_off[l]] == k) {
                        J.child[J.nch++] = arr(l);
                        height[k] = std::max(height[k], height[l] + 1);
                    }
                J.out = arr(k);
                if (by_height.size() <= height[k]) by_height.resize(height[k] + 1);
                by_height[height[k]].push_back(J);
            }
        }
        std::vector<WsumJob> all;
        h->wjob_level.assign(1, 0);
        for (auto& v : by_height) {
            all.insert(all.end(), v.begin(), v.end());
            h->wjob_level.push_back((uint32_t)all.size());
        }
        if (h->d_wjobs) CK(cudaFree(h->d_wjobs));
        h->d_wjobs = nullptr;
        CK(cudaMalloc(&h->d_wjobs, std::max<size_t>(all.size(), 1) * sizeof(WsumJob)));
        CK(cudaMemcpy(h->d_wjobs, all.data(), all.size() * sizeof(WsumJob), cudaMemcpyHostToDevice));
        h->wjobs_for = h->d_wsum;
    }
    for (size_t lv = 0; lv + 1 < h->wjob_level.size(); ++lv) {
        const uint32_t j0 = h->wjob_level[lv], nj = h->wjob_level[lv + 1] - j0;
        if (!nj) continue;
        const dim3 grid((unsigned)std::max<uint32_t>((uint32_t)h->num_sms * 2, (uint32_t)h->num_sms * 8 / nj), nj);
        k_wsum<<<grid, 256, 0, h->stream>>>(h->rec, h->dvcap, h->pool, h->d_dval, h->dv, h->d_wjobs, j0);
        LAUNCHED();
    }
    CK(cudaGetLastError());
    return CGB_OK;
}

// Level-sum table of a DFS launch (none when no plan uses level sums);
// lsum_clear zeroes it on the stream before each launch.
void lsum_bind(const cgb_handle* h, bool any, DfsArgs& da) {
    const bool on = any && h->d_lsum;
    da.lsum_tab = on ? h->d_lsum : nullptr;
    da.lsum_mask = on ? h->lsum_slots - 1 : 0;
}
cgb_status lsum_clear(cgb_handle* h, const DfsArgs& da) {
    if (da.lsum_tab)
        CK(cudaMemsetAsync(da.lsum_tab, 0, ((size_t)da.lsum_mask + 1) * 2 * sizeof(unsigned long long), h->stream));
    return CGB_OK;
}

// Compacts the pool into pool_alt (allocating or growing it to new_cap words)
// and swaps.  Synchronous.
cgb_status compact_pool(cgb_handle* h, unsigned long long new_cap) {
    const uint64_t n = (uint64_t)h->nd * h->dv;
    if (new_cap < h->pool_cap) new_cap = h->pool_cap;
    uint32_t* sizes = nullptr;
    unsigned long long* offs = nullptr;
    unsigned long long live = 0;
    CK(cudaMalloc(&sizes, std::max<uint64_t>(n, 1) * sizeof(uint32_t)));
    CK(cudaMalloc(&offs, (n + 1) * sizeof(unsigned long long)));
    CK(cudaMemsetAsync(offs, 0, (n + 1) * sizeof(unsigned long long), h->stream));
    if (n > 0) {
        k_rec_sizes<<<grid_for(h, n), 256, 0, h->stream>>>(h->rec, h->dvcap, h->dv, h->nd, sizes, nullptr);
        LAUNCHED();
        k_u32_to_u64<<<grid_for(h, n), 256, 0, h->stream>>>(sizes, offs, n);
        LAUNCHED();
    }
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, offs, offs, (int64_t)n + 1, h->stream));
    if (grow_temp(h, tb) != CGB_OK) return CGB_ERR_OOM;
    CK(cub::DeviceScan::ExclusiveSum(h->d_temp, tb, offs, offs, (int64_t)n + 1, h->stream));
    LAUNCHED();
    CK(cudaMemcpyAsync(&live, offs + n, sizeof(live), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // the destination must hold every live run plus the headroom requested
    while (new_cap < live + (16ull << 20)) new_cap *= 2;
    uint32_t* dst = nullptr;
    if (h->pool_alt && new_cap == h->pool_cap) {
        dst = h->pool_alt;
    } else {
        if (h->pool_alt) CK(cudaFree(h->pool_alt));
        h->pool_alt = nullptr;
        CK(cudaMalloc(&dst, new_cap * sizeof(uint32_t)));
    }
    if (n > 0) {
        k_compact<<<grid_for(h, n * 32), 256, 0, h->stream>>>(h->rec, h->dvcap, h->dv, h->nd, h->pool, dst, offs);
        LAUNCHED();
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaFree(sizes));
    CK(cudaFree(offs));
    uint32_t* old = h->pool;
    h->pool = dst;
    if (new_cap == h->pool_cap) {
        h->pool_alt = old;
    } else {
        CK(cudaFree(old));
        h->pool_alt = nullptr;
        h->pool_cap = new_cap;
    }
    h->h_pool_top = live;
    h->h_live = (long long)live;
    unsigned long long sc[2] = {live, live};
    CK(cudaMemcpyAsync(h->d_scal, sc, sizeof(sc), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CGB_OK;
}

// Ensures the pool can absorb a merge of n_edits edits in the worst case.
cgb_status reserve_pool(cgb_handle* h, uint64_t n_edits) {
    const unsigned long long need = (unsigned long long)std::max<long long>(h->h_live, 0) + 4ull * n_edits + 64;
    if (h->h_pool_top + need <= h->pool_cap) return CGB_OK;
    unsigned long long cap = h->pool_cap;
    while ((unsigned long long)std::max<long long>(h->h_live, 0) + need > cap * 3 / 4) cap = cap * 2;
    return compact_pool(h, cap);
}

// Sorts packed keys in place (alt buffer used as ping-pong); returns sorted pointer.
cgb_status radix_sort(cgb_handle* h, uint64_t*& keys, uint64_t*& alt, uint64_t n, int end_bit) {
    if (n == 0) return CGB_OK;
    cub::DoubleBuffer<uint64_t> db(keys, alt);
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)n, 0, end_bit, h->stream));
    if (grow_temp(h, tb) != CGB_OK) return CGB_ERR_OOM;
    CK(cub::DeviceRadixSort::SortKeys(h->d_temp, tb, db, (int64_t)n, 0, end_bit, h->stream));
    LAUNCHED();
    if (db.Current() != keys) std::swap(keys, alt);
    return CGB_OK;
}

// Run-length segments of du over n sorted entries; offsets by exclusive scan.
cgb_status segment(cgb_handle* h, const uint32_t* du, uint64_t n, uint32_t* run_du, uint32_t* run_len,
                   uint32_t* run_off, int* num_runs) {
    size_t tb = 0;
    CK(cub::DeviceRunLengthEncode::Encode(nullptr, tb, du, run_du, run_len, num_runs, (int64_t)n, h->stream));
    size_t tb2 = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, run_len, run_off, (int64_t)n, h->stream));
    if (grow_temp(h, std::max(tb, tb2)) != CGB_OK) return CGB_ERR_OOM;
    CK(cub::DeviceRunLengthEncode::Encode(h->d_temp, tb, du, run_du, run_len, num_runs, (int64_t)n, h->stream));
    LAUNCHED();
    // scanning n entries (runs beyond num_runs hold garbage but are never read)
    CK(cub::DeviceScan::ExclusiveSum(h->d_temp, tb2, run_len, run_off, (int64_t)n, h->stream));
    LAUNCHED();
    return CGB_OK;
}

// Grow-only per-batch buffers (reallocated only when a batch is larger than any before).
cgb_status ensure_edit_buffers(cgb_handle* h, uint64_t n) {
    if (n <= h->edits_cap && h->d_edits) return CGB_OK;
    size_t nc = std::max<size_t>(n + n / 2, 1 << 16);
    CK(cudaStreamSynchronize(h->stream));
    void* olds[] = {h->d_edits, h->d_edits_alt, h->d_du, h->d_run_du, h->d_run_len, h->d_run_off,
                    h->d_small_runs, h->d_big_runs, h->d_tiny_runs};
    for (void* p : olds) if (p) CK(cudaFree(p));
    CK(cudaMalloc(&h->d_tiny_runs, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_small_runs, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_big_runs, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_edits, nc * sizeof(uint64_t)));
    CK(cudaMalloc(&h->d_edits_alt, nc * sizeof(uint64_t)));
    CK(cudaMalloc(&h->d_du, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_run_du, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_run_len, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_run_off, nc * sizeof(uint32_t)));
    h->edits_cap = nc;
    h->runs_cap = nc;
    return CGB_OK;
}

cgb_status ensure_delta_buffers(cgb_handle* h, uint64_t n) {
    if (n <= h->dkeys_cap && h->d_dkeys) return CGB_OK;
    size_t nc = std::max<size_t>(n + n / 2, 1 << 16);
    CK(cudaStreamSynchronize(h->stream));
    void* olds[] = {h->d_dkeys, h->d_dkeys_alt, h->d_dval, h->d_ddu, h->d_drun_du, h->d_drun_len, h->d_drun_off};
    for (void* p : olds) if (p) CK(cudaFree(p));
    CK(cudaMalloc(&h->d_dkeys, nc * sizeof(uint64_t)));
    CK(cudaMalloc(&h->d_dkeys_alt, nc * sizeof(uint64_t)));
    CK(cudaMalloc(&h->d_dval, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_ddu, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_drun_du, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_drun_len, nc * sizeof(uint32_t)));
    CK(cudaMalloc(&h->d_drun_off, nc * sizeof(uint32_t)));
    h->dkeys_cap = nc;
    h->druns_cap = nc;
    return CGB_OK;
}

// Applies edits = adds0 (ext keys, device) + adds1 + removes to the index.
cgb_status apply_edits(cgb_handle* h, const uint64_t* adds0, uint64_t n0, const uint64_t* adds1, uint64_t n1,
                       const uint64_t* rems, uint64_t n2) {
    const uint64_t n = n0 + n1 + n2;
    if (n == 0) return CGB_OK;
    cgb_status s;
    if ((s = reserve_pool(h, n)) != CGB_OK) return s;
    if ((s = ensure_edit_buffers(h, n)) != CGB_OK) return s;
    PackInfo pi{bits_for(h->dv), h->nd, h->dv, h->mq ? 1u : 0u};
    unsigned int* d_err = (unsigned int*)(h->d_scal + 2);
    if (n0) { k_pack_edits<<<grid_for(h, n0), 256, 0, h->stream>>>(adds0, n0, 0, pi, h->d_edits, d_err, h->d_self); LAUNCHED(); }
    if (n1) { k_pack_edits<<<grid_for(h, n1), 256, 0, h->stream>>>(adds1, n1, 0, pi, h->d_edits + n0, d_err, h->d_self); LAUNCHED(); }
    if (n2) { k_pack_edits<<<grid_for(h, n2), 256, 0, h->stream>>>(rems, n2, 1, pi, h->d_edits + n0 + n1, d_err, h->d_self); LAUNCHED(); }
    CK(cudaGetLastError());
    // valid keys use 2B+6 bits; one more bit makes the all-ones invalid marker sort last
    if ((s = radix_sort(h, h->d_edits, h->d_edits_alt, n, 2 * (int)pi.B + 7)) != CGB_OK) return s;
    k_extract_du<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_edits, n, pi.B + 1, h->d_du);
    LAUNCHED();
    if ((s = segment(h, h->d_du, n, h->d_run_du, h->d_run_len, h->d_run_off, h->d_num_runs)) != CGB_OK) return s;
    MergeArgs ma;
    ma.rec = h->rec;
    ma.dvcap = h->dvcap;
    ma.pool = h->pool;
    ma.pool_top = h->d_scal + 0;
    ma.pool_cap = h->pool_cap;
    ma.live_words = (long long*)(h->d_scal + 1);
    ma.edits = h->d_edits;
    ma.run_du = h->d_run_du;
    ma.run_len = h->d_run_len;
    ma.run_off = h->d_run_off;
    ma.num_runs = h->d_num_runs;
    ma.small_runs = h->d_small_runs;
    ma.big_runs = h->d_big_runs;
    ma.tiny_runs = h->d_tiny_runs;
    ma.list_ctr = h->d_list_ctr;
    ma.B = pi.B;
    ma.err = d_err;
    ma.stats = h->d_stats;
    // bit sets are kept current by the merge once built (k_rb_fill_new, k_rb_edits)
    const bool rb = h->rb_valid && !(h->cfg.flags & CGB_FLAG_NO_RUN_BITS);
    ma.rb_slot = rb ? h->d_rb_slot : nullptr;
    ma.rb_sel = h->d_rb_sel;
    ma.rb_ctr = h->d_rb_ctr;
    ma.rb_new = h->d_rb_new;
    ma.rb_cap = h->rb_cap;
    ma.rb_min_len = h->rb_min_len;
    if (rb) {
        if ((s = grow(h, h->d_rb_new, h->rb_new_cap, std::max<size_t>(h->rb_cap, 1))) != CGB_OK) return s;
        ma.rb_new = h->d_rb_new;
        CK(cudaMemsetAsync(h->d_rb_ctr + 1, 0, sizeof(unsigned int), h->stream));
    }
    CK(cudaMemsetAsync(h->d_list_ctr, 0, 3 * sizeof(unsigned int), h->stream));
    k_merge_classify<<<grid_for(h, n), 256, 0, h->stream>>>(ma);
    LAUNCHED();
    k_merge_tiny<<<grid_for(h, n), 256, 0, h->stream>>>(ma);
    LAUNCHED();
    const int mg = std::max(1, std::min<int>((int)((n * 32 + 255) / 256), h->num_sms * 16));
    k_merge_runs<<<mg, 256, 0, h->stream>>>(ma);
    LAUNCHED();
    // hub runs: one CTA each (at most n / kBigRun of them)
    const int bg = (int)std::max<uint64_t>(1, std::min<uint64_t>(n / kBigRun + 1, (uint64_t)h->num_sms * 2));
    k_merge_big<<<bg, kMergeWarps * 32, 0, h->stream>>>(ma);
    LAUNCHED();
    if (rb) {
        k_rb_fill_new<<<h->num_sms * 4, 256, 0, h->stream>>>(h->rec, h->dvcap, h->pool, h->d_rb_sel, h->d_rb_new,
                                                           h->d_rb_ctr, h->d_rb_bits, h->rb_words);
        LAUNCHED();
        k_rb_edits<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_edits, n, pi.B, h->dvcap, h->d_rb_slot,
                                                           h->d_rb_bits, h->rb_words);
        LAUNCHED();
    }
    CK(cudaGetLastError());
    return CGB_OK;
}

// Builds the run bit sets in full: a slot for every run of at least
// rb_min_len entries while the budget lasts (later merges keep them current).
cgb_status rebuild_run_bits(cgb_handle* h) {
    cgb_status s;
    h->rb_words = (h->dvcap + 31) / 32;
    // as many bit sets as the budget holds, never more than records exist
    h->rb_cap = (uint32_t)std::min<size_t>(kRunBitsBytes / 4 / std::max(h->rb_words, 1u),
                                           std::max<size_t>((size_t)h->nd * h->dvcap, 1));
    const uint32_t cap = h->rb_cap;
    if ((s = grow(h, h->d_rb_slot, h->rb_slot_cap, (size_t)h->nd * h->dvcap)) != CGB_OK) return s;
    if ((s = grow(h, h->d_rb_sel, h->rb_sel_cap, (size_t)cap)) != CGB_OK) return s;
    if ((s = grow(h, h->d_rb_bits, h->rb_bits_cap, (size_t)cap * h->rb_words)) != CGB_OK) return s;
    CK(cudaMemsetAsync(h->d_rb_ctr, 0, 2 * sizeof(unsigned int), h->stream));
    k_rb_select<<<grid_for(h, (uint64_t)h->nd * h->dvcap), 256, 0, h->stream>>>(
        h->rec, h->dvcap, h->nd, h->rb_min_len, cap, h->d_rb_slot, h->d_rb_sel, h->d_rb_ctr);
    LAUNCHED();
    k_rb_zero<<<h->num_sms * 8, 256, 0, h->stream>>>(h->d_rb_bits, h->rb_words, cap, h->d_rb_ctr);
    LAUNCHED();
    k_rb_fill<<<h->num_sms * 8, 256, 0, h->stream>>>(h->rec, h->dvcap, h->pool, h->d_rb_sel, cap, h->d_rb_ctr,
                                                     h->d_rb_bits, h->rb_words);
    LAUNCHED();
    CK(cudaGetLastError());
    h->rb_valid = true;
    return CGB_OK;
}

cgb_status sync_scalars(cgb_handle* h) {
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_scal + 4, h->d_counts, kMaxQE * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaMemcpyAsync(h->h_scal + 4 + kMaxQE, h->d_stats, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaMemcpyAsync(h->h_scal + 12 + kMaxQE, h->d_rb_ctr, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // every slot claimed: rebuild on the next batch, so today's long runs get them
    if (h->rb_valid && (uint32_t)h->h_scal[12 + kMaxQE] >= h->rb_cap) h->rb_valid = false;
    h->h_pool_top = h->h_scal[0];
    h->h_live = (long long)h->h_scal[1];
    return CGB_OK;
}

cgb_status flush_pending(cgb_handle* h) {
    if (h->n_pending == 0) return CGB_OK;
    cgb_status s = apply_edits(h, h->d_pending, h->n_pending, nullptr, 0, nullptr, 0);
    if (s != CGB_OK) return s;
    h->n_pending = 0;
    return sync_scalars(h);
}

}  // namespace

extern "C" {

void cgb_default_config(cgb_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
}

cgb_status cgb_create(const cgb_config* cfg, cgb_handle** out) {
    if (!out) return CGB_ERR_ARG;
    *out = nullptr;
    cgb_handle* h = new cgb_handle();
    if (cfg) h->cfg = *cfg; else cgb_default_config(&h->cfg);
    h->device = h->cfg.device;
    if (const char* e = std::getenv("CGB_RUN_BITS_MIN_LEN")) h->rb_min_len = (uint32_t)std::max(1l, std::atol(e));
    if (const char* e = std::getenv("CGB_PAIR_LANE_MAX")) h->pair_lane_max = (uint32_t)std::max(0l, std::atol(e));
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cgb_status s = fail(h, CGB_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
        *out = h;
        return s;
    }
    if (h->device < 0 || h->device >= ndev) { *out = h; return fail(h, CGB_ERR_ARG, "bad device %d", h->device); }
#define CKC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { *out = h; return fail(h, CGB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); } } while (0)
    CKC(cudaSetDevice(h->device));
    CKC(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    CKC(cudaMalloc(&h->d_scal, 4 * sizeof(unsigned long long)));
    CKC(cudaMemset(h->d_scal, 0, 4 * sizeof(unsigned long long)));
    CKC(cudaMalloc(&h->d_self, sizeof(unsigned int)));
    CKC(cudaMemset(h->d_self, 0, sizeof(unsigned int)));
    CKC(cudaMallocHost(&h->h_scal, (16 + kMaxQE) * sizeof(unsigned long long)));
    CKC(cudaMalloc(&h->d_num_runs, 2 * sizeof(int)));
    CKC(cudaMalloc(&h->d_list_ctr, 3 * sizeof(unsigned int)));
    CKC(cudaMalloc(&h->d_rb_ctr, 2 * sizeof(unsigned int)));
    CKC(cudaMemset(h->d_rb_ctr, 0, 2 * sizeof(unsigned int)));
    CKC(cudaMalloc(&h->d_rev, kMaxDir));
    CKC(cudaMalloc(&h->d_seed, (3 * kMaxQE + 2) * sizeof(uint32_t)));
    CKC(cudaMalloc(&h->d_counts, kMaxQE * sizeof(unsigned long long)));
    CKC(cudaMalloc(&h->d_stats, 8 * sizeof(unsigned long long)));
    CKC(cudaMalloc(&h->d_tasks, (size_t)kTaskCap * kTaskWords * sizeof(uint32_t)));
    CKC(cudaMalloc(&h->d_qctr, 8 * sizeof(unsigned int)));
    CKC(cudaMemset(h->d_tasks, 0, (size_t)kTaskCap * kTaskWords * sizeof(uint32_t)));
    CKC(cudaMalloc(&h->d_qe_dirs, 2 * kMaxQE));
    CKC(cudaMalloc(&h->d_edge_ok, kMaxQE));
    CKC(cudaMalloc(&h->d_plans, sizeof(EdgePlan) * kMaxQE));
    CKC(cudaMalloc(&h->d_vbplans, sizeof(cgb::VbPlan) * kMaxQE));
    CKC(cudaMalloc(&h->d_dir_edge, kMaxDir));
    for (auto& ev : h->ev) CKC(cudaEventCreate(&ev));
#undef CKC
    *out = h;
    return CGB_OK;
}

void cgb_destroy(cgb_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void* ptrs[] = {h->rec, h->pool, h->pool_alt, h->d_scal, h->d_self, h->d_keys_in, h->d_pending, h->d_edits,
                    h->d_edits_alt, h->d_du, h->d_run_du, h->d_run_len, h->d_run_off, h->d_num_runs,
                    h->d_dkeys, h->d_dkeys_alt, h->d_dval, h->d_ddu, h->d_drun_du, h->d_drun_len, h->d_drun_off,
                    h->d_seed, h->d_counts, h->d_stats, h->d_tasks, h->d_qctr, h->d_temp, h->d_qe_dirs, h->d_edge_ok,
                    h->d_vb, h->d_rb_slot, h->d_rb_sel, h->d_rb_bits, h->d_rb_ctr, h->d_rb_new, h->d_small_runs,
                    h->d_big_runs, h->d_tiny_runs, h->d_list_ctr, h->d_rev, h->d_touched, h->d_plans,
                    h->d_vbplans, h->d_dir_edge, h->d_lsum, h->d_wsum, h->d_wjobs};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    for (auto& ev : h->ev)
        if (ev) cudaEventDestroy(ev);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char* cgb_last_error(const cgb_handle* h) { return h ? h->err.c_str() : "null handle"; }

cgb_status cgb_load_query(cgb_handle* h, uint32_t qv, const uint32_t* labels, uint32_t qe, const uint32_t* edges) {
    if (!h || !edges) return CGB_ERR_ARG;
    if (h->have_index) return fail(h, CGB_ERR_STATE, "query must be loaded before the index");
    std::string e = cgb::build_query_meta(qv, qe, edges, labels, h->q);
    if (!e.empty()) return fail(h, CGB_ERR_ARG, "%s", e.c_str());
    h->nd = h->q.nd;
    uint8_t dirs[2 * kMaxQE];
    for (uint32_t i = 0; i < h->q.qe; ++i) { dirs[2 * i] = h->q.qe_dir[i][0]; dirs[2 * i + 1] = h->q.qe_dir[i][1]; }
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpy(h->d_qe_dirs, dirs, 2 * h->q.qe, cudaMemcpyHostToDevice));
    uint8_t rev[kMaxDir];
    std::memset(rev, 255, sizeof(rev));
    for (uint32_t d = 0; d < h->q.nd; ++d) rev[d] = h->q.eidx[h->q.dir_dst[d] * kMaxQV + h->q.dir_src[d]];
    CK(cudaMemcpy(h->d_rev, rev, kMaxDir, cudaMemcpyHostToDevice));
    h->have_query = true;
    return CGB_OK;
}

cgb_status cgb_load_query_file(cgb_handle* h, const char* path) {
    if (!h || !path) return CGB_ERR_ARG;
    std::vector<uint32_t> labels, edges;
    uint32_t qv = 0;
    std::string e = cgb::parse_query_file(path, labels, edges, qv);
    if (!e.empty()) return fail(h, CGB_ERR_IO, "%s", e.c_str());
    return cgb_load_query(h, qv, labels.data(), (uint32_t)(edges.size() / 2), edges.data());
}

uint32_t cgb_query_dir(const cgb_handle* h, uint32_t a, uint32_t b) {
    if (!h || !h->have_query || a >= h->q.qv || b >= h->q.qv) return 255;
    return h->q.eidx[a * kMaxQV + b];
}

cgb_status cgb_build_index(cgb_handle* h, const uint64_t* keys, uint64_t n, uint32_t dv_count) {
    if (!h) return CGB_ERR_ARG;
    if (!h->have_query) return fail(h, CGB_ERR_STATE, "load a query first");
    if (h->have_index) return fail(h, CGB_ERR_STATE, "index already built");
    if (dv_count > CGB_MAX_VID) return fail(h, CGB_ERR_LIMIT, "dv_count %u exceeds 2^27-1", dv_count);
    if (n && !keys) return CGB_ERR_ARG;
    CK(cudaSetDevice(h->device));
    // planner statistics (calig_helper_gamma.cu:304-311): entries and
    // non-empty vertices per direction -> mean run length
    std::vector<uint64_t> card(h->nd, 0), nodes(h->nd, 0);
    {
        std::vector<uint8_t> seen((size_t)h->nd * std::max<uint32_t>(dv_count, 1), 0);
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t d = (uint32_t)(keys[i] >> 59), u = (uint32_t)((keys[i] >> 32) & 0x07FFFFFFu);
            uint32_t v = (uint32_t)keys[i];
            if (d >= h->nd || u >= dv_count || v >= dv_count)
                return fail(h, CGB_ERR_ARG, "key %llu out of range (dir %u u %u v %u, dv %u)",
                            (unsigned long long)i, d, u, v, dv_count);
            card[d]++;
            uint8_t& s = seen[(size_t)d * dv_count + u];
            if (!s) { s = 1; nodes[d]++; }
        }
    }
    float avg[kMaxDir] = {0};
    for (uint32_t d = 0; d < h->nd; ++d) avg[d] = nodes[d] ? (float)card[d] / (float)nodes[d] : 0.f;
    cgb::plan_edges(h->q, avg, h->plans, !(h->cfg.flags & CGB_FLAG_ENUMERATE_TAIL),
                    !(h->cfg.flags & CGB_FLAG_PLAIN_CORE_ORDER), !(h->cfg.flags & CGB_FLAG_NO_SEED_GROUPS),
                    !(h->cfg.flags & CGB_FLAG_WARP_TAIL), !(h->cfg.flags & CGB_FLAG_NO_LEVEL_SUM), true);
    h->n_wsum = 0;
    h->wjobs_for = nullptr;  // the plans changed: rebuild the level-sum jobs
    for (uint32_t e = 0; e < h->q.qe; ++e)
        if (h->plans[e].sum_dense) {
            h->plans[e].wslot = (uint8_t)h->n_wsum;
            h->n_wsum += h->plans[e].n_core - h->plans[e].sum_from;
        }
    CK(cudaMemcpy(h->d_plans, h->plans, sizeof(EdgePlan) * kMaxQE, cudaMemcpyHostToDevice));
    {
        // valid-bit plans from the reference's starting edge
        cgb::select_starting_edge(h->q, card.data(), avg, h->vb_start);
        cgb::VbPlan vbp[kMaxQE];
        std::memset(vbp, 0, sizeof(vbp));
        h->vb_plan_error = cgb::plan_valid_bits(h->q, h->vb_start, vbp);
        if (!h->vb_plan_error.empty() && (h->cfg.flags & (CGB_FLAG_VALID_BITS | CGB_FLAG_MASK_PRUNE)))
            return fail(h, CGB_ERR_ARG, "valid bits: %s", h->vb_plan_error.c_str());
        CK(cudaMemcpy(h->d_vbplans, vbp, sizeof(vbp), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->d_dir_edge, h->q.dir_to_edge, sizeof(h->q.dir_to_edge), cudaMemcpyHostToDevice));
    }

    h->dv = dv_count;
    cgb_status s;
    if ((s = ensure_dvcap(h, std::max<uint32_t>(dv_count, 1))) != CGB_OK) return s;
    unsigned long long cap = h->cfg.pool_words;
    // out-of-place merges write every touched run anew, so the pool carries
    // headroom for many batches between compactions (HBM is plentiful)
    if (cap == 0) cap = std::max<unsigned long long>(4ull * n + (128ull << 20), 192ull << 20);
    CK(cudaMalloc(&h->pool, cap * sizeof(uint32_t)));
    h->pool_cap = cap;
    h->h_pool_top = 0;
    h->h_live = 0;
    CK(cudaMemsetAsync(h->d_scal, 0, 4 * sizeof(unsigned long long), h->stream));
    if ((s = grow(h, h->d_keys_in, h->keys_in_cap, std::max<uint64_t>(n, 1))) != CGB_OK) return s;
    if (n) CK(cudaMemcpyAsync(h->d_keys_in, keys, n * sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream));
    if ((s = apply_edits(h, h->d_keys_in, n, nullptr, 0, nullptr, 0)) != CGB_OK) return s;
    if ((s = sync_scalars(h)) != CGB_OK) return s;
    if (h->h_scal[2]) return fail(h, CGB_ERR_ARG, "invalid keys (error bits %llu)", h->h_scal[2]);
    h->have_index = true;
    return CGB_OK;
}

cgb_status cgb_apply_batch_device(cgb_handle* h, uint32_t dv_count, const uint64_t* ins, uint64_t n_ins,
                                  const uint64_t* del, uint64_t n_del, const uint64_t* delta, uint64_t n_delta,
                                  const uint8_t* edge_ok, void* stream, uint64_t* out_count) {
    if (!h || !out_count) return CGB_ERR_ARG;
    *out_count = 0;
    if (!h->have_index) return fail(h, CGB_ERR_STATE, "build the index first");
    if (dv_count < h->dv) return fail(h, CGB_ERR_ARG, "dv_count must not decrease (%u < %u)", dv_count, h->dv);
    if (dv_count > CGB_MAX_VID) return fail(h, CGB_ERR_LIMIT, "dv_count exceeds 2^27-1");
    if ((n_ins && !ins) || (n_del && !del) || (n_delta && !delta)) return CGB_ERR_ARG;
    if (n_ins > kMaxBatchKeys || n_del > kMaxBatchKeys) return fail(h, CGB_ERR_LIMIT, "edit batch too large");
    if (n_delta > 0xffffffffull) return fail(h, CGB_ERR_LIMIT, "delta batch too large");
    CK(cudaSetDevice(h->device));
    cudaStream_t user = (cudaStream_t)stream;
    if (user && user != h->stream) {
        // order this batch after the caller's prior work on `user`
        CK(cudaEventRecord(h->ev[4], user));
        CK(cudaStreamWaitEvent(h->stream, h->ev[4], 0));
    }
    cgb_status s;
    if ((s = ensure_dvcap(h, dv_count)) != CGB_OK) return s;
    h->dv = dv_count;
    const uint32_t B = bits_for(dv_count);
    PackInfo pi{B, h->nd, dv_count};
    unsigned int* d_err = (unsigned int*)(h->d_scal + 2);
    CK(cudaMemsetAsync(h->d_scal + 2, 0, 2 * sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->d_counts, 0, kMaxQE * sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->d_stats, 0, 8 * sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->d_qctr, 0, 8 * sizeof(unsigned int), h->stream));
    CK(cudaEventRecord(h->ev[0], h->stream));

    // 1. index update: pending delta (add) + ins (add) + del (remove)
    if ((s = apply_edits(h, h->d_pending, h->n_pending, ins, n_ins, del, n_del)) != CGB_OK) return s;
    h->n_pending = 0;
    CK(cudaEventRecord(h->ev[1], h->stream));

    // 2. delta lists
    const bool match = n_delta > 0;
    if (match) {
        if ((s = ensure_delta_buffers(h, n_delta)) != CGB_OK) return s;
        uint32_t* du = h->d_ddu;
        k_pack_delta<<<grid_for(h, n_delta), 256, 0, h->stream>>>(delta, n_delta, pi, h->d_dkeys, d_err, h->d_self);
        LAUNCHED();
        if ((s = radix_sort(h, h->d_dkeys, h->d_dkeys_alt, n_delta, 2 * (int)B + 6)) != CGB_OK) return s;
        k_delta_values<<<grid_for(h, n_delta), 256, 0, h->stream>>>(h->d_dkeys, n_delta, (1ull << B) - 1, h->d_dval);
        LAUNCHED();
        k_extract_du<<<grid_for(h, n_delta), 256, 0, h->stream>>>(h->d_dkeys, n_delta, B, du);
        LAUNCHED();
        if ((s = segment(h, du, n_delta, h->d_drun_du, h->d_drun_len, h->d_drun_off, h->d_num_runs + 1)) != CGB_OK)
            return s;
        k_delta_recs<<<grid_for(h, n_delta), 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                                   h->d_drun_off, h->d_num_runs + 1, B, 0);
        LAUNCHED();
        if (edge_ok) CK(cudaMemcpyAsync(h->d_edge_ok, edge_ok, h->q.qe, cudaMemcpyHostToDevice, h->stream));
        k_seed_ranges<<<1, 32, 0, h->stream>>>(h->d_dkeys, n_delta, B, h->q.qe, h->d_plans, h->d_qe_dirs, h->d_edge_ok,
                                               edge_ok ? 1 : 0, h->d_seed, h->d_seed + kMaxQE);
        LAUNCHED();
        CK(cudaGetLastError());
        const bool vb_on = (h->cfg.flags & (CGB_FLAG_VALID_BITS | CGB_FLAG_MASK_PRUNE)) != 0;
        h->vb_stride = 0;
        if (vb_on) {
            // 2b. valid bits: fill, endpoints from the delta keys, then one
            // launch per indexing-order position (all query edges at once)
            const uint32_t stride = (dv_count + 31) / 32, qv = h->q.qv, qe = h->q.qe;
            if ((s = grow(h, h->d_vb, h->vb_cap, (size_t)qe * qv * stride)) != CGB_OK) return s;
            CK(cudaEventRecord(h->ev[6], h->stream));
            const size_t words = (size_t)qe * qv * stride;
            k_vb_fill<<<(unsigned)std::min<size_t>((words + 255) / 256, (size_t)h->num_sms * 16), 256, 0,
                        h->stream>>>(h->d_vbplans, h->d_vb, qe, qv, stride);
            LAUNCHED();
            k_vb_seed<<<grid_for(h, n_delta), 256, 0, h->stream>>>(h->d_vbplans, h->d_dir_edge, h->d_dkeys, n_delta,
                                                                   B, h->d_vb, qv, stride);
            LAUNCHED();
            const dim3 g((unsigned)std::min<uint32_t>((stride + 7) / 8, (uint32_t)h->num_sms * 8), qe);
            for (uint32_t d = 2; d < qv; ++d) {
                k_vb_depth<<<g, 256, 0, h->stream>>>(h->d_vbplans, h->rec, h->dvcap, h->pool, h->d_dval, dv_count,
                                                     h->d_vb, qv, stride, d);
                LAUNCHED();
            }
            CK(cudaGetLastError());
            h->vb_stride = stride;
        }
        CK(cudaEventRecord(h->ev[2], h->stream));

        // 2c. bit sets of the long old runs (this batch's index): built in full
        // once (and after the record table grows), since then kept current by
        // every merge; rebuilt when the slots ran out so that the longest runs
        // of today's index hold them
        const bool rb_on = !(h->cfg.flags & CGB_FLAG_NO_RUN_BITS);
        if (rb_on && !h->rb_valid && (s = rebuild_run_bits(h)) != CGB_OK) return s;

        // 3. matching
        DfsArgs da;
        da.rec = h->rec;
        da.dvcap = h->dvcap;
        da.pool = h->pool;
        da.dval = h->d_dval;
        da.dkeys = h->d_dkeys;
        da.B = B;
        da.qe = h->q.qe;
        da.seed_lo = h->d_seed;
        da.seed_pre = h->d_seed + kMaxQE;
        da.counts = h->d_counts;
        da.work_next = (unsigned int*)(h->d_scal + 3);
        da.err = d_err;
        da.stats = h->d_stats;
        da.tasks = h->d_tasks;
        da.task_cap = kTaskCap;
        da.qctr = h->d_qctr;
        do {  // the tag's epoch field must never be 0 (the ring starts zeroed)
            ++h->dfs_epoch;
        } while ((h->dfs_epoch & 0xfffffu) == 0);
        da.epoch = h->dfs_epoch;
        da.force_split = (h->cfg.flags & CGB_FLAG_FORCE_SPLIT) ? 1u : 0u;
        da.num_shards = h->cfg.num_shards ? h->cfg.num_shards : 1u;
        da.steal = (h->cfg.flags & CGB_FLAG_NO_STEAL) ? 0u : 1u;
        da.tail_cache = (h->cfg.flags & CGB_FLAG_NO_TAIL_CACHE) ? 0u : 1u;
        da.pair_lane_max = h->pair_lane_max;
        da.shard = h->cfg.shard_index < da.num_shards ? h->cfg.shard_index : 0u;
        da.self_seen = h->d_self;
        da.vb = (h->cfg.flags & CGB_FLAG_MASK_PRUNE) ? h->d_vb : nullptr;
        da.vb_stride = h->vb_stride;
        da.qv = h->q.qv;
        da.rb_slot = rb_on ? h->d_rb_slot : nullptr;
        da.rb_bits = h->d_rb_bits;
        da.rb_words = h->rb_words;
        da.plans = h->d_plans;
        da.epoch_ptr = nullptr;
        da.touched = nullptr;
        const bool footprint = (h->cfg.flags & CGB_FLAG_FOOTPRINT) != 0;
        const uint64_t nrec = (uint64_t)h->nd * h->dvcap;
        if (footprint) {
            if ((s = grow(h, h->d_touched, h->touched_cap, (size_t)(nrec + 31) / 32)) != CGB_OK) return s;
            CK(cudaMemsetAsync(h->d_touched, 0, ((nrec + 31) / 32) * sizeof(uint32_t), h->stream));
            da.touched = h->d_touched;
        }
        da.budget_ns = h->cfg.dfs_budget_ms ? (unsigned long long)h->cfg.dfs_budget_ms * 1000000ull
                                            : 600ull * 1000000000ull;
        // persistent grid: exactly the blocks that can be resident at once
        if (h->dfs_occupancy == 0) {
            int occ = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_dfs_count<false>, kDfsWarps * 32, 0));
            h->dfs_occupancy = std::max(occ, 1);
        }
        int bps = h->dfs_occupancy;
        if (h->cfg.dfs_blocks_per_sm) bps = std::min(bps, (int)h->cfg.dfs_blocks_per_sm);
        bool any_sum = false;
        for (uint32_t e = 0; e < h->q.qe; ++e)
            any_sum |= (h->plans[e].sum_from != 0 && !h->plans[e].sum_dense) || h->plans[e].memo_from != 0;
        da.wsum = nullptr;
        if (h->n_wsum && !da.vb && da.tail_cache) {
            if ((s = dense_level_sums(h)) != CGB_OK) return s;
            da.wsum = h->d_wsum;
        }
        lsum_bind(h, any_sum, da);
        if ((s = lsum_clear(h, da)) != CGB_OK) return s;
        bool uses_sums = false;
        for (uint32_t e = 0; e < h->q.qe; ++e)
            uses_sums |= h->plans[e].sum_from != 0 || h->plans[e].tail_lane == 2 || h->plans[e].memo_from != 0 ||
                         h->plans[e].pair_last != 0;
        const dim3 grid(h->num_sms * bps), block(kDfsWarps * 32);
        if (footprint && uses_sums) k_dfs_count<false, true, true><<<grid, block, 0, h->stream>>>(da);
        else if (footprint) k_dfs_count<false, true, false><<<grid, block, 0, h->stream>>>(da);
        else if (uses_sums) k_dfs_count<false, false, true><<<grid, block, 0, h->stream>>>(da);
        else k_dfs_count<false, false, false><<<grid, block, 0, h->stream>>>(da);
        LAUNCHED();
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->ev[3], h->stream));
        if (footprint) {  // stats[4] := the launch's footprint (bytes of distinct records and lists)
            CK(cudaMemsetAsync(h->d_stats + 4, 0, sizeof(unsigned long long), h->stream));
            k_footprint<<<grid_for(h, nrec), 256, 0, h->stream>>>(h->rec, nrec, h->d_touched, h->d_stats + 4);
            LAUNCHED();
        }

        // 4. clear delta records; this delta becomes the pending merge-back
        k_delta_recs<<<grid_for(h, n_delta), 256, 0, h->stream>>>(h->rec, h->dvcap, h->d_drun_du, h->d_drun_len,
                                                                   h->d_drun_off, h->d_num_runs + 1, B, 1);
        LAUNCHED();
        if ((s = grow(h, h->d_pending, h->pending_cap, n_delta)) != CGB_OK) return s;
        CK(cudaMemcpyAsync(h->d_pending, delta, n_delta * sizeof(uint64_t), cudaMemcpyDeviceToDevice, h->stream));
        h->n_pending = n_delta;
    } else {
        CK(cudaEventRecord(h->ev[2], h->stream));
        CK(cudaEventRecord(h->ev[3], h->stream));
    }
    CK(cudaEventRecord(h->ev[5], h->stream));
    if ((s = sync_scalars(h)) != CGB_OK) return s;
    float t01 = 0, t12 = 0, t23 = 0, t03 = 0;
    cudaEventElapsedTime(&t01, h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&t12, h->ev[1], h->ev[2]);
    cudaEventElapsedTime(&t23, h->ev[2], h->ev[3]);
    cudaEventElapsedTime(&t03, h->ev[0], h->ev[5]);
    h->last_vb_ms = 0;
    if (h->vb_stride) cudaEventElapsedTime(&h->last_vb_ms, h->ev[6], h->ev[2]);
    h->last_t[0] = t01; h->last_t[1] = t12; h->last_t[2] = t23; h->last_t[3] = t03;
    for (int i = 0; i < 8; ++i) h->last_stats[i] = h->h_scal[4 + kMaxQE + i];
    if (h->h_scal[2]) {
        h->n_pending = 0;
        h->rb_valid = false;  // a rejected batch may have left runs and bit sets apart
        cgb_status st = (h->h_scal[2] & 24u) ? CGB_ERR_TIMEOUT : (h->h_scal[2] & 4u) ? CGB_ERR_OOM : CGB_ERR_ARG;
        return fail(h, st,
                    "batch rejected: error bits %llu (1/2 = key out of range, 4 = pool exhausted, "
                    "8 = matching exceeded its time budget, 16 = a queued task was never published)",
                    h->h_scal[2]);
    }
    uint64_t total = 0;
    for (uint32_t e = 0; e < h->q.qe; ++e) { h->last_counts[e] = h->h_scal[4 + e]; total += h->h_scal[4 + e]; }
    for (int i = 0; i < 8; ++i) h->last_stats[i] = h->h_scal[4 + kMaxQE + i];
    *out_count = total;
    if (h->cfg.flags & CGB_FLAG_NO_MERGE_BACK_DEFER) {
        if ((s = flush_pending(h)) != CGB_OK) return s;
    }
    return CGB_OK;
}

cgb_status cgb_apply_batch(cgb_handle* h, uint32_t dv_count, const uint64_t* ins, uint64_t n_ins,
                           const uint64_t* del, uint64_t n_del, const uint64_t* delta, uint64_t n_delta,
                           const uint8_t* edge_ok, uint64_t* out_count) {
    if (!h || !out_count) return CGB_ERR_ARG;
    if ((n_ins && !ins) || (n_del && !del) || (n_delta && !delta)) return CGB_ERR_ARG;
    // bounded before the sum below, which must not wrap
    if (n_ins > kMaxBatchKeys || n_del > kMaxBatchKeys || n_delta > kMaxBatchKeys)
        return fail(h, CGB_ERR_LIMIT, "batch too large");
    CK(cudaSetDevice(h->device));
    const uint64_t n = n_ins + n_del + n_delta;
    cgb_status s;
    if ((s = grow(h, h->d_keys_in, h->keys_in_cap, std::max<uint64_t>(n, 1))) != CGB_OK) return s;
    uint64_t* d = h->d_keys_in;
    if (n_ins) CK(cudaMemcpyAsync(d, ins, n_ins * 8, cudaMemcpyHostToDevice, h->stream));
    if (n_del) CK(cudaMemcpyAsync(d + n_ins, del, n_del * 8, cudaMemcpyHostToDevice, h->stream));
    if (n_delta) CK(cudaMemcpyAsync(d + n_ins + n_del, delta, n_delta * 8, cudaMemcpyHostToDevice, h->stream));
    return cgb_apply_batch_device(h, dv_count, d, n_ins, d + n_ins, n_del, d + n_ins + n_del, n_delta, edge_ok,
                                  nullptr, out_count);
}

cgb_status cgb_last_edge_counts(const cgb_handle* h, uint64_t* out, uint32_t cap) {
    if (!h || !out) return CGB_ERR_ARG;
    for (uint32_t e = 0; e < cap && e < h->q.qe; ++e) out[e] = h->last_counts[e];
    return CGB_OK;
}

cgb_status cgb_last_timings(const cgb_handle* h, float* t4) {
    if (!h || !t4) return CGB_ERR_ARG;
    for (int i = 0; i < 4; ++i) t4[i] = h->last_t[i];
    return CGB_OK;
}

uint64_t cgb_kernel_launches(const cgb_handle* h) { return h ? h->launches : 0; }

cgb_status cgb_last_stats(const cgb_handle* h, uint64_t* out8) {
    if (!h || !out8) return CGB_ERR_ARG;
    for (int i = 0; i < 8; ++i) out8[i] = h->last_stats[i];
    return CGB_OK;
}

void* cgb_stream(const cgb_handle* h) { return h ? (void*)h->stream : nullptr; }

cgb_status cgb_plan_anchor(const cgb_handle* h, uint32_t ei, uint32_t* qvertex) {
    if (!h || !qvertex) return CGB_ERR_ARG;
    if (!h->have_index) return CGB_ERR_STATE;
    if (ei >= h->q.qe) return CGB_ERR_ARG;
    *qvertex = h->plans[ei].vs[0];
    return CGB_OK;
}

cgb_status cgb_plan_info(const cgb_handle* h, uint32_t ei, uint32_t* out4) {
    if (!h || !out4) return CGB_ERR_ARG;
    if (!h->have_index) return CGB_ERR_STATE;
    if (ei >= h->q.qe) return CGB_ERR_ARG;
    const EdgePlan& P = h->plans[ei];
    out4[0] = P.n_core;
    out4[1] = P.sum_from;
    out4[2] = P.sum_dense;
    out4[3] = P.tail_lane | (uint32_t)P.memo_from << 8 | (uint32_t)P.memo_pos << 16;
    return CGB_OK;
}

cgb_status cgb_check_symmetry(cgb_handle* h, uint64_t* n_asym) {
    if (!h || !n_asym) return CGB_ERR_ARG;
    *n_asym = 0;
    if (!h->have_index) return fail(h, CGB_ERR_STATE, "no index");
    CK(cudaSetDevice(h->device));
    cgb_status s;
    if ((s = flush_pending(h)) != CGB_OK) return s;
    unsigned long long* d_bad = nullptr;
    CK(cudaMalloc(&d_bad, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), h->stream));
    const uint64_t n = (uint64_t)h->nd * h->dv;
    if (n) {
        k_asymmetry<<<grid_for(h, n * 32), 256, 0, h->stream>>>(h->rec, h->dvcap, h->dv, h->nd, h->pool, h->d_rev, d_bad);
        LAUNCHED();
    }
    unsigned long long bad = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_bad);
    CK(e);
    *n_asym = bad;
    return CGB_OK;
}

cgb_status cgb_starting_edge(const cgb_handle* h, uint32_t* out2) {
    if (!h || !out2) return CGB_ERR_ARG;
    if (!h->have_index) return CGB_ERR_STATE;
    out2[0] = h->vb_start[0];
    out2[1] = h->vb_start[1];
    return CGB_OK;
}

cgb_status cgb_valid_bits(cgb_handle* h, uint32_t* out, uint64_t cap, uint64_t* n_words, float* ms) {
    if (!h || !n_words) return CGB_ERR_ARG;
    *n_words = 0;
    if (!h->vb_stride) return fail(h, CGB_ERR_STATE, "no valid bits: enable CGB_FLAG_VALID_BITS and match a batch");
    const uint64_t n = (uint64_t)h->q.qe * h->q.qv * h->vb_stride;
    *n_words = n;
    if (ms) *ms = h->last_vb_ms;
    if (!out) return CGB_OK;
    if (cap < n) return fail(h, CGB_ERR_ARG, "buffer holds %llu of %llu words", (unsigned long long)cap,
                             (unsigned long long)n);
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(out, h->d_vb, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CGB_OK;
}

cgb_status cgb_read_index(cgb_handle* h, uint64_t* out, uint64_t cap, uint64_t* n_out) {
    if (!h || !n_out) return CGB_ERR_ARG;
    if (!h->have_index) return fail(h, CGB_ERR_STATE, "no index");
    CK(cudaSetDevice(h->device));
    cgb_status s;
    if ((s = flush_pending(h)) != CGB_OK) return s;
    const uint64_t n = (uint64_t)h->nd * h->dv;
    uint32_t* lens = nullptr;
    unsigned long long* offs = nullptr;
    CK(cudaMalloc(&lens, std::max<uint64_t>(n, 1) * sizeof(uint32_t)));
    CK(cudaMalloc(&offs, (n + 1) * sizeof(unsigned long long)));
    CK(cudaMemsetAsync(offs, 0, (n + 1) * sizeof(unsigned long long), h->stream));
    if (n) {
        k_rec_sizes<<<grid_for(h, n), 256, 0, h->stream>>>(h->rec, h->dvcap, h->dv, h->nd, nullptr, lens);
        LAUNCHED();
        k_u32_to_u64<<<grid_for(h, n), 256, 0, h->stream>>>(lens, offs, n);
        LAUNCHED();
    }
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, offs, offs, (int64_t)n + 1, h->stream));
    if ((s = grow_temp(h, tb)) != CGB_OK) return s;
    CK(cub::DeviceScan::ExclusiveSum(h->d_temp, tb, offs, offs, (int64_t)n + 1, h->stream));
    LAUNCHED();
    unsigned long long total = 0;
    CK(cudaMemcpyAsync(&total, offs + n, sizeof(total), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n_out = total;
    if (out && cap >= total && total > 0) {
        uint64_t* d_out = nullptr;
        CK(cudaMalloc(&d_out, total * sizeof(uint64_t)));
        k_dump<<<grid_for(h, n * 32), 256, 0, h->stream>>>(h->rec, h->dvcap, h->dv, h->nd, h->pool, offs, d_out);
        LAUNCHED();
        CK(cudaMemcpyAsync(out, d_out, total * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaFree(d_out));
    } else if (out && cap < total) {
        CK(cudaFree(lens));
        CK(cudaFree(offs));
        return fail(h, CGB_ERR_ARG, "output capacity %llu < %llu", (unsigned long long)cap, total);
    }
    CK(cudaFree(lens));
    CK(cudaFree(offs));
    return CGB_OK;
}

}  // extern "C"

#include "multiquery.cuh"
