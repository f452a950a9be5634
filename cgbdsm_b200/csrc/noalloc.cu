// Index update without device allocation: cgb_merge_keys_noalloc.
//
// Some callers cannot allocate device memory: code that runs while a CUDA
// graph is being captured (cudaMalloc is not a capturable operation), hosts
// that hand out all device memory through their own allocator or cap it per
// tenant, and plugins that are not allowed to grow a process's footprint after
// start-up.  For them this entry point applies one batch of index edits with
// set semantics, out = (old U ins) \ del, where the index is given as one flat
// sorted key array.  The caller passes inputs and outputs in device memory;
// every temporary (packed edits, radix-sort double buffer, sort and scan temp
// space, per-tile counts) lives in one file-scope static device array of
// kScratchBytes, which every GPU that loads this library holds until the
// process exits.
//
// Set-up: the scratch array's device address is obtained once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on
// that device (and again if that device's context was reset since); make that
// first call before any stream capture.
// Sharing: every call uses the same array and it keeps the last call's
// contents; calls whose work overlaps on the GPU (different streams, or
// different host threads, on one device) race on it and must be ordered by
// the caller.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cstdint>
#include <mutex>

#include "cgbdsm.h"

namespace {

constexpr uint64_t kMaxEdits = CGB_NOALLOC_MAX_EDITS;
constexpr uint32_t kTile = 2048;           // merged positions per block and step
constexpr uint32_t kMaxTiles = 1u << 16;   // per-tile counts kept in scratch
constexpr uint64_t kMaxMerged = (uint64_t)kMaxTiles * kTile;  // old keys + edits per call (2^27)
constexpr size_t kSortTempBytes = 6u << 20;
constexpr size_t kScanTempBytes = 1u << 20;
// layout: [edits A][edits B][sort temp][scan temp][tile counts + 1][error word]
constexpr size_t kOffA = 0;
constexpr size_t kOffB = kOffA + kMaxEdits * 8;
constexpr size_t kOffSort = kOffB + kMaxEdits * 8;
constexpr size_t kOffScan = kOffSort + kSortTempBytes;
constexpr size_t kOffTiles = kOffScan + kScanTempBytes;
constexpr size_t kOffErr = kOffTiles + (size_t)(kMaxTiles + 1) * 8;
constexpr size_t kScratchBytes = kOffErr + 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;

__device__ __forceinline__ bool unpack_ext(uint64_t k, uint32_t dv, uint32_t& d, uint32_t& u, uint32_t& v) {
    d = (uint32_t)(k >> 59);
    u = (uint32_t)((k >> 32) & 0x07FFFFFFu);
    v = (uint32_t)k;
    return u < dv && v < dv;
}

// edits -> ((d,u,v) << 1 | op), invalid keys -> all ones + error word
__global__ void k_na_pack(const uint64_t* ins, uint64_t n_ins, const uint64_t* del, uint64_t n_del, uint32_t dv,
                          uint32_t B, uint64_t* out, unsigned int* err) {
    const uint64_t n = n_ins + n_del;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const bool is_del = i >= n_ins;
        const uint64_t k = is_del ? del[i - n_ins] : ins[i];
        uint32_t d, u, v;
        if (unpack_ext(k, dv, d, u, v)) {
            out[i] = (((uint64_t)d << (2 * B)) | ((uint64_t)u << B) | v) << 1 | (is_del ? 1u : 0u);
        } else {
            out[i] = ~0ull;
            atomicOr(err, 1u);
        }
    }
}

struct Merged {
    const uint64_t* X;  // old keys, external format, sorted
    uint64_t xl;
    const uint64_t* Y;  // packed edits, sorted
    uint64_t yl;
    uint32_t B;
    __device__ __forceinline__ uint64_t xv(uint64_t i) const {  // old key -> packed (d,u,v)
        const uint64_t k = X[i];
        return ((k >> 59) << (2 * B)) | (((k >> 32) & 0x07FFFFFFull) << B) | (k & 0xFFFFFFFFull);
    }
    __device__ __forceinline__ uint64_t yv(uint64_t j) const { return Y[j] >> 1; }
    // merge-path split of diagonal k: X wins ties (old before add before remove)
    __device__ uint64_t split(uint64_t k) const {
        uint64_t lo = k > yl ? k - yl : 0, hi = k < xl ? k : xl;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (xv(mid) <= yv(k - 1 - mid)) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    }
};

__device__ __forceinline__ uint64_t to_ext(uint64_t p, uint32_t B) {
    const uint64_t vm = (1ull << B) - 1ull;
    return ((p >> (2 * B)) << 59) | (((p >> B) & vm) << 32) | (p & vm);
}

constexpr uint32_t kThreads = 256;
constexpr uint32_t kItems = kTile / kThreads;  // merged entries per thread
constexpr uint64_t kEnd = ~0ull;               // beyond every packed value

// Tiled merge path.  Block b merges the entries [b * kTile, (b + 1) * kTile):
// two splits per tile (its ends), the tile's part of X and Y staged in
// shared memory (X converted to the packed order, Y with its op bit), then
// each thread splits its own kItems entries inside the tile and merges them
// serially.  An entry is emitted when it is the last of its value group and
// not a remove.  Pass 1 (kWrite = false) stores each tile's emitted count;
// pass 2 writes the entries at the scanned tile offsets.
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_na_merge(Merged M, unsigned long long* tile_cnt,
                                                      const unsigned long long* tile_off, uint64_t* out) {
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    __shared__ uint64_t s_e[kTile];    // [0, nx): X (packed), [nx, nx + ny): Y (packed << 1 | op)
    __shared__ uint64_t s_split[3];    // i0, i1, value of the entry after the tile
    __shared__ typename Scan::TempStorage s_scan;
    const uint64_t total = M.xl + M.yl;
    const uint64_t k0 = (uint64_t)blockIdx.x * kTile;
    const uint64_t k1 = k0 + kTile < total ? k0 + kTile : total;
    if (threadIdx.x == 0) s_split[0] = M.split(k0);
    if (threadIdx.x == 32) {
        const uint64_t i1 = M.split(k1), j1 = k1 - i1;
        s_split[1] = i1;
        uint64_t nxt = kEnd;
        if (i1 < M.xl) nxt = M.xv(i1);
        if (j1 < M.yl && M.yv(j1) < nxt) nxt = M.yv(j1);
        s_split[2] = nxt;
    }
    __syncthreads();
    const uint64_t i0 = s_split[0], i1 = s_split[1];
    const uint64_t j0 = k0 - i0;
    const uint32_t nx = (uint32_t)(i1 - i0), nt = (uint32_t)(k1 - k0), ny = nt - nx;
    for (uint32_t t = threadIdx.x; t < nt; t += kThreads)
        s_e[t] = t < nx ? M.xv(i0 + t) : M.Y[j0 + (t - nx)];
    __syncthreads();
    const uint64_t* sx = s_e;
    const uint64_t* sy = s_e + nx;
    // this thread's entries [a0, a1) of the tile
    const uint32_t a0 = min(threadIdx.x * kItems, nt), a1 = min(a0 + kItems, nt);
    uint32_t lo = a0 > ny ? a0 - ny : 0, hi = a0 < nx ? a0 : nx;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sx[mid] <= (sy[a0 - 1 - mid] >> 1)) lo = mid + 1;
        else hi = mid;
    }
    uint32_t i = lo, j = a0 - lo;
    uint64_t val[kItems + 1];
    bool rem[kItems];
#pragma unroll
    for (uint32_t q = 0; q <= kItems; ++q) {
        if (a0 + q < a1 || (q > 0 && a0 + q == a1 && a1 < nt)) {
            const bool fx = i < nx && (j >= ny || sx[i] <= (sy[j] >> 1));
            if (fx) { val[q] = sx[i++]; if (q < kItems) rem[q] = false; }
            else { val[q] = sy[j] >> 1; if (q < kItems) rem[q] = (sy[j] & 1ull) != 0; ++j; }
        } else {
            val[q] = (a0 + q == nt) ? s_split[2] : kEnd;
            if (q < kItems) rem[q] = true;
        }
    }
    uint32_t cnt = 0;
#pragma unroll
    for (uint32_t q = 0; q < kItems; ++q)
        cnt += (a0 + q < a1 && val[q] != val[q + 1] && !rem[q] && val[q] != (~0ull >> 1)) ? 1u : 0u;
    uint32_t before = 0, all = 0;
    Scan(s_scan).ExclusiveSum(cnt, before, all);
    if (!kWrite) {
        if (threadIdx.x == 0) tile_cnt[blockIdx.x] = all;
        return;
    }
    uint64_t o = tile_off[blockIdx.x] + before;
#pragma unroll
    for (uint32_t q = 0; q < kItems; ++q)
        if (a0 + q < a1 && val[q] != val[q + 1] && !rem[q] && val[q] != (~0ull >> 1)) out[o++] = to_ext(val[q], M.B);
}

__global__ void k_na_finish(const unsigned long long* tile_off, uint32_t tiles, const unsigned int* err,
                            uint64_t* out_n) {
    *out_n = (*err) ? ~0ull : (uint64_t)tile_off[tiles];
}

inline uint32_t bits_for(uint32_t dv) {
    uint32_t b = 1;
    while ((1ull << b) < (uint64_t)dv) ++b;
    return b;
}

// Device address of the scratch array for the current device and context.
// The host-side name g_noalloc_scratch is only a stand-in: the address must
// be asked for with cudaGetSymbolAddress, with the device current.  It is
// looked up again when the device's context changes (after a
// cudaDeviceReset), which the driver's context id shows; that check makes no
// allocation and no stream operation.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

bool current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_ctx = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_ctx = (CtxGetCurrentFn)f1;
            get_id = (CtxGetIdFn)f2;
        }
    }
    void* ctx = nullptr;
    if (!get_ctx || !get_id || get_ctx(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0;
}

unsigned char* scratch_address(int dev) {
    static unsigned char* addr[64] = {};
    static unsigned long long ctx_id[64] = {};
    unsigned long long id = 0;
    const bool have_id = current_context_id(&id);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!addr[dev] || (have_id && id != ctx_id[dev])) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return nullptr;
        addr[dev] = (unsigned char*)p;
        ctx_id[dev] = have_id ? id : 0;
    }
    return addr[dev];
}

}  // namespace

extern "C" cgb_status cgb_merge_keys_noalloc(const uint64_t* old_keys_device, uint64_t n_old,
                                             const uint64_t* ins_device, uint64_t n_ins,
                                             const uint64_t* del_device, uint64_t n_del, uint32_t dv_count,
                                             uint64_t* out_device, uint64_t* out_n_device, void* stream) {
    if (!out_device || !out_n_device || (n_old && !old_keys_device) || (n_ins && !ins_device) ||
        (n_del && !del_device))
        return CGB_ERR_ARG;
    // more edits than the scratch array holds, or more merged keys than its
    // tile counts cover (tested without forming sums that could wrap)
    if (n_ins > kMaxEdits || n_del > kMaxEdits - n_ins) return CGB_ERR_LIMIT;
    if (n_old > kMaxMerged - (n_ins + n_del)) return CGB_ERR_LIMIT;
    if (dv_count == 0 || dv_count > CGB_MAX_VID) return CGB_ERR_ARG;
    // an error left by earlier work on this thread is reported, not cleared
    if (cudaPeekAtLastError() != cudaSuccess) return CGB_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CGB_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t B = bits_for(dv_count);
    const uint64_t ne = n_ins + n_del;
    const uint64_t total = n_old + ne;
    const uint64_t ntiles = total ? (total + kTile - 1) / kTile : 1;
    // temporary sizes first (host-only queries): every limit is checked before
    // any work is enqueued
    size_t sort_need = 0, scan_need = 0;
    if (ne) {
        cub::DoubleBuffer<uint64_t> probe(nullptr, nullptr);
        if (cub::DeviceRadixSort::SortKeys(nullptr, sort_need, probe, (int64_t)ne, 0, (int)(2 * B + 7), st) !=
            cudaSuccess)
            return CGB_ERR_CUDA;
        if (sort_need > kSortTempBytes) return CGB_ERR_LIMIT;
    }
    {
        unsigned long long* none = nullptr;
        if (cub::DeviceScan::ExclusiveSum(nullptr, scan_need, none, none, (int64_t)ntiles + 1, st) != cudaSuccess)
            return CGB_ERR_CUDA;
        if (scan_need > kScanTempBytes) return CGB_ERR_LIMIT;
    }
    unsigned char* scratch = scratch_address(dev);
    if (!scratch) return CGB_ERR_CUDA;
    uint64_t* A = (uint64_t*)(scratch + kOffA);
    uint64_t* Bf = (uint64_t*)(scratch + kOffB);
    unsigned long long* tiles = (unsigned long long*)(scratch + kOffTiles);
    unsigned int* err = (unsigned int*)(scratch + kOffErr);
    if (cudaMemsetAsync(err, 0, sizeof(unsigned int), st) != cudaSuccess) return CGB_ERR_CUDA;
    if (ne) {
        k_na_pack<<<(int)((ne + 255) / 256 < 4096 ? (ne + 255) / 256 : 4096), 256, 0, st>>>(
            ins_device, n_ins, del_device, n_del, dv_count, B, A, err);
        if (cudaGetLastError() != cudaSuccess) return CGB_ERR_CUDA;
        cub::DoubleBuffer<uint64_t> db(A, Bf);
        if (cub::DeviceRadixSort::SortKeys(scratch + kOffSort, sort_need, db, (int64_t)ne, 0, (int)(2 * B + 7), st) !=
            cudaSuccess)
            return CGB_ERR_CUDA;
        A = db.Current();
    }
    Merged M{old_keys_device, n_old, A, ne, B};
    if (total) {
        k_na_merge<false><<<(unsigned)ntiles, kThreads, 0, st>>>(M, tiles, nullptr, nullptr);
        if (cudaGetLastError() != cudaSuccess) return CGB_ERR_CUDA;
    } else if (cudaMemsetAsync(tiles, 0, sizeof(unsigned long long), st) != cudaSuccess) {
        return CGB_ERR_CUDA;
    }
    if (cudaMemsetAsync(tiles + ntiles, 0, sizeof(unsigned long long), st) != cudaSuccess) return CGB_ERR_CUDA;
    if (cub::DeviceScan::ExclusiveSum(scratch + kOffScan, scan_need, tiles, tiles, (int64_t)ntiles + 1, st) !=
        cudaSuccess)
        return CGB_ERR_CUDA;
    if (total) {
        k_na_merge<true><<<(unsigned)ntiles, kThreads, 0, st>>>(M, nullptr, tiles, out_device);
        if (cudaGetLastError() != cudaSuccess) return CGB_ERR_CUDA;
    }
    k_na_finish<<<1, 1, 0, st>>>(tiles, (uint32_t)ntiles, err, out_n_device);
    return cudaGetLastError() == cudaSuccess ? CGB_OK : CGB_ERR_CUDA;
}
