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
// that device; make that first call before any stream capture.
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
unsigned char* g_scratch_addr[64] = {};

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
    // element k of the merge: value, whether it is a remove, and the next value
    __device__ void at(uint64_t k, uint64_t& val, bool& rem, bool& last) const {
        uint64_t i = split(k), j = k - i;
        const bool fx = i < xl && (j >= yl || xv(i) <= yv(j));
        if (fx) { val = xv(i); rem = false; ++i; }
        else { val = yv(j); rem = (Y[j] & 1ull) != 0; ++j; }
        last = true;
        if (k + 1 < xl + yl) {
            const uint64_t nv = (i < xl && (j >= yl || xv(i) <= yv(j))) ? xv(i) : yv(j);
            last = nv != val;
        }
    }
};

__device__ __forceinline__ uint64_t to_ext(uint64_t p, uint32_t B) {
    const uint64_t vm = (1ull << B) - 1ull;
    return ((p >> (2 * B)) << 59) | (((p >> B) & vm) << 32) | (p & vm);
}

// pass 1: per-tile number of emitted keys; pass 2: write them at scanned offsets
template <bool kWrite>
__global__ void k_na_merge(Merged M, uint64_t per_tile, unsigned long long* tile_cnt,
                           const unsigned long long* tile_off, uint64_t* out) {
    __shared__ unsigned int s_warp[32];
    const uint64_t total = M.xl + M.yl;
    const uint64_t t0 = (uint64_t)blockIdx.x * per_tile;
    const uint64_t t1 = t0 + per_tile < total ? t0 + per_tile : total;
    unsigned long long base = kWrite ? tile_off[blockIdx.x] : 0;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t k0 = t0; k0 < t1; k0 += blockDim.x) {
        const uint64_t k = k0 + threadIdx.x;
        bool emit = false;
        uint64_t val = 0;
        if (k < t1) {
            bool rem, last;
            M.at(k, val, rem, last);
            emit = last && !rem && val != (~0ull >> 1);
        }
        const unsigned int bal = __ballot_sync(0xffffffffu, emit);
        if (lane == 0) s_warp[wid] = __popc(bal);
        __syncthreads();
        unsigned int before = 0, sum = 0;
        for (uint32_t w2 = 0; w2 < blockDim.x / 32; ++w2) {
            if (w2 < wid) before += s_warp[w2];
            sum += s_warp[w2];
        }
        if (kWrite && emit) out[base + before + __popc(bal & ((1u << lane) - 1u))] = to_ext(val, M.B);
        base += sum;
        __syncthreads();
    }
    if (!kWrite && threadIdx.x == 0) tile_cnt[blockIdx.x] = base;
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

}  // namespace

extern "C" cgb_status cgb_merge_keys_noalloc(const uint64_t* old_keys_device, uint64_t n_old,
                                             const uint64_t* ins_device, uint64_t n_ins,
                                             const uint64_t* del_device, uint64_t n_del, uint32_t dv_count,
                                             uint64_t* out_device, uint64_t* out_n_device, void* stream) {
    if (!out_device || !out_n_device || (n_old && !old_keys_device) || (n_ins && !ins_device) ||
        (n_del && !del_device))
        return CGB_ERR_ARG;
    // more edits than the scratch array holds (tested without forming n_ins + n_del, which could wrap)
    if (n_ins > kMaxEdits || n_del > kMaxEdits - n_ins) return CGB_ERR_LIMIT;
    if (dv_count == 0 || dv_count > CGB_MAX_VID) return CGB_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CGB_ERR_CUDA;
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[dev]) {
            // the host-side symbol is only a stand-in: the device address must be asked for
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CGB_ERR_CUDA;
            g_scratch_addr[dev] = (unsigned char*)p;
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t* A = (uint64_t*)(scratch + kOffA);
    uint64_t* Bf = (uint64_t*)(scratch + kOffB);
    unsigned long long* tiles = (unsigned long long*)(scratch + kOffTiles);
    unsigned int* err = (unsigned int*)(scratch + kOffErr);
    const uint32_t B = bits_for(dv_count);
    const uint64_t ne = n_ins + n_del;
    if (cudaMemsetAsync(err, 0, sizeof(unsigned int), st) != cudaSuccess) return CGB_ERR_CUDA;
    if (ne) {
        k_na_pack<<<(int)((ne + 255) / 256 < 4096 ? (ne + 255) / 256 : 4096), 256, 0, st>>>(
            ins_device, n_ins, del_device, n_del, dv_count, B, A, err);
        cub::DoubleBuffer<uint64_t> db(A, Bf);
        size_t need = 0;
        if (cub::DeviceRadixSort::SortKeys(nullptr, need, db, (int64_t)ne, 0, (int)(2 * B + 7), st) != cudaSuccess)
            return CGB_ERR_CUDA;
        if (need > kSortTempBytes) return CGB_ERR_LIMIT;
        if (cub::DeviceRadixSort::SortKeys(scratch + kOffSort, need, db, (int64_t)ne, 0, (int)(2 * B + 7), st) !=
            cudaSuccess)
            return CGB_ERR_CUDA;
        A = db.Current();
    }
    const uint64_t total = n_old + ne;
    uint64_t ntiles = (total + kTile - 1) / kTile;
    if (ntiles == 0) ntiles = 1;
    if (ntiles > kMaxTiles) ntiles = kMaxTiles;
    const uint64_t per_tile = (total + ntiles - 1) / ntiles ? (total + ntiles - 1) / ntiles : 1;
    Merged M{old_keys_device, n_old, A, ne, B};
    k_na_merge<false><<<(unsigned)ntiles, 256, 0, st>>>(M, per_tile, tiles, nullptr, nullptr);
    size_t scan_need = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, scan_need, tiles, tiles, (int64_t)ntiles + 1, st) != cudaSuccess)
        return CGB_ERR_CUDA;
    if (scan_need > kScanTempBytes) return CGB_ERR_LIMIT;
    if (cudaMemsetAsync(tiles + ntiles, 0, sizeof(unsigned long long), st) != cudaSuccess) return CGB_ERR_CUDA;
    if (cub::DeviceScan::ExclusiveSum(scratch + kOffScan, scan_need, tiles, tiles, (int64_t)ntiles + 1, st) !=
        cudaSuccess)
        return CGB_ERR_CUDA;
    k_na_merge<true><<<(unsigned)ntiles, 256, 0, st>>>(M, per_tile, nullptr, tiles, out_device);
    k_na_finish<<<1, 1, 0, st>>>(tiles, (uint32_t)ntiles, err, out_n_device);
    return cudaGetLastError() == cudaSuccess ? CGB_OK : CGB_ERR_CUDA;
}
