// Exclusive prefix sum of 32-bit counts into 64-bit offsets (subsystem (d)):
// the per-point list offsets of the neighbour table.  Replaces the
// reference's key sort + kernelUniqueKeys + second sort + host range
// stitching (GPU.cu:863-980, kernel.cu:79-105, GPU.cu:1143-1214): with exact
// per-point counts the table is laid out by one scan.
//
// Three phases over tiles of kScanTile elements: tile sums, a single-block
// scan of the tile sums, and the tile-local scans with the tile prefix added.
// Thread t of a tile owns its elements [16 t, 16 t + 16): four 16-byte loads
// when the arrays are 16-byte aligned, one block-wide scan of the 256 thread
// sums, then 16 sequential outputs per thread.
// out has n+1 entries; out[n] is the total.
#include <cstdint>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>

#include "../../include/gpuselfjoin.h"
#include "gsj_kernels.h"
#include "gsj_scan.h"

namespace gsj {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint64_t kScanTile = (uint64_t)kScanThreads * kScanItems;
constexpr int kTileSumThreads = 1024;  // the single block scanning the tile sums

__device__ __forceinline__ unsigned long long warp_incl_scan(unsigned long long x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Block-wide exclusive scan of one value per thread (THREADS threads);
// returns the exclusive prefix and writes the block total to *total.
template <int THREADS>
__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long* total) {
    __shared__ unsigned long long wsum[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long inc = warp_incl_scan(v, lane);
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < THREADS / 32 ? wsum[lane] : 0ull;
        w = warp_incl_scan(w, lane);
        if (lane < THREADS / 32) wsum[lane] = w;
    }
    __syncthreads();
    const unsigned long long before = warp ? wsum[warp - 1] : 0ull;
    *total = wsum[THREADS / 32 - 1];
    __syncthreads();
    return before + inc - v;
}

// Elements [e0, e0 + kScanItems) (zero past n); vec: in is 16-byte aligned.
__device__ __forceinline__ void load_items(const uint32_t* __restrict__ in, uint64_t e0, uint64_t n, bool vec,
                                           uint32_t (&v)[kScanItems]) {
    if (vec && e0 + kScanItems <= n) {
        const uint4* p = reinterpret_cast<const uint4*>(in + e0);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) {
            const uint4 x = p[q];
            v[4 * q] = x.x;
            v[4 * q + 1] = x.y;
            v[4 * q + 2] = x.z;
            v[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++) v[i] = e0 + (uint64_t)i < n ? in[e0 + i] : 0u;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const uint32_t* __restrict__ in, uint64_t n, bool vec,
                                                            unsigned long long* __restrict__ tsum) {
    const uint64_t e0 = blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_items(in, e0, n, vec, v);
    unsigned long long s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) s += v[i];
    unsigned long long tot;
    block_excl_scan<kScanThreads>(s, &tot);
    if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

// One block: tsum[i] becomes the exclusive prefix of the tile sums, tsum[ntiles]
// the total.  Each thread takes 4 consecutive sums per round of 4096.
__global__ void __launch_bounds__(kTileSumThreads) k_scan_tile_sums(unsigned long long* __restrict__ tsum,
                                                                    uint64_t ntiles) {
    unsigned long long carry = 0;
    for (uint64_t b0 = 0; b0 < ntiles; b0 += 4u * kTileSumThreads) {
        const uint64_t i0 = b0 + 4u * threadIdx.x;
        unsigned long long v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = i0 + j < ntiles ? tsum[i0 + j] : 0ull;
        unsigned long long tot;
        unsigned long long ex = block_excl_scan<kTileSumThreads>(v[0] + v[1] + v[2] + v[3], &tot);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (i0 + j < ntiles) tsum[i0 + j] = carry + ex;
            ex += v[j];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) tsum[ntiles] = carry;
}

// OutT is uint64_t (list offsets) or uint32_t (slot offsets, digit offsets:
// the caller guarantees that the total fits).  vin / vout: in / out are
// 16-byte aligned (a thread's 16 elements are then 4 aligned vectors in and
// 4 or 8 out).
template <typename OutT>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const uint32_t* __restrict__ in, uint64_t n, bool vin,
                                                            const unsigned long long* __restrict__ tsum,
                                                            uint64_t ntiles, OutT* __restrict__ out, bool vout) {
    const uint64_t e0 = blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_items(in, e0, n, vin, v);
    unsigned long long s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) s += v[i];
    unsigned long long tot;
    unsigned long long pre = tsum[blockIdx.x] + block_excl_scan<kScanThreads>(s, &tot);
    OutT o[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        o[i] = (OutT)pre;
        pre += v[i];
    }
    if (vout && e0 + kScanItems <= n) {
        if constexpr (sizeof(OutT) == 8) {
            ulonglong2* p = reinterpret_cast<ulonglong2*>(out + e0);
#pragma unroll
            for (int q = 0; q < kScanItems / 2; q++) p[q] = make_ulonglong2(o[2 * q], o[2 * q + 1]);
        } else {
            uint4* p = reinterpret_cast<uint4*>(out + e0);
#pragma unroll
            for (int q = 0; q < kScanItems / 4; q++) p[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++)
            if (e0 + (uint64_t)i < n) out[e0 + i] = o[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = (OutT)tsum[ntiles];
}

size_t scan_u32_u64_temp_bytes(uint64_t n) { return ((n + kScanTile - 1) / kScanTile + 1) * sizeof(unsigned long long); }

template <typename OutT>
static cudaError_t scan_any(const uint32_t* in, OutT* out, uint64_t n, void* temp, cudaStream_t st) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    unsigned long long* tsum = static_cast<unsigned long long*>(temp);
    if (ntiles == 0) return cudaMemsetAsync(out, 0, sizeof(OutT), st);
    const bool vin = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
    const bool vout = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    k_tile_sums<<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, vin, tsum);
    k_scan_tile_sums<<<1, kTileSumThreads, 0, st>>>(tsum, ntiles);
    k_tile_scan<OutT><<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, vin, tsum, ntiles, out, vout);
    return cudaGetLastError();
}

cudaError_t scan_u32_u64(const uint32_t* in, uint64_t* out, uint64_t n, void* temp, cudaStream_t st) {
    return scan_any<uint64_t>(in, out, n, temp, st);
}

cudaError_t scan_u32_u32(const uint32_t* in, uint32_t* out, uint64_t n, void* temp, cudaStream_t st) {
    return scan_any<uint32_t>(in, out, n, temp, st);
}

// ---------------------------------------------------------------- launch shapes
namespace {
struct OccKey {
    int dev;
    const void* kern;
    int threads;
    size_t smem;
    bool operator<(const OccKey& o) const {
        if (dev != o.dev) return dev < o.dev;
        if (kern != o.kern) return kern < o.kern;
        if (threads != o.threads) return threads < o.threads;
        return smem < o.smem;
    }
};
std::mutex g_occ_mu;
std::map<OccKey, int> g_occ;
}  // namespace

cudaError_t blocks_per_sm(const void* kern, int threads, size_t smem, int* per_sm) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const OccKey key{dev, kern, threads, smem};
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(key);
        if (it != g_occ.end()) {
            *per_sm = it->second;
            return cudaSuccess;
        }
    }
    int api = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&api, kern, threads, smem);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    int smem_sm = 0, resv = 0, regs_sm = 0, thr_sm = 0;
    if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess &&
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) == cudaSuccess) {
        const long long blk_smem = (long long)smem + resv + (long long)fa.sharedSizeBytes;
        const long long warp_regs = ((long long)fa.numRegs * 32 + 255) / 256 * 256;
        const long long blk_regs = warp_regs * ((threads + 31) / 32);
        long long fit = (long long)thr_sm / threads;
        if (blk_smem > 0 && smem_sm / blk_smem < fit) fit = smem_sm / blk_smem;
        if (blk_regs > 0 && regs_sm / blk_regs < fit) fit = regs_sm / blk_regs;
        if (fit > api) api = (int)fit;
    } else {
        cudaGetLastError();
    }
    *per_sm = api;
    std::lock_guard<std::mutex> lk(g_occ_mu);
    g_occ[key] = api;
    return cudaSuccess;
}

// ---------------------------------------------------------------- no allocation
// Scratch of gsj_list_offsets_noalloc: the per-tile sums of the scan live in
// a fixed array in the library's device image instead of memory obtained
// from cudaMalloc.  64 KiB hold the sums of 8191 tiles (plus the total), so
// one call covers up to 8191 * 4096 = 33,550,336 counts.  Every device that
// loads the library keeps this array until the process exits.
constexpr size_t kNoAllocScratchBytes = 64u * 1024u;
constexpr uint64_t kNoAllocMaxTiles = kNoAllocScratchBytes / sizeof(unsigned long long) - 1u;
constexpr uint64_t kNoAllocMaxCounts = kNoAllocMaxTiles * kScanTile;
static __device__ __align__(256) unsigned long long g_noalloc_tile_sums[kNoAllocScratchBytes / sizeof(unsigned long long)];

int report_error(int code, const std::string& msg);

}  // namespace gsj

namespace {
// Device address of g_noalloc_tile_sums, looked up once per device.  On the
// host the symbol name only stands for the device array; a kernel must be
// given the address that cudaGetSymbolAddress returns for the current device.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};
}  // namespace

extern "C" int gsj_list_offsets_noalloc(const uint32_t* d_counts, uint64_t n, uint64_t* d_offsets, void* stream) {
    using namespace gsj;
    if (!d_offsets || (n && !d_counts)) return report_error(GSJ_ERR_INVALID, "null device pointer");
    if (n > kNoAllocMaxCounts)
        return report_error(GSJ_ERR_INVALID, "gsj_list_offsets_noalloc: " + std::to_string(n) +
                                                 " counts exceed the fixed scratch limit of " +
                                                 std::to_string(kNoAllocMaxCounts));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return report_error(GSJ_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return report_error(GSJ_ERR_INVALID, "gsj_list_offsets_noalloc: device ordinal " + std::to_string(dev) +
                                                 " beyond the " + std::to_string(kMaxDevices) +
                                                 " devices whose scratch address is cached");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_tile_sums);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                return report_error(GSJ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
        }
        scratch = g_noalloc_addr[dev];
    }
    // Every tile sum the scan reads is written earlier in the same call, so the
    // previous call's contents need no clearing.
    e = scan_u32_u64(d_counts, d_offsets, n, scratch, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return report_error(GSJ_ERR_CUDA, std::string("list offsets scan: ") + cudaGetErrorString(e));
    return GSJ_OK;
}
