// Stable LSD radix sort and run-length encoding (subsystems (a) and (d)).
//
// Replaces the library sorts of the index build: the reference builds its
// grid on the host with a std::set and per-cell vectors (main.cu:690-857) and
// sorts its result pairs with thrust::sort_by_key (GPU.cu:863-880).  Here the
// (cell id, point id) keys are sorted on the device by this sort, which orders
// points by cell with ties in ascending point id - the reference's per-cell
// order (main.cu:741-763).
//
// Each digit pass (8-bit digits, or 9-bit where that saves a pass) is a
// reduce-then-scan over tiles of kSortTile keys:
//   k_radix_hist     per-tile digit counts, written digit-major
//   scan_u32_u32     exclusive scan of the counts: the global offset of each
//                    (digit, tile) run
//   k_radix_scatter  the tile is ranked stably in shared memory (per-warp
//                    match_any groups, in index order), then written out in
//                    sorted order, so each digit's run of the tile is stored
//                    by consecutive threads to consecutive addresses.
// Stability: keys are ranked by (warp, round, lane) = their index order within
// the tile, and tiles are laid out in order within each digit.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_scan.h"
#include "gsj_sort.h"

namespace gsj {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;                           // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;    // keys per tile
constexpr int kWarpKeys = kSortTile / kSortWarps;       // keys per warp (8 rounds of 32)
constexpr int kMaxBins = 512;  // digits of 8 or 9 bits
static_assert(kMaxBins % kSortThreads == 0, "whole digits per thread in the tile prefix");

__device__ __forceinline__ unsigned lanemask_lt_s() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename K, int BINS>
__device__ __forceinline__ uint32_t digit_of(K key, int shift) {
    return (uint32_t)(key >> shift) & (uint32_t)(BINS - 1);
}

template <typename K, int BINS>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const K* __restrict__ keys, uint64_t n, int shift,
                                                             uint32_t* __restrict__ hist, uint32_t ntiles) {
    __shared__ uint32_t h[kSortWarps][BINS];
    for (int i = threadIdx.x; i < kSortWarps * BINS; i += kSortThreads) (&h[0][0])[i] = 0u;
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int i = 0; i < kSortItems; i++) {
        const uint64_t e = base + (uint64_t)i * kSortThreads + threadIdx.x;
        if (e < n) atomicAdd(&h[warp][digit_of<K, BINS>(keys[e], shift)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < BINS; d += kSortThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) s += h[w][d];
        hist[(uint64_t)d * ntiles + blockIdx.x] = s;
    }
}

template <typename K, bool VALS, int BINS>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const K* __restrict__ kin,
                                                                const uint32_t* __restrict__ vin,
                                                                K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                                uint64_t n, int shift,
                                                                const uint32_t* __restrict__ offs, uint32_t ntiles) {
    extern __shared__ __align__(16) unsigned char sort_smem[];
    K* skeys = reinterpret_cast<K*>(sort_smem);
    uint32_t* svals = reinterpret_cast<uint32_t*>(sort_smem + sizeof(K) * kSortTile);
    constexpr int DPT = BINS / kSortThreads;       // digits per thread in the tile prefix
    __shared__ uint32_t wcnt[kSortWarps][BINS];    // per-warp digit counts, then their exclusive prefix
    __shared__ uint32_t tile_off[BINS];            // exclusive prefix of the tile's digit counts
    __shared__ uint32_t gbase[BINS];               // global offset of the digit's run minus tile_off
    __shared__ uint32_t wsum[kSortWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = lanemask_lt_s();
    for (int i = threadIdx.x; i < kSortWarps * BINS; i += kSortThreads) (&wcnt[0][0])[i] = 0u;
    __syncthreads();

    const uint64_t base = (uint64_t)blockIdx.x * kSortTile + (uint64_t)warp * kWarpKeys;
    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];  // digit << 16 | rank within the warp's keys of that digit
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
        const uint64_t e = base + (uint64_t)r * 32u + lane;
        const bool valid = e < n;
        key[r] = valid ? kin[e] : K(0);
        if (VALS) val[r] = valid ? vin[e] : 0u;
        const uint32_t d = valid ? digit_of<K, BINS>(key[r], shift) : (uint32_t)BINS;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t c = 0;
        if (lane == leader && valid) {
            c = wcnt[warp][d];
            wcnt[warp][d] = c + (uint32_t)__popc(peers);
        }
        c = __shfl_sync(0xffffffffu, c, leader);
        rank[r] = (d << 16) | (c + (uint32_t)__popc(peers & lt));
        __syncwarp();
    }
    __syncthreads();
    // per digit (DPT consecutive digits a thread): prefix over the warps, then
    // over the digits
    {
        const int d0 = threadIdx.x * DPT;
        uint32_t pd[DPT];
        uint32_t p = 0;
#pragma unroll
        for (int dd = 0; dd < DPT; dd++) {
            uint32_t q = 0;
#pragma unroll
            for (int w = 0; w < kSortWarps; w++) {
                const uint32_t t = wcnt[w][d0 + dd];
                wcnt[w][d0 + dd] = q;
                q += t;
            }
            pd[dd] = q;
            p += q;
        }
        uint32_t x = p;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        uint32_t before = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++)
            if (w < warp) before += wsum[w];
        uint32_t ex = before + x - p;
#pragma unroll
        for (int dd = 0; dd < DPT; dd++) {
            const int d = d0 + dd;
            tile_off[d] = ex;
            gbase[d] = offs[(uint64_t)d * ntiles + blockIdx.x] - ex;  // modulo 2^32, re-added below
            ex += pd[dd];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
        const uint32_t d = rank[r] >> 16;
        if (d < (uint32_t)BINS) {
            const uint32_t idx = tile_off[d] + wcnt[warp][d] + (rank[r] & 0xffffu);
            skeys[idx] = key[r];
            if (VALS) svals[idx] = val[r];
        }
    }
    __syncthreads();
    const uint64_t tbase = (uint64_t)blockIdx.x * kSortTile;
    const uint32_t cnt = (uint32_t)((n - tbase) < (uint64_t)kSortTile ? (n - tbase) : (uint64_t)kSortTile);
    for (uint32_t i = threadIdx.x; i < cnt; i += kSortThreads) {
        const K kk = skeys[i];
        const uint32_t g = gbase[digit_of<K, BINS>(kk, shift)] + i;
        kout[g] = kk;
        if (VALS) vout[g] = svals[i];
    }
}

template <typename K>
__global__ void k_run_flags(const K* __restrict__ keys, uint64_t n, uint32_t* __restrict__ flags) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

template <typename K>
__global__ void k_run_compact(const K* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ flags,
                              const uint32_t* __restrict__ pos, uint64_t* __restrict__ run_key,
                              uint32_t* __restrict__ run_start) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n && flags[i]) {
        run_key[pos[i]] = (uint64_t)keys[i];
        run_start[pos[i]] = (uint32_t)i;
    }
    if (i == 0) run_start[pos[n]] = (uint32_t)n;
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

inline uint64_t tiles_of(uint64_t n) { return (n + kSortTile - 1) / kSortTile; }

}  // namespace

size_t radix_sort_temp_bytes(uint64_t n) {
    const uint64_t nt = tiles_of(n);
    const size_t hist = (size_t)kMaxBins * nt * sizeof(uint32_t);
    const size_t hist_al = (2 * hist + sizeof(uint32_t) + 255) / 256 * 256;
    return hist_al + scan_u32_u64_temp_bytes((uint64_t)kMaxBins * nt) + 256;
}

template <typename K>
cudaError_t radix_sort(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int begin_bit,
                       int end_bit, void* temp, bool* in_alt, int* launches, cudaStream_t st) {
    *in_alt = false;
    if (n <= 1 || begin_bit >= end_bit) return cudaSuccess;
    if (n >= (1ull << 32)) return cudaErrorInvalidValue;
    const uint64_t nt = tiles_of(n);
    const size_t hist_bytes = (size_t)kMaxBins * nt * sizeof(uint32_t);
    uint32_t* hist = static_cast<uint32_t*>(temp);
    uint32_t* offs = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(temp) + hist_bytes);
    void* stemp = static_cast<unsigned char*>(temp) + (2 * hist_bytes + sizeof(uint32_t) + 255) / 256 * 256;
    const size_t smem = sizeof(K) * kSortTile + (vals ? sizeof(uint32_t) * kSortTile : 0);
    cudaError_t e;
    for (const void* f : {(const void*)k_radix_scatter<K, true, 256>, (const void*)k_radix_scatter<K, false, 256>,
                          (const void*)k_radix_scatter<K, true, 512>, (const void*)k_radix_scatter<K, false, 512>}) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    // digits of 8 bits, or of 9 where that saves a pass (25 key bits: 9 + 8 + 8)
    const int B = end_bit - begin_bit;
    const int p8 = (B + 7) / 8, p9 = (B + 8) / 9;
    const int passes = p9 < p8 ? p9 : p8;
    const int nine = p9 < p8 ? B - 8 * passes : 0;  // passes with 9-bit digits
    K *ki = keys, *ko = keys_alt;
    uint32_t *vi = vals, *vo = vals_alt;
    bool alt = false;
    int shift = begin_bit;
    for (int pass = 0; pass < passes; pass++) {
        const bool wide = pass < nine;
        const uint32_t bins = wide ? 512u : 256u;
        if (wide) k_radix_hist<K, 512><<<(unsigned)nt, kSortThreads, 0, st>>>(ki, n, shift, hist, (uint32_t)nt);
        else k_radix_hist<K, 256><<<(unsigned)nt, kSortThreads, 0, st>>>(ki, n, shift, hist, (uint32_t)nt);
        e = scan_u32_u32(hist, offs, (uint64_t)bins * nt, stemp, st);
        if (e != cudaSuccess) return e;
        if (wide) {
            if (vals) k_radix_scatter<K, true, 512><<<(unsigned)nt, kSortThreads, smem, st>>>(ki, vi, ko, vo, n, shift, offs, (uint32_t)nt);
            else k_radix_scatter<K, false, 512><<<(unsigned)nt, kSortThreads, smem, st>>>(ki, nullptr, ko, nullptr, n, shift, offs, (uint32_t)nt);
        } else {
            if (vals) k_radix_scatter<K, true, 256><<<(unsigned)nt, kSortThreads, smem, st>>>(ki, vi, ko, vo, n, shift, offs, (uint32_t)nt);
            else k_radix_scatter<K, false, 256><<<(unsigned)nt, kSortThreads, smem, st>>>(ki, nullptr, ko, nullptr, n, shift, offs, (uint32_t)nt);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (launches) *launches += 5;
        shift += wide ? 9 : 8;
        K* tk = ki;
        ki = ko;
        ko = tk;
        uint32_t* tv = vi;
        vi = vo;
        vo = tv;
        alt = !alt;
    }
    *in_alt = alt;
    return cudaSuccess;
}

template cudaError_t radix_sort<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint64_t, int, int, void*,
                                          bool*, int*, cudaStream_t);
template cudaError_t radix_sort<uint64_t>(uint64_t*, uint64_t*, uint32_t*, uint32_t*, uint64_t, int, int, void*,
                                          bool*, int*, cudaStream_t);

// flags[n + 1], then pos[n + 1] from the next 16-byte boundary (the scan moves
// whole 16-byte vectors only between aligned arrays), then the scan's scratch.
static uint64_t runs_pos_offset(uint64_t n) { return (n + 1 + 3) & ~3ull; }

static size_t runs_arrays_bytes(uint64_t n) {
    return ((runs_pos_offset(n) + n + 1) * sizeof(uint32_t) + 255) / 256 * 256;
}

size_t runs_temp_bytes(uint64_t n) { return runs_arrays_bytes(n) + scan_u32_u64_temp_bytes(n) + 256; }

template <typename K>
cudaError_t run_length(const K* keys, uint64_t n, uint64_t* run_key, uint32_t* run_start, uint32_t* d_nruns,
                       void* temp, cudaStream_t st) {
    if (n == 0) return cudaMemsetAsync(d_nruns, 0, sizeof(uint32_t), st);
    uint32_t* flags = static_cast<uint32_t*>(temp);
    uint32_t* pos = flags + runs_pos_offset(n);
    void* stemp = static_cast<unsigned char*>(temp) + runs_arrays_bytes(n);
    k_run_flags<K><<<blocks_for(n, 256), 256, 0, st>>>(keys, n, flags);
    cudaError_t e = scan_u32_u32(flags, pos, n, stemp, st);
    if (e != cudaSuccess) return e;
    k_run_compact<K><<<blocks_for(n, 256), 256, 0, st>>>(keys, n, flags, pos, run_key, run_start);
    e = cudaMemcpyAsync(d_nruns, pos + n, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template cudaError_t run_length<uint32_t>(const uint32_t*, uint64_t, uint64_t*, uint32_t*, uint32_t*, void*,
                                          cudaStream_t);
template cudaError_t run_length<uint64_t>(const uint64_t*, uint64_t, uint64_t*, uint32_t*, uint32_t*, void*,
                                          cudaStream_t);

}  // namespace gsj
