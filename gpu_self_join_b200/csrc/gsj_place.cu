// Pair keys -> neighbour table (subsystem (d)).
//
// The reference sorts its (query id, neighbour id) result pairs by key with
// thrust::sort_by_key and finds the list boundaries with kernelUniqueKeys and
// a second sort (GPU.cu:863-980, kernel.cu:79-105).  Here the warp, tile and
// screen paths emit packed keys (query id << shift | neighbour id) in an
// arbitrary order, and the table is built without a global sort:
//   k_pair_count   list lengths: one atomic per run of equal queries in a warp
//   scan           list offsets
//   k_pair_place   each neighbour id goes to its query's list (a per-query
//                  cursor, one atomic per run of equal queries in a warp)
//   list sort      every list ascending, which also makes the table
//                  independent of the emission order: a warp per list held in
//                  registers (bitonic network) up to kWarpSortMax entries, a
//                  CTA per list (LSD radix passes through a scratch copy) above.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_kernels.h"
#include "gsj_place.h"
#include "gsj_scan.h"

namespace gsj {

namespace {

constexpr unsigned long long kPadKey = ~0ull;  // unused entries of reserved blocks
constexpr uint32_t kWarpSortMax = 256;         // 8 entries per lane
constexpr int kBlockSortThreads = 256;

__device__ __forceinline__ unsigned lanemask_lt_p() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void k_pair_count(const unsigned long long* __restrict__ keys, uint64_t nkeys, uint32_t shift,
                             uint32_t* __restrict__ counts) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < nkeys; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const unsigned long long kk = i < nkeys ? keys[i] : kPadKey;
        const bool v = kk != kPadKey;
        const uint32_t q = v ? (uint32_t)(kk >> shift) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, q);
        if (v && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&counts[q], (uint32_t)__popc(peers));
    }
}

__global__ void k_pair_place(const unsigned long long* __restrict__ keys, uint64_t nkeys, uint32_t shift,
                             const uint64_t* __restrict__ offsets, uint32_t* __restrict__ cursor,
                             uint32_t* __restrict__ table, uint64_t cap, uint32_t* __restrict__ err) {
    const uint64_t mask = (1ull << shift) - 1ull;
    const unsigned lt = lanemask_lt_p();
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < nkeys; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const unsigned long long kk = i < nkeys ? keys[i] : kPadKey;
        const bool v = kk != kPadKey;
        const uint32_t q = v ? (uint32_t)(kk >> shift) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, q);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (v && lane == leader) base = atomicAdd(&cursor[q], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (v) {
            const uint64_t pos = offsets[q] + base + (uint32_t)__popc(peers & lt);
            if (pos < offsets[q + 1] && pos < cap) table[pos] = (uint32_t)(kk & mask);
            else *err = 1u;
        }
    }
}

// Bitonic sort of one list of up to 32*E entries held as E registers per lane
// (entry r*32 + lane), padded with 0xffffffff; lists whose length lies in
// (lo, 32*E] are sorted by this instantiation.
template <int E>
__global__ void __launch_bounds__(256) k_list_sort_warp(uint32_t* __restrict__ table,
                                                        const uint64_t* __restrict__ offsets, uint32_t nlists,
                                                        uint32_t lo) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    constexpr uint32_t P = 32u * E;
    for (uint32_t l0 = gw * 32u; l0 < nlists; l0 += nw * 32u) {
        // the lengths of 32 consecutive lists, then the lists of this size class one by one
        const uint32_t li = l0 + (uint32_t)lane;
        uint64_t b = 0, e = 0;
        if (li < nlists) {
            b = offsets[li];
            e = offsets[li + 1];
        }
        const uint64_t len = e - b;
        unsigned mine = __ballot_sync(FULL, li < nlists && len > lo && len <= P);
        while (mine) {
            const int j = __ffs(mine) - 1;
            mine &= mine - 1u;
            const uint64_t base = __shfl_sync(FULL, b, j);
            const uint32_t n = (uint32_t)__shfl_sync(FULL, len, j);
            uint32_t v[E];
#pragma unroll
            for (int r = 0; r < E; r++) {
                const uint32_t i = (uint32_t)r * 32u + (uint32_t)lane;
                v[r] = i < n ? table[base + i] : 0xffffffffu;
            }
#pragma unroll
            for (uint32_t k = 2; k <= P; k <<= 1) {
#pragma unroll
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
#pragma unroll
                    for (int r = 0; r < E; r++) {
                        const uint32_t i = (uint32_t)r * 32u + (uint32_t)lane;
                        const bool up = (i & k) == 0u;
                        if (jj >= 32u) {
                            const int pr = r ^ (int)(jj >> 5);
                            if (pr > r) {
                                const uint32_t a = v[r], c = v[pr];
                                const bool sw = up ? (a > c) : (a < c);
                                v[r] = sw ? c : a;
                                v[pr] = sw ? a : c;
                            }
                        } else {
                            const uint32_t o = __shfl_xor_sync(FULL, v[r], (int)jj);
                            const bool lower = (i & jj) == 0u;
                            v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < E; r++) {
                const uint32_t i = (uint32_t)r * 32u + (uint32_t)lane;
                if (i < n) table[base + i] = v[r];
            }
        }
    }
}

// One CTA per list longer than kWarpSortMax: LSD radix passes of 8 bits over
// the list's entries (ids below 2^bits), alternating between the table and
// the same range of `scratch`; the pass count is even, so the sorted list ends
// in the table.  Each pass: a digit histogram of the whole list, then its
// tiles in order, each ranked stably (per-warp match_any groups in index
// order) and written at the running offset of its digit.
__global__ void __launch_bounds__(kBlockSortThreads) k_list_sort_block(uint32_t* __restrict__ table,
                                                                       uint32_t* __restrict__ scratch,
                                                                       const uint64_t* __restrict__ offsets,
                                                                       const uint32_t* __restrict__ long_lists,
                                                                       uint32_t nlong, int passes) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t run[256];
    __shared__ uint32_t wcnt[kBlockSortThreads / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = lanemask_lt_p();
    for (uint32_t li = blockIdx.x; li < nlong; li += gridDim.x) {
        const uint32_t l = long_lists[li];
        const uint64_t b = offsets[l];
        const uint32_t n = (uint32_t)(offsets[l + 1] - b);
        uint32_t* src = table + b;
        uint32_t* dst = scratch + b;
        for (int p = 0; p < passes; p++) {
            const int shift = 8 * p;
            hist[threadIdx.x] = 0u;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < n; i += kBlockSortThreads) atomicAdd(&hist[(src[i] >> shift) & 255u], 1u);
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t acc = 0;
                for (int d = 0; d < 256; d++) {
                    run[d] = acc;
                    acc += hist[d];
                }
            }
            __syncthreads();
            for (uint32_t t0 = 0; t0 < n; t0 += kBlockSortThreads) {
                for (int d = threadIdx.x; d < (kBlockSortThreads / 32) * 256; d += kBlockSortThreads)
                    (&wcnt[0][0])[d] = 0u;
                __syncthreads();
                const uint32_t i = t0 + threadIdx.x;
                const bool v = i < n;
                const uint32_t x = v ? src[i] : 0u;
                const uint32_t dg = v ? ((x >> shift) & 255u) : 256u;
                const unsigned peers = __match_any_sync(0xffffffffu, dg);
                const uint32_t rk = (uint32_t)__popc(peers & lt);
                if (v && lane == __ffs(peers) - 1) wcnt[warp][dg] = (uint32_t)__popc(peers);
                __syncthreads();
                uint32_t before = 0;
                if (v)
                    for (int w = 0; w < warp; w++) before += wcnt[w][dg];
                if (v) dst[run[dg] + before + rk] = x;
                __syncthreads();
                {
                    uint32_t tot = 0;
#pragma unroll
                    for (int w = 0; w < kBlockSortThreads / 32; w++) tot += wcnt[w][threadIdx.x];
                    run[threadIdx.x] += tot;
                }
                __syncthreads();
            }
            uint32_t* t = src;
            src = dst;
            dst = t;
        }
    }
}

__global__ void k_long_lists(const uint64_t* __restrict__ offsets, uint32_t nlists, uint32_t lo,
                             uint32_t* __restrict__ out, uint32_t* __restrict__ nout) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nlists && offsets[i + 1] - offsets[i] > lo) out[atomicAdd(nout, 1u)] = i;
}

inline unsigned grid_for(uint64_t n, unsigned t, uint64_t cap) {
    uint64_t b = (n + t - 1) / t;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

}  // namespace

size_t place_temp_bytes(uint64_t nlists) {
    return (nlists + 64) * sizeof(uint32_t) + scan_u32_u64_temp_bytes(nlists) + 256;
}

cudaError_t sort_short_lists(uint32_t* table, const uint64_t* offsets, uint32_t nlists, int num_sms, int* launches,
                             cudaStream_t st) {
    if (nlists == 0) return cudaSuccess;
    const unsigned g = grid_for((uint64_t)nlists * 32u, 256, (uint64_t)num_sms * 64);
    k_list_sort_warp<1><<<g, 256, 0, st>>>(table, offsets, nlists, 1u);
    k_list_sort_warp<2><<<g, 256, 0, st>>>(table, offsets, nlists, 32u);
    k_list_sort_warp<4><<<g, 256, 0, st>>>(table, offsets, nlists, 64u);
    k_list_sort_warp<8><<<g, 256, 0, st>>>(table, offsets, nlists, 128u);
    if (launches) *launches += 4;
    return cudaGetLastError();
}

cudaError_t find_long_lists(const uint64_t* offsets, uint32_t nlists, void* temp, uint32_t* d_nlong,
                            uint32_t* h_nlong, int* launches, cudaStream_t st) {
    *h_nlong = 0;
    if (nlists == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(d_nlong, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_long_lists<<<grid_for(nlists, 256, ~0ull), 256, 0, st>>>(offsets, nlists, kWarpSortMax,
                                                              static_cast<uint32_t*>(temp), d_nlong);
    if (launches) *launches += 1;
    e = cudaMemcpyAsync(h_nlong, d_nlong, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t sort_long_lists(uint32_t* table, uint32_t* scratch, const uint64_t* offsets, const void* temp,
                            uint32_t nlong, uint32_t id_bits, int num_sms, int* launches, cudaStream_t st) {
    if (nlong == 0) return cudaSuccess;
    int passes = (int)((id_bits + 7u) / 8u);
    passes += passes & 1;  // even: the sorted list ends in the table
    k_list_sort_block<<<grid_for(nlong, 1, (uint64_t)num_sms * 8), kBlockSortThreads, 0, st>>>(
        table, scratch, offsets, static_cast<const uint32_t*>(temp), nlong, passes);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

cudaError_t place_pairs(const unsigned long long* keys, uint64_t nkeys, uint32_t shift, uint32_t nlists,
                        uint32_t* counts, uint64_t* offsets, uint32_t* table, uint64_t cap, uint32_t* cursor,
                        uint32_t* err, void* temp, int num_sms, int* launches, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counts, 0, ((size_t)nlists + 1) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(cursor, 0, (size_t)nlists * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const unsigned g = grid_for(nkeys, 256, (uint64_t)num_sms * 32);
    if (nkeys) k_pair_count<<<g, 256, 0, st>>>(keys, nkeys, shift, counts);
    e = scan_u32_u64(counts, offsets, nlists, temp, st);
    if (e != cudaSuccess) return e;
    if (nkeys) k_pair_place<<<g, 256, 0, st>>>(keys, nkeys, shift, offsets, cursor, table, cap, err);
    if (launches) *launches += 5;
    return cudaGetLastError();
}

}  // namespace gsj
