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
//                  CTA per list (bitonic network in registers, shuffles and
//                  shared memory) up to kCtaSortMax, above that a CTA per list
//                  of LSD radix passes through a scratch copy.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_kernels.h"
#include "gsj_place.h"
#include "gsj_scan.h"

namespace gsj {

namespace {

constexpr unsigned long long kPadKey = ~0ull;  // unused entries of reserved blocks
constexpr uint32_t kWarpSortMax = 256;         // 8 entries per lane
constexpr int kCtaSortThreads = 256;
constexpr uint32_t kCtaSortMax = 4096;         // 16 entries per thread
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

// Bitonic sort of one list of n <= 32*E entries held as E registers per lane
// (entry r*32 + lane), padded with 0xffffffff.  Called by a whole warp.
template <int E>
__device__ __forceinline__ void warp_bitonic(uint32_t* __restrict__ list, uint32_t n, int lane) {
    const unsigned FULL = 0xffffffffu;
    constexpr uint32_t P = 32u * E;
    uint32_t v[E];
#pragma unroll
    for (int r = 0; r < E; r++) {
        const uint32_t i = (uint32_t)r * 32u + (uint32_t)lane;
        v[r] = i < n ? list[i] : 0xffffffffu;
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
        if (i < n) list[i] = v[r];
    }
}

// Every list of min_len+1..kWarpSortMax entries sorted by one warp (the
// network sized to the list: 32, 64, 128 or 256 entries); lists above
// kWarpSortMax are gathered into long_lists (*nlong, warp-aggregated), those
// above kCtaSortMax counted in *nvery.  List l: table[offsets[l] ..
// offsets[l+1]).
template <typename OffT>
__global__ void __launch_bounds__(256) k_list_sort_short(uint32_t* __restrict__ table,
                                                         const OffT* __restrict__ offsets, uint32_t nlists,
                                                         uint32_t min_len, uint32_t* __restrict__ long_lists,
                                                         uint32_t* __restrict__ nlong) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt_p();
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t l0 = gw * 32u; l0 < nlists; l0 += nw * 32u) {
        // the lengths of 32 consecutive lists, then the short ones one by one
        const uint32_t li = l0 + (uint32_t)lane;
        uint64_t b = 0, e = 0;
        if (li < nlists) {
            b = (uint64_t)offsets[li];
            e = (uint64_t)offsets[li + 1];
        }
        const uint64_t len = e - b;
        const unsigned lng = __ballot_sync(FULL, len > kWarpSortMax);
        if (lng) {
            uint32_t at = 0;
            if (lane == 0) at = atomicAdd(nlong, (uint32_t)__popc(lng));
            at = __shfl_sync(FULL, at, 0);
            if ((lng >> lane) & 1u) long_lists[at + (uint32_t)__popc(lng & lt)] = li;
            const unsigned vl = __ballot_sync(FULL, len > kCtaSortMax);
            if (vl && lane == 0) atomicAdd(nlong + 1, (uint32_t)__popc(vl));
        }
        unsigned mine = __ballot_sync(FULL, len > min_len && len > 1u && len <= kWarpSortMax);
        while (mine) {
            const int j = __ffs(mine) - 1;
            mine &= mine - 1u;
            uint32_t* list = table + __shfl_sync(FULL, b, j);
            const uint32_t n = (uint32_t)__shfl_sync(FULL, len, j);
            if (n <= 32u) warp_bitonic<1>(list, n, lane);
            else if (n <= 64u) warp_bitonic<2>(list, n, lane);
            else if (n <= 128u) warp_bitonic<4>(list, n, lane);
            else warp_bitonic<8>(list, n, lane);
        }
    }
}

// Bitonic sort of one list of n <= 256*E entries by the whole CTA
// (kCtaSortThreads threads), entry r*256 + t in register r of thread t.
// Exchange distances below 32 use shuffles; the others go through one of two
// shared-memory buffers (alternated by *buf, so each such stage needs one
// barrier: a buffer is rewritten only after every thread passed the barrier
// that followed its last read).
template <int E>
__device__ __forceinline__ void cta_bitonic(uint32_t* __restrict__ list, uint32_t n, uint32_t (*sb)[kCtaSortMax],
                                            int& buf) {
    const unsigned FULL = 0xffffffffu;
    const uint32_t t = threadIdx.x;
    constexpr uint32_t P = (uint32_t)kCtaSortThreads * E;
    uint32_t v[E];
#pragma unroll
    for (int r = 0; r < E; r++) {
        const uint32_t i = (uint32_t)r * kCtaSortThreads + t;
        v[r] = i < n ? list[i] : 0xffffffffu;
    }
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32u) {
                uint32_t* s = sb[buf];
                buf ^= 1;
#pragma unroll
                for (int r = 0; r < E; r++) s[(uint32_t)r * kCtaSortThreads + t] = v[r];
                __syncthreads();
#pragma unroll
                for (int r = 0; r < E; r++) {
                    const uint32_t i = (uint32_t)r * kCtaSortThreads + t;
                    const uint32_t o = s[i ^ j];
                    const bool up = (i & k) == 0u, lower = (i & j) == 0u;
                    v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
                }
            } else {
#pragma unroll
                for (int r = 0; r < E; r++) {
                    const uint32_t i = (uint32_t)r * kCtaSortThreads + t;
                    const uint32_t o = __shfl_xor_sync(FULL, v[r], (int)j);
                    const bool up = (i & k) == 0u, lower = (i & j) == 0u;
                    v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < E; r++) {
        const uint32_t i = (uint32_t)r * kCtaSortThreads + t;
        if (i < n) list[i] = v[r];
    }
}

// A CTA per list of kWarpSortMax+1 .. kCtaSortMax entries (longer lists are
// left to k_list_sort_block).
template <typename OffT>
__global__ void __launch_bounds__(kCtaSortThreads) k_list_sort_cta(uint32_t* __restrict__ table,
                                                                   const OffT* __restrict__ offsets,
                                                                   const uint32_t* __restrict__ long_lists,
                                                                   uint32_t nlong) {
    __shared__ uint32_t sb[2][kCtaSortMax];
    int buf = 0;
    for (uint32_t li = blockIdx.x; li < nlong; li += gridDim.x) {
        const uint32_t l = long_lists[li];
        const uint64_t b = (uint64_t)offsets[l];
        const uint32_t n = (uint32_t)((uint64_t)offsets[l + 1] - b);
        if (n > kCtaSortMax) continue;
        if (n <= 512u) cta_bitonic<2>(table + b, n, sb, buf);
        else if (n <= 1024u) cta_bitonic<4>(table + b, n, sb, buf);
        else if (n <= 2048u) cta_bitonic<8>(table + b, n, sb, buf);
        else cta_bitonic<16>(table + b, n, sb, buf);
    }
}

// One CTA per list longer than kCtaSortMax: LSD radix passes of 8 bits over
// the list's entries (ids below 2^bits), alternating between the table and
// the same range of `scratch`; the pass count is even, so the sorted list ends
// in the table.  Each pass: a digit histogram of the whole list, then its
// tiles in order, each ranked stably (per-warp match_any groups in index
// order) and written at the running offset of its digit.
template <typename OffT>
__global__ void __launch_bounds__(kBlockSortThreads) k_list_sort_block(uint32_t* __restrict__ table,
                                                                       uint32_t* __restrict__ scratch,
                                                                       const OffT* __restrict__ offsets,
                                                                       const uint32_t* __restrict__ long_lists,
                                                                       uint32_t nlong, int passes) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t run[256];
    __shared__ uint32_t wcnt[kBlockSortThreads / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = lanemask_lt_p();
    for (uint32_t li = blockIdx.x; li < nlong; li += gridDim.x) {
        const uint32_t l = long_lists[li];
        const uint64_t b = (uint64_t)offsets[l];
        const uint32_t n = (uint32_t)((uint64_t)offsets[l + 1] - b);
        if (n <= kCtaSortMax) continue;  // block-uniform: sorted by k_list_sort_cta
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

inline unsigned grid_for(uint64_t n, unsigned t, uint64_t cap) {
    uint64_t b = (n + t - 1) / t;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

}  // namespace

size_t place_temp_bytes(uint64_t nlists) {
    return (nlists + 64) * sizeof(uint32_t) + scan_u32_u64_temp_bytes(nlists) + 256;
}

template <typename OffT>
cudaError_t sort_short_lists(uint32_t* table, const OffT* offsets, uint32_t nlists, uint32_t min_len, void* temp,
                             uint32_t* d_nlong, uint32_t* h_nlong, uint32_t* h_nvery, int num_sms, int* launches,
                             cudaStream_t st) {
    *h_nlong = *h_nvery = 0;
    if (nlists == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(d_nlong, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const unsigned g = grid_for((uint64_t)nlists, 256, (uint64_t)num_sms * 64);
    k_list_sort_short<OffT><<<g, 256, 0, st>>>(table, offsets, nlists, min_len, static_cast<uint32_t*>(temp), d_nlong);
    if (launches) *launches += 1;
    uint32_t h[2];
    e = cudaMemcpyAsync(h, d_nlong, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    *h_nlong = h[0];
    *h_nvery = h[1];
    return e;
}

template <typename OffT>
cudaError_t sort_long_lists(uint32_t* table, uint32_t* scratch, const OffT* offsets, const void* temp,
                            uint32_t nlong, uint32_t nvery, uint32_t id_bits, int num_sms, int* launches,
                            cudaStream_t st) {
    if (nlong == 0) return cudaSuccess;
    const uint32_t* ll = static_cast<const uint32_t*>(temp);
    if (nlong > nvery) {
        k_list_sort_cta<OffT><<<grid_for(nlong - nvery, 1, (uint64_t)num_sms * 6), kCtaSortThreads, 0, st>>>(
            table, offsets, ll, nlong);
        if (launches) *launches += 1;
    }
    if (nvery) {
        if (!scratch) return cudaErrorInvalidValue;
        int passes = (int)((id_bits + 7u) / 8u);
        passes += passes & 1;  // even: the sorted list ends in the table
        k_list_sort_block<OffT><<<grid_for(nvery, 1, (uint64_t)num_sms * 8), kBlockSortThreads, 0, st>>>(
            table, scratch, offsets, ll, nlong, passes);
        if (launches) *launches += 1;
    }
    return cudaGetLastError();
}

template cudaError_t sort_short_lists<uint64_t>(uint32_t*, const uint64_t*, uint32_t, uint32_t, void*, uint32_t*,
                                                uint32_t*, uint32_t*, int, int*, cudaStream_t);
template cudaError_t sort_short_lists<uint32_t>(uint32_t*, const uint32_t*, uint32_t, uint32_t, void*, uint32_t*,
                                                uint32_t*, uint32_t*, int, int*, cudaStream_t);
template cudaError_t sort_long_lists<uint64_t>(uint32_t*, uint32_t*, const uint64_t*, const void*, uint32_t,
                                               uint32_t, uint32_t, int, int*, cudaStream_t);
template cudaError_t sort_long_lists<uint32_t>(uint32_t*, uint32_t*, const uint32_t*, const void*, uint32_t,
                                               uint32_t, uint32_t, int, int*, cudaStream_t);

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
