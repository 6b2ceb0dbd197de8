// GPU brute-force neighbour count: the reference's algorithm 1
// (kernelBruteForce, kernel.cu:486-515, driven by
// makeDistanceTableGPUBruteForce, GPU.cu:1285-1440).  Every point is tested
// against every point, self included, with the reference's arithmetic for
// its loop `runningDist += (c - q)*(c - q)` over the dimensions in order (the
// sequential model of gsj_dist.cuh with the pinned contraction policy) and
// `sqrt(runningDist) <= eps` as `s <= thr`.  The reference accumulates one
// global total; here each point's count is written as well, which makes the
// kernel an exact-count check of the grid join on small inputs.
//
// Layout: a CTA of 256 queries walks all points in tiles of kBfTile rows
// staged in shared memory; every thread keeps its own count (no atomics but
// one per CTA for the total).
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_dist.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

namespace {

constexpr int kBfThreads = 256;
constexpr int kBfTile = 64;

template <typename T, int POL>
__global__ void __launch_bounds__(kBfThreads) k_bruteforce(const T* __restrict__ pts, uint32_t N, uint32_t n, T thr,
                                                           uint32_t rows, uint32_t* __restrict__ counts,
                                                           unsigned long long* __restrict__ total) {
    extern __shared__ __align__(16) unsigned char bsm[];
    T* tile = reinterpret_cast<T*>(bsm);  // [rows][n]
    const uint32_t q = blockIdx.x * kBfThreads + threadIdx.x;
    const bool active = q < N;
    const T* qrow = pts + (size_t)(active ? q : 0u) * n;
    uint32_t cnt = 0;
    for (uint32_t c0 = 0; c0 < N; c0 += rows) {
        const uint32_t m = min(rows, N - c0);
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < m * n; e += kBfThreads) tile[e] = pts[(size_t)c0 * n + e];
        __syncthreads();
        if (active) {
            for (uint32_t j = 0; j < m; j++) {
                const T* c = tile + (size_t)j * n;
                Acc<T, POL> s;
                for (uint32_t l = 0; l < n; l++) s.add_prod(FP<T>::sub(c[l], __ldg(qrow + l)));
                if (s.v <= thr) cnt++;
            }
        }
    }
    if (active) counts[q] = cnt;
    unsigned long long t = cnt;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31u) == 0u && t) atomicAdd(total, t);
}

}  // namespace

template <typename T>
cudaError_t launch_bruteforce(const T* pts, uint32_t N, uint32_t n, T thr, uint32_t* counts,
                              unsigned long long* total, cudaStream_t st) {
    if (N == 0) return cudaSuccess;
    if (n == 0) return cudaErrorInvalidValue;
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    // candidate rows per tile: kBfTile, fewer for very wide points
    const size_t row_bytes = (size_t)n * sizeof(T);
    const size_t limit = 160u * 1024u;
    uint32_t rows = (uint32_t)kBfTile;
    if ((size_t)rows * row_bytes > limit) rows = (uint32_t)(limit / row_bytes);
    if (rows == 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)rows * row_bytes;
    auto kern = k_bruteforce<T, POL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = (N + kBfThreads - 1) / kBfThreads;
    kern<<<blocks, kBfThreads, smem, st>>>(pts, N, n, thr, rows, counts, total);
    return cudaGetLastError();
}

template cudaError_t launch_bruteforce<float>(const float*, uint32_t, uint32_t, float, uint32_t*,
                                              unsigned long long*, cudaStream_t);
template cudaError_t launch_bruteforce<double>(const double*, uint32_t, uint32_t, double, uint32_t*,
                                               unsigned long long*, cudaStream_t);

}  // namespace gsj
