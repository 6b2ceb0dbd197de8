// The SORT variant of the grid traversal (params.h:46; GPU.cu:351-395 sorts the
// points of each cell, kernel.cu:400-467 prunes the scan of each neighbour
// cell).  The points of every cell are ordered by their value in the sort
// dimension - the first non-indexed dimension, or dim 0 when every dimension
// is indexed - and each query evaluates, per neighbour cell:
//   sort dimension indexed: the cell's points from the side nearer the query
//     (descending when the cell lies below the query's cell in dim 0,
//     ascending above), up to the first point farther than eps in dim 0; all
//     points of a cell level with the query's in dim 0;
//   sort dimension not indexed: the points from the position the reference's
//     stepping search reaches (a halving step from the middle, clamped, then up
//     to two steps back while within eps), while the point's value minus the
//     query's stays below eps (strict).
// The window is the reference's, so the reported pairs are its pairs - the
// second rule can skip a boundary pair that the unpruned scan reports.
//
// One thread per query (the reference's own work split), the full
// neighbourhood; a count pass writes the list lengths, the fill pass writes
// every list at its offset in candidate order.  A compatibility path: every
// switch of the reference is accepted, and its lists are the reference's.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_dist.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

namespace {

template <typename T, int MODEL, int POL, bool FILL>
__global__ void __launch_bounds__(128) k_sort_join(const JoinArgs<T> a, const uint32_t* __restrict__ slot_cell,
                                                   uint32_t noff, uint32_t* __restrict__ counts_by_id) {
    const uint32_t N = a.n_points;
    const uint32_t n = a.n, npad = a.npad, k = a.g.k;
    const T eps = a.eps, thr = a.thr;
    const bool indexed = n == k;
    const uint32_t sd = indexed ? 0u : k;
    unsigned long long cand = 0;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
        const T* p = a.pts + (size_t)s * npad;
        const uint32_t cell = slot_cell[s];
        const uint64_t key = a.cell_key[cell];
        uint32_t own[kMaxK];
#pragma unroll
        for (int j = 0; j < kMaxK; j++) own[j] = j < (int)k ? (uint32_t)((key / a.g.mult[j]) % a.g.ncells[j]) : 0u;
        uint32_t lowmask, highmask, oddmask;
        cell_masks(own, a.g, lowmask, highmask, oddmask);
        const uint32_t id = a.ids[s];
        uint32_t cnt = 0;
        uint32_t* list = FILL ? a.table + a.offsets[id] : nullptr;
        const uint32_t len_cap = FILL ? (uint32_t)(a.offsets[id + 1] - a.offsets[id]) : 0u;
        auto eval = [&](uint32_t slot) {
            cand++;
            const T d2 = sqdist_lane<T, MODEL, POL>(p, a.pts + (size_t)slot * npad, n, a.ilp);
            if (d2 <= thr) {
                if constexpr (FILL) {
                    if (cnt < len_cap) list[cnt] = a.ids[slot];
                    else *a.err_flag = 1u;
                }
                cnt++;
            }
        };
        for (uint32_t o = 0; o < noff; o++) {
            uint64_t lin;
            if (!nb_offset<T, false>(a, o, key, lowmask, highmask, oddmask, lin)) continue;
            uint32_t start, num;
            if (!lookup_range(a, lin, start, num)) continue;
            if (indexed) {
                // the neighbour's step in dim 0 is digit 0 of the offset
                const int dl0 = (int)(o % 3u) - 1;
                const bool mid = dl0 == 0, left = dl0 < 0;
                for (uint32_t kk = 0; kk < num; kk++) {
                    const uint32_t pos = left ? num - 1u - kk : kk;
                    const T dv = FP<T>::sub(a.pts[(size_t)(start + pos) * npad], p[0]);
                    if (!mid && fabs(dv) > eps) break;
                    eval(start + pos);
                }
            } else {
                const int length = (int)num - 1;
                auto db = [&](int pos) { return a.pts[(size_t)(start + (uint32_t)pos) * npad + sd]; };
                int idx = length / 2;
                for (int step = (length + 3) / 4; step > 1; step = (step + 1) / 2) {
                    if (FP<T>::sub(p[sd], db(idx)) >= eps) {
                        idx += step;
                        if (idx > length) idx = length;
                    } else {
                        idx -= step;
                        if (idx < 0) {
                            idx = 0;
                            step = 0;
                        }
                    }
                }
                if (idx > 0 && FP<T>::sub(p[sd], db(idx - 1)) <= eps) idx--;
                if (idx > 0 && FP<T>::sub(p[sd], db(idx - 1)) <= eps) idx--;
                while (idx <= length && FP<T>::sub(db(idx), p[sd]) < eps) {
                    eval(start + (uint32_t)idx);
                    idx++;
                }
            }
        }
        if (!FILL) counts_by_id[id] = cnt;
        else if (cnt != len_cap) *a.err_flag = 1u;
    }
    if (!FILL) {
        for (int off = 16; off > 0; off >>= 1) cand += __shfl_down_sync(0xffffffffu, cand, off);
        if ((threadIdx.x & 31) == 0 && cand) atomicAdd(a.cand_cnt, cand);
    }
}

template <typename T, int MODEL, int POL>
cudaError_t sort_launch(const JoinArgs<T>& a, const uint32_t* slot_cell, uint32_t noff, uint32_t* counts_by_id,
                        bool fill, int num_sms, cudaStream_t st) {
    uint64_t blocks = ((uint64_t)a.n_points + 127) / 128;
    const uint64_t cap = (uint64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    if (fill) k_sort_join<T, MODEL, POL, true><<<(unsigned)blocks, 128, 0, st>>>(a, slot_cell, noff, counts_by_id);
    else k_sort_join<T, MODEL, POL, false><<<(unsigned)blocks, 128, 0, st>>>(a, slot_cell, noff, counts_by_id);
    return cudaGetLastError();
}

// Values of the sort dimension by slot: out[s] = in[ids[s]][col] (input layout).
template <typename T>
__global__ void k_sort_values(const T* __restrict__ in, uint64_t N, uint32_t n, uint32_t col,
                              const uint32_t* __restrict__ ids, T* __restrict__ out) {
    const uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s < N) out[s] = in[(uint64_t)ids[s] * n + col];
}

}  // namespace

template <typename T>
cudaError_t launch_sort_join(const JoinArgs<T>& a, const uint32_t* slot_cell, uint32_t* counts_by_id, int model,
                             bool fill, int num_sms, cudaStream_t st) {
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    uint32_t noff = 1;
    for (uint32_t j = 0; j < a.g.k; j++) noff *= 3u;
    if (model == kSeq) return sort_launch<T, kSeq, POL>(a, slot_cell, noff, counts_by_id, fill, num_sms, st);
    if (model == kIlp) return sort_launch<T, kIlp, POL>(a, slot_cell, noff, counts_by_id, fill, num_sms, st);
    return sort_launch<T, kIlpSc, POL>(a, slot_cell, noff, counts_by_id, fill, num_sms, st);
}

template <typename T>
cudaError_t launch_sort_values(const T* in, uint64_t N, uint32_t n, uint32_t col, const uint32_t* ids, T* out,
                               cudaStream_t st) {
    if (N == 0) return cudaSuccess;
    k_sort_values<T><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(in, N, n, col, ids, out);
    return cudaGetLastError();
}

template cudaError_t launch_sort_join<float>(const JoinArgs<float>&, const uint32_t*, uint32_t*, int, bool, int,
                                             cudaStream_t);
template cudaError_t launch_sort_join<double>(const JoinArgs<double>&, const uint32_t*, uint32_t*, int, bool, int,
                                              cudaStream_t);
template cudaError_t launch_sort_values<float>(const float*, uint64_t, uint32_t, uint32_t, const uint32_t*, float*,
                                               cudaStream_t);
template cudaError_t launch_sort_values<double>(const double*, uint64_t, uint32_t, uint32_t, const uint32_t*,
                                                double*, cudaStream_t);

}  // namespace gsj
