// Thread-per-query join for dense low-dimensional grids (k <= 3).
//
// Low-dimensional workloads have tiny cells (a 2-D mixture of 20M points
// averages 3 points per non-empty cell), so any per-cell set-up done by a
// whole warp costs more than the distance tests.  Here each thread owns one
// query slot; the slots of a warp are consecutive in cell order, so the lanes
// of one cell walk identical candidate ranges (broadcast loads) and lanes of
// neighbouring cells walk overlapping ones.  The neighbour rows come from the
// cell plan (k_cell_plan): 3^(k-1) contiguous slot ranges, the full
// neighbourhood of kernel.cu:292-302.  Every thread therefore finds exactly
// its own neighbour set and counts it (k_rows_tpq); the fill pass (k_fill_q32)
// spreads each query's candidates over a warp instead.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_dist.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

template <typename T, int NT, int POL>
__global__ void __launch_bounds__(256) k_rows_tpq(const JoinArgs<T> a, const uint32_t* __restrict__ slot_cell,
                                                  uint32_t nrows) {
    const uint32_t N = a.n_points;
    const uint32_t npad = a.npad;
    unsigned long long cand = 0;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
        const uint32_t cell = slot_cell[s];
        T q[NT];
#pragma unroll
        for (int l = 0; l < NT; l++) q[l] = a.pts[(size_t)s * npad + l];
        uint32_t cnt = 0;
        for (uint32_t r = 0; r < nrows; r++) {
            const uint2 e = a.plan[(size_t)cell * nrows + r];
            cand += e.y;
            for (uint32_t i = 0; i < e.y; i++) {
                const uint32_t c = e.x + i;
                T cr[NT];
#pragma unroll
                for (int l = 0; l < NT; l++) cr[l] = a.pts[(size_t)c * npad + l];
                const T d2 = sqdist_seq_reg<T, NT, POL>(q, cr);
                if (d2 <= a.thr) cnt++;
            }
        }
        a.fwd_cnt[s] = cnt;
        a.rev_cnt[s] = 0u;
    }
    // one atomic per warp for the candidate statistic
    for (int o = 16; o > 0; o >>= 1) cand += __shfl_down_sync(0xffffffffu, cand, o);
    if ((threadIdx.x & 31) == 0 && cand) atomicAdd(a.cand_cnt, cand);
}

__device__ __forceinline__ unsigned lanemask_lt_q() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Fill pass of dense low-dimensional grids: a warp per 32 consecutive query
// slots.  Lane j loads query j's coordinates, list cursor and the NR row
// ranges of its cell in one parallel round; then the warp takes the queries
// one after another, spreads the query's candidates over the lanes (32 per
// tile) and writes its hits with one ballot per tile at consecutive positions
// of the query's list.  Consecutive queries usually share a cell; while they
// do, up to G candidate tiles stay in registers.  No per-cell set-up, no
// shared memory, every list written by one warp in candidate order.
template <typename T, int NT, int NR, int POL>
__global__ void __launch_bounds__(256) k_fill_q32(const JoinArgs<T> a, const uint32_t* __restrict__ slot_cell) {
    constexpr int G = 4;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt_q();
    const uint32_t N = a.n_points;
    const uint32_t npad = a.npad;
    const uint64_t gwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (uint64_t s0 = gw * 32u; s0 < N; s0 += gwarps * 32u) {
        const uint32_t s = (uint32_t)s0 + lane;
        const uint32_t nq = min(32u, N - (uint32_t)s0);
        // lane j: query j's cell, coordinates, list (pointer + length from the count pass)
        uint32_t my_cell = 0xffffffffu, my_lo[NR], my_cnt[NR], my_len = 0;
        T myq[NT];
        uint32_t* my_list = a.table;
        if ((uint32_t)lane < nq) {
            my_cell = slot_cell[s];
#pragma unroll
            for (int l = 0; l < NT; l++) myq[l] = a.pts[(size_t)s * npad + l];
            const unsigned long long off = a.offsets[a.ids[s]];
            my_len = a.fwd_cnt[s] + a.rev_cnt[s];
            if (off + my_len <= a.table_cap) my_list = a.table + off;
            else {
                my_len = 0;
                *a.err_flag = 1u;
            }
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const uint2 e = a.plan[(size_t)my_cell * NR + r];
                my_lo[r] = e.x;
                my_cnt[r] = e.y;
            }
        } else {
#pragma unroll
            for (int l = 0; l < NT; l++) myq[l] = T(0);
#pragma unroll
            for (int r = 0; r < NR; r++) my_lo[r] = my_cnt[r] = 0u;
        }
        uint32_t cached = 0xffffffffu, total = 0, ntile = 0;
        uint32_t lo[NR], pre[NR + 1];
        T cx[G][NT];
        uint32_t cid[G];
        bool cval[G];
#pragma unroll
        for (int r = 0; r < NR; r++) lo[r] = pre[r] = 0u;
        pre[NR] = 0u;
#pragma unroll
        for (int t = 0; t < G; t++) {
            cid[t] = 0u;
            cval[t] = false;
#pragma unroll
            for (int l = 0; l < NT; l++) cx[t][l] = T(0);
        }
        for (uint32_t j = 0; j < nq; j++) {
            const uint32_t cell = __shfl_sync(FULL, my_cell, j);
            if (cell != cached) {
                cached = cell;
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    lo[r] = __shfl_sync(FULL, my_lo[r], j);
                    pre[r + 1] = pre[r] + __shfl_sync(FULL, my_cnt[r], j);
                }
                total = pre[NR];
                ntile = (total + 31u) / 32u;
                if (ntile <= (uint32_t)G) {
#pragma unroll
                    for (int t = 0; t < G; t++) {
                        const uint32_t f = (uint32_t)t * 32u + lane;
                        cval[t] = f < total;
                        uint32_t slot = 0;
                        if (cval[t]) {
                            uint32_t st = lo[0], p = 0;
#pragma unroll
                            for (int rr = 1; rr < NR; rr++)
                                if (f >= pre[rr]) {
                                    st = lo[rr];
                                    p = pre[rr];
                                }
                            slot = st + (f - p);
                            cid[t] = a.ids[slot];
                        }
#pragma unroll
                        for (int l = 0; l < NT; l++) cx[t][l] = a.pts[(size_t)slot * npad + l];
                    }
                }
            }
            T q[NT];
#pragma unroll
            for (int l = 0; l < NT; l++) q[l] = __shfl_sync(FULL, myq[l], j);
            uint32_t* list = reinterpret_cast<uint32_t*>(
                __shfl_sync(FULL, reinterpret_cast<unsigned long long>(my_list), j));
            const uint32_t len = __shfl_sync(FULL, my_len, j);
            uint32_t run = 0;  // entries of this list written so far
            if (ntile <= (uint32_t)G) {
#pragma unroll
                for (int t = 0; t < G; t++) {
                    if ((uint32_t)t < ntile) {
                        const T d2 = sqdist_seq_reg<T, NT, POL>(q, cx[t]);
                        const bool hit = cval[t] && (d2 <= a.thr);
                        const unsigned b = __ballot_sync(FULL, hit);
                        const uint32_t pos = run + __popc(b & lt);
                        if (hit && pos < len) list[pos] = cid[t];
                        run += __popc(b);
                    }
                }
            } else {
                for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
                    const uint32_t f = t0 + lane;
                    const bool v = f < total;
                    uint32_t slot = 0, c_id = 0;
                    if (v) {
                        uint32_t st = lo[0], p = 0;
#pragma unroll
                        for (int rr = 1; rr < NR; rr++)
                            if (f >= pre[rr]) {
                                st = lo[rr];
                                p = pre[rr];
                            }
                        slot = st + (f - p);
                        c_id = a.ids[slot];
                    }
                    T c[NT];
#pragma unroll
                    for (int l = 0; l < NT; l++) c[l] = a.pts[(size_t)slot * npad + l];
                    const T d2 = sqdist_seq_reg<T, NT, POL>(q, c);
                    const bool hit = v && (d2 <= a.thr);
                    const unsigned b = __ballot_sync(FULL, hit);
                    const uint32_t pos = run + __popc(b & lt);
                    if (hit && pos < len) list[pos] = c_id;
                    run += __popc(b);
                }
            }
            // the count pass and this pass must agree on every list
            if (lane == 0 && run != len) *a.err_flag = 1u;
        }
    }
}

template <typename T, int NT, int NR>
static cudaError_t launch_fill_q32_nt(const JoinArgs<T>& a, const uint32_t* slot_cell, int num_sms, cudaStream_t st) {
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    auto kern = k_fill_q32<T, NT, NR, POL>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)num_sms * per_sm * 4;
    const uint64_t needed = ((uint64_t)a.n_points + 255) / 256;
    if (blocks > needed) blocks = needed ? needed : 1;
    kern<<<(unsigned)blocks, 256, 0, st>>>(a, slot_cell);
    return cudaGetLastError();
}

template <typename T, int NR>
static cudaError_t fill_q32_nr(const JoinArgs<T>& a, const uint32_t* slot_cell, int num_sms, cudaStream_t st) {
    switch (a.n) {
        case 1: return launch_fill_q32_nt<T, 1, NR>(a, slot_cell, num_sms, st);
        case 2: return launch_fill_q32_nt<T, 2, NR>(a, slot_cell, num_sms, st);
        case 3: return launch_fill_q32_nt<T, 3, NR>(a, slot_cell, num_sms, st);
        case 4: return launch_fill_q32_nt<T, 4, NR>(a, slot_cell, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_fill_q32(const JoinArgs<T>& a, const uint32_t* slot_cell, int num_sms, cudaStream_t st) {
    if (!tpq_supported(a)) return cudaErrorInvalidValue;
    if (a.g.k == 1) return fill_q32_nr<T, 1>(a, slot_cell, num_sms, st);
    if (a.g.k == 2) return fill_q32_nr<T, 3>(a, slot_cell, num_sms, st);
    return fill_q32_nr<T, 9>(a, slot_cell, num_sms, st);
}

template cudaError_t launch_fill_q32<float>(const JoinArgs<float>&, const uint32_t*, int, cudaStream_t);
template cudaError_t launch_fill_q32<double>(const JoinArgs<double>&, const uint32_t*, int, cudaStream_t);

// Slot -> cell index map (one thread per cell writes its slots).
__global__ void k_slot_cell(const uint32_t* __restrict__ cell_start, uint32_t M, uint32_t* __restrict__ slot_cell) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    for (uint32_t s = cell_start[c]; s < cell_start[c + 1]; s++) slot_cell[s] = c;
}

cudaError_t launch_slot_cell(const uint32_t* cell_start, uint32_t M, uint32_t* slot_cell, cudaStream_t st) {
    k_slot_cell<<<(M + 255) / 256, 256, 0, st>>>(cell_start, M, slot_cell);
    return cudaGetLastError();
}

template <typename T, int NT>
static cudaError_t launch_tpq_nt(const JoinArgs<T>& a, const uint32_t* slot_cell, uint32_t nrows, int num_sms,
                                 cudaStream_t st) {
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    auto kern = k_rows_tpq<T, NT, POL>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)num_sms * per_sm;
    const uint64_t needed = ((uint64_t)a.n_points + 255) / 256;
    if (blocks > needed) blocks = needed ? needed : 1;
    kern<<<(unsigned)blocks, 256, 0, st>>>(a, slot_cell, nrows);
    return cudaGetLastError();
}

template <typename T>
bool tpq_supported(const JoinArgs<T>& a) {
    return a.n >= 1 && a.n <= 4 && a.ilp == 0 && a.g.k <= 3 && a.plan != nullptr;
}

template <typename T>
cudaError_t launch_count_tpq(const JoinArgs<T>& a, const uint32_t* slot_cell, int num_sms, cudaStream_t st) {
    if (!tpq_supported(a)) return cudaErrorInvalidValue;
    const uint32_t nrows = a.g.k == 1 ? 1u : (a.g.k == 2 ? 3u : 9u);
    switch (a.n) {
        case 1: return launch_tpq_nt<T, 1>(a, slot_cell, nrows, num_sms, st);
        case 2: return launch_tpq_nt<T, 2>(a, slot_cell, nrows, num_sms, st);
        case 3: return launch_tpq_nt<T, 3>(a, slot_cell, nrows, num_sms, st);
        case 4: return launch_tpq_nt<T, 4>(a, slot_cell, nrows, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

template bool tpq_supported<float>(const JoinArgs<float>&);
template bool tpq_supported<double>(const JoinArgs<double>&);
template cudaError_t launch_count_tpq<float>(const JoinArgs<float>&, const uint32_t*, int, cudaStream_t);
template cudaError_t launch_count_tpq<double>(const JoinArgs<double>&, const uint32_t*, int, cudaStream_t);

}  // namespace gsj
