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
// its own neighbour set, which it counts (pass kCount) or appends to its list
// (pass kFill).
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_dist.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

template <typename T, int NT, int POL, int PASS>
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
        unsigned long long cur = 0;
        if (PASS == kFill) cur = a.offsets[a.ids[s]];
        for (uint32_t r = 0; r < nrows; r++) {
            const uint2 e = a.plan[(size_t)cell * nrows + r];
            if (PASS == kCount) cand += e.y;
            for (uint32_t i = 0; i < e.y; i++) {
                const uint32_t c = e.x + i;
                T cr[NT];
#pragma unroll
                for (int l = 0; l < NT; l++) cr[l] = a.pts[(size_t)c * npad + l];
                const T d2 = sqdist_seq_reg<T, NT, POL>(q, cr);
                if (d2 <= a.thr) {
                    if (PASS == kCount) {
                        cnt++;
                    } else {
                        if (cur < a.table_cap) a.table[cur] = a.ids[c];
                        else *a.err_flag = 1u;
                        cur++;
                    }
                }
            }
        }
        if (PASS == kCount) {
            a.fwd_cnt[s] = cnt;
            a.rev_cnt[s] = 0u;
        }
    }
    if (PASS == kCount) {
        // one atomic per warp for the candidate statistic
        for (int o = 16; o > 0; o >>= 1) cand += __shfl_down_sync(0xffffffffu, cand, o);
        if ((threadIdx.x & 31) == 0 && cand) atomicAdd(a.cand_cnt, cand);
    }
}

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

template <typename T, int NT, int PASS>
static cudaError_t launch_tpq_nt(const JoinArgs<T>& a, const uint32_t* slot_cell, uint32_t nrows, int num_sms,
                                 cudaStream_t st) {
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    auto kern = k_rows_tpq<T, NT, POL, PASS>;
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
cudaError_t launch_join_tpq(const JoinArgs<T>& a, int pass, const uint32_t* slot_cell, int num_sms,
                            cudaStream_t st) {
    if (!tpq_supported(a)) return cudaErrorInvalidValue;
    const uint32_t nrows = a.g.k == 1 ? 1u : (a.g.k == 2 ? 3u : 9u);
    switch (a.n * 2 + (pass == kFill ? 1 : 0)) {
        case 2: return launch_tpq_nt<T, 1, kCount>(a, slot_cell, nrows, num_sms, st);
        case 3: return launch_tpq_nt<T, 1, kFill>(a, slot_cell, nrows, num_sms, st);
        case 4: return launch_tpq_nt<T, 2, kCount>(a, slot_cell, nrows, num_sms, st);
        case 5: return launch_tpq_nt<T, 2, kFill>(a, slot_cell, nrows, num_sms, st);
        case 6: return launch_tpq_nt<T, 3, kCount>(a, slot_cell, nrows, num_sms, st);
        case 7: return launch_tpq_nt<T, 3, kFill>(a, slot_cell, nrows, num_sms, st);
        case 8: return launch_tpq_nt<T, 4, kCount>(a, slot_cell, nrows, num_sms, st);
        case 9: return launch_tpq_nt<T, 4, kFill>(a, slot_cell, nrows, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

template bool tpq_supported<float>(const JoinArgs<float>&);
template bool tpq_supported<double>(const JoinArgs<double>&);
template cudaError_t launch_join_tpq<float>(const JoinArgs<float>&, int, const uint32_t*, int, cudaStream_t);
template cudaError_t launch_join_tpq<double>(const JoinArgs<double>&, int, const uint32_t*, int, cudaStream_t);

}  // namespace gsj
