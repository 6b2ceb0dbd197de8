// Join of dense low-dimensional grids (k <= 3, n <= 4): the ROWS path.
//
// Low-dimensional workloads have tiny cells (a 2-D mixture of 20M points
// averages 3 points per non-empty cell), so any per-cell set-up done by a
// whole warp costs more than the distance tests.  Each query's candidates are
// the 3^(k-1) contiguous slot ranges of its cell plan (k_cell_plan), the full
// neighbourhood of kernel.cu:292-302, taken in a fixed order: candidate f of
// query s is the f-th slot of the concatenated ranges.
//
//   k_rows_count  one thread per query slot (the slots of a warp are
//                 consecutive in cell order, so lanes of one cell walk the same
//                 ranges: broadcast loads).  It evaluates every candidate in the
//                 reference's arithmetic and records the decisions as a bit
//                 mask (bit f of the query's words), the list length by slot and
//                 by point id.
//   k_rows_fill   a warp per 32 consecutive query slots, two queries at a time
//                 (one per half-warp).  A half-warp replays its query's bit mask
//                 - no second distance pass - one mask word per step: lane l
//                 takes bits 2l and 2l + 1, loads the ids of those candidates
//                 whose bit is set, and stores them at the query's next free list
//                 positions, so each word's hits are written by the half's lanes
//                 to consecutive places of the point-id-ordered table.
// Both kernels claim their 32-slot chunks dynamically (one atomic per warp,
// the next claim issued before the current chunk is processed), since chunk
// costs vary with the local density by orders of magnitude.
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

#include "gsj_common.cuh"
#include "gsj_dist.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

namespace {

// Next 32-slot chunk of the warp (lane 0 claims; the caller broadcasts it).
__device__ __forceinline__ uint32_t claim32(uint32_t* ctr, int lane) {
    uint32_t v = 0;
    if (lane == 0) v = atomicAdd(ctr, 32u);
    return v;
}

}  // namespace

// Coordinates of one point row (NT values of a row padded to npad = 1, 2 or
// 4 entries, so the vector forms are aligned).
template <typename T, int NT>
__device__ __forceinline__ void load_row(const T* __restrict__ p, T (&r)[NT]) {
    if constexpr (std::is_same<T, float>::value && NT == 2) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        r[0] = v.x;
        r[1] = v.y;
    } else if constexpr (std::is_same<T, float>::value && NT >= 3) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        r[0] = v.x;
        r[1] = v.y;
        r[2] = v.z;
        if constexpr (NT == 4) r[3] = v.w;
    } else if constexpr (std::is_same<T, double>::value && NT >= 2) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        r[0] = v.x;
        r[1] = v.y;
        if constexpr (NT >= 3) {
            const double2 w = *reinterpret_cast<const double2*>(p + 2);
            r[2] = w.x;
            if constexpr (NT == 4) r[3] = w.y;
        }
    } else {
#pragma unroll
        for (int l = 0; l < NT; l++) r[l] = p[l];
    }
}

template <typename T, int NT, int NR, int POL>
__global__ void __launch_bounds__(256) k_rows_count(const JoinArgs<T> a, const uint32_t* __restrict__ slot_cell,
                                                    const uint64_t* __restrict__ bitoff, uint32_t* __restrict__ bits,
                                                    uint32_t* __restrict__ counts_by_id) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t N = a.n_points;
    const uint32_t npad = a.npad;
    const T thr = a.thr;
    unsigned long long cand = 0;
    uint32_t cur = __shfl_sync(FULL, claim32(a.work_counter, lane), 0);
    while (cur < N) {
        const uint32_t nxt = claim32(a.work_counter, lane);  // in flight while this chunk runs
        const uint32_t s = cur + (uint32_t)lane;
        if (s < N) {
            const uint32_t cell = slot_cell[s];
            T q[NT];
            load_row<T, NT>(a.pts + (size_t)s * npad, q);
            uint64_t wp = bitoff[s];
            uint32_t cnt = 0, word = 0, b = 0;  // b: next bit of the current mask word
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const uint2 e = a.plan[(size_t)cell * NR + r];
                const T* cp = a.pts + (size_t)e.x * npad;
                uint32_t left = e.y;
                cand += left;
                while (left) {
                    // candidates up to the end of the current mask word
                    const uint32_t m = min(left, 32u - b);
#pragma unroll 4
                    for (uint32_t u = 0; u < m; u++) {
                        T cr[NT];
                        load_row<T, NT>(cp, cr);
                        cp += npad;
                        const T d2 = sqdist_seq_reg<T, NT, POL>(q, cr);
                        word |= (d2 <= thr ? 1u : 0u) << (b + u);
                    }
                    b += m;
                    left -= m;
                    if (b == 32u) {
                        bits[wp++] = word;
                        cnt += (uint32_t)__popc(word);
                        word = 0u;
                        b = 0u;
                    }
                }
            }
            if (b) {
                bits[wp] = word;
                cnt += (uint32_t)__popc(word);
            }
            a.fwd_cnt[s] = cnt;
            counts_by_id[a.ids[s]] = cnt;
        }
        cur = __shfl_sync(FULL, nxt, 0);
    }
    // one atomic per warp for the candidate statistic
    for (int o = 16; o > 0; o >>= 1) cand += __shfl_down_sync(FULL, cand, o);
    if (lane == 0 && cand) atomicAdd(a.cand_cnt, cand);
}

// Queries: the slots qslots[0 .. nq) (all slots 0 .. nq-1 when qslots is
// null); the list of point id i goes to a.table[offsets[i] - base].
// Per-query parameters of the fill, staged in shared memory by the lane that
// loaded them and read back by the whole warp (one broadcast per 16 bytes).
template <int NR>
struct alignas(16) FillQuery {
    unsigned long long dst;  // list place in the table (relative to the batch base)
    unsigned long long bo;   // first mask word
    uint32_t cnt, nw;        // list length, mask words
    uint32_t lo[NR];         // first slot of each candidate row
    uint32_t pre[NR];        // candidates before each row
};

template <int NR>
__global__ void __launch_bounds__(256) k_rows_fill(const JoinArgs<float> a, const uint32_t* __restrict__ slot_cell,
                                                   const uint64_t* __restrict__ bitoff,
                                                   const uint32_t* __restrict__ bits,
                                                   const uint32_t* __restrict__ qslots, uint32_t nq, uint64_t base) {
    __shared__ FillQuery<NR> qp[8][32];  // blockDim.x <= 256
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    FillQuery<NR>* wq = qp[threadIdx.x >> 5];
    uint32_t cur = __shfl_sync(FULL, claim32(a.work_counter, lane), 0);
    while (cur < nq) {
        const uint32_t nxt = claim32(a.work_counter, lane);
        const uint32_t j = cur + (uint32_t)lane;
        const uint32_t nv = min(32u, nq - cur);
        // lane j: query j's list length, mask words, list place and candidate rows
        FillQuery<NR> f{};
        if (j < nq) {
            const uint32_t s = qslots ? qslots[j] : j;
            f.cnt = a.fwd_cnt[s];
            f.bo = bitoff[s];
            f.nw = (uint32_t)(bitoff[s + 1] - f.bo);
            f.dst = a.offsets[a.ids[s]] - base;
            if (f.dst + f.cnt > a.table_cap) {
                *a.err_flag = 1u;
                f.cnt = 0u;
            }
            const uint32_t cell = slot_cell[s];
            uint32_t p = 0;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const uint2 e = a.plan[(size_t)cell * NR + r];
                f.lo[r] = e.x;
                f.pre[r] = p;
                p += e.y;
            }
        }
        __syncwarp();  // the previous chunk's reads of wq are done
        wq[lane] = f;
        __syncwarp();
        // two queries at a time, one per half-warp: lane l of a half takes bits
        // 2l and 2l + 1 of each of its query's mask words
        const uint32_t h = (uint32_t)lane >> 4, hl = (uint32_t)lane & 15u;
        for (uint32_t qi = 0; qi < nv; qi += 2u) {
            const FillQuery<NR> q = wq[qi + h];  // entries past nv are zero (no words)
            const uint32_t qnw = q.cnt ? q.nw : 0u;
            uint32_t* list = a.table + q.dst;
            const uint32_t* qb = bits + q.bo;
            const uint32_t nwmax = max(__shfl_sync(FULL, qnw, 0), __shfl_sync(FULL, qnw, 16));
            uint32_t run = 0;  // entries of this half's list written so far
            for (uint32_t t0 = 0; t0 < nwmax; t0 += 16u) {
                const uint32_t myw = (t0 + hl < qnw) ? qb[t0 + hl] : 0u;
                const uint32_t tn = min(16u, nwmax - t0);
                for (uint32_t tt = 0; tt < tn; tt++) {
                    const uint32_t w = __shfl_sync(FULL, myw, (int)(h * 16u + tt));
                    if (__ballot_sync(FULL, w != 0u) == 0u) continue;
#pragma unroll
                    for (uint32_t bs = 0; bs < 2u; bs++) {
                        const uint32_t bit = 2u * hl + bs;
                        if ((w >> bit) & 1u) {
                            const uint32_t f = (t0 + tt) * 32u + bit;
                            uint32_t st = q.lo[0] + f;
#pragma unroll
                            for (int r = 1; r < NR; r++)
                                if (f >= q.pre[r]) st = q.lo[r] + (f - q.pre[r]);
                            list[run + (uint32_t)__popc(w & ((1u << bit) - 1u))] = a.ids[st];
                        }
                    }
                    run += (uint32_t)__popc(w);
                }
            }
        }
        cur = __shfl_sync(FULL, nxt, 0);
    }
}

// Resident CTAs of a kernel, for persistent grids.
static int resident_blocks(const void* kern, int threads, size_t smem, int num_sms) {
    int per_sm = 0;
    if (blocks_per_sm(kern, threads, smem, &per_sm) != cudaSuccess || per_sm < 1) per_sm = 1;
    return num_sms * per_sm;
}

template <typename T, int NT, int NR>
static cudaError_t launch_count_nt(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff,
                                   uint32_t* bits, uint32_t* counts_by_id, int num_sms, cudaStream_t st) {
    constexpr int POL = sizeof(T) == 8 ? kPolF64 : kPolF32;
    auto kern = k_rows_count<T, NT, NR, POL>;
    const int threads = a.shape_threads ? (int)a.shape_threads : 256;
    uint64_t blocks = (uint64_t)resident_blocks((const void*)kern, threads, 0, num_sms);
    const uint64_t needed = ((uint64_t)a.n_points + threads - 1) / threads;
    if (blocks > needed) blocks = needed ? needed : 1;
    kern<<<(unsigned)blocks, threads, 0, st>>>(a, slot_cell, bitoff, bits, counts_by_id);
    return cudaGetLastError();
}

template <typename T, int NR>
static cudaError_t count_nr(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff, uint32_t* bits,
                            uint32_t* counts_by_id, int num_sms, cudaStream_t st) {
    switch (a.n) {
        case 1: return launch_count_nt<T, 1, NR>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
        case 2: return launch_count_nt<T, 2, NR>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
        case 3: return launch_count_nt<T, 3, NR>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
        case 4: return launch_count_nt<T, 4, NR>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
bool tpq_supported(const JoinArgs<T>& a) {
    return a.n >= 1 && a.n <= 4 && a.ilp == 0 && a.g.k <= 3 && a.plan != nullptr;
}

template <typename T>
cudaError_t launch_rows_count(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff, uint32_t* bits,
                              uint32_t* counts_by_id, int num_sms, cudaStream_t st) {
    if (!tpq_supported(a)) return cudaErrorInvalidValue;
    if (a.g.k == 1) return count_nr<T, 1>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
    if (a.g.k == 2) return count_nr<T, 3>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
    return count_nr<T, 9>(a, slot_cell, bitoff, bits, counts_by_id, num_sms, st);
}

template <int NR>
static cudaError_t fill_nr(const JoinArgs<float>& a, const uint32_t* slot_cell, const uint64_t* bitoff,
                           const uint32_t* bits, const uint32_t* qslots, uint32_t nq, uint64_t base, int num_sms,
                           cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    auto kern = k_rows_fill<NR>;
    const int threads = a.shape_threads ? (int)a.shape_threads : 256;
    uint64_t blocks = (uint64_t)resident_blocks((const void*)kern, threads, 0, num_sms);
    const uint64_t needed = ((uint64_t)nq + threads - 1) / threads;
    if (blocks > needed) blocks = needed ? needed : 1;
    kern<<<(unsigned)blocks, threads, 0, st>>>(a, slot_cell, bitoff, bits, qslots, nq, base);
    return cudaGetLastError();
}

// The fill pass reads no coordinates: the table, offsets, ids and plan are
// independent of the coordinate type, so both precisions share one kernel
// (JoinArgs<float> view of the same buffers).
template <typename T>
cudaError_t launch_rows_fill(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff,
                             const uint32_t* bits, const uint32_t* qslots, uint32_t nq, uint64_t base, int num_sms,
                             cudaStream_t st) {
    if (!tpq_supported(a)) return cudaErrorInvalidValue;
    JoinArgs<float> f{};
    f.ids = a.ids;
    f.plan = a.plan;
    f.work_counter = a.work_counter;
    f.n_points = a.n_points;
    f.fwd_cnt = a.fwd_cnt;
    f.offsets = a.offsets;
    f.table = a.table;
    f.table_cap = a.table_cap;
    f.err_flag = a.err_flag;
    f.shape_threads = a.shape_threads;
    if (a.g.k == 1) return fill_nr<1>(f, slot_cell, bitoff, bits, qslots, nq, base, num_sms, st);
    if (a.g.k == 2) return fill_nr<3>(f, slot_cell, bitoff, bits, qslots, nq, base, num_sms, st);
    return fill_nr<9>(f, slot_cell, bitoff, bits, qslots, nq, base, num_sms, st);
}

template bool tpq_supported<float>(const JoinArgs<float>&);
template bool tpq_supported<double>(const JoinArgs<double>&);
template cudaError_t launch_rows_count<float>(const JoinArgs<float>&, const uint32_t*, const uint64_t*, uint32_t*,
                                              uint32_t*, int, cudaStream_t);
template cudaError_t launch_rows_count<double>(const JoinArgs<double>&, const uint32_t*, const uint64_t*, uint32_t*,
                                               uint32_t*, int, cudaStream_t);
template cudaError_t launch_rows_fill<float>(const JoinArgs<float>&, const uint32_t*, const uint64_t*,
                                             const uint32_t*, const uint32_t*, uint32_t, uint64_t, int, cudaStream_t);
template cudaError_t launch_rows_fill<double>(const JoinArgs<double>&, const uint32_t*, const uint64_t*,
                                              const uint32_t*, const uint32_t*, uint32_t, uint64_t, int,
                                              cudaStream_t);

// ---------------------------------------------------------------- result batches
// Batch b of the host-result pipeline holds the point ids [bound[b],
// bound[b+1]): its lists are the table range [boff[b], boff[b+1]) with boff[b]
// = offsets[bound[b]].  bound[b] = the last id whose list starts at or below
// b * step, so with step = segment capacity minus the longest list every batch
// fits one segment; bound[0] = 0, bound[nb] = N.
__global__ void k_batch_bounds(const uint64_t* __restrict__ offsets, uint32_t N, uint64_t step, uint32_t nb,
                               uint32_t* __restrict__ bound, unsigned long long* __restrict__ boff) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    if (b == 0 || b == nb) {
        bound[b] = b == 0 ? 0u : N;
        boff[b] = b == 0 ? 0ull : offsets[N];
        return;
    }
    const unsigned long long target = (unsigned long long)b * step;
    uint32_t lo = 0, hi = N;  // first i in [0, N) with offsets[i] > target (N if none)
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (offsets[mid] > target) hi = mid;
        else lo = mid + 1u;
    }
    bound[b] = lo > 0 ? lo - 1u : 0u;
    boff[b] = offsets[bound[b]];
}

// Batch index of every slot's point id (binary search over the bounds), and
// the slot index as the value of the stable sort by batch.
__global__ void k_slot_batch(const uint32_t* __restrict__ ids, uint32_t N, const uint32_t* __restrict__ bound,
                             uint32_t nb, uint32_t* __restrict__ bkey, uint32_t* __restrict__ slot) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint32_t id = ids[s];
    uint32_t lo = 0, hi = nb;  // last b with bound[b] <= id
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) / 2u;
        if (bound[mid] <= id) lo = mid;
        else hi = mid;
    }
    bkey[s] = lo;
    slot[s] = s;
}

// Start of each batch's slots in the batch-sorted slot list: gstart[b] =
// first position whose batch key is >= b, gstart[nb] = N.
__global__ void k_group_starts(const uint32_t* __restrict__ sorted_bkey, uint32_t N, uint32_t nb,
                               uint32_t* __restrict__ gstart) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    uint32_t lo = 0, hi = N;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (sorted_bkey[mid] >= b) hi = mid;
        else lo = mid + 1u;
    }
    gstart[b] = lo;
}

// *out = max(in[0 .. n)) (*out zeroed by the caller).
__global__ void k_max_u32(const uint32_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ out) {
    uint32_t m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, in[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

cudaError_t launch_batch_bounds(const uint64_t* offsets, uint32_t N, uint64_t step, uint32_t nb, uint32_t* bound,
                                unsigned long long* boff, cudaStream_t st) {
    k_batch_bounds<<<(nb + 1 + 127) / 128, 128, 0, st>>>(offsets, N, step, nb, bound, boff);
    return cudaGetLastError();
}

cudaError_t launch_slot_batch(const uint32_t* ids, uint32_t N, const uint32_t* bound, uint32_t nb, uint32_t* bkey,
                              uint32_t* slot, cudaStream_t st) {
    k_slot_batch<<<(N + 255) / 256, 256, 0, st>>>(ids, N, bound, nb, bkey, slot);
    return cudaGetLastError();
}

cudaError_t launch_group_starts(const uint32_t* sorted_bkey, uint32_t N, uint32_t nb, uint32_t* gstart,
                                cudaStream_t st) {
    k_group_starts<<<(nb + 1 + 127) / 128, 128, 0, st>>>(sorted_bkey, N, nb, gstart);
    return cudaGetLastError();
}

cudaError_t launch_max_u32(const uint32_t* in, uint64_t n, uint32_t* out, cudaStream_t st) {
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    k_max_u32<<<(unsigned)(blocks ? blocks : 1), 256, 0, st>>>(in, n, out);
    return cudaGetLastError();
}

// Slot -> cell map and the bit-mask words of each slot's query: every query
// of cell c has the same candidates, ceil(sum of its plan rows / 32) words.
__global__ void k_slot_cell(const uint32_t* __restrict__ cell_start, uint32_t M, const uint2* __restrict__ plan,
                            uint32_t nrows, uint32_t* __restrict__ slot_cell, uint32_t* __restrict__ swords) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    uint64_t tot = 0;
    if (swords)
        for (uint32_t r = 0; r < nrows; r++) tot += plan[(size_t)c * nrows + r].y;
    const uint32_t w = (uint32_t)((tot + 31u) / 32u);
    for (uint32_t s = cell_start[c]; s < cell_start[c + 1]; s++) {
        slot_cell[s] = c;
        if (swords) swords[s] = w;
    }
}

cudaError_t launch_slot_cell(const uint32_t* cell_start, uint32_t M, const uint2* plan, uint32_t nrows,
                             uint32_t* slot_cell, uint32_t* swords, cudaStream_t st) {
    k_slot_cell<<<(M + 255) / 256, 256, 0, st>>>(cell_start, M, plan, nrows, slot_cell, swords);
    return cudaGetLastError();
}

}  // namespace gsj
