// Tile join for high-dimensional float data with populated cells.
//
// Replaces, for 5 <= n <= kTileMaxN float data, the reference's per-query
// traversal (kernelNDGridIndexGlobal / evaluateCell / evalPoint,
// kernel.cu:132-480) and its pair buffers + sort (GPU.cu:863-980).  A CTA owns
// a work item: up to kTileQ = 64 consecutive query slots of one cell.  It
//   1. enumerates the cell's 3^k neighbour offsets once (threads in parallel,
//      dense slot-prefix table or hash table, unicomp half-space with STAMP)
//      and compacts the non-empty ones in offset order;
//   2. keeps the 64 queries in shared memory, dimension-major;
//   3. walks the concatenated candidate slots 64 at a time: the candidate rows
//      are staged dimension-major in shared memory, and every thread evaluates
//      a 4 x 4 block of (query, candidate) pairs in registers with the
//      reference's exact arithmetic for the configured ILP/SHORTCIRCUIT model.
// Every model's running value only grows (every term is a rounded square,
// every step a monotone rounding), so a warp stops a tile as soon as all its
// pairs are above the threshold; that never changes a decision and is the
// reference's SHORTCIRCUIT taken further.
// Hits become packed (query id, candidate id) keys, appended with one atomic
// per warp and tile into a pair buffer; with STAMP a hit in another cell also
// yields the reverse pair (kernel.cu:367-375).  The buffer is then sorted on
// the device (the neighbour table in point-id order, each list ascending).
// The same kernel, without appending, samples every `stride`-th item to size
// the buffer (the role of the reference's batch estimator, GPU.cu:57-268);
// the full pass always counts every pair, so a buffer that turns out too
// small is re-sized exactly and the pass re-run.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

namespace {

constexpr int kTQ = kTileQ;   // queries per item
constexpr int kTC = 64;       // candidates per tile
constexpr int kThreads = 256; // 16 x 16 threads, 4 x 4 pairs each
constexpr uint32_t kNoSlot = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt_t() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct TileSmem {
    uint32_t qs, cs, nbs, nbp, cslot, cid, qid, misc, total;
};

__host__ __device__ inline TileSmem tile_smem(uint32_t npad, uint32_t noff) {
    TileSmem t{};
    uint32_t o = 0;
    t.qs = o;
    o += npad * kTQ * 4u;
    t.cs = o;
    o += npad * kTC * 4u;
    t.nbs = o;
    o += noff * 4u;
    t.nbp = o;
    o += (noff + 1u) * 4u;
    t.cslot = o;
    o += kTC * 4u;
    t.cid = o;
    o += kTC * 4u;
    t.qid = o;
    o += kTQ * 4u;
    t.misc = o;
    o += 16u * 4u;
    t.total = (o + 15u) & ~15u;
    return t;
}

// Squared distances of the thread's 4 x 4 pairs in the reference's order
// (float: a fused square-accumulate chain, see gsj_dist.cuh, kPolF32).
template <int MODEL>
__device__ __forceinline__ void tile_dists(const float* __restrict__ qs, const float* __restrict__ cs, uint32_t n,
                                           uint32_t ilp, float thr, int tx, int ty, unsigned valid,
                                           float (&acc)[4][4]) {
    const unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    auto all_dead = [&](const float (&v)[4][4]) {
        bool alive = false;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) alive |= ((valid >> (i * 4 + j)) & 1u) && !(v[i][j] > thr);
        return __all_sync(FULL, !alive);
    };
    if (MODEL == kSeq || MODEL == kIlpSc) {
        // kSeq: s = fma(d, d, s) over l.  kIlpSc (kernel.cu:320-334): the first
        // dim of every ILP block is fused into s, the others are squared on
        // their own and added.
        uint32_t p = 0;
        for (uint32_t l = 0; l < n; l++) {
            const float4 qa = *reinterpret_cast<const float4*>(qs + (size_t)l * kTQ + ty * 4);
            const float4 ca = *reinterpret_cast<const float4*>(cs + (size_t)l * kTC + tx * 4);
            const float qv[4] = {qa.x, qa.y, qa.z, qa.w};
            const float cv[4] = {ca.x, ca.y, ca.z, ca.w};
            const bool fused = MODEL == kSeq || p == 0;
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const float d = __fsub_rn(cv[j], qv[i]);
                    acc[i][j] = fused ? __fmaf_rn(d, d, acc[i][j]) : __fadd_rn(acc[i][j], __fmaf_rn(d, d, 0.f));
                }
            if (MODEL == kIlpSc && ++p == ilp) p = 0;
            if ((l & 7u) == 7u && l + 1 < n && all_dead(acc)) break;
        }
    } else {
        // kIlp (kernel.cu:312-341): r_j = fma chain over l == j (mod ILP), then
        // s = r_0 + r_1 + ... in j order.
        for (uint32_t jb = 0; jb < ilp && jb < n; jb++) {
            float r[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) r[i][j] = 0.f;
            for (uint32_t l = jb; l < n; l += ilp) {
                const float4 qa = *reinterpret_cast<const float4*>(qs + (size_t)l * kTQ + ty * 4);
                const float4 ca = *reinterpret_cast<const float4*>(cs + (size_t)l * kTC + tx * 4);
                const float qv[4] = {qa.x, qa.y, qa.z, qa.w};
                const float cv[4] = {ca.x, ca.y, ca.z, ca.w};
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float d = __fsub_rn(cv[j], qv[i]);
                        r[i][j] = __fmaf_rn(d, d, r[i][j]);
                    }
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = jb == 0 ? r[i][j] : __fadd_rn(acc[i][j], r[i][j]);
            if (jb + 1 < ilp && jb + 1 < n && all_dead(acc)) break;
        }
    }
}

template <int MODEL, bool STAMP>
__global__ void __launch_bounds__(kThreads) k_tile_join(const JoinArgs<float> a, const TileOut o, uint32_t noff,
                                                        uint32_t nvisit) {
    extern __shared__ __align__(16) unsigned char tsm[];
    const uint32_t n = a.n, npad = a.npad, k = a.g.k;
    const TileSmem L = tile_smem(npad, noff);
    float* qs = reinterpret_cast<float*>(tsm + L.qs);
    float* cs = reinterpret_cast<float*>(tsm + L.cs);
    uint32_t* nb_start = reinterpret_cast<uint32_t*>(tsm + L.nbs);
    uint32_t* nb_pref = reinterpret_cast<uint32_t*>(tsm + L.nbp);
    uint32_t* c_slot = reinterpret_cast<uint32_t*>(tsm + L.cslot);
    uint32_t* c_id = reinterpret_cast<uint32_t*>(tsm + L.cid);
    uint32_t* q_id = reinterpret_cast<uint32_t*>(tsm + L.qid);
    uint32_t* misc = reinterpret_cast<uint32_t*>(tsm + L.misc);  // [0] item, [2] total, [4..11] warp counts
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tid & 15, ty = tid >> 4;
    const unsigned lt = lanemask_lt_t();
    unsigned long long cand_total = 0;

    for (;;) {
        __syncthreads();  // the previous item is done with shared memory
        if (tid == 0) misc[0] = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t vi = misc[0];
        if (vi >= nvisit) break;
        const uint2 wi = a.items[(size_t)vi * o.stride];
        const uint32_t cell = wi.x;
        const uint32_t cs0 = a.cell_start[cell], ce = a.cell_start[cell + 1];
        const uint32_t q0 = cs0 + wi.y * (uint32_t)kTQ;
        const uint32_t qn = min((uint32_t)kTQ, ce - q0);

        // ---- own cell coordinates (the key formula, main.cu:744)
        uint32_t own[kMaxK];
#pragma unroll
        for (int j = 0; j < kMaxK; j++)
            own[j] = (j < (int)k) ? FP<float>::to_uint_rz(FP<float>::div(
                                        FP<float>::sub(a.pts[(size_t)cs0 * npad + j], a.minv[j]), a.eps))
                                  : 0u;
        // ---- neighbour cells in offset order (kernel.cu:180-303; stamploops.h)
        uint32_t nnb = 0;
        uint32_t lowmask, highmask, oddmask;
        cell_masks(own, a.g, lowmask, highmask, oddmask);
        const uint64_t own_lin = a.cell_key[cell];
        for (uint32_t base = 0; base < noff; base += kThreads) {
            const uint32_t off = base + tid;
            uint64_t lin = 0;
            const bool ok = off < noff && nb_offset<float, STAMP>(a, off, own_lin, lowmask, highmask, oddmask, lin);
            uint32_t st = 0, cnt = 0;
            const bool found = ok && lookup_range(a, lin, st, cnt);
            const unsigned m = __ballot_sync(FULL, found);
            if (lane == 0) misc[4 + warp] = __popc(m);
            __syncthreads();
            uint32_t before = 0, all = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; w++) {
                const uint32_t cw = misc[4 + w];
                before += (w < warp) ? cw : 0u;
                all += cw;
            }
            if (found) {
                const uint32_t pos = nnb + before + __popc(m & lt);
                nb_start[pos] = st;
                nb_pref[pos] = cnt;
            }
            nnb += all;
            __syncthreads();  // misc is rewritten next round
        }
        // ---- exclusive prefix of the candidate counts (warp 0)
        if (warp == 0) {
            uint32_t run = 0;
            for (uint32_t b = 0; b < nnb; b += 32) {
                const uint32_t i = b + lane;
                const uint32_t v = i < nnb ? nb_pref[i] : 0u;
                uint32_t x = v;
#pragma unroll
                for (int s = 1; s < 32; s <<= 1) {
                    const uint32_t y = __shfl_up_sync(FULL, x, s);
                    if (lane >= s) x += y;
                }
                if (i < nnb) nb_pref[i] = run + x - v;
                run += __shfl_sync(FULL, x, 31);
            }
            if (lane == 0) {
                nb_pref[nnb] = run;
                misc[2] = run;
            }
        }
        // ---- query tile, dimension-major; rows >= qn are zero and never valid
        for (uint32_t e = tid; e < (uint32_t)kTQ * npad; e += kThreads) {
            const uint32_t i = e / npad, l = e - i * npad;
            qs[(size_t)l * kTQ + i] = i < qn ? a.pts[(size_t)(q0 + i) * npad + l] : 0.f;
        }
        if (tid < kTQ) q_id[tid] = (uint32_t)tid < qn ? a.ids[q0 + tid] : 0u;
        __syncthreads();
        const uint32_t total = misc[2];
        cand_total += (unsigned long long)total * qn;
        unsigned qvalid = 0;
#pragma unroll
        for (int i = 0; i < 4; i++)
            if ((uint32_t)(ty * 4 + i) < qn) qvalid |= 0xfu << (i * 4);

        for (uint32_t t0 = 0; t0 < total; t0 += kTC) {
            // candidate slots of this tile (binary search over the prefix)
            if (tid < kTC) {
                const uint32_t f = t0 + tid;
                uint32_t slot = kNoSlot, cid = 0;
                if (f < total) {
                    uint32_t lo = 0, hi = nnb;  // nb_pref[lo] <= f < nb_pref[hi]
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (nb_pref[mid] <= f) lo = mid;
                        else hi = mid;
                    }
                    slot = nb_start[lo] + (f - nb_pref[lo]);
                    cid = a.ids[slot];
                }
                c_slot[tid] = slot;
                c_id[tid] = cid;
            }
            __syncthreads();
            // candidate rows, dimension-major (float4 reads of the padded rows)
            const uint32_t n4 = npad >> 2;
            for (uint32_t e = tid; e < (uint32_t)kTC * n4; e += kThreads) {
                const uint32_t j = e & (kTC - 1), l4 = e / kTC;
                const uint32_t slot = c_slot[j];
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (slot != kNoSlot) v = *reinterpret_cast<const float4*>(a.pts + (size_t)slot * npad + 4u * l4);
                float* dst = cs + (size_t)(4u * l4) * kTC + j;
                dst[0] = v.x;
                dst[kTC] = v.y;
                dst[2 * kTC] = v.z;
                dst[3 * kTC] = v.w;
            }
            __syncthreads();
            unsigned cvalid = 0;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (t0 + (uint32_t)(tx * 4 + j) < total) cvalid |= 0x1111u << j;
            const unsigned valid = qvalid & cvalid;
            float acc[4][4];
            tile_dists<MODEL>(qs, cs, n, a.ilp, a.thr, tx, ty, valid, acc);
            unsigned hit = 0;
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (((valid >> (i * 4 + j)) & 1u) && acc[i][j] <= a.thr) hit |= 1u << (i * 4 + j);
            if (__any_sync(FULL, hit != 0u)) {
                // cross: candidate outside the own cell (its reverse pair is
                // not produced by any other item under unicomp)
                unsigned cross = 0;
                if (STAMP) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const uint32_t sl = c_slot[tx * 4 + j];
                        if (sl != kNoSlot && (sl < cs0 || sl >= ce)) cross |= 0x1111u << j;
                    }
                }
                const uint32_t cnt = (uint32_t)__popc(hit) + (uint32_t)__popc(hit & cross);
                uint32_t x = cnt;
#pragma unroll
                for (int s = 1; s < 32; s <<= 1) {
                    const uint32_t y = __shfl_up_sync(FULL, x, s);
                    if (lane >= s) x += y;
                }
                const uint32_t wtotal = __shfl_sync(FULL, x, 31);
                unsigned long long base = 0;
                if (lane == 31) base = atomicAdd(o.cursor, (unsigned long long)wtotal);
                base = __shfl_sync(FULL, base, 31);
                if (o.emit && cnt) {
                    unsigned long long p = base + (x - cnt);
                    unsigned h = hit;
                    while (h) {
                        const int b = __ffs(h) - 1;
                        h &= h - 1u;
                        const uint64_t qid = q_id[ty * 4 + (b >> 2)], cid = c_id[tx * 4 + (b & 3)];
                        if (p < o.cap) o.pairs[p] = (qid << o.shift) | cid;
                        p++;
                        if (STAMP && ((cross >> b) & 1u)) {
                            if (p < o.cap) o.pairs[p] = (cid << o.shift) | qid;
                            p++;
                        }
                    }
                }
            }
            __syncthreads();  // the next tile overwrites c_slot / cs
        }
    }
    if (tid == 0 && cand_total && o.emit) atomicAdd(a.cand_cnt, cand_total);
}

template <int MODEL, bool STAMP>
cudaError_t launch_tile_one(const JoinArgs<float>& a, const TileOut& o, uint32_t noff, uint32_t nvisit, int num_sms,
                            cudaStream_t st) {
    auto kern = k_tile_join<MODEL, STAMP>;
    const TileSmem L = tile_smem(a.npad, noff);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return e;
    // the whole unified L1/shared array as shared memory, so that the CTAs the
    // occupancy calculation counts on are resident together
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = blocks_per_sm((const void*)kern, kThreads, L.total, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (a.shape_per_sm && (int)a.shape_per_sm < per_sm) per_sm = (int)a.shape_per_sm;
    uint64_t blocks = (uint64_t)num_sms * per_sm;
    if (blocks > nvisit) blocks = nvisit ? nvisit : 1;
    kern<<<(unsigned)blocks, kThreads, L.total, st>>>(a, o, noff, nvisit);
    return cudaGetLastError();
}

// Packed sorted pairs -> neighbour table + list lengths.  Keys are sorted, so
// the lanes of a warp that share a query add their count with one atomic.
__global__ void k_pairs_to_table(const unsigned long long* __restrict__ keys, uint64_t R, uint32_t shift,
                                 uint32_t* __restrict__ table, uint32_t* __restrict__ counts) {
    const uint64_t mask = (1ull << shift) - 1ull;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < R; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool v = i < R;
        const unsigned act = __ballot_sync(0xffffffffu, v);
        if (!v) continue;
        const unsigned long long kk = keys[i];
        table[i] = (uint32_t)(kk & mask);
        const uint32_t q = (uint32_t)(kk >> shift);
        const unsigned peers = __match_any_sync(act, q);
        if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&counts[q], (uint32_t)__popc(peers));
    }
}

}  // namespace

bool tile_supported(uint32_t n, uint32_t npad, uint32_t k, int model, uint32_t ilp) {
    return n >= 5 && n <= (uint32_t)kTileMaxN && (npad & 3u) == 0 && k >= 1 && k <= 6 &&
           (model == kSeq || model == kIlpSc || (model == kIlp && ilp >= 1));
}

cudaError_t launch_tile_join(const JoinArgs<float>& a, const TileOut& o, bool stamp, int model, uint32_t nvisit,
                             int num_sms, cudaStream_t st) {
    if (!tile_supported(a.n, a.npad, a.g.k, model, a.ilp) || o.stride == 0) return cudaErrorInvalidValue;
    if (nvisit == 0) return cudaSuccess;
    if ((uint64_t)(nvisit - 1) * o.stride >= a.num_items) return cudaErrorInvalidValue;
    uint32_t noff = 1;
    for (uint32_t j = 0; j < a.g.k; j++) noff *= 3u;
    switch (model * 2 + (stamp ? 1 : 0)) {
        case kSeq * 2: return launch_tile_one<kSeq, false>(a, o, noff, nvisit, num_sms, st);
        case kSeq * 2 + 1: return launch_tile_one<kSeq, true>(a, o, noff, nvisit, num_sms, st);
        case kIlp * 2: return launch_tile_one<kIlp, false>(a, o, noff, nvisit, num_sms, st);
        case kIlp * 2 + 1: return launch_tile_one<kIlp, true>(a, o, noff, nvisit, num_sms, st);
        case kIlpSc * 2: return launch_tile_one<kIlpSc, false>(a, o, noff, nvisit, num_sms, st);
        case kIlpSc * 2 + 1: return launch_tile_one<kIlpSc, true>(a, o, noff, nvisit, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pairs_to_table(const unsigned long long* keys, uint64_t R, uint32_t shift, uint32_t* table,
                                  uint32_t* counts, int num_sms, cudaStream_t st) {
    if (R == 0) return cudaSuccess;
    uint64_t blocks = (R + 255) / 256;
    const uint64_t cap = (uint64_t)num_sms * 32;
    if (blocks > cap) blocks = cap;
    k_pairs_to_table<<<(unsigned)blocks, 256, 0, st>>>(keys, R, shift, table, counts);
    return cudaGetLastError();
}

}  // namespace gsj
