// Candidate-cell distance join (subsystem (b)).
//
// Replaces kernelNDGridIndexGlobal / evaluateCell / evalPoint
// (kernel.cu:132-480, kernelloops.h, stamploops.h).  The reference runs one
// thread per query point, repeats the neighbour-cell search (2 binary searches
// per cell) for every query, and appends every hit with a global atomicAdd.
// Here one warp owns a work item: up to 32 consecutive query slots of one
// non-empty cell.  The warp
//   1. enumerates the cell's 3^k neighbour offsets once, lanes in parallel,
//      resolving each through the dense cell table or the hash table, and
//      compacts the non-empty ones (ballot) into a per-warp list in shared
//      memory - with STAMP only the unicomp half-space of stamploops.h;
//   2. stages the queries in shared memory;
//   3. walks the concatenated candidate slots 32 at a time, one candidate per
//      lane (rows are contiguous in the cell-sorted layout), and tests every
//      query against the 32 candidates with the reference's exact arithmetic
//      (s <= thr is sqrt(s) <= eps, see gsj_threshold_*).
// Every hit becomes a packed (query id, candidate id) key appended to the pair
// buffer (emit_keys), with STAMP also the reverse key of a hit in another cell
// (the reference emits (q,c) twice there, kernel.cu:367-375); the buffer is
// sorted into the neighbour table afterwards (the reference's pair buffers +
// sort_by_key, GPU.cu:863-980).  One traversal per join; a sampling run over
// every stride-th item sizes the buffer first.
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_fp.cuh"
#include "gsj_dist.cuh"
#include "gsj_kernels.h"

namespace gsj {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__host__ __device__ constexpr uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

__host__ __device__ constexpr uint32_t npad_for(uint32_t n, uint32_t tsize) {
    return n <= 2 ? n : ((n + (16u / tsize) - 1u) / (16u / tsize)) * (16u / tsize);
}

struct WarpSmem {
    uint32_t q_off, qid_off, nbs_off, nbp_off, cand_off, total;
};

__host__ __device__ inline WarpSmem warp_smem_layout(uint32_t npad, uint32_t tsize, uint32_t nb_cap, bool generic) {
    WarpSmem w{};
    uint32_t o = 0;
    w.q_off = o;
    o = align16(o + 32u * npad * tsize);
    w.qid_off = o;
    o = align16(o + 32u * 4u);
    w.nbs_off = o;
    o = align16(o + nb_cap * 4u);
    w.nbp_off = o;
    o = align16(o + (nb_cap + 1u) * 4u);
    w.cand_off = o;
    if (generic) o = align16(o + 32u * (npad + 1u) * tsize);
    w.total = o;
    return w;
}

// The warp appends its hits as packed (query id << shift |
// candidate id) keys, and with unicomp the reverse key of a hit in another
// cell, into blocks of kEmitBlk entries it reserves on o.cursor (unused tails
// padded with kUndecidedPad, which sorts after every key); emitted counts the
// keys exactly.  hit / cr are this lane's flags, b / cb their ballots.
constexpr uint32_t kEmitBlk = (uint32_t)kScreenBlockSlack;

__device__ __forceinline__ void emit_keys(const TileOut& o, unsigned long long& blk_base, uint32_t& blk_used,
                                          unsigned long long& emitted, bool hit, bool cr, unsigned b, unsigned cb,
                                          unsigned lt, int lane, uint64_t qid, uint64_t cid) {
    const uint32_t cnt = (uint32_t)__popc(b) + (uint32_t)__popc(cb);
    emitted += cnt;
    if (!o.emit) return;
    if (blk_used + cnt > kEmitBlk) {
        for (uint32_t e = blk_used + (uint32_t)lane; e < kEmitBlk; e += 32u)
            if (blk_base + e < o.cap) o.pairs[blk_base + e] = kUndecidedPad;
        unsigned long long nb = 0;
        if (lane == 0) nb = atomicAdd(o.cursor, (unsigned long long)kEmitBlk);
        blk_base = __shfl_sync(0xffffffffu, nb, 0);
        blk_used = 0;
    }
    if (hit) {
        unsigned long long p = blk_base + blk_used + (unsigned)__popc(b & lt) + (unsigned)__popc(cb & lt);
        if (p < o.cap) o.pairs[p] = (qid << o.shift) | cid;
        p++;
        if (cr && p < o.cap) o.pairs[p] = (cid << o.shift) | qid;
    }
    blk_used += cnt;
}

// Slot of candidate f = f0 + lane in the concatenated neighbour ranges
// (nb_pref: exclusive prefix of the range sizes, nb_pref[nnb] = total).  `ent`
// is the range holding f0 (warp-uniform).  Every range holds at least one
// candidate, so the warp's 32 candidates lie in ranges ent .. ent + 31: lane j
// loads nb_pref[ent + j] and each lane finds its range with a 5-step search
// over those values; `ent` then moves to the range of f0 + 32 (at most one
// range past lane 31's).
__device__ __forceinline__ uint32_t cand_slot(const uint32_t* nb_start, const uint32_t* nb_pref, uint32_t nnb,
                                              uint32_t& ent, uint32_t f0, uint32_t lane, uint32_t total) {
    const unsigned FULL = 0xffffffffu;
    const uint32_t f = f0 + lane;
    const uint32_t p = ent + lane <= nnb ? nb_pref[ent + lane] : 0xffffffffu;
    uint32_t lo = 0;
#pragma unroll
    for (uint32_t step = 16; step >= 1; step >>= 1) {
        const uint32_t c = lo + step;
        if (__shfl_sync(FULL, p, c) <= f) lo = c;
    }
    const uint32_t my = ent + lo;
    const uint32_t pf = __shfl_sync(FULL, p, lo);
    const uint32_t e31 = __shfl_sync(FULL, my, 31);
    ent = (e31 + 1u <= nnb && nb_pref[e31 + 1u] <= f0 + 32u) ? e31 + 1u : e31;
    return f < total ? nb_start[my] + (f - pf) : 0u;
}

// 4 CTAs of 8 warps per SM for float data (at most 64 registers a thread; the
// 6-D register path spills 36 bytes): on the 6-D mixture the emit stage went
// from 38.7 to 34.7 ms against 3 CTAs at 80 registers, the candidate-row loads
// being latency-bound.
template <typename T, int NT, int MODEL, int POL, bool STAMP, bool ROWS>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_join(const JoinArgs<T> a, uint32_t nb_cap, uint32_t noff,
                                              const TileOut o, uint32_t nvisit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr bool GENERIC = (NT == 0);
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t npad = a.npad;
    const WarpSmem L = warp_smem_layout(npad, sizeof(T), nb_cap, GENERIC);
    unsigned char* wb = smem_raw + (size_t)warp * L.total;
    T* q_s = reinterpret_cast<T*>(wb + L.q_off);
    uint32_t* qid_s = reinterpret_cast<uint32_t*>(wb + L.qid_off);
    uint32_t* nb_start = reinterpret_cast<uint32_t*>(wb + L.nbs_off);
    uint32_t* nb_pref = reinterpret_cast<uint32_t*>(wb + L.nbp_off);
    T* cand_s = reinterpret_cast<T*>(wb + L.cand_off);
    const unsigned lt = lanemask_lt();
    const uint32_t k = a.g.k;
    unsigned long long cand_total = 0;
    unsigned long long blk_base = 0, emitted = 0;
    uint32_t blk_used = kEmitBlk;

    // Work items are claimed one at a time: items in cell order are as heavy
    // as their cells are dense, so claiming runs of consecutive items left one
    // warp with a run of the densest cells long after the others had finished
    // (on a 5M-point 6-D Gaussian mixture the heaviest run of 32 items held 7.5x
    // a warp's mean share).  The next claim is issued before the current item
    // is processed and read after it, so its latency hides behind the item.
    // Item i is items[i * o.stride] (a stride above 1 samples every stride-th item).
    uint32_t claim = 0;
    if (lane == 0) claim = atomicAdd(a.work_counter, 1u);
    for (;;) {
        const uint32_t item = __shfl_sync(FULL, claim, 0);
        if (item >= nvisit) break;
        if (lane == 0) claim = atomicAdd(a.work_counter, 1u);
        const uint2 wi = a.items[(size_t)item * o.stride];
        const uint32_t cell = wi.x;
        const uint32_t cs = a.cell_start[cell], ce = a.cell_start[cell + 1];
        const uint32_t q0 = cs + wi.y * kQChunk;
        const uint32_t qn = min((uint32_t)kQChunk, ce - q0);

        uint32_t nnb = 0;
        if constexpr (ROWS) {
            // ---- dense grid, k <= 3: the cell plan holds, per neighbour row, the
            // slot range of cells x-1..x+1 (one contiguous range, see
            // k_cell_plan) and the parities of the own coordinates.
            const uint32_t nrows = k == 1 ? 1u : (k == 2 ? 3u : 9u);
            uint2 e = make_uint2(0u, 0u);
            if ((uint32_t)lane < nrows) e = a.plan[(size_t)cell * nrows + lane];
            if (STAMP) {
                // stamploops.h: own row -> its dim-0 neighbours only when x is odd;
                // another row -> all three cells when the own coordinate of its
                // highest differing dim is odd
                const uint32_t par = a.plan_par[cell];
                const int d1 = k >= 2 ? (int)(lane % 3) - 1 : 0;
                const int d2 = k >= 3 ? (int)(lane / 3) - 1 : 0;
                if (d1 == 0 && d2 == 0) {
                    if (!(par & 1u)) e = make_uint2(cs, ce - cs);
                } else if (!((par >> (d2 != 0 ? 2 : 1)) & 1u)) {
                    e.y = 0u;
                }
            }
            const bool found = (uint32_t)lane < nrows && e.y != 0u;
            const unsigned m = __ballot_sync(FULL, found);
            if (found) {
                const uint32_t pos = __popc(m & lt);
                nb_start[pos] = e.x;
                nb_pref[pos] = e.y;
            }
            nnb = __popc(m);
        } else {
            // ---- own cell coordinates, from the first query of the cell with the
            // formula the keys were built with (main.cu:744, kernel.cu:184)
            uint32_t own[kMaxK];
#pragma unroll
            for (int j = 0; j < kMaxK; j++)
                own[j] = (j < (int)k) ? FP<T>::to_uint_rz(FP<T>::div(FP<T>::sub(a.pts[(size_t)cs * npad + j], a.minv[j]),
                                                                       a.eps))
                                      : 0u;
            // ---- neighbour cells (kernel.cu:180-303; stamploops.h for STAMP)
            uint32_t lowmask, highmask, oddmask;
            cell_masks(own, a.g, lowmask, highmask, oddmask);
            const uint64_t own_lin = a.cell_key[cell];
            for (uint32_t base = 0; base < noff; base += 32) {
                const uint32_t o = base + lane;
                uint64_t lin = 0;
                const bool ok = o < noff && nb_offset<T, STAMP>(a, o, own_lin, lowmask, highmask, oddmask, lin);
                uint32_t st = 0, cnt = 0;
                const bool found = ok && lookup_range(a, lin, st, cnt);
                const unsigned m = __ballot_sync(FULL, found);
                if (found) {
                    const uint32_t pos = nnb + __popc(m & lt);
                    nb_start[pos] = st;
                    nb_pref[pos] = cnt;
                }
                nnb += __popc(m);
            }
        }
        __syncwarp();
        // exclusive prefix of candidate counts over the list
        uint32_t run = 0;
        for (uint32_t base = 0; base < nnb; base += 32) {
            const uint32_t i = base + lane;
            const uint32_t v = i < nnb ? nb_pref[i] : 0u;
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, x, o);
                if (lane >= o) x += y;
            }
            if (i < nnb) nb_pref[i] = run + x - v;
            run += __shfl_sync(FULL, x, 31);
        }
        const uint32_t total = run;
        if (lane == 0) nb_pref[nnb] = total;

        // ---- queries
        for (uint32_t e = lane; e < qn * npad; e += 32) q_s[e] = a.pts[(size_t)q0 * npad + e];
        if (lane < qn) qid_s[lane] = a.ids[q0 + lane];
        __syncwarp();
        cand_total += (unsigned long long)total * qn;
        const uint64_t my_qid = lane < qn ? qid_s[lane] : 0u;

        if constexpr (!GENERIC) {
            // ---- register path (n <= 8): up to G tiles of 32 candidates live in
            // registers; queries outside, tiles inside, so each query's
            // coordinates are loaded once per group of tiles.
            constexpr int G = 4;
            constexpr int NR = NT > 0 ? NT : 1;
            uint32_t ent = 0;
            for (uint32_t g0 = 0; g0 < total; g0 += 32u * G) {
                T cx[G][NR];
                uint32_t cid[G];
                bool cval[G], ccross[G];
                const uint32_t ntile = min((uint32_t)G, (total - g0 + 31u) / 32u);
#pragma unroll
                for (int t = 0; t < G; t++) {
                    const uint32_t f = g0 + (uint32_t)t * 32u + lane;
                    cval[t] = f < total;
                    cid[t] = 0u;
                    ccross[t] = false;
                    if ((uint32_t)t >= ntile) continue;
                    const uint32_t slot = cand_slot(nb_start, nb_pref, nnb, ent, g0 + (uint32_t)t * 32u, lane, total);
                    if (cval[t]) cid[t] = a.ids[slot];
                    ccross[t] = STAMP && cval[t] && (slot < cs || slot >= ce);  // outside the own cell
                    const T* row = a.pts + (size_t)slot * npad;
#pragma unroll
                    for (int l = 0; l < NR; l++) cx[t][l] = row[l];
                }
                for (uint32_t j = 0; j < qn; j++) {
                    T q[NR];
#pragma unroll
                    for (int l = 0; l < NR; l++) q[l] = q_s[(size_t)j * npad + l];
                    const uint64_t qid = __shfl_sync(FULL, my_qid, j);
#pragma unroll
                    for (int t = 0; t < G; t++) {
                        if ((uint32_t)t < ntile) {
                            const T s = sqdist_seq_reg<T, NR, POL>(q, cx[t]);
                            const bool hit = cval[t] && (s <= a.thr);
                            const unsigned b = __ballot_sync(FULL, hit);
                            if (b) {
                                const bool cr = STAMP && ccross[t] && hit;
                                const unsigned cb = __ballot_sync(FULL, cr);
                                emit_keys(o, blk_base, blk_used, emitted, hit, cr, b, cb, lt, lane, qid, cid[t]);
                            }
                        }
                    }
                }
            }
        } else {
            // ---- generic n: one tile of 32 candidate rows staged in shared memory
            uint32_t ent = 0;
            for (uint32_t t0 = 0; t0 < total; t0 += 32) {
                const uint32_t f = t0 + lane;
                const bool valid = f < total;
                const uint32_t slot = cand_slot(nb_start, nb_pref, nnb, ent, t0, lane, total);
                uint32_t corig = 0;
                bool cross = false;
                if (valid) {
                    cross = STAMP && (slot < cs || slot >= ce);  // outside the own cell
                    corig = a.ids[slot];
                }
                {
                    const T* row = a.pts + (size_t)slot * npad;
                    T* dst = cand_s + (size_t)lane * (npad + 1u);
                    for (uint32_t l = 0; l < a.n; l++) dst[l] = row[l];
                    __syncwarp();
                }
                for (uint32_t j = 0; j < qn; j++) {
                    const T* q = q_s + (size_t)j * npad;
                    const T s =
                        sqdist_generic<T, MODEL, POL>(q, cand_s + (size_t)lane * (npad + 1u), a.n, a.ilp, a.thr, valid);
                    const bool hit = valid && (s <= a.thr);
                    const unsigned b = __ballot_sync(FULL, hit);
                    if (b) {
                        const bool cr = STAMP && cross && hit;
                        const unsigned cb = __ballot_sync(FULL, cr);
                        emit_keys(o, blk_base, blk_used, emitted, hit, cr, b, cb, lt, lane,
                                  __shfl_sync(FULL, my_qid, j), corig);
                    }
                }
                __syncwarp();
            }
        }
        __syncwarp();
    }
    if (lane == 0 && cand_total && o.emit) atomicAdd(a.cand_cnt, cand_total);
    if (o.emit && blk_used < kEmitBlk)
        for (uint32_t e = blk_used + (uint32_t)lane; e < kEmitBlk; e += 32u)
            if (blk_base + e < o.cap) o.pairs[blk_base + e] = kUndecidedPad;
    if (lane == 0 && emitted) atomicAdd(o.rechecks, emitted);
}

// ------------------------------------------------------------------ launch
template <typename T, int NT, int MODEL, int POL, bool STAMP, bool ROWS>
static cudaError_t launch_one(const JoinArgs<T>& a, uint32_t nb_cap, uint32_t noff, const TileOut& o,
                              uint32_t nvisit, int num_sms, cudaStream_t st) {
    auto kern = k_join<T, NT, MODEL, POL, STAMP, ROWS>;
    const WarpSmem L = warp_smem_layout(a.npad, sizeof(T), nb_cap, NT == 0);
    const uint32_t max_smem = 200u * 1024u;
    int warps = (int)(max_smem / L.total);
    if (warps > 8) warps = 8;
    if (a.shape_warps && (int)a.shape_warps < warps) warps = (int)a.shape_warps;
    if (warps < 1) return cudaErrorInvalidValue;
    const int threads = warps * 32;
    const size_t smem = (size_t)warps * L.total;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the whole unified L1/shared array as shared memory, so that the CTAs the
    // occupancy calculation counts on are resident together
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = blocks_per_sm((const void*)kern, threads, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (a.shape_per_sm && (int)a.shape_per_sm < per_sm) per_sm = (int)a.shape_per_sm;
    const uint64_t needed = ((uint64_t)nvisit + warps - 1) / warps;
    uint64_t blocks = (uint64_t)num_sms * per_sm;
    if (blocks > needed) blocks = needed ? needed : 1;
    // every warp claims once past the last item: the counter must not wrap
    const uint64_t total_warps = blocks * (uint64_t)warps;
    if ((uint64_t)nvisit + total_warps >= 0xffffffffull) return cudaErrorInvalidValue;
    kern<<<(unsigned)blocks, threads, smem, st>>>(a, nb_cap, noff, o, nvisit);
    return cudaGetLastError();
}

template <typename T, int MODEL, int POL, bool STAMP>
static cudaError_t dispatch_nt(const JoinArgs<T>& a, bool rows, uint32_t nb_cap, uint32_t noff, const TileOut& o,
                               uint32_t nvisit, int num_sms, cudaStream_t st) {
    if (rows) {
        // low-dimensional dense grids (k <= 3): registers for n <= 4
        if (MODEL == kSeq && a.npad == npad_for(a.n, sizeof(T))) {
            switch (a.n) {
                case 1: return launch_one<T, 1, MODEL, POL, STAMP, true>(a, nb_cap, noff, o, nvisit, num_sms, st);
                case 2: return launch_one<T, 2, MODEL, POL, STAMP, true>(a, nb_cap, noff, o, nvisit, num_sms, st);
                case 3: return launch_one<T, 3, MODEL, POL, STAMP, true>(a, nb_cap, noff, o, nvisit, num_sms, st);
                case 4: return launch_one<T, 4, MODEL, POL, STAMP, true>(a, nb_cap, noff, o, nvisit, num_sms, st);
                default: break;
            }
        }
        return launch_one<T, 0, MODEL, POL, STAMP, true>(a, nb_cap, noff, o, nvisit, num_sms, st);
    }
    if (MODEL == kSeq && a.npad == npad_for(a.n, sizeof(T))) {
        switch (a.n) {
            case 6: return launch_one<T, 6, MODEL, POL, STAMP, false>(a, nb_cap, noff, o, nvisit, num_sms, st);
            case 8: return launch_one<T, 8, MODEL, POL, STAMP, false>(a, nb_cap, noff, o, nvisit, num_sms, st);
            default: break;
        }
    }
    return launch_one<T, 0, MODEL, POL, STAMP, false>(a, nb_cap, noff, o, nvisit, num_sms, st);
}

template <typename T, bool STAMP>
static cudaError_t dispatch_model(const JoinArgs<T>& a, int model, bool rows, uint32_t nb_cap, uint32_t noff,
                                  const TileOut& o, uint32_t nvisit, int num_sms, cudaStream_t st) {
    constexpr int P = sizeof(T) == 8 ? kPolF64 : kPolF32;
    switch (model) {
        case kSeq: return dispatch_nt<T, kSeq, P, STAMP>(a, rows, nb_cap, noff, o, nvisit, num_sms, st);
        case kIlp: return dispatch_nt<T, kIlp, P, STAMP>(a, rows, nb_cap, noff, o, nvisit, num_sms, st);
        case kIlpSc: return dispatch_nt<T, kIlpSc, P, STAMP>(a, rows, nb_cap, noff, o, nvisit, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_join_emit(const JoinArgs<T>& a, const TileOut& o, uint32_t nvisit, int model, bool stamp, bool rows,
                             int num_sms, cudaStream_t st) {
    uint32_t noff = 1;
    for (uint32_t j = 0; j < a.g.k; j++) noff *= 3u;
    if (rows && (a.g.k > 3 || !a.ds)) return cudaErrorInvalidValue;
    if (o.stride == 0) return cudaErrorInvalidValue;
    if (nvisit == 0) return cudaSuccess;
    if ((uint64_t)(nvisit - 1) * o.stride >= a.num_items) return cudaErrorInvalidValue;
    const uint32_t nb_cap = rows ? 32u : noff;
    return stamp ? dispatch_model<T, true>(a, model, rows, nb_cap, noff, o, nvisit, num_sms, st)
                 : dispatch_model<T, false>(a, model, rows, nb_cap, noff, o, nvisit, num_sms, st);
}

template cudaError_t launch_join_emit<float>(const JoinArgs<float>&, const TileOut&, uint32_t, int, bool, bool, int,
                                             cudaStream_t);
template cudaError_t launch_join_emit<double>(const JoinArgs<double>&, const TileOut&, uint32_t, int, bool, bool, int,
                                              cudaStream_t);

}  // namespace gsj
