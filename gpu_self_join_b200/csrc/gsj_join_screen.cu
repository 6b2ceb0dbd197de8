// Tensor-core screened tile join for high-dimensional float data.
//
// Same work decomposition and output as the tile join (gsj_join_tile.cu): a
// CTA owns up to kScreenQ = 128 consecutive query slots of one cell, walks the
// concatenated candidate slots of the cell's neighbour cells (3^k offsets,
// kernel.cu:180-303) 128 at a time and appends every pair within eps as a
// packed (query id, candidate id) key.  What changes is how a pair is decided:
//
//   1. Once per join (k_screen_rows), every point is centred on the data mean
//      o and rounded to BF16, c^ = bf16(fl(c - o)), and stored with its norm
//      as a row [c^, |c^|^2_hi, |c^|^2_lo] (slot order).  Candidate tiles are
//      copied from these rows (cp.async, 16-byte chunks) into K-major
//      shared-memory tiles (8 x 16-byte core matrices, no swizzle); the query
//      tile holds [-2 q^, 1, 1], so the product carries the candidate norm.
//   2. One thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M = N =
//      128, K = 16 per instruction) over the padded dimensions; the 128 x 128
//      values |c^_j|^2 - 2 q^_i.c^_j accumulate in tensor memory (exact
//      BF16 products; -2 q^ is exact in BF16).
//   3. Every consumer thread reads its query's row (tcgen05.ld 32x32b) and
//      rejects candidate j when that value exceeds
//      G_i = (R0 + kE (|q^_i| + max_j |c^_j|))^2 + c1 (|q^_i|^2 + 2 max_j |c^_j|^2) - |q^_i|^2,
//      the maximum over the 32 candidates of j's column group.
//      The bound is proven, not tuned: R0^2 covers the rounding of the
//      reference's own FP32 sum (at most 2n+8 roundings of non-negative
//      terms), kE the BF16 rounding of both centred points and of the centring
//      (|x - bf16(x)| <= 2^-8 |x|), c1 the FP32 accumulation (K + 32 steps of
//      2^-20) and the two-term BF16 split of the norm (2^-16).  A pair within
//      eps by the reference's arithmetic is therefore never rejected.
//   4. Every pair not rejected is appended to a list of undecided pairs;
//      k_screen_recheck recomputes each in the reference's exact FP32 order
//      from the original coordinates (ILP/SHORTCIRCUIT model,
//      kernel.cu:307-365) and keeps it iff s <= thr.
// The emitted pair set is the plain path's, bit for bit.  Non-finite values
// only make the test inconclusive, which sends the pair to the exact check.
//
// Synchronisation: warps 8-11 produce candidate tiles (slot search, cp.async of
// the rows) and one of their threads issues the MMA, warps 0-7 consume;
// candidate tiles rotate through kStages buffers and two accumulators
// alternate, handed over by mbarriers only (staged: every producer thread's
// slots and landed rows of a buffer; full: MMA commit + the issuer's release;
// empty and free: the consumer arrivals), so the producer warps never wait for
// one another.  Every wait is a bounded poll by one thread whose outcome is
// shared before any warp-collective; on time-out the error flag is raised and
// the CTA stops.  Tensor memory (2 x 128 columns) is allocated once
// per CTA; the shared-memory request keeps at most 2 CTAs (512 columns) on an
// SM; it is released before exit.
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

namespace {

constexpr int kSQ = kScreenQ;        // queries per item = MMA M
constexpr int kSC = 128;             // candidates per tile = MMA N
constexpr int kSThreads = 384;      // warps 0-7 consume, warps 8-11 produce
constexpr int kProd0 = 256;         // first producer thread
constexpr uint32_t kTmemCols = 128;  // FP32 accumulator columns (N)
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kMinSmem = 80u * 1024u;  // at most 2 CTAs (2 x 256 TMEM columns) per SM
constexpr uint32_t kWaitPolls = 1u << 20;
constexpr uint32_t kBlk = (uint32_t)kScreenBlockSlack;  // undecided-pair entries a consumer warp reserves
constexpr uint32_t kStages = 3;     // candidate tiles in flight (the accumulators alternate in 2)

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bit 4),
// A and B BF16 (bits 7 and 10), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kSC >> 3) << 17) |
                            ((uint32_t)(kSQ >> 4) << 24);

__device__ __forceinline__ unsigned lanemask_lt_s() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8 rows
// x 16 bytes; LBO = byte distance between K-adjacent core matrices, SBO =
// between row-group-adjacent ones; version 1 (bit 46).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Byte offset of element (r, k) of a K-major tile with kpad columns.
__device__ __forceinline__ uint32_t core_off(uint32_t r, uint32_t kc, uint32_t kpad) {
    return ((r >> 3) * (kpad >> 3) + kc) * 128u + (r & 7u) * 16u;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// try_wait suspends the thread in hardware until the phase completes or an
// implementation-defined time passes; the loop bounds the total wait.
__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool bar_wait_bounded(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitPolls; it++)
        if (bar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// The reference's squared distance in its exact order, one thread, stopping
// as soon as the running value (which only grows) is above thr.
template <int MODEL>
__device__ float exact_sqdist(const float* __restrict__ q, const float* __restrict__ c, uint32_t n, uint32_t ilp,
                              float thr) {
    if (MODEL == kSeq || MODEL == kIlpSc) {
        float s = 0.f;
        uint32_t p = 0;
        for (uint32_t l = 0; l < n; l++) {
            const float d = __fsub_rn(c[l], q[l]);
            s = (MODEL == kSeq || p == 0) ? __fmaf_rn(d, d, s) : __fadd_rn(s, __fmaf_rn(d, d, 0.f));
            if (MODEL == kIlpSc && ++p == ilp) p = 0;
            if (s > thr) break;
        }
        return s;
    } else {
        float s = 0.f;
        for (uint32_t j = 0; j < ilp && j < n; j++) {
            float r = 0.f;
            for (uint32_t l = j; l < n; l += ilp) {
                const float d = __fsub_rn(c[l], q[l]);
                r = __fmaf_rn(d, d, r);
            }
            s = j == 0 ? r : __fadd_rn(s, r);
            if (s > thr) break;
        }
        return s;
    }
}

// Same arithmetic, rows read as float4 blocks of 32 dimensions loaded before
// use (npad is a multiple of 4 here); the ILP model without SHORTCIRCUIT
// walks its dimensions with stride ILP and keeps the scalar form.
template <int MODEL>
__device__ float exact_sqdist4(const float* __restrict__ q, const float* __restrict__ c, uint32_t n, uint32_t ilp,
                               float thr) {
    if (MODEL == kIlp) return exact_sqdist<MODEL>(q, c, n, ilp, thr);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* c4 = reinterpret_cast<const float4*>(c);
    float s = 0.f;
    uint32_t p = 0;
    for (uint32_t l0 = 0; l0 < n; l0 += 32u) {
        float4 qa[8], ca[8];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            if (l0 + 4u * b < n) {
                qa[b] = q4[(l0 >> 2) + b];
                ca[b] = c4[(l0 >> 2) + b];
            } else {
                qa[b] = ca[b] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const float qv[4] = {qa[b].x, qa[b].y, qa[b].z, qa[b].w};
            const float cv[4] = {ca[b].x, ca[b].y, ca[b].z, ca[b].w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                if (l0 + 4u * b + (uint32_t)e < n) {
                    const float d = __fsub_rn(cv[e], qv[e]);
                    s = (MODEL == kSeq || p == 0) ? __fmaf_rn(d, d, s) : __fadd_rn(s, __fmaf_rn(d, d, 0.f));
                    if (MODEL == kIlpSc && ++p == ilp) p = 0;
                }
            }
        }
        if (s > thr) break;
    }
    return s;
}

struct ScreenSmem {
    uint32_t a, b, nbs, nbp, cslot, cwmax, qid, qinfo, misc, total;
};

__host__ __device__ inline ScreenSmem screen_smem(uint32_t kpad, uint32_t noff) {
    ScreenSmem t{};
    uint32_t o = 0;
    t.a = o;
    o += (uint32_t)kSQ * kpad * 2u;
    t.b = o;  // kStages candidate tiles
    o += kStages * (uint32_t)kSC * kpad * 2u;
    t.nbs = o;
    o += noff * 4u;
    t.nbp = o;
    o += (noff + 1u) * 4u;
    o = (o + 15u) & ~15u;
    t.cslot = o;  // [kStages][kSC]
    o += kStages * kSC * 4u;
    t.cwmax = o;  // [kStages][8] per 32-candidate group: largest norm [0..3], its square root [4..7]
    o += kStages * 8u * 4u;
    t.qid = o;
    o += kSQ * 4u;
    o = (o + 15u) & ~15u;
    t.qinfo = o;  // float4 per query: |q^|^2, R0 + kE |q^|, c1 |q^|^2, valid
    o += kSQ * 16u;
    t.misc = o;   // [0] item [1] failed [2] total [4] tmem [8..19] warp counts
                  // [24..31] mbarriers full0 full1 empty0 empty1, [32..37] free0 free1 free2
    o += 48u * 4u;
    t.total = (o + 127u) & ~127u;
    return t;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// The CTA is warp-specialised: warps 8-11 produce (candidate slots, centred
// BF16 candidate rows with the norm folded in, the MMA), warps 0-7 consume
// (tensor-memory rows, the screen, the undecided-pair appends).  Candidate
// tiles rotate through kStages buffers and two accumulators alternate;
// mbarriers staged[b] (rows in place), full[s] (MMA done), empty[s]
// (accumulator read) and free[b] (buffer read) hand them over.
//
// With the norm folded into the product (A row, the query = [-2 q^, 1, 1];
// B row, the candidate = [c^, |c^|^2_hi, |c^|^2_lo]), the accumulator holds
// |c^_j|^2 - 2 q^_i.c^_j directly and the screen is one comparison per pair.
template <int MODEL, bool STAMP>
__global__ void __launch_bounds__(kSThreads, 2) k_tile_screen(const JoinArgs<float> a, const TileOut o,
                                                              const ScreenConst sc, uint32_t noff, uint32_t nvisit) {
    extern __shared__ __align__(1024) unsigned char ssm[];
    const uint32_t n = a.n, npad = a.npad, k = a.g.k, kpad = sc.kpad;
    const ScreenSmem L = screen_smem(kpad, noff);
    unsigned char* A = ssm + L.a;
    uint32_t* nb_start = reinterpret_cast<uint32_t*>(ssm + L.nbs);
    uint32_t* nb_pref = reinterpret_cast<uint32_t*>(ssm + L.nbp);
    uint32_t* c_slot = reinterpret_cast<uint32_t*>(ssm + L.cslot);
    float* cwmax = reinterpret_cast<float*>(ssm + L.cwmax);
    uint32_t* q_id = reinterpret_cast<uint32_t*>(ssm + L.qid);
    float4* qinfo = reinterpret_cast<float4*>(ssm + L.qinfo);
    uint32_t* misc = reinterpret_cast<uint32_t*>(ssm + L.misc);
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = lanemask_lt_s();
    const uint32_t sbo = (kpad >> 3) * 128u;
    const uint32_t a_addr = smem_u32(A);
    const uint32_t full0 = smem_u32(misc + 24), full1 = smem_u32(misc + 26);
    const uint32_t empty0 = smem_u32(misc + 28), empty1 = smem_u32(misc + 30);
    const uint32_t free0 = smem_u32(misc + 32);  // free_b = free0 + 8 b
    const uint32_t staged0 = smem_u32(misc + 38);  // staged_b = staged0 + 8 b

    // ---- set-up: mbarriers, tensor memory (two accumulators)
    if (tid == 0) {
        misc[1] = 0u;
        // full[s]: the MMA's commit + the issuing thread's release of the tile's metadata
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(full0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(full1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 256;" ::"r"(empty0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 256;" ::"r"(empty1) : "memory");
        // free[b]: the consumers are done with stage b (candidate tile, slots, norm bound)
        for (uint32_t b = 0; b < kStages; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 256;" ::"r"(free0 + 8u * b) : "memory");
        // staged[b]: the 128 producer threads' slots and rows of stage b are in place
        for (uint32_t b = 0; b < kStages; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(staged0 + 8u * b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(misc + 4)),
                     "r"(2u * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = misc[4];
    uint32_t tiles_done = 0;  // tiles of earlier items (the mbarrier phases)
    unsigned long long cand_total = 0;
    // consumer warps: the reserved block of undecided-pair entries and the count
    unsigned long long blk_base = 0, und_count = 0;
    uint32_t blk_used = kBlk;

    for (;;) {
        __syncthreads();
        if (tid == 0) misc[0] = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t vi = misc[0];
        if (vi >= nvisit || misc[1]) break;
        const uint2 wi = a.items[(size_t)vi * o.stride];
        const uint32_t cell = wi.x;
        const uint32_t cs0 = a.cell_start[cell], ce = a.cell_start[cell + 1];
        const uint32_t q0 = cs0 + wi.y * (uint32_t)kSQ;
        const uint32_t qn = min((uint32_t)kSQ, ce - q0);

        // ---- neighbour cells in offset order (as the tile join)
        uint32_t own[kMaxK];
#pragma unroll
        for (int j = 0; j < kMaxK; j++)
            own[j] = (j < (int)k) ? FP<float>::to_uint_rz(FP<float>::div(
                                        FP<float>::sub(a.pts[(size_t)cs0 * npad + j], a.minv[j]), a.eps))
                                  : 0u;
        uint32_t nnb = 0;
        uint32_t lowmask, highmask, oddmask;
        cell_masks(own, a.g, lowmask, highmask, oddmask);
        const uint64_t own_lin = a.cell_key[cell];
        for (uint32_t base = 0; base < noff; base += kSThreads) {
            const uint32_t off = base + tid;
            uint64_t lin = 0;
            const bool ok = off < noff && nb_offset<float, STAMP>(a, off, own_lin, lowmask, highmask, oddmask, lin);
            uint32_t st = 0, cnt = 0;
            const bool found = ok && lookup_range(a, lin, st, cnt);
            const unsigned m = __ballot_sync(FULL, found);
            if (lane == 0) misc[8 + warp] = __popc(m);
            __syncthreads();
            uint32_t before = 0, all = 0;
#pragma unroll
            for (int w = 0; w < kSThreads / 32; w++) {
                const uint32_t cw = misc[8 + w];
                before += (w < warp) ? cw : 0u;
                all += cw;
            }
            if (found) {
                const uint32_t pos = nnb + before + __popc(m & lt);
                nb_start[pos] = st;
                nb_pref[pos] = cnt;
            }
            nnb += all;
            __syncthreads();
        }
        if (warp == 0) {
            uint32_t run = 0;
            for (uint32_t b0 = 0; b0 < nnb; b0 += 32) {
                const uint32_t i = b0 + lane;
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
        // ---- query tile [-2 q^, 1, 1] from the precomputed rows [q^, |q^|^2_hi, |q^|^2_lo]
        const uint32_t kch = kpad >> 3;  // 16-byte chunks per row
        if (tid < kSQ) {
            const bool valid = (uint32_t)tid < qn;
            q_id[tid] = valid ? a.ids[q0 + tid] : 0u;
            const float nrm = valid ? sc.norms[q0 + tid] : 0.f;
            qinfo[tid] = make_float4(nrm, __fmaf_ru(sc.ke, __fsqrt_ru(nrm), sc.r0), __fmul_ru(sc.c1, nrm),
                                     valid ? 1.f : 0.f);
        }
        for (uint32_t e = tid; e < (uint32_t)kSQ * kch; e += kSThreads) {
            const uint32_t r = e / kch, kc = e - r * kch;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r < qn) v = sc.rows[(size_t)(q0 + r) * kch + kc];
            uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int h = 0; h < 4; h++) {
                __nv_bfloat162 b = *reinterpret_cast<__nv_bfloat162*>(&w[h]);
                float2 f = __bfloat1622float2(b);
                const uint32_t col = kc * 8u + 2u * (uint32_t)h;
                f.x = col < n ? -2.f * f.x : (col < n + 2u && r < qn ? 1.f : 0.f);
                f.y = col + 1u < n ? -2.f * f.y : (col + 1u < n + 2u && r < qn ? 1.f : 0.f);
                b = __floats2bfloat162_rn(f.x, f.y);
                w[h] = *reinterpret_cast<uint32_t*>(&b);
            }
            *reinterpret_cast<uint4*>(A + core_off(r, kc, kpad)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        fence_async_smem();
        __syncthreads();
        const uint32_t total = misc[2];
        const uint32_t T = (total + kSC - 1u) / kSC;
        cand_total += (unsigned long long)total * qn;

        if (tid >= kProd0) {
            // ================= producer warps: stage tile t + 1 (slots, cp.async of
            // the rows) before publishing tile t (copies landed); one thread then
            // issues tile t's MMA
            const uint32_t pt = (uint32_t)tid - (uint32_t)kProd0;  // candidate row of the tile
            uint32_t e = 0;  // neighbour range of this thread's current candidate (f grows by kSC per tile)
            float wm_cur = 0.f, wm_next = 0.f;  // candidate norms of the last two prepared tiles
            const uint32_t wbase = (uint32_t)(warp - 8) * 32u;  // this warp's first row of the tile
            // stage tile t: this warp's 32 slots and rows (no barrier with the other
            // producer warps: the stage is free once its consumers released it)
            auto prepare = [&](uint32_t t) -> bool {
                const uint32_t g = tiles_done + t, b = g % kStages;
                if (g >= kStages) {
                    bool ok = true;
                    if (lane == 0) ok = bar_wait_bounded(free0 + 8u * b, ((g / kStages) - 1u) & 1u);
                    if (!__shfl_sync(FULL, ok ? 1u : 0u, 0)) return false;
                }
                const uint32_t f = t * kSC + pt;
                uint32_t slot = kNone;
                wm_cur = wm_next;
                wm_next = 0.f;
                if (f < total) {
                    while (nb_pref[e + 1] <= f) e++;
                    slot = nb_start[e] + (f - nb_pref[e]);
                    // |c^|^2 in FP32 bounds the folded hi + lo terms (reduced when the
                    // tile is published, so that the load's latency is not waited for here)
                    wm_next = sc.norms[slot];
                }
                c_slot[b * kSC + pt] = slot;
                const uint32_t dst = smem_u32(ssm + L.b) + b * ((uint32_t)kSC * kpad * 2u);
                if (kch <= 4u) {
                    // short rows (up to 32 values): each thread copies its own row
                    const bool valid = slot != kNone;
                    const uint4* src = sc.rows + (size_t)(valid ? slot : 0u) * kch;
                    for (uint32_t kc = 0; kc < kch; kc++)
                        cp_async16(dst + core_off(pt, kc, kpad), src + kc, valid ? 16u : 0u);
                } else {
                    // longer rows: the warp's 32 rows, consecutive lanes on consecutive
                    // chunks of a row
                    for (uint32_t j = 0; j < kch; j++) {
                        const uint32_t idx = j * 32u + (uint32_t)lane;
                        const uint32_t r = idx / kch, kc = idx - r * kch;
                        const uint32_t sl = __shfl_sync(FULL, slot, (int)r);
                        const bool valid = sl != kNone;
                        cp_async16(dst + core_off(wbase + r, kc, kpad),
                                   sc.rows + (size_t)(valid ? sl : 0u) * kch + kc, valid ? 16u : 0u);
                    }
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
                return true;
            };
            // tile t's rows landed (this thread's copies): publish slots, norm bound and rows
            auto publish = [&](uint32_t t, bool next_pending) {
                const uint32_t g = tiles_done + t, b = g % kStages;
                float wm = next_pending ? wm_cur : wm_next;
#pragma unroll
                for (int sh = 16; sh > 0; sh >>= 1) wm = fmaxf(wm, __shfl_xor_sync(FULL, wm, sh));
                if (lane == 0) {
                    cwmax[b * 8u + (uint32_t)(warp - 8)] = wm;
                    cwmax[b * 8u + 4u + (uint32_t)(warp - 8)] = __fsqrt_ru(wm);
                }
                if (next_pending) asm volatile("cp.async.wait_group 1;" ::: "memory");
                else asm volatile("cp.async.wait_group 0;" ::: "memory");
                fence_async_smem();
                bar_arrive(staged0 + 8u * b);
            };
            // one thread: tile t staged by all producers and its accumulator free -> MMA
            auto issue = [&](uint32_t t) -> bool {
                const uint32_t g = tiles_done + t, b = g % kStages, s = g & 1u;
                if (!bar_wait_bounded(staged0 + 8u * b, (g / kStages) & 1u)) return false;
                if (g >= 2 && !bar_wait_bounded((s ? empty1 : empty0), ((g >> 1) - 1u) & 1u)) return false;
                fence_after();
                const uint32_t b_addr = smem_u32(ssm + L.b) + b * ((uint32_t)kSC * kpad * 2u);
                for (uint32_t ks = 0; ks < (kpad >> 4); ks++)
                    mma_bf16(tmem + s * kTmemCols, smem_desc(a_addr + ks * 256u, 128u, sbo),
                             smem_desc(b_addr + ks * 256u, 128u, sbo), ks > 0 ? 1u : 0u);
                mma_commit((s ? full1 : full0));
                bar_arrive((s ? full1 : full0));
                return true;
            };
            bool ok = T == 0 || prepare(0);
            for (uint32_t t = 0; ok && t < T; t++) {
                if (t + 1 < T) ok = prepare(t + 1);
                if (!ok) break;
                publish(t, t + 1 < T);
                if (warp == 8) {
                    bool r = true;
                    if (lane == 0) r = issue(t);
                    ok = __shfl_sync(FULL, r ? 1u : 0u, 0) != 0u;
                }
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            if (!ok) misc[1] = 1u;
        } else {
            // ================= consumer warps: query row i = TMEM lane i; warps w and
            // w + 4 share lane quarter w % 4 and split the columns
            const uint32_t quarter = (uint32_t)warp & 3u, colbase = ((uint32_t)warp >> 2) * ((uint32_t)kSC / 2u);
            const uint32_t i = quarter * 32u + (uint32_t)lane;
            const float4 qi = qinfo[i];
            const bool qvalid = qi.w != 0.f;
            for (uint32_t t = 0; t < T; t++) {
                const uint32_t g = tiles_done + t, s = g & 1u;
                bool ok = true;
                if (lane == 0) ok = bar_wait_bounded((s ? full1 : full0), (g >> 1) & 1u);
                ok = __shfl_sync(FULL, ok ? 1u : 0u, 0) != 0u;
                if (!ok) {
                    misc[1] = 1u;
                    break;
                }
                fence_after();
                const uint32_t b = g % kStages;
                const uint32_t nvalid = min((uint32_t)kSC, total - t * kSC);
                // a warp whose 32 query rows are all empty still waits for every tile
                // (its arrivals keep the phases of empty[] in order) but skips the work
                const uint32_t col_end = (quarter * 32u < qn) ? colbase + (uint32_t)kSC / 2u : colbase;
                for (uint32_t c32 = colbase; c32 < col_end; c32 += 32u) {
                  // G_i from the group's largest candidate norm (an upper bound of each of
                  // its 32 columns' bounds; the group's candidates are one producer warp's)
                  const float cmax = cwmax[b * 8u + (c32 >> 5)], rcmax = cwmax[b * 8u + 4u + (c32 >> 5)];
                  const float tt = __fmaf_ru(sc.ke, rcmax, qi.y);
                  const float G =
                      __fsub_ru(__fmaf_ru(tt, tt, __fadd_ru(qi.z, __fmul_ru(sc.c1, __fmul_ru(2.f, cmax)))), qi.x);
                  float d32[32];
                  tmem_ld32(tmem + s * kTmemCols + ((quarter * 32u) << 16) + c32, d32);
                  // common case: every value of the 32 columns above G (NaN counts as undecided)
                  bool all_out = true;
#pragma unroll
                  for (int jj = 0; jj < 32; jj++) all_out = all_out && (d32[jj] > G);
                  if (__all_sync(FULL, !qvalid || all_out || c32 >= nvalid)) continue;
                  for (uint32_t h16 = 0; h16 < 2u; h16++) {
                    const uint32_t col0 = c32 + 16u * h16;
                    unsigned und = 0;
                    if (qvalid) {
#pragma unroll
                        for (int jj = 0; jj < 16; jj++) und |= (d32[16 * h16 + jj] > G) ? 0u : (1u << jj);
                        if (col0 + 16u > nvalid) und &= (col0 >= nvalid) ? 0u : ((1u << (nvalid - col0)) - 1u);
                    }
                    if (!__any_sync(FULL, und != 0u)) continue;
                    // the undecided pairs (query slot | cross << 31, candidate slot) go to
                    // the exact check (k_screen_recheck), one atomic per warp and chunk
                    const uint32_t nu = (uint32_t)__popc(und);
                    uint32_t x = nu;
#pragma unroll
                    for (int sh = 1; sh < 32; sh <<= 1) {
                        const uint32_t y = __shfl_up_sync(FULL, x, sh);
                        if (lane >= sh) x += y;
                    }
                    const uint32_t wtotal = __shfl_sync(FULL, x, 31);
                    und_count += wtotal;
                    if (o.emit) {
                        if (blk_used + wtotal > kBlk) {
                            // pad the rest of the warp's block, reserve the next one
                            for (uint32_t e2 = blk_used + (uint32_t)lane; e2 < kBlk; e2 += 32u)
                                if (blk_base + e2 < o.cap) o.pairs[blk_base + e2] = kUndecidedPad;
                            unsigned long long nb = 0;
                            if (lane == 0) nb = atomicAdd(o.cursor, (unsigned long long)kBlk);
                            blk_base = __shfl_sync(FULL, nb, 0);
                            blk_used = 0;
                        }
                        unsigned long long p = blk_base + blk_used + (x - nu);
                        blk_used += wtotal;
                        const unsigned long long qword = (unsigned long long)(q0 + i);
                        unsigned uu = und;
                        while (uu) {
                            const int bb = __ffs(uu) - 1;
                            uu &= uu - 1u;
                            const uint32_t sl = c_slot[b * kSC + col0 + (uint32_t)bb];
                            const unsigned long long cr = (STAMP && (sl < cs0 || sl >= ce)) ? (1ull << 31) : 0ull;
                            if (p < o.cap) o.pairs[p] = ((qword | cr) << 32) | sl;
                            p++;
                        }
                    }
                  }
                }
                fence_before();
                bar_arrive((s ? empty1 : empty0));
                bar_arrive(free0 + 8u * b);
            }
        }
        tiles_done += T;
    }
    // ---- the consumer warps' last blocks and their exact undecided counts
    if (tid < kProd0) {
        if (o.emit && blk_used < kBlk)
            for (uint32_t e2 = blk_used + (uint32_t)lane; e2 < kBlk; e2 += 32u)
                if (blk_base + e2 < o.cap) o.pairs[blk_base + e2] = kUndecidedPad;
        if (lane == 0 && und_count) atomicAdd(o.rechecks, und_count);
    }
    // ---- tear-down: every MMA this CTA issued has been waited for (the last
    // tiles by the epilogue), unless a wait timed out
    if (misc[1] && tid == 0) *a.err_flag = 2u;
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2u * kTmemCols)
                     : "memory");
    if (tid == 0 && o.emit && cand_total) atomicAdd(a.cand_cnt, cand_total);
}

template <int MODEL, bool STAMP>
cudaError_t launch_screen_one(const JoinArgs<float>& a, const TileOut& o, const ScreenConst& sc, uint32_t noff,
                              uint32_t nvisit, int num_sms, cudaStream_t st) {
    auto kern = k_tile_screen<MODEL, STAMP>;
    const ScreenSmem L = screen_smem(sc.kpad, noff);
    const uint32_t smem = L.total > kMinSmem ? L.total : kMinSmem;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the whole unified L1/shared array as shared memory, so that the CTAs the
    // occupancy calculation counts on are resident together
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = blocks_per_sm((const void*)kern, kSThreads, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    // tensor memory: 2 accumulators of 128 columns per CTA, 512 columns per SM
    if ((uint32_t)per_sm * 2u * kTmemCols > 512u) per_sm = (int)(512u / (2u * kTmemCols));
    if (a.shape_per_sm && (int)a.shape_per_sm < per_sm) per_sm = (int)a.shape_per_sm;
    uint64_t blocks = (uint64_t)num_sms * per_sm;
    if (blocks > nvisit) blocks = nvisit ? nvisit : 1;
    kern<<<(unsigned)blocks, kSThreads, smem, st>>>(a, o, sc, noff, nvisit);
    return cudaGetLastError();
}

}  // namespace

// The exact check of the pairs the screen could not reject: the reference's
// arithmetic for the configured model (kernel.cu:307-365), s <= thr; a hit
// appends (query id, candidate id), and with the cross flag (unicomp, the
// candidate outside the query's cell) also the reverse pair.
template <int MODEL, bool STAMP>
__global__ void __launch_bounds__(256) k_screen_recheck(const float* __restrict__ pts, const uint32_t* __restrict__ ids,
                                                        uint32_t n, uint32_t npad, uint32_t ilp, float thr,
                                                        uint32_t npoints, const unsigned long long* __restrict__ unc,
                                                        unsigned long long nunc, const TileOut o) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lt = lanemask_lt_s();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < nunc; i0 += stride) {
        const uint64_t e = i0 + threadIdx.x;
        bool hit = false, cross = false;
        uint32_t qs = 0, cs = 0;
        const unsigned long long w = e < nunc ? unc[e] : kUndecidedPad;
        const uint32_t qw = (uint32_t)(w >> 32);
        if (w != kUndecidedPad && (qw & 0x7fffffffu) < npoints && (uint32_t)w < npoints) {
            cs = (uint32_t)w;
            qs = qw & 0x7fffffffu;
            const float d = exact_sqdist4<MODEL>(pts + (size_t)qs * npad, pts + (size_t)cs * npad, n, ilp, thr);
            hit = d <= thr;
            cross = STAMP && hit && (qw >> 31) != 0u;
        }
        const unsigned hb = __ballot_sync(FULL, hit), cb = __ballot_sync(FULL, cross);
        if (hb == 0u) continue;
        const uint32_t wtotal = (uint32_t)__popc(hb) + (uint32_t)__popc(cb);
        unsigned long long base = 0;
        if ((threadIdx.x & 31u) == 0u) base = atomicAdd(o.cursor, (unsigned long long)wtotal);
        base = __shfl_sync(FULL, base, 0);
        if (hit) {
            unsigned long long p = base + (unsigned)__popc(hb & lt) + (unsigned)__popc(cb & lt);
            const uint64_t qid = ids[qs], cid = ids[cs];
            if (p < o.cap) o.pairs[p] = (qid << o.shift) | cid;
            p++;
            if (cross && p < o.cap) o.pairs[p] = (cid << o.shift) | qid;
        }
    }
}

template <int MODEL, bool STAMP>
cudaError_t launch_recheck_one(const JoinArgs<float>& a, const unsigned long long* unc, unsigned long long nunc,
                               const TileOut& o, int num_sms, cudaStream_t st) {
    uint64_t blocks = (nunc + 255) / 256;
    const uint64_t cap = (uint64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_screen_recheck<MODEL, STAMP><<<(unsigned)blocks, 256, 0, st>>>(a.pts, a.ids, a.n, a.npad, a.ilp, a.thr,
                                                                     a.n_points, unc, nunc, o);
    return cudaGetLastError();
}

// Per-block FP64 column sums and counts of the finite values over a fixed row
// range (deterministic).  Non-finite coordinates are left out of the centre,
// so that only their own rows (and pairs) become inconclusive for the screen.
__global__ void k_col_partial(const float* __restrict__ pts, uint32_t N, uint32_t n, uint32_t npad,
                              double* __restrict__ partial) {
    const uint32_t per = (N + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = blockIdx.x * per, r1 = min(N, r0 + per);
    for (uint32_t d = threadIdx.x; d < n; d += blockDim.x) {
        double acc = 0.0, cnt = 0.0;
        for (uint32_t r = r0; r < r1; r++) {
            const float v = pts[(size_t)r * npad + d];
            if (isfinite(v)) {
                acc += (double)v;
                cnt += 1.0;
            }
        }
        partial[((size_t)blockIdx.x * n + d) * 2] = acc;
        partial[((size_t)blockIdx.x * n + d) * 2 + 1] = cnt;
    }
}

__global__ void k_col_mean(const double* __restrict__ partial, uint32_t nblocks, uint32_t n,
                           float* __restrict__ centre) {
    for (uint32_t d = threadIdx.x; d < n; d += blockDim.x) {
        double acc = 0.0, cnt = 0.0;
        for (uint32_t b = 0; b < nblocks; b++) {
            acc += partial[((size_t)b * n + d) * 2];
            cnt += partial[((size_t)b * n + d) * 2 + 1];
        }
        const double m = cnt > 0.0 ? acc / cnt : 0.0;
        centre[d] = isfinite(m) ? (float)m : 0.f;
    }
}

// Row s: x' = fl(x - centre), c^ = bf16(x'), |c^|^2 in FP32 (sequential
// fused sum of the exact squares), split into two BF16 terms.
__global__ void k_screen_rows(const float* __restrict__ pts, uint32_t N, uint32_t n, uint32_t npad, uint32_t kpad,
                              const float* __restrict__ centre, uint4* __restrict__ rows, float* __restrict__ norms) {
    const uint32_t kch = kpad >> 3;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
        const float* x = pts + (size_t)s * npad;
        float nrm = 0.f;
        for (uint32_t kc = 0; kc < kch; kc++) {
            uint32_t w[4];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const uint32_t l = kc * 8u + 2u * (uint32_t)h;
                const float x0 = l < n ? __fsub_rn(x[l], centre[l]) : 0.f;
                const float x1 = l + 1u < n ? __fsub_rn(x[l + 1u], centre[l + 1u]) : 0.f;
                const __nv_bfloat162 b = __floats2bfloat162_rn(x0, x1);
                const float2 f = __bfloat1622float2(b);
                nrm = __fmaf_rn(f.x, f.x, nrm);
                nrm = __fmaf_rn(f.y, f.y, nrm);
                w[h] = *reinterpret_cast<const uint32_t*>(&b);
            }
            rows[(size_t)s * kch + kc] = make_uint4(w[0], w[1], w[2], w[3]);
        }
        // the norm terms go to columns n and n + 1
        const __nv_bfloat16 hi = __float2bfloat16_rn(nrm);
        const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(nrm, __bfloat162float(hi)));
        __nv_bfloat16* rb = reinterpret_cast<__nv_bfloat16*>(rows + (size_t)s * kch);
        rb[n] = hi;
        rb[n + 1u] = lo;
        norms[s] = nrm;
    }
}

cudaError_t launch_screen_prep(const float* pts, uint32_t N, uint32_t n, uint32_t npad, uint32_t kpad,
                               double* partial, float* centre, uint4* rows, float* norms, cudaStream_t st) {
    if (N == 0) return cudaSuccess;
    if (kpad < n + 2u || (kpad & 7u)) return cudaErrorInvalidValue;
    k_col_partial<<<kScreenPrepBlocks, 128, 0, st>>>(pts, N, n, npad, partial);
    k_col_mean<<<1, 128, 0, st>>>(partial, kScreenPrepBlocks, n, centre);
    uint64_t blocks = ((uint64_t)N + 255) / 256;
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    k_screen_rows<<<(unsigned)blocks, 256, 0, st>>>(pts, N, n, npad, kpad, centre, rows, norms);
    return cudaGetLastError();
}

bool screen_supported(uint32_t n, uint32_t npad, uint32_t k, int model, uint32_t ilp, float thr) {
    // n + 2 columns: the dimensions and the folded candidate norm
    return tile_supported(n, npad, k, model, ilp) && n >= 16 && n + 2u <= kTileMaxN && thr >= 1e-30f &&
           thr <= 1e30f;
}

ScreenConst make_screen_const(uint32_t n, float thr) {
    ScreenConst sc{};
    sc.kpad = (n + 2u + 15u) & ~15u;
    // R0 >= sqrt(thr / (1 - (2n + 8) 2^-24)), plus room for the FP32 evaluation of G
    const double r0 = std::sqrt((double)thr) * (1.0 + (2.0 * n + 8.0) * 0x1p-24 + 0x1p-19);
    sc.r0 = std::nextafter((float)r0, INFINITY);
    // BF16 rounding of a centred coordinate: |x - bf16(x)| <= 2^-8 |x|, plus
    // the centring subtraction and the square root of the norm
    sc.ke = 0x1p-8f * 1.0045f;
    // FP32 accumulation (K + 32 steps of 2^-20) and the two-term split of the
    // folded candidate norm (2^-16)
    sc.c1 = (float)(sc.kpad + 48u) * 0x1p-20f;
    return sc;
}

cudaError_t launch_screen_recheck(const JoinArgs<float>& a, const unsigned long long* unc, unsigned long long nunc,
                                  const TileOut& o, bool stamp, int model, int num_sms, cudaStream_t st) {
    if (nunc == 0) return cudaSuccess;
    if ((a.npad & 3u) || !unc) return cudaErrorInvalidValue;
    switch (model * 2 + (stamp ? 1 : 0)) {
        case kSeq * 2: return launch_recheck_one<kSeq, false>(a, unc, nunc, o, num_sms, st);
        case kSeq * 2 + 1: return launch_recheck_one<kSeq, true>(a, unc, nunc, o, num_sms, st);
        case kIlp * 2: return launch_recheck_one<kIlp, false>(a, unc, nunc, o, num_sms, st);
        case kIlp * 2 + 1: return launch_recheck_one<kIlp, true>(a, unc, nunc, o, num_sms, st);
        case kIlpSc * 2: return launch_recheck_one<kIlpSc, false>(a, unc, nunc, o, num_sms, st);
        case kIlpSc * 2 + 1: return launch_recheck_one<kIlpSc, true>(a, unc, nunc, o, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_tile_screen(const JoinArgs<float>& a, const TileOut& o, const ScreenConst& sc, bool stamp,
                               int model, uint32_t nvisit, int num_sms, cudaStream_t st) {
    if (!screen_supported(a.n, a.npad, a.g.k, model, a.ilp, a.thr) || o.stride == 0 || sc.kpad < a.n + 2u ||
        !sc.rows || !sc.norms ||
        (sc.kpad & 15u) || sc.kpad > kTileMaxN)
        return cudaErrorInvalidValue;
    if (nvisit == 0) return cudaSuccess;
    if ((uint64_t)(nvisit - 1) * o.stride >= a.num_items) return cudaErrorInvalidValue;
    uint32_t noff = 1;
    for (uint32_t j = 0; j < a.g.k; j++) noff *= 3u;
    switch (model * 2 + (stamp ? 1 : 0)) {
        case kSeq * 2: return launch_screen_one<kSeq, false>(a, o, sc, noff, nvisit, num_sms, st);
        case kSeq * 2 + 1: return launch_screen_one<kSeq, true>(a, o, sc, noff, nvisit, num_sms, st);
        case kIlp * 2: return launch_screen_one<kIlp, false>(a, o, sc, noff, nvisit, num_sms, st);
        case kIlp * 2 + 1: return launch_screen_one<kIlp, true>(a, o, sc, noff, nvisit, num_sms, st);
        case kIlpSc * 2: return launch_screen_one<kIlpSc, false>(a, o, sc, noff, nvisit, num_sms, st);
        case kIlpSc * 2 + 1: return launch_screen_one<kIlpSc, true>(a, o, sc, noff, nvisit, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gsj
