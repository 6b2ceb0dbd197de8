// Host orchestration and C ABI of the B200 self-join (include/gpuselfjoin.h).
//
// One gsj_join() call replaces the mode-3 body of main.cu:178-262 together
// with distanceTableNDGridBatches (GPU.cu:270-1088) and the table export of
// main.cu:514-542:
//   H2D of the dataset (when it lives on the host)
//   REORDER statistic on the device, dimension order on the host (std::sort
//     with the reference comparator, main.cu:1040)
//   grid extents: device min/max, scalar tail on the host (main.cu:925-946)
//   index: cell keys -> radix sort -> runs -> cell table -> work items
//   join, one of four paths (gsj_stats.join_path):
//     ROWS   (dense, k <= 3, n <= 4): count pass -> list offsets -> fill pass
//     WARP, TILE, SCREEN: one pass appending packed (query, candidate) keys,
//       sized by a sampling pass -> radix sort -> table + offsets
// The result stays on the device in the context's pool until fetched.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <thread>
#include <type_traits>
#include <vector>


#include "../../include/gpuselfjoin.h"
#include "gsj_common.cuh"
#include "gsj_kernels.h"
#include "gsj_model.h"
#include "gsj_place.h"
#include "gsj_scan.h"
#include "gsj_sort.h"

// Build-time defaults, same macro names as the reference's params.h.
#ifndef GPUNUMDIM
#define GPUNUMDIM 0 /* 0: any dimensionality accepted at run time */
#endif
#ifndef NUMINDEXEDDIM
#define NUMINDEXEDDIM 6
#endif
#ifndef REORDER
#define REORDER 0
#endif
#ifndef SHORTCIRCUIT
#define SHORTCIRCUIT 0
#endif
#ifndef ILP
#define ILP 0
#endif
#ifndef STAMP
#define STAMP 0
#endif
// LINEARSTAMP (kernel.cu:272-289) visits the own cell and the neighbour cells
// of larger linear id: another half of the cross-cell pairs than STAMP's
// parity rule, the same pair set.  It selects the unicomp traversal here.
#ifndef LINEARSTAMP
#define LINEARSTAMP 0
#endif
#ifndef QUERYREORDER
#define QUERYREORDER 0
#endif
#ifndef SORT
#define SORT 0
#endif

using namespace gsj;

namespace {

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
};

struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
};

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Model of the distance arithmetic from the ILP / SHORTCIRCUIT switches.
int model_of(const gsj_config& c) {
    if (c.ilp == 0) return kSeq;
    return c.shortcircuit ? kIlpSc : kIlp;
}

template <typename T>
T threshold_of(T eps);

template <>
float threshold_of<float>(float eps) {
    if (std::isnan(eps) || eps < 0.0f) return -INFINITY;
    if (std::isinf(eps)) return INFINITY;
    float s = (float)((double)eps * (double)eps);
    while (s > 0.0f && std::sqrt(s) > eps) s = std::nextafter(s, 0.0f);
    for (;;) {
        const float nx = std::nextafter(s, INFINITY);
        if (std::sqrt(nx) <= eps) s = nx;
        else break;
    }
    return s;
}

template <>
double threshold_of<double>(double eps) {
    if (std::isnan(eps) || eps < 0.0) return -INFINITY;
    if (std::isinf(eps)) return INFINITY;
    double s = eps * eps;
    if (std::isinf(s)) s = DBL_MAX;
    while (s > 0.0 && std::sqrt(s) > eps) s = std::nextafter(s, 0.0);
    for (;;) {
        const double nx = std::nextafter(s, INFINITY);
        if (std::sqrt(nx) <= eps) s = nx;
        else break;
    }
    return s;
}

// SORT's per-cell element and order (GPU.cu:51-54): kept as the reference
// declares them so that std::sort orders ties the same way.
template <typename T>
struct key_val_sort {
    unsigned int pid;
    T value_at_dim;
};
template <typename T>
bool compareByPointValue(const key_val_sort<T>& a, const key_val_sort<T>& b) {
    return a.value_at_dim < b.value_at_dim;
}

template <typename T>
struct dim_reorder_sort {  // structs.h:37-41
    unsigned int dim;
    T variance;
};
template <typename T>
bool compareByDimVariance(const dim_reorder_sort<T>& a, const dim_reorder_sort<T>& b) {  // main.cu:33-36
    return a.variance > b.variance;
}

// Scalars of a join in the context's `misc` buffer (at least 512 bytes):
// min/max per indexed dim (2 kMaxK values of T), then 32-bit words: run count,
// work counter, error flag, candidate counter (64-bit), pair cursors (2 x
// 64-bit); the pair placement's error flag and long-list count at words
// 4 kMaxK + 20 and + 24, the longest list at + 28 (bytes 240, 256 and 272).
constexpr size_t kMiscWords = 128;

uint32_t npad_of(uint32_t n, uint32_t tsize) {
    return n <= 2 ? n : ((n + (16u / tsize) - 1u) / (16u / tsize)) * (16u / tsize);
}

}  // namespace

struct gsj_context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaEvent_t tev[8] = {};  // stage timing: index, count, fill (start/end), estimate start/end
    // device pool
    Buf in, pts, ids, keys, keys2, vals, cell_key, cell_start, dense, dcnt, plan, plan_par, slot_cell, hkeys, hvals, order,
        sizes, nchunks,
        item_off, items, fwd, swords, counts, offsets, table, temp, scan_temp, misc, var, perm, minarr,
        minmax_part, pairs, srows, snorms, spartial, scentre, unc, table2, nbtab, bitoff, hitbits, ptemp, sortv;
    PinnedBuf stage[2];
    PinnedBuf hmisc;
    // host-result pipeline: copy streams, per-segment events, pinned staging
    static constexpr int kMaxSeg = 8;
    cudaStream_t cst[kMaxSeg] = {};
    cudaEvent_t seg_filled[kMaxSeg] = {}, seg_copied[kMaxSeg] = {};
    PinnedBuf hseg[kMaxSeg];
    Buf segs, bounds, bkeys;
    bool table_on_device = true;  // false after a batched host-result join
    // learned result-count model and the last join's cell table (its features)
    Buf mw, mm1, mm2, mx, my, mxt, myt, mtmp;
    bool model_ready = false;    // weights initialised
    bool model_trained = false;  // trained on at least one join
    uint32_t model_t = 0;        // Adam steps taken
    double model_unc_ratio = 0;  // undecided / result pairs of the screen's training join (0: none)
    struct {
        bool valid = false;
        uint32_t M = 0, n = 0;
        float log2_eps = 0;
        JoinArgs<float> lookup{};
    } last;
    // tuned launch shapes by (path, dim, density_log2)
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, gsj_tuning> tuning;
    const gsj_tuning* forced = nullptr;  // the autotuner's candidate, in place of the table
    // last result
    bool have_result = false;
    uint64_t N = 0, R = 0;
    std::string err;
    gsj_stats stats{};
};

namespace {

std::mutex g_err_mu;
std::string g_err_default;

int fail(gsj_context* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err_default = msg;
    return code;
}

#define GSJ_CUDA(ctx, call)                                                                               \
    do {                                                                                                  \
        cudaError_t _e = (call);                                                                          \
        if (_e != cudaSuccess)                                                                            \
            return fail((ctx), _e == cudaErrorMemoryAllocation ? GSJ_ERR_NOMEM : GSJ_ERR_CUDA,            \
                        std::string(#call) + ": " + cudaGetErrorString(_e));                              \
    } while (0)

// Grow-only device allocation.
template <typename X>
int dev_get(gsj_context* c, Buf& b, size_t count, X** out) {
    const size_t bytes = std::max<size_t>(count * sizeof(X), 256);
    if (b.cap < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
        size_t want = bytes + bytes / 2;  // headroom: a stream of growing joins re-allocates rarely
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            e = cudaMalloc(&b.p, bytes);
            want = bytes;
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GSJ_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
        b.cap = want;
    }
    *out = static_cast<X*>(b.p);
    return GSJ_OK;
}

int pinned_get(gsj_context* c, PinnedBuf& b, size_t bytes) {
    if (b.cap < bytes) {
        if (b.p) cudaFreeHost(b.p);
        b.p = nullptr;
        b.cap = 0;
        if (cudaMallocHost(&b.p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GSJ_ERR_NOMEM, "pinned host allocation failed");
        }
        b.cap = bytes;
    }
    return GSJ_OK;
}

#define GSJ_TRY(x)                    \
    do {                              \
        int _r = (x);                 \
        if (_r != GSJ_OK) return _r;  \
    } while (0)

bool host_is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Parallel host memcpy (the copy-out of staged results into pageable memory).
void par_memcpy(void* dst, const void* src, size_t bytes) {
    const size_t kMin = 8u << 20;
    unsigned nt = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16u);
    if (bytes < kMin || nt == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        const size_t b = t * per;
        if (b >= bytes) break;
        const size_t len = std::min(per, bytes - b);
        th.emplace_back([=] { std::memcpy((char*)dst + b, (const char*)src + b, len); });
    }
    for (auto& x : th) x.join();
}

// Device -> host copy through two pinned staging buffers on alternating
// streams, so the PCIe transfer of chunk i+1 overlaps the copy-out of chunk i.
int d2h_staged(gsj_context* c, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return GSJ_OK;
    if (host_is_pinned(dst)) {
        GSJ_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st));
        GSJ_CUDA(c, cudaStreamSynchronize(c->st));
        return GSJ_OK;
    }
    const size_t chunk = 64u << 20;
    GSJ_TRY(pinned_get(c, c->stage[0], chunk));
    GSJ_TRY(pinned_get(c, c->stage[1], chunk));
    const size_t nch = (bytes + chunk - 1) / chunk;
    cudaStream_t ss[2] = {c->st, c->st2};
    for (size_t i = 0; i < nch && i < 2; i++) {
        const size_t off = i * chunk, len = std::min(chunk, bytes - off);
        GSJ_CUDA(c, cudaMemcpyAsync(c->stage[i].p, (const char*)src + off, len, cudaMemcpyDeviceToHost, ss[i]));
        GSJ_CUDA(c, cudaEventRecord(c->ev[i], ss[i]));
    }
    for (size_t i = 0; i < nch; i++) {
        const int b = (int)(i & 1);
        const size_t off = i * chunk, len = std::min(chunk, bytes - off);
        GSJ_CUDA(c, cudaEventSynchronize(c->ev[b]));
        par_memcpy((char*)dst + off, c->stage[b].p, len);
        const size_t nx = i + 2;
        if (nx < nch) {
            const size_t off2 = nx * chunk, len2 = std::min(chunk, bytes - off2);
            GSJ_CUDA(c, cudaMemcpyAsync(c->stage[b].p, (const char*)src + off2, len2, cudaMemcpyDeviceToHost, ss[b]));
            GSJ_CUDA(c, cudaEventRecord(c->ev[b], ss[b]));
        }
    }
    return GSJ_OK;
}

int h2d_copy(gsj_context* c, void* dst, const void* src, size_t bytes) {
    GSJ_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
    return GSJ_OK;
}

template <typename X>
int d2h_small(gsj_context* c, X* dst, const X* src, size_t count) {
    GSJ_CUDA(c, cudaMemcpyAsync(dst, src, count * sizeof(X), cudaMemcpyDeviceToHost, c->st));
    GSJ_CUDA(c, cudaStreamSynchronize(c->st));
    return GSJ_OK;
}

// Entries a block-reserving pass may take for `real` entries: each warp
// reserves blocks of kScreenBlockSlack entries and abandons its block (padding
// the tail) when the next chunk of at most `max_chunk` entries does not fit,
// so every abandoned block holds at least kScreenBlockSlack - (max_chunk - 1)
// real entries; each of the `warps` warps may end with one partly filled block.
uint64_t reserve_bound(uint64_t real, uint64_t warps, uint32_t max_chunk) {
    const uint64_t per = kScreenBlockSlack - (max_chunk - 1u);
    return ((real + per - 1u) / per + warps) * kScreenBlockSlack;
}

// Capacity of attempt `attempt` of a block-reserving pass: the estimate first;
// after a short buffer the previous pass's own reservation `used` with room
// for a different block-filling order; then the proven bound.  The first pass
// runs with no buffer at all under GSJ_FLAG_EXACT_SIZE.
uint64_t retry_cap(int attempt, uint64_t estimate, uint64_t used, uint64_t bound) {
    if (attempt == 0) return estimate;
    if (attempt == 1) return std::min(bound, used + used / 8u + (1u << 16));
    return bound;
}

int validate(gsj_context* c, const gsj_config& cfg, uint64_t N) {
    if (cfg.dim == 0) return fail(c, GSJ_ERR_INVALID, "dim must be >= 1");
    if (cfg.dim > 4096) return fail(c, GSJ_ERR_INVALID, "dim above 4096 is not supported");
    if (cfg.indexed_dims == 0 || cfg.indexed_dims > cfg.dim)
        return fail(c, GSJ_ERR_INVALID, "indexed_dims must satisfy 1 <= k <= dim (main.cu:70)");
    if (cfg.indexed_dims > 8) return fail(c, GSJ_ERR_INVALID, "indexed_dims above 8 is not supported");
    if (cfg.ilp > (uint32_t)kMaxIlp) return fail(c, GSJ_ERR_INVALID, "ILP above 64 is not supported");
    if (cfg.dtype != GSJ_FLOAT32 && cfg.dtype != GSJ_FLOAT64) return fail(c, GSJ_ERR_INVALID, "unknown dtype");
    if (N >= (1ull << 31)) return fail(c, GSJ_ERR_INVALID, "at most 2^31-1 points per join");
    return GSJ_OK;
}

// ------------------------------------------------------------------ lists ascending
// Sorts every list of the table ascending (ids below N): a warp per list up
// to 256 entries, a CTA bitonic network up to 4096, CTA radix passes with a
// scratch copy of the table above.
int sort_table_lists(gsj_context* c, uint32_t* table, const uint64_t* offsets, uint64_t N, uint64_t R) {
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    int nl = 0;
    void* temp = nullptr;
    GSJ_TRY(dev_get(c, c->ptemp, place_temp_bytes(N), (unsigned char**)&temp));
    uint32_t* d_nlong = reinterpret_cast<uint32_t*>(c->misc.p) + 4 * kMaxK + 24;
    uint32_t nlong = 0, nvery = 0;
    GSJ_CUDA(c, sort_short_lists<uint64_t>(table, offsets, (uint32_t)N, 1u, temp, d_nlong, &nlong, &nvery,
                                           c->num_sms, &nl, st));
    if (nlong) {
        uint32_t* scratch = nullptr;
        if (nvery) GSJ_TRY(dev_get(c, c->table2, R, &scratch));
        uint32_t id_bits = 1;
        while (id_bits < 32 && ((N - 1) >> id_bits)) id_bits++;
        GSJ_CUDA(c, sort_long_lists<uint64_t>(table, scratch, offsets, temp, nlong, nvery, id_bits, c->num_sms, &nl,
                                              st));
    }
    S.kernel_launches += (uint64_t)nl;
    return GSJ_OK;
}

// ------------------------------------------------------------------ pair keys -> table
// Builds the neighbour table from `nkeys` packed (query id << shift |
// candidate id) keys (entries equal to ~0 are unused block tails): list
// lengths, offsets, placement, then every list sorted ascending.  Fills the
// stage times and the result state.  cand: the device candidate counter.
int pairs_to_csr(gsj_context* c, unsigned long long* pairs, uint64_t nkeys, uint64_t R, uint32_t shift, uint64_t N,
                 uint32_t* counts, uint64_t* offsets, const unsigned long long* cand) {
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    GSJ_CUDA(c, cudaEventRecord(c->tev[4], st));
    uint32_t *table = nullptr, *cursor = nullptr;
    GSJ_TRY(dev_get(c, c->table, R ? R : 1, &table));
    GSJ_TRY(dev_get(c, c->fwd, N, &cursor));
    void* temp = nullptr;
    GSJ_TRY(dev_get(c, c->ptemp, place_temp_bytes(N), (unsigned char**)&temp));
    uint32_t* d_err = reinterpret_cast<uint32_t*>(c->misc.p) + 4 * kMaxK + 20;
    GSJ_CUDA(c, cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st));
    int nl = 0;
    GSJ_CUDA(c, place_pairs(pairs, nkeys, shift, (uint32_t)N, counts, offsets, table, R, cursor, d_err, temp,
                            c->num_sms, &nl, st));
    S.kernel_launches += (uint64_t)nl;
    GSJ_TRY(sort_table_lists(c, table, offsets, N, R));
    GSJ_CUDA(c, cudaEventRecord(c->tev[5], st));
    uint64_t total = 0;
    GSJ_TRY(d2h_small(c, &total, offsets + N, 1));
    if (total != R) return fail(c, GSJ_ERR_STATE, "list lengths disagree with the pair count");
    uint32_t err = 0;
    GSJ_TRY(d2h_small(c, &err, d_err, 1));
    if (err) return fail(c, GSJ_ERR_STATE, "pair placement left a list (internal error)");
    unsigned long long ncand = 0;
    GSJ_TRY(d2h_small(c, &ncand, cand, 1));
    {
        float ms = 0;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[0], c->tev[1]));
        S.dev_ms_index = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[2], c->tev[3]));
        S.dev_ms_count = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[4], c->tev[5]));
        S.dev_ms_fill = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[6], c->tev[7]));
        S.dev_ms_estimate = ms;
    }
    S.candidates = ncand;
    S.total_pairs = R;
    c->R = R;
    c->have_result = true;
    return GSJ_OK;
}

// ------------------------------------------------------------------ learned estimate
// Pairs the exact pass of the last indexed join will produce, predicted by the
// context's model from the per-cell features (requires model_trained).
int learned_estimate(gsj_context* c, double* est) {
    cudaStream_t st = c->st;
    const uint32_t M = c->last.M;
    float* X = nullptr;
    GSJ_TRY(dev_get(c, c->mx, (size_t)M * kModelFeatures, &X));
    double* d_est = nullptr;
    GSJ_TRY(dev_get(c, c->mtmp, 4, &d_est));
    GSJ_CUDA(c, cudaMemsetAsync(d_est, 0, sizeof(double), st));
    c->stats.kernel_launches += 2;
    GSJ_CUDA(c, model_features(c->last.lookup, M, c->last.log2_eps, c->last.n, X, st));
    GSJ_CUDA(c, model_predict(X, M, static_cast<const float*>(c->mw.p), nullptr, c->last.lookup.cell_start,
                              (float)c->last.lookup.n_points, d_est, st));
    GSJ_TRY(d2h_small(c, est, d_est, 1));
    return GSJ_OK;
}

// ------------------------------------------------------------------ warp join (emit)
// The warp-per-item traversal in one pass: k_join appends every
// pair as a packed key (sampling pass over every kSampleStride-th item to size
// the buffer; a short buffer is re-sized exactly and the pass repeated), then
// the keys are sorted into the table.
template <typename T>
int emit_join(gsj_context* c, JoinArgs<T>& a, uint64_t N, bool stamp, int model, bool rows, bool exact_size,
              bool learned, uint32_t* counts, uint64_t* offsets, unsigned long long* cursor, double t_join,
              double t_start) {
    constexpr uint32_t kSampleStride = 64;
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    uint32_t shift = 1;
    while (shift < 32 && ((N - 1) >> shift)) shift++;
    const uint32_t ni = a.num_items;
    TileOut o{};
    o.cursor = cursor;       // entries reserved (blocks)
    o.rechecks = cursor + 1; // keys emitted (exact)
    o.shift = shift;
    unsigned long long* cand = reinterpret_cast<unsigned long long*>(a.work_counter + 2);
    // a warp appends at most 64 keys at once (32 hits and their reverse keys);
    // at most 64 warps per SM are resident
    const uint64_t warps = (uint64_t)c->num_sms * 64u;
    const uint64_t slack = warps * kScreenBlockSlack;
    auto reset = [&]() -> int {
        GSJ_CUDA(c, cudaMemsetAsync(a.work_counter, 0, 4 * sizeof(uint32_t), st));
        GSJ_CUDA(c, cudaMemsetAsync(cursor, 0, 2 * sizeof(unsigned long long), st));
        return GSJ_OK;
    };
    GSJ_CUDA(c, cudaEventRecord(c->tev[2], st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[6], st));
    double est = 0.0;
    if (learned) {
        GSJ_TRY(learned_estimate(c, &est));
    } else if (!exact_size) {
        // sampled estimator: the exact pass over every kSampleStride-th item
        const uint32_t nsample = (ni + kSampleStride - 1) / kSampleStride;
        GSJ_TRY(reset());
        o.emit = false;
        o.stride = kSampleStride;
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_join_emit<T>(a, o, nsample, model, stamp, rows, c->num_sms, st));
        unsigned long long sampled = 0;
        GSJ_TRY(d2h_small(c, &sampled, o.rechecks, 1));
        est = nsample ? (double)sampled * (double)ni / (double)nsample : 0.0;
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[7], st));
    S.estimate = (uint64_t)est;
    const uint64_t estimate = exact_size ? 0u : (uint64_t)(est * 1.25) + N + (1u << 16) + slack;
    uint64_t cap = estimate;
    unsigned long long* pairs = nullptr;
    unsigned long long used = 0, R = 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        cap = retry_cap(attempt, estimate, used, reserve_bound(R, warps, 64u));
        GSJ_TRY(dev_get(c, c->pairs, cap ? cap : 1, &pairs));
        GSJ_TRY(reset());
        o.emit = true;
        o.stride = 1;
        o.pairs = pairs;
        o.cap = cap;
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_join_emit<T>(a, o, ni, model, stamp, rows, c->num_sms, st));
        GSJ_TRY(d2h_small(c, &used, cursor, 1));
        GSJ_TRY(d2h_small(c, &R, o.rechecks, 1));
        if (used <= cap) break;
        if (attempt == 2) return fail(c, GSJ_ERR_STATE, "warp join: pair buffer short at its proven bound");
        c->stats.reruns++;
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[3], st));
    GSJ_TRY(pairs_to_csr(c, pairs, used, R, shift, N, counts, offsets, cand));
    S.join_path = GSJ_PATH_WARP;
    S.ms_join = now_ms() - t_join;
    S.ms_total = now_ms() - t_start;
    return GSJ_OK;
}

// ------------------------------------------------------------------ tile join
// Count, pair buffer, sort and table of the tile join (high-dimensional float
// data).  A sampling pass over every kSampleStride-th item sizes the pair
// buffer; the full pass counts every pair even past the buffer, so a short
// buffer is re-sized to the exact count and the pass repeated.
int tile_join(gsj_context* c, JoinArgs<float>& a, uint64_t N, bool stamp, int model, bool screen, bool exact_size,
              bool learned, uint32_t* counts, uint64_t* offsets, unsigned long long* cursor, double t_join,
              double t_start) {
    constexpr uint32_t kSampleStride = 64;
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    uint32_t shift = 1;
    while (shift < 32 && ((N - 1) >> shift)) shift++;
    const uint32_t ni = a.num_items;
    TileOut o{};
    o.cursor = cursor;
    o.shift = shift;
    o.rechecks = cursor + 1;  // the screen's exact count of undecided pairs
    // the screen's consumer warps reserve blocks (a warp appends at most
    // 32 x 16 undecided pairs at once; at most 64 warps per SM are resident);
    // the tile join appends exactly
    const uint64_t warps = (uint64_t)c->num_sms * 64u;
    const uint64_t slack = screen ? warps * kScreenBlockSlack : 0u;
    unsigned long long* cand = reinterpret_cast<unsigned long long*>(a.work_counter + 2);
    a.err_flag = a.work_counter + 1;
    ScreenConst sc = make_screen_const(a.n, a.thr);
    auto reset = [&]() -> int {
        // work counter, error flag and candidate statistic, then the cursor and rechecks
        GSJ_CUDA(c, cudaMemsetAsync(a.work_counter, 0, 4 * sizeof(uint32_t), st));
        GSJ_CUDA(c, cudaMemsetAsync(cursor, 0, 2 * sizeof(unsigned long long), st));
        return GSJ_OK;
    };
    auto launch = [&](uint32_t nvisit) -> cudaError_t {
        return screen ? launch_tile_screen(a, o, sc, stamp, model, nvisit, c->num_sms, st)
                      : launch_tile_join(a, o, stamp, model, nvisit, c->num_sms, st);
    };
    GSJ_CUDA(c, cudaEventRecord(c->tev[2], st));
    if (screen) {
        // centred BF16 rows and norms of all points, read by every candidate tile
        uint4* rows = nullptr;
        float *norms = nullptr, *centre = nullptr;
        double* partial = nullptr;
        GSJ_TRY(dev_get(c, c->srows, N * (sc.kpad / 8), &rows));
        GSJ_TRY(dev_get(c, c->snorms, N, &norms));
        GSJ_TRY(dev_get(c, c->spartial, (size_t)kScreenPrepBlocks * a.n * 2, &partial));
        GSJ_TRY(dev_get(c, c->scentre, a.n, &centre));
        S.kernel_launches += 3;
        GSJ_CUDA(c, launch_screen_prep(a.pts, (uint32_t)N, a.n, a.npad, sc.kpad, partial, centre, rows, norms, st));
        sc.rows = rows;
        sc.norms = norms;
    }
    // ---- estimate of the exact pass's entries (pairs, or the screen's undecided pairs)
    if (learned && screen && !(c->model_unc_ratio > 0.0)) learned = false;  // no screened training join yet
    GSJ_CUDA(c, cudaEventRecord(c->tev[6], st));
    double est = 0.0;
    if (learned) {
        GSJ_TRY(learned_estimate(c, &est));
        if (screen) est *= c->model_unc_ratio;
    } else if (!exact_size) {
        // sampled estimator: the exact pass over every kSampleStride-th item
        const uint32_t nsample = (ni + kSampleStride - 1) / kSampleStride;
        GSJ_TRY(reset());
        o.emit = false;
        o.stride = kSampleStride;
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch(nsample));
        unsigned long long sampled = 0;
        GSJ_TRY(d2h_small(c, &sampled, screen ? o.rechecks : cursor, 1));
        uint32_t err = 0;
        GSJ_TRY(d2h_small(c, &err, a.err_flag, 1));
        if (err) return fail(c, GSJ_ERR_CUDA, "tile join: tensor-core wait timed out");
        est = nsample ? (double)sampled * (double)ni / (double)nsample : 0.0;
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[7], st));
    S.estimate = (uint64_t)est;
    const uint64_t estimate = exact_size ? 0u : (uint64_t)(est * 1.25) + N + (1u << 16) + slack;
    uint64_t cap = estimate;
    // ---- full pass (repeated with a larger buffer if the buffer was short):
    // the tile join's hits, or the screen's undecided pairs
    unsigned long long *list = nullptr, *pairs = nullptr;
    unsigned long long U = 0, R = 0, nlist = 0, used = 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        cap = retry_cap(attempt, estimate, used, screen ? reserve_bound(U, warps, 512u) : U);
        GSJ_TRY(dev_get(c, screen ? c->unc : c->pairs, cap ? cap : 1, &list));
        GSJ_TRY(reset());
        o.emit = true;
        o.stride = 1;
        o.pairs = list;
        o.cap = cap;
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch(ni));
        // entries written (pairs), or reserved (undecided blocks)
        GSJ_TRY(d2h_small(c, &used, cursor, 1));
        U = used;
        if (screen) GSJ_TRY(d2h_small(c, &U, o.rechecks, 1));
        uint32_t err = 0;
        GSJ_TRY(d2h_small(c, &err, a.err_flag, 1));
        if (err) return fail(c, GSJ_ERR_CUDA, "tile join: tensor-core wait timed out");
        if (used <= cap) {
            nlist = used;
            break;
        }
        if (attempt == 2) return fail(c, GSJ_ERR_STATE, "tile join: pair buffer short at its proven bound");
        c->stats.reruns++;
    }
    if (screen) {
        // exact check of the undecided pairs; each yields at most one pair, two with unicomp
        const uint64_t pcap = stamp ? 2 * U : U;
        GSJ_TRY(dev_get(c, c->pairs, pcap ? pcap : 1, &pairs));
        GSJ_CUDA(c, cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), st));
        TileOut ro = o;
        ro.pairs = pairs;
        ro.cap = pcap;
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_screen_recheck(a, list, nlist, ro, stamp, model, c->num_sms, st));
        GSJ_TRY(d2h_small(c, &R, cursor, 1));
        if (R > pcap) return fail(c, GSJ_ERR_STATE, "screened join: more pairs than undecided candidates");
    } else {
        pairs = list;
        R = U;
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[3], st));
    GSJ_TRY(pairs_to_csr(c, pairs, R, R, shift, N, counts, offsets, cand));
    S.screen_rechecks = screen ? U : 0;
    S.join_path = screen ? GSJ_PATH_SCREEN : GSJ_PATH_TILE;
    S.ms_join = now_ms() - t_join;
    S.ms_total = now_ms() - t_start;
    return GSJ_OK;
}

// ------------------------------------------------------------------ host results
// Destination of gsj_join_host.
struct HostOut {
    uint32_t* counts;  // numNeighbors[N], host
    uint32_t* table;   // neighborTable, host, `cap` entries
    uint64_t cap;
};

int ensure_copy_streams(gsj_context* c, int nseg) {
    for (int i = 0; i < nseg; i++) {
        if (!c->cst[i]) GSJ_CUDA(c, cudaStreamCreateWithFlags(&c->cst[i], cudaStreamNonBlocking));
        if (!c->seg_filled[i]) GSJ_CUDA(c, cudaEventCreateWithFlags(&c->seg_filled[i], cudaEventDisableTiming));
        if (!c->seg_copied[i]) GSJ_CUDA(c, cudaEventCreateWithFlags(&c->seg_copied[i], cudaEventDisableTiming));
    }
    return GSJ_OK;
}

// ROWS path, results to the host: the table is filled in batches of point-id
// ranges whose lists fit one device segment; each batch's segment is copied to
// the host on its own copy stream while the compute stream fills the next
// segment.  offsets/counts are final (the count pass is exact), so every batch
// has a known place in the host table.
template <typename T>
int rows_to_host(gsj_context* c, JoinArgs<T>& a, const gsj_config& cfg, uint64_t N, uint64_t R,
                 const uint32_t* slot_cell, const uint64_t* bitoff, const uint32_t* hitbits, const uint32_t* counts,
                 const uint64_t* offsets, const HostOut& ho) {
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    uint32_t* ctr = a.work_counter;
    // numNeighbors to the host (overlaps the batches when the destination is pinned)
    const bool counts_pinned = host_is_pinned(ho.counts);
    const bool table_pinned = host_is_pinned(ho.table);
    GSJ_CUDA(c, cudaEventRecord(c->ev[0], st));
    if (counts_pinned) {
        GSJ_CUDA(c, cudaStreamWaitEvent(c->st2, c->ev[0], 0));
        GSJ_CUDA(c, cudaMemcpyAsync(ho.counts, counts, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st2));
    }
    // batch plan: segments of seg_cap entries, each batch at most seg_cap
    uint64_t seg_cap = cfg.buffer_pairs ? cfg.buffer_pairs : 100000000ull;
    const uint32_t min_b = cfg.min_batches ? cfg.min_batches : 3u;
    uint32_t lmax = 0;
    {
        uint32_t* d_lmax = reinterpret_cast<uint32_t*>(c->misc.p) + 4 * kMaxK + 28;
        GSJ_CUDA(c, cudaMemsetAsync(d_lmax, 0, sizeof(uint32_t), st));
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_max_u32(counts, N, d_lmax, st));
        GSJ_TRY(d2h_small(c, &lmax, d_lmax, 1));
    }
    if (seg_cap < 2ull * lmax) seg_cap = 2ull * lmax;  // the longest list must fit with room
    uint64_t step = seg_cap - lmax;
    const uint64_t even = (R + min_b - 1) / min_b;
    if (even >= 1 && even < step) step = even;
    // a batch holds fewer than step + lmax entries: no segment needs more
    seg_cap = std::min<uint64_t>(seg_cap, step + lmax);
    const uint64_t nb64 = R ? (R + step - 1) / step : 1;
    if (nb64 > 65535) return fail(c, GSJ_ERR_INVALID, "more than 65535 result batches: raise buffer_pairs");
    const uint32_t nb = (uint32_t)nb64;
    S.batches = nb;
    // bound[nb+1] and gstart[nb+1] (32-bit), then boff[nb+1] (64-bit)
    unsigned long long* bbuf = nullptr;
    GSJ_TRY(dev_get(c, c->bounds, 2ull * (nb + 1), &bbuf));
    uint32_t* bound = reinterpret_cast<uint32_t*>(bbuf);
    uint32_t* gstart = bound + (nb + 1);
    unsigned long long* boff = bbuf + (nb + 1);
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_batch_bounds(offsets, (uint32_t)N, step, nb, bound, boff, st));
    // the query slots grouped by batch (a stable sort keeps slot order inside a batch)
    uint32_t *bkey = nullptr, *bkey2 = nullptr, *qs = nullptr, *qs2 = nullptr;
    GSJ_TRY(dev_get(c, c->bkeys, 4ull * N, &bkey));
    bkey2 = bkey + N;
    qs = bkey + 2 * N;
    qs2 = bkey + 3 * N;
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_slot_batch(a.ids, (uint32_t)N, bound, nb, bkey, qs, st));
    int kb = 1;
    while (kb < 32 && ((nb - 1) >> kb)) kb++;
    void* temp = nullptr;
    GSJ_TRY(dev_get(c, c->temp, radix_sort_temp_bytes(N), (unsigned char**)&temp));
    bool alt = false;
    int nl = 0;
    if (nb > 1) GSJ_CUDA(c, radix_sort<uint32_t>(bkey, bkey2, qs, qs2, N, 0, kb, temp, &alt, &nl, st));
    S.kernel_launches += (uint64_t)nl;
    const uint32_t* sorted_key = alt ? bkey2 : bkey;
    const uint32_t* qslots = alt ? qs2 : qs;
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_group_starts(sorted_key, (uint32_t)N, nb, gstart, st));
    std::vector<uint32_t> h_gs(nb + 1);
    std::vector<unsigned long long> h_bo(nb + 1);
    GSJ_CUDA(c, cudaMemcpyAsync(h_gs.data(), gstart, (nb + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GSJ_CUDA(c, cudaMemcpyAsync(h_bo.data(), boff, (nb + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                st));
    GSJ_CUDA(c, cudaStreamSynchronize(st));
    if (h_bo[nb] != R) return fail(c, GSJ_ERR_STATE, "result batches do not cover the table (internal error)");
    // segments in flight
    const int nseg = (int)std::min<uint32_t>(nb, std::min<uint32_t>(cfg.streams ? cfg.streams : 3u,
                                                                      (uint32_t)gsj_context::kMaxSeg));
    GSJ_TRY(ensure_copy_streams(c, nseg));
    uint32_t* segs = nullptr;
    GSJ_TRY(dev_get(c, c->segs, (size_t)nseg * seg_cap, &segs));
    if (!table_pinned)
        for (int i = 0; i < nseg; i++) GSJ_TRY(pinned_get(c, c->hseg[i], seg_cap * sizeof(uint32_t)));
    a.offsets = offsets;
    a.table_cap = seg_cap;
    a.err_flag = ctr + 1;
    GSJ_CUDA(c, cudaEventRecord(c->tev[4], st));
    // pageable destinations: the staged batches are copied out in order
    uint32_t next_out = 0;
    auto drain = [&](uint32_t upto) -> int {
        for (; next_out < upto; next_out++) {
            const int sg = (int)(next_out % (uint32_t)nseg);
            GSJ_CUDA(c, cudaEventSynchronize(c->seg_copied[sg]));
            const uint64_t rb = h_bo[next_out + 1] - h_bo[next_out];
            par_memcpy(ho.table + h_bo[next_out], c->hseg[sg].p, rb * sizeof(uint32_t));
        }
        return GSJ_OK;
    };
    for (uint32_t b = 0; b < nb; b++) {
        const int sg = (int)(b % (uint32_t)nseg);
        if (b >= (uint32_t)nseg) {
            if (!table_pinned) GSJ_TRY(drain(b - (uint32_t)nseg + 1));  // frees the staging buffer
            GSJ_CUDA(c, cudaStreamWaitEvent(st, c->seg_copied[sg], 0));
        }
        uint32_t* seg = segs + (size_t)sg * seg_cap;
        a.table = seg;
        GSJ_CUDA(c, cudaMemsetAsync(ctr, 0, sizeof(uint32_t), st));
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_rows_fill<T>(a, slot_cell, bitoff, hitbits, qslots + h_gs[b], h_gs[b + 1] - h_gs[b],
                                        h_bo[b], c->num_sms, st));
        GSJ_CUDA(c, cudaEventRecord(c->seg_filled[sg], st));
        const uint64_t rb = h_bo[b + 1] - h_bo[b];
        GSJ_CUDA(c, cudaStreamWaitEvent(c->cst[sg], c->seg_filled[sg], 0));
        if (rb)
            GSJ_CUDA(c, cudaMemcpyAsync(table_pinned ? (void*)(ho.table + h_bo[b]) : c->hseg[sg].p, seg,
                                        rb * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->cst[sg]));
        GSJ_CUDA(c, cudaEventRecord(c->seg_copied[sg], c->cst[sg]));
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[5], st));
    if (!table_pinned) GSJ_TRY(drain(nb));
    for (int i = 0; i < nseg; i++) GSJ_CUDA(c, cudaStreamSynchronize(c->cst[i]));
    GSJ_CUDA(c, cudaStreamSynchronize(st));
    if (counts_pinned) GSJ_CUDA(c, cudaStreamSynchronize(c->st2));
    else GSJ_TRY(d2h_staged(c, ho.counts, counts, N * sizeof(uint32_t)));
    return GSJ_OK;
}

// ------------------------------------------------------------------ SORT path
// The reference's SORT traversal (kernel.cu:400-467), thread per query: count
// pass, list offsets, fill pass writing every list in candidate order.
template <typename T>
int sort_join(gsj_context* c, JoinArgs<T>& a, uint64_t N, int model, uint32_t* counts, uint64_t* offsets,
              const uint32_t* cell_start, uint32_t M, double t_join, double t_start) {
    gsj_stats& S = c->stats;
    cudaStream_t st = c->st;
    uint32_t* slot_cell = nullptr;
    GSJ_TRY(dev_get(c, c->slot_cell, N, &slot_cell));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_slot_cell(cell_start, M, nullptr, 0, slot_cell, nullptr, st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[2], st));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_sort_join<T>(a, slot_cell, counts, model, false, c->num_sms, st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[3], st));
    void* stemp = nullptr;
    GSJ_TRY(dev_get(c, c->scan_temp, scan_u32_u64_temp_bytes(N), (unsigned char**)&stemp));
    S.kernel_launches += 3;
    GSJ_CUDA(c, scan_u32_u64(counts, offsets, N, stemp, st));
    uint64_t R = 0;
    GSJ_TRY(d2h_small(c, &R, offsets + N, 1));
    uint32_t* table = nullptr;
    GSJ_TRY(dev_get(c, c->table, R ? R : 1, &table));
    a.offsets = offsets;
    a.table = table;
    a.table_cap = R;
    a.err_flag = a.work_counter + 1;
    GSJ_CUDA(c, cudaEventRecord(c->tev[4], st));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_sort_join<T>(a, slot_cell, counts, model, true, c->num_sms, st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[5], st));
    GSJ_CUDA(c, cudaStreamSynchronize(st));
    uint32_t err = 0;
    GSJ_TRY(d2h_small(c, &err, a.err_flag, 1));
    if (err) return fail(c, GSJ_ERR_STATE, "SORT fill pass disagreed with its count pass (internal error)");
    unsigned long long ncand = 0;
    GSJ_TRY(d2h_small(c, &ncand, a.cand_cnt, 1));
    {
        float ms = 0;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[0], c->tev[1]));
        S.dev_ms_index = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[2], c->tev[3]));
        S.dev_ms_count = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[4], c->tev[5]));
        S.dev_ms_fill = ms;
    }
    S.candidates = ncand;
    S.total_pairs = R;
    S.join_path = GSJ_PATH_SORT;
    c->R = R;
    c->have_result = true;
    S.ms_join = now_ms() - t_join;
    S.ms_total = now_ms() - t_start;
    return GSJ_OK;
}

// ------------------------------------------------------------------ join
template <typename T>
int run_join(gsj_context* c, const void* data, uint64_t N, double eps_d, const gsj_config& cfg, int on_dev,
             const HostOut* ho) {
    const double t_start = now_ms();
    gsj_stats& S = c->stats;
    S = gsj_stats{};
    S.num_points = N;
    c->have_result = false;
    c->table_on_device = true;
    c->last.valid = false;
    S.batches = 1;
    c->N = N;
    c->R = 0;
    const T eps = (T)eps_d;
    const uint32_t n = cfg.dim, k = cfg.indexed_dims;
    const uint32_t npad = npad_of(n, sizeof(T));
    cudaStream_t st = c->st;

    uint32_t *counts = nullptr;
    uint64_t* offsets = nullptr;
    GSJ_TRY(dev_get(c, c->counts, N + 1, &counts));
    GSJ_TRY(dev_get(c, c->offsets, N + 1, &offsets));
    if (N == 0) {
        GSJ_CUDA(c, cudaMemsetAsync(offsets, 0, sizeof(uint64_t), st));
        GSJ_CUDA(c, cudaStreamSynchronize(st));
        c->have_result = true;
        S.ms_total = now_ms() - t_start;
        return GSJ_OK;
    }

    // ---- input
    const T* d_in = nullptr;
    if (on_dev) {
        d_in = static_cast<const T*>(data);
    } else {
        T* p = nullptr;
        GSJ_TRY(dev_get(c, c->in, N * n, &p));
        const double t0 = now_ms();
        GSJ_TRY(h2d_copy(c, p, data, N * n * sizeof(T)));
        GSJ_CUDA(c, cudaStreamSynchronize(st));
        S.ms_h2d = now_ms() - t0;
        d_in = p;
    }
    const double t_index = now_ms();
    GSJ_CUDA(c, cudaEventRecord(c->tev[0], st));

    // ---- REORDER (main.cu:981-1075): statistic on the device, order on the host
    std::vector<uint32_t> perm(n);
    for (uint32_t j = 0; j < n; j++) perm[j] = j;
    if (cfg.reorder) {
        T* d_var = nullptr;
        GSJ_TRY(dev_get(c, c->var, n, &d_var));
        const T inv_sample = (T)(1.0 / (100 * 1.0));
        const T denom = (T)N * inv_sample;
        S.kernel_launches += 1;
    GSJ_CUDA(c, launch_variance<T>(d_in, N, n, denom, d_var, st));
        std::vector<T> var(n);
        GSJ_TRY(d2h_small(c, var.data(), d_var, n));
        std::vector<dim_reorder_sort<T>> dv(n);
        for (uint32_t j = 0; j < n; j++) dv[j] = {j, var[j]};
        std::sort(dv.begin(), dv.end(), compareByDimVariance<T>);
        for (uint32_t j = 0; j < n; j++) perm[j] = dv[j].dim;
    }
    uint32_t* d_perm = nullptr;
    GSJ_TRY(dev_get(c, c->perm, n, &d_perm));
    GSJ_CUDA(c, cudaMemcpyAsync(d_perm, perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));

    // ---- grid extents (main.cu:891-948)
    const uint32_t nparts = (uint32_t)std::min<uint64_t>((N + 255) / 256, (uint64_t)c->num_sms * 4);
    T *d_part = nullptr, *d_mm = nullptr;
    GSJ_TRY(dev_get(c, c->minmax_part, (size_t)nparts * 2 * k, &d_part));
    GSJ_TRY(dev_get(c, c->misc, kMiscWords, &d_mm));
    S.kernel_launches += 2;
    GSJ_CUDA(c, launch_minmax<T>(d_in, N, n, k, d_perm, d_part, nparts, d_mm, st));
    std::vector<T> mm(2 * k);
    GSJ_TRY(d2h_small(c, mm.data(), d_mm, 2 * k));
    std::vector<T> minArr(k), maxArr(k);
    GridGeom g{};
    g.k = k;
    uint64_t totalCells = 1;
    if (!(eps > T(0)) || std::isinf(eps))
        return fail(c, GSJ_ERR_INVALID, "epsilon must be positive and finite");
    long double cells_prod = 1.0L;
    for (uint32_t j = 0; j < k; j++) {
        minArr[j] = mm[j] - eps;
        maxArr[j] = mm[k + j] + eps;
        const T q = (maxArr[j] - minArr[j]) / eps;
        const T cq = std::ceil(q);
        if (!(cq >= T(1)) || !(cq < T(4294967296.0)))
            return fail(c, GSJ_ERR_INVALID, "grid dimension out of range (non-finite data or epsilon too small)");
        g.ncells[j] = (uint32_t)cq;
        cells_prod *= (long double)g.ncells[j];
    }
    // the reference's uint64 linear ids (main.cu:867-883) alias once the grid
    // has 2^64 cells or more; such grids are rejected instead
    if (cells_prod >= 18446744073709551615.0L)
        return fail(c, GSJ_ERR_INVALID, "grid has 2^64 cells or more (epsilon too small for this data)");
    uint64_t mult = 1;
    for (uint32_t j = 0; j < k; j++) {
        g.mult[j] = mult;
        mult *= g.ncells[j];
        totalCells = (j == 0) ? g.ncells[0] : totalCells * g.ncells[j];
    }
    S.total_cells = totalCells;
    // neighbour offsets in the kernels' order (digit j of o is dim j's step + 1):
    // linear-id delta, moved-down / moved-up dims, highest moved dim
    uint4* d_nbtab = nullptr;
    {
        uint32_t noff = 1;
        for (uint32_t j = 0; j < k; j++) noff *= 3u;
        std::vector<uint4> tab(noff);
        for (uint32_t o = 0; o < noff; o++) {
            long long delta = 0;
            uint32_t down = 0, up = 0, hd = 0xffu, t = o;
            for (uint32_t j = 0; j < k; j++) {
                const int dl = (int)(t % 3u) - 1;
                t /= 3u;
                delta += (long long)dl * (long long)g.mult[j];
                if (dl < 0) down |= 1u << j;
                if (dl > 0) up |= 1u << j;
                if (dl != 0) hd = j;
            }
            const uint64_t d = (uint64_t)delta;
            tab[o] = make_uint4((uint32_t)d, (uint32_t)(d >> 32), down | (up << 16), hd);
        }
        GSJ_TRY(dev_get(c, c->nbtab, noff, &d_nbtab));
        GSJ_CUDA(c, cudaMemcpyAsync(d_nbtab, tab.data(), noff * sizeof(uint4), cudaMemcpyHostToDevice, st));
    }
    T* d_min = nullptr;
    GSJ_TRY(dev_get(c, c->minarr, k, &d_min));
    GSJ_CUDA(c, cudaMemcpyAsync(d_min, minArr.data(), k * sizeof(T), cudaMemcpyHostToDevice, st));

    // ---- cell keys + radix sort (subsystem (a)): points ordered by cell, ties
    // by point id (a stable sort of keys generated in point-id order).  (A
    // counting sort through the dense slot table was measured slower on the 2-D
    // workload: its scatter of ids to random slots took 1.2 ms at 20M points,
    // more than the four coalesced radix passes.)
    uint64_t *keys = nullptr, *keys2 = nullptr;
    uint32_t *vals = nullptr, *ids = nullptr;
    GSJ_TRY(dev_get(c, c->keys, N, &keys));
    GSJ_TRY(dev_get(c, c->keys2, N, &keys2));
    GSJ_TRY(dev_get(c, c->vals, N, &vals));
    GSJ_TRY(dev_get(c, c->ids, N, &ids));
    int bits = 1;
    while (bits < 64 && (totalCells - 1) >> bits) bits++;
    const bool key32 = bits <= 32;
    void* temp = nullptr;
    GSJ_TRY(dev_get(c, c->temp, std::max(radix_sort_temp_bytes(N), runs_temp_bytes(N)), (unsigned char**)&temp));
    bool in_alt = false;
    int nl = 0;
    // the number of non-empty cells (word 0) and the out-of-range flag of the
    // cell keys (word 1)
    uint32_t* d_nruns = reinterpret_cast<uint32_t*>(d_mm + 2 * kMaxK);
    GSJ_CUDA(c, cudaMemsetAsync(d_nruns, 0, 2 * sizeof(uint32_t), st));
    S.kernel_launches += 1;
    if (key32) {
        uint32_t* k32 = reinterpret_cast<uint32_t*>(keys);
        uint32_t* k32b = reinterpret_cast<uint32_t*>(keys2);
        GSJ_CUDA(c, (launch_cell_keys<T, uint32_t>(d_in, N, n, d_perm, g, d_min, eps, k32, vals, d_nruns + 1, st)));
        GSJ_CUDA(c, radix_sort<uint32_t>(k32, k32b, vals, ids, N, 0, bits, temp, &in_alt, &nl, st));
    } else {
        GSJ_CUDA(c, (launch_cell_keys<T, uint64_t>(d_in, N, n, d_perm, g, d_min, eps, keys, vals, d_nruns + 1, st)));
        GSJ_CUDA(c, radix_sort<uint64_t>(keys, keys2, vals, ids, N, 0, bits, temp, &in_alt, &nl, st));
    }
    S.kernel_launches += (uint64_t)nl;
    if (!in_alt) {
        // an even number of passes (or none) leaves the result in the first buffers
        std::swap(c->keys, c->keys2);
        std::swap(c->vals, c->ids);
        std::swap(keys, keys2);
        std::swap(vals, ids);
    }

    // ---- runs of equal keys = non-empty cells: cell_key[M], cell_start[M+1]
    uint64_t* cell_key = nullptr;
    uint32_t* cell_start = nullptr;
    GSJ_TRY(dev_get(c, c->cell_key, N, &cell_key));
    GSJ_TRY(dev_get(c, c->cell_start, N + 1, &cell_start));
    S.kernel_launches += 5;
    if (key32)
        GSJ_CUDA(c, run_length<uint32_t>(reinterpret_cast<const uint32_t*>(keys2), N, cell_key, cell_start, d_nruns,
                                         temp, st));
    else
        GSJ_CUDA(c, run_length<uint64_t>(keys2, N, cell_key, cell_start, d_nruns, temp, st));
    uint32_t runs[2] = {0, 0};
    GSJ_TRY(d2h_small(c, runs, d_nruns, 2));
    if (runs[1])
        return fail(c, GSJ_ERR_INVALID,
                    "a coordinate maps to the grid's extent (epsilon below the resolution of the data's type)");
    const uint32_t M = runs[0];
    S.nonempty_cells = M;

    // ---- SORT (GPU.cu:351-395): each cell's points ordered by their value in the
    // sort dimension with std::sort and the reference's comparator, on the host
    // as the reference does (the tie order is std::sort's)
    if (cfg.sort && N > 1) {
        const uint32_t sd = n > k ? k : 0u;
        T* d_sv = reinterpret_cast<T*>(vals);  // the sort's value buffer is free now
        if (sizeof(T) > sizeof(uint32_t)) GSJ_TRY(dev_get(c, c->sortv, N, &d_sv));
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_sort_values<T>(d_in, N, n, perm[sd], ids, d_sv, st));
        std::vector<T> hv(N);
        std::vector<uint32_t> hid(N), hcs(M + 1);
        GSJ_CUDA(c, cudaMemcpyAsync(hv.data(), d_sv, N * sizeof(T), cudaMemcpyDeviceToHost, st));
        GSJ_CUDA(c, cudaMemcpyAsync(hid.data(), ids, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GSJ_CUDA(c, cudaMemcpyAsync(hcs.data(), cell_start, (M + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GSJ_CUDA(c, cudaStreamSynchronize(st));
        const unsigned nt = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16u);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; t++)
            th.emplace_back([&, t] {
                std::vector<key_val_sort<T>> tmp;
                for (uint64_t cc = t; cc < M; cc += nt) {
                    tmp.clear();
                    for (uint32_t s2 = hcs[cc]; s2 < hcs[cc + 1]; s2++) tmp.push_back({hid[s2], hv[s2]});
                    std::sort(tmp.begin(), tmp.end(), compareByPointValue<T>);
                    for (size_t x = 0; x < tmp.size(); x++) hid[hcs[cc] + x] = tmp[x].pid;
                }
            });
        for (auto& x : th) x.join();
        GSJ_CUDA(c, cudaMemcpyAsync(ids, hid.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        GSJ_CUDA(c, cudaStreamSynchronize(st));
    }

    // ---- points in cell order
    T* pts = nullptr;
    GSJ_TRY(dev_get(c, c->pts, N * npad, &pts));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_gather_points<T>(d_in, N, n, npad, d_perm, ids, pts, st));

    // ---- cell lookup: on dense grids a slot-prefix table over every linear
    // cell id (cell L holds slots [ds[L], ds[L+1])), else a hash table of the
    // non-empty cells
    uint32_t *ds = nullptr, *dcnt = nullptr;
    unsigned long long* hkeys = nullptr;
    uint32_t* hvals = nullptr;
    uint64_t hmask = 0;
    const uint64_t dense_limit = std::max<uint64_t>(1u << 24, 8ull * N);
    const bool dense = totalCells <= dense_limit && totalCells < (1ull << 30);
    if (dense) {
        GSJ_TRY(dev_get(c, c->dense, totalCells + 1, &ds));
        GSJ_TRY(dev_get(c, c->dcnt, totalCells + 1, &dcnt));
        GSJ_CUDA(c, cudaMemsetAsync(dcnt, 0, (totalCells + 1) * sizeof(uint32_t), st));
    } else {
        uint64_t hcap = 1024;
        while (hcap < 2ull * M) hcap <<= 1;
        hmask = hcap - 1;
        GSJ_TRY(dev_get(c, c->hkeys, hcap, &hkeys));
        GSJ_TRY(dev_get(c, c->hvals, hcap, &hvals));
        GSJ_CUDA(c, cudaMemsetAsync(hkeys, 0xff, hcap * sizeof(unsigned long long), st));
    }
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_cell_tables(cell_key, cell_start, M, dcnt, hkeys, hvals, hmask, st));
    if (dense) {
        // the slot-prefix table: ds[L] = points in cells below L (ds[totalCells] = N)
        GSJ_TRY(dev_get(c, c->temp, scan_u32_u64_temp_bytes(totalCells), (unsigned char**)&temp));
        S.kernel_launches += 3;
        GSJ_CUDA(c, scan_u32_u32(dcnt, ds, totalCells, temp, st));
    }
    // Dense low-dimensional grids use the row-range traversal driven by a
    // per-cell plan of neighbour-row slot ranges.
    const bool rows = dense && k <= 3;
    uint2* plan = nullptr;
    uint8_t* plan_par = nullptr;
    if (rows) {
        const uint32_t nrows = k == 1 ? 1u : (k == 2 ? 3u : 9u);
        GSJ_TRY(dev_get(c, c->plan, (size_t)M * nrows, &plan));
        GSJ_TRY(dev_get(c, c->plan_par, M, &plan_par));
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_cell_plan(cell_key, M, g, ds, plan, plan_par, st));
    }
    uint32_t* slot_cell = nullptr;
    uint64_t* bitoff = nullptr;
    const bool tpq = rows && cfg.ilp == 0 && n <= 4 && !cfg.sort;
    if (tpq) {
        // slot -> cell, and the hit-mask layout: slot s's query owns words
        // [bitoff[s], bitoff[s+1]) of the count pass's bit masks
        uint32_t* swords = nullptr;
        const uint32_t nrows = k == 1 ? 1u : (k == 2 ? 3u : 9u);
        GSJ_TRY(dev_get(c, c->slot_cell, N, &slot_cell));
        GSJ_TRY(dev_get(c, c->swords, N, &swords));
        GSJ_TRY(dev_get(c, c->bitoff, N + 1, &bitoff));
        GSJ_TRY(dev_get(c, c->scan_temp, scan_u32_u64_temp_bytes(N), (unsigned char**)&temp));
        S.kernel_launches += 4;
        GSJ_CUDA(c, launch_slot_cell(cell_start, M, plan, nrows, slot_cell, swords, st));
        GSJ_CUDA(c, scan_u32_u64(swords, bitoff, N, temp, st));
    }

    // High-dimensional float data with populated cells (at least 8 points per
    // non-empty cell on average) takes the tile join; everything else the
    // warp-per-item passes.
    // From 16 dimensions on, the tile join screens pairs with BF16 dot
    // products on the tensor cores (GSJ_FLAG_PLAIN turns the screen off).
    const int model = model_of(cfg);
    bool tile = false, screen = false;
    if constexpr (std::is_same<T, float>::value) {
        tile = !cfg.sort && tile_supported(n, npad, k, model, cfg.ilp) && N >= 8ull * M;
        screen = tile && !(cfg.flags & GSJ_FLAG_PLAIN) &&
                 screen_supported(n, npad, k, model, cfg.ilp, threshold_of<float>(eps));
    }
    const uint32_t qchunk = screen ? (uint32_t)kScreenQ : tile ? (uint32_t)kTileQ : (uint32_t)kQChunk;
    // launch shape: the autotuner's candidate, else the table's entry for this
    // (path, dim, density), else the launchers' defaults
    const uint32_t path_id = cfg.sort ? GSJ_PATH_SORT
                             : tpq    ? GSJ_PATH_ROWS
                             : screen ? GSJ_PATH_SCREEN
                             : tile   ? GSJ_PATH_TILE
                                      : GSJ_PATH_WARP;
    uint32_t dlog = 0;
    while (dlog < 31 && (N / std::max<uint32_t>(M, 1u)) >> (dlog + 1)) dlog++;
    S.density_log2 = dlog;
    gsj_tuning shape{};
    if (c->forced) {
        shape = *c->forced;
        S.tuned = 1;
    } else {
        auto it = c->tuning.find(std::make_tuple(path_id, n, dlog));
        if (it != c->tuning.end()) {
            shape = it->second;
            S.tuned = 1;
        }
    }

    // ---- work items (QUERYREORDER: heaviest cells first, GPU.cu:1491-1525).
    // The ROWS path has none: its passes claim 32 consecutive query slots at a
    // time, and the order in which queries run changes no result.
    uint32_t num_items = 0;
    uint2* items = nullptr;
    if (tpq) {
        S.work_items = ((uint64_t)N + 31u) / 32u;
    } else {
        uint32_t *order = nullptr, *nchunks = nullptr, *item_off = nullptr;
        GSJ_TRY(dev_get(c, c->nchunks, M + 1, &nchunks));
        GSJ_TRY(dev_get(c, c->item_off, M + 1, &item_off));
        if (cfg.query_reorder) {
            uint32_t *sizes = nullptr, *sizes2 = nullptr, *iota = nullptr;
            GSJ_TRY(dev_get(c, c->sizes, 2 * (size_t)M, &sizes));
            sizes2 = sizes + M;
            GSJ_TRY(dev_get(c, c->order, 2 * (size_t)M, &order));
            iota = order + M;
            // stable descending sort by cell size (ties keep ascending cell order):
            // an ascending sort of the complemented sizes
            S.kernel_launches += 2;
            GSJ_CUDA(c, launch_item_counts(cell_start, nullptr, M, qchunk, nchunks, sizes, st));
            GSJ_CUDA(c, launch_iota(iota, M, st));
            GSJ_TRY(dev_get(c, c->temp, radix_sort_temp_bytes(M), (unsigned char**)&temp));
            bool alt = false;
            int nl2 = 0;
            GSJ_CUDA(c, radix_sort<uint32_t>(sizes, sizes2, iota, order, M, 0, 32, temp, &alt, &nl2, st));
            S.kernel_launches += (uint64_t)nl2;
            if (!alt) {
                // the sorted cell indices are in iota (order + M): move them to order[0, M)
                GSJ_CUDA(c, cudaMemcpyAsync(order, iota, (size_t)M * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
            }
            S.kernel_launches += 1;
            GSJ_CUDA(c, launch_item_counts(cell_start, order, M, qchunk, nchunks, nullptr, st));
        } else {
            S.kernel_launches += 1;
            GSJ_CUDA(c, launch_item_counts(cell_start, nullptr, M, qchunk, nchunks, nullptr, st));
        }
        GSJ_TRY(dev_get(c, c->temp, scan_u32_u64_temp_bytes(M), (unsigned char**)&temp));
        S.kernel_launches += 3;
        GSJ_CUDA(c, scan_u32_u32(nchunks, item_off, M, temp, st));
        GSJ_TRY(d2h_small(c, &num_items, item_off + M, 1));
        S.work_items = num_items;
        GSJ_TRY(dev_get(c, c->items, num_items, &items));
        S.kernel_launches += 1;
        GSJ_CUDA(c, launch_make_items(order, nchunks, item_off, M, items, st));
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[1], st));
    GSJ_CUDA(c, cudaStreamSynchronize(st));
    const double t_join = now_ms();
    S.ms_index = t_join - t_index;

    // ---- join arguments (every path); per-slot list lengths of the ROWS path
    uint32_t* fwd = nullptr;
    if (tpq) GSJ_TRY(dev_get(c, c->fwd, N, &fwd));
    uint32_t* ctr = reinterpret_cast<uint32_t*>(d_mm + 2 * kMaxK) + 2;  // work counter
    unsigned long long* cand = reinterpret_cast<unsigned long long*>(reinterpret_cast<uint32_t*>(d_mm + 2 * kMaxK) + 4);
    GSJ_CUDA(c, cudaMemsetAsync(ctr, 0, 4 * sizeof(uint32_t), st));
    JoinArgs<T> a{};
    a.pts = pts;
    a.ids = ids;
    a.cell_start = cell_start;
    a.cell_key = cell_key;
    a.ds = ds;
    a.plan = plan;
    a.plan_par = plan_par;
    a.hkeys = reinterpret_cast<const uint64_t*>(hkeys);
    a.hvals = hvals;
    a.hmask = hmask;
    a.items = items;
    a.num_items = num_items;
    a.nbtab = d_nbtab;
    a.work_counter = ctr;
    a.n = n;
    a.npad = npad;
    a.n_points = (uint32_t)N;
    a.ilp = cfg.ilp;
    a.g = g;
    a.thr = threshold_of<T>(eps);
    a.eps = eps;
    for (uint32_t j = 0; j < k; j++) a.minv[j] = minArr[j];
    a.fwd_cnt = fwd;
    a.cand_cnt = cand;
    a.shape_threads = shape.threads;
    a.shape_warps = shape.warps;
    a.shape_per_sm = shape.ctas_per_sm;
    const bool stamp = cfg.stamp != 0 && !(cfg.flags & GSJ_FLAG_NO_UNICOMP);
    const bool exact_size = (cfg.flags & GSJ_FLAG_EXACT_SIZE) != 0;
    // the cell table of this join, for the model's features (estimate now,
    // training after the join)
    c->last.valid = true;
    c->last.M = M;
    c->last.n = n;
    c->last.log2_eps = (float)std::log2((double)eps);
    c->last.lookup = JoinArgs<float>{};
    c->last.lookup.cell_start = cell_start;
    c->last.lookup.cell_key = cell_key;
    c->last.lookup.ds = ds;
    c->last.lookup.hkeys = reinterpret_cast<const uint64_t*>(hkeys);
    c->last.lookup.hvals = hvals;
    c->last.lookup.hmask = hmask;
    c->last.lookup.g = g;
    c->last.lookup.n_points = (uint32_t)N;
    c->last.lookup.ids = ids;
    const bool learned = !exact_size && cfg.estimator == GSJ_EST_LEARNED && c->model_trained;
    if (cfg.sort) return sort_join<T>(c, a, N, model, counts, offsets, cell_start, M, t_join, t_start);
    if constexpr (std::is_same<T, float>::value) {
        if (tile) {
            unsigned long long* cursor = reinterpret_cast<unsigned long long*>(ctr + 4);
            return tile_join(c, a, N, stamp, model, screen, exact_size, learned, counts, offsets, cursor, t_join,
                             t_start);
        }
    }
    // Every other grid except the thread-per-query rows: one emit pass + pair sort.
    if (!tpq) {
        unsigned long long* cursor = reinterpret_cast<unsigned long long*>(ctr + 4);
        return emit_join<T>(c, a, N, stamp, model, rows, exact_size, learned, counts, offsets, cursor, t_join,
                            t_start);
    }
    // Dense low-dimensional grids (the ROWS path): the distance work is cheap
    // and the cells too small for per-cell warp work, so one thread per query
    // evaluates its full neighbourhood once, recording the decisions as a bit
    // mask; the fill pass replays the masks into the table.
    uint32_t* hitbits = nullptr;
    {
        uint64_t nwords = 0;
        GSJ_TRY(d2h_small(c, &nwords, bitoff + N, 1));
        GSJ_TRY(dev_get(c, c->hitbits, nwords ? nwords : 1, &hitbits));
    }
    GSJ_CUDA(c, cudaEventRecord(c->tev[2], st));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_rows_count<T>(a, slot_cell, bitoff, hitbits, counts, c->num_sms, st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[3], st));

    // ---- list offsets (counts are by point id)
    void* stemp = nullptr;
    GSJ_TRY(dev_get(c, c->scan_temp, scan_u32_u64_temp_bytes(N), (unsigned char**)&stemp));
    S.kernel_launches += 3;
    GSJ_CUDA(c, scan_u32_u64(counts, offsets, N, stemp, st));
    uint64_t R = 0;
    GSJ_TRY(d2h_small(c, &R, offsets + N, 1));
    unsigned long long ncand = 0;
    GSJ_TRY(d2h_small(c, &ncand, cand, 1));
    S.candidates = ncand;

    // ---- fill pass: into the device table, or in batches to the host
    if (ho) {
        c->table_on_device = false;
        if (ho->cap < R) {
            GSJ_TRY(d2h_staged(c, ho->counts, counts, N * sizeof(uint32_t)));
            S.total_pairs = R;
            c->R = R;
            return GSJ_ERR_OVERFLOW;
        }
        gsj_config pcfg = cfg;
        if (shape.streams) pcfg.streams = shape.streams;
        GSJ_TRY(rows_to_host<T>(c, a, pcfg, N, R, slot_cell, bitoff, hitbits, counts, offsets, *ho));
        {
            float ms = 0;
            GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[0], c->tev[1]));
            S.dev_ms_index = ms;
            GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[2], c->tev[3]));
            S.dev_ms_count = ms;
            GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[4], c->tev[5]));
            S.dev_ms_fill = ms;
        }
        uint32_t errflag = 0;
        GSJ_TRY(d2h_small(c, &errflag, ctr + 1, 1));
        if (errflag) return fail(c, GSJ_ERR_STATE, "fill pass: a list would leave its segment (internal error)");
        S.ms_join = now_ms() - t_join;
        S.total_pairs = R;
        S.join_path = GSJ_PATH_ROWS;
        c->R = R;
        c->have_result = true;
        S.ms_total = now_ms() - t_start;
        return GSJ_OK;
    }
    uint32_t* table = nullptr;
    GSJ_TRY(dev_get(c, c->table, R ? R : 1, &table));
    GSJ_CUDA(c, cudaMemsetAsync(ctr, 0, sizeof(uint32_t), st));
    a.offsets = offsets;
    a.table = table;
    a.table_cap = R;
    a.err_flag = ctr + 1;  // zeroed with the counters before the count pass
    GSJ_CUDA(c, cudaEventRecord(c->tev[4], st));
    S.kernel_launches += 1;
    GSJ_CUDA(c, launch_rows_fill<T>(a, slot_cell, bitoff, hitbits, nullptr, (uint32_t)N, 0, c->num_sms, st));
    GSJ_CUDA(c, cudaEventRecord(c->tev[5], st));
    GSJ_CUDA(c, cudaStreamSynchronize(st));
    {
        float ms = 0;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[0], c->tev[1]));
        S.dev_ms_index = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[2], c->tev[3]));
        S.dev_ms_count = ms;
        GSJ_CUDA(c, cudaEventElapsedTime(&ms, c->tev[4], c->tev[5]));
        S.dev_ms_fill = ms;
    }
    uint32_t errflag = 0;
    GSJ_TRY(d2h_small(c, &errflag, ctr + 1, 1));
    if (errflag) return fail(c, GSJ_ERR_STATE, "fill pass: a list would leave the table (internal error)");
    if ((cfg.flags & GSJ_FLAG_SORT_LISTS) && R > 1) {
        // every list ascending
        GSJ_TRY(sort_table_lists(c, table, offsets, N, R));
        GSJ_CUDA(c, cudaStreamSynchronize(st));
    }
    S.ms_join = now_ms() - t_join;
    S.total_pairs = R;
    S.join_path = GSJ_PATH_ROWS;
    c->R = R;
    c->have_result = true;
    S.ms_total = now_ms() - t_start;
    return GSJ_OK;
}

}  // namespace

namespace gsj {
// Error reporting for entry points defined in other translation units.
int report_error(int code, const std::string& msg) { return fail(nullptr, code, msg); }
}  // namespace gsj

// ====================================================================== C ABI
extern "C" {

static std::mutex g_cfg_mu;
static bool g_cfg_set = false;
static gsj_config g_cfg;

void gsj_default_config(gsj_config* cfg) {
    if (!cfg) return;
    {
        std::lock_guard<std::mutex> lk(g_cfg_mu);
        if (g_cfg_set) {
            *cfg = g_cfg;
            return;
        }
    }
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->dim = GPUNUMDIM;
    cfg->indexed_dims = NUMINDEXEDDIM;
#ifdef GSJ_DTYPE_DOUBLE
    cfg->dtype = GSJ_FLOAT64;
#else
    cfg->dtype = GSJ_FLOAT32;
#endif
    cfg->reorder = REORDER;
    cfg->shortcircuit = SHORTCIRCUIT;
    cfg->ilp = ILP;
    cfg->stamp = (STAMP || LINEARSTAMP) ? 1 : 0;
    cfg->query_reorder = QUERYREORDER;
    cfg->sort = SORT;
    cfg->device = 0;
    cfg->flags = GSJ_FLAG_QUIET;
}

int gsj_set_default_config(const gsj_config* cfg) {
    if (!cfg) return fail(nullptr, GSJ_ERR_INVALID, "null config");
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    g_cfg = *cfg;
    g_cfg_set = true;
    return GSJ_OK;
}

int gsj_create(gsj_context** out, int device) {
    if (!out) return fail(nullptr, GSJ_ERR_INVALID, "null context pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, GSJ_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(nullptr, GSJ_ERR_INVALID, "device ordinal out of range");
    gsj_context* c = new gsj_context();
    c->device = device;
    GSJ_CUDA(c, cudaSetDevice(device));
    GSJ_CUDA(c, cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    GSJ_CUDA(c, cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    GSJ_CUDA(c, cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
    GSJ_CUDA(c, cudaEventCreateWithFlags(&c->ev[0], cudaEventDisableTiming));
    GSJ_CUDA(c, cudaEventCreateWithFlags(&c->ev[1], cudaEventDisableTiming));
    for (auto& e : c->tev) GSJ_CUDA(c, cudaEventCreate(&e));
    *out = c;
    return GSJ_OK;
}

int gsj_destroy(gsj_context* c) {
    if (!c) return GSJ_OK;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->st2) cudaStreamSynchronize(c->st2);
    Buf* bufs[] = {&c->in,       &c->pts,   &c->ids,    &c->keys,      &c->keys2,   &c->vals,      &c->cell_key,
                   &c->cell_start, &c->dense, &c->dcnt, &c->plan, &c->plan_par, &c->slot_cell, &c->hkeys,
                   &c->hvals,
                   &c->order,    &c->sizes,
                   &c->nchunks,  &c->item_off, &c->items, &c->fwd,     &c->swords,     &c->counts,    &c->offsets,
                   &c->table, &c->temp,   &c->scan_temp, &c->misc,    &c->var,       &c->perm,
                   &c->minarr,   &c->minmax_part, &c->pairs, &c->srows, &c->snorms,
                   &c->spartial, &c->scentre, &c->unc, &c->table2, &c->nbtab, &c->bitoff, &c->hitbits, &c->ptemp, &c->sortv};
    for (Buf* b : bufs)
        if (b->p) cudaFree(b->p);
    for (auto* pb : {&c->stage[0], &c->stage[1], &c->hmisc})
        if (pb->p) cudaFreeHost(pb->p);
    for (int i = 0; i < gsj_context::kMaxSeg; i++) {
        if (c->cst[i]) cudaStreamSynchronize(c->cst[i]);
        if (c->hseg[i].p) cudaFreeHost(c->hseg[i].p);
        if (c->seg_filled[i]) cudaEventDestroy(c->seg_filled[i]);
        if (c->seg_copied[i]) cudaEventDestroy(c->seg_copied[i]);
        if (c->cst[i]) cudaStreamDestroy(c->cst[i]);
    }
    for (Buf* b : {&c->segs, &c->bounds, &c->bkeys, &c->mw, &c->mm1, &c->mm2, &c->mx, &c->my, &c->mxt, &c->myt,
                   &c->mtmp})
        if (b->p) cudaFree(b->p);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->tev)
        if (e) cudaEventDestroy(e);
    if (c->st) cudaStreamDestroy(c->st);
    if (c->st2) cudaStreamDestroy(c->st2);
    delete c;
    return GSJ_OK;
}

int gsj_join(gsj_context* c, const void* data, uint64_t num_points, double eps, const gsj_config* cfg,
             int data_on_device, gsj_stats* stats) {
    if (!c || !cfg) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!data && num_points) return fail(c, GSJ_ERR_INVALID, "null data");
    GSJ_TRY(validate(c, *cfg, num_points));
    if (cfg->device != c->device) return fail(c, GSJ_ERR_INVALID, "config device differs from the context's device");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    int r = cfg->dtype == GSJ_FLOAT32 ? run_join<float>(c, data, num_points, eps, *cfg, data_on_device, nullptr)
                                      : run_join<double>(c, data, num_points, eps, *cfg, data_on_device, nullptr);
    if (stats) *stats = c->stats;
    return r;
}

int gsj_join_host(gsj_context* c, const void* data, uint64_t num_points, double eps, const gsj_config* cfg,
                  int data_on_device, uint32_t* num_neighbors, uint32_t* neighbor_table, uint64_t cap,
                  uint64_t* total_pairs, gsj_stats* stats) {
    if (!c || !cfg || !total_pairs) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!data && num_points) return fail(c, GSJ_ERR_INVALID, "null data");
    if (!num_neighbors && num_points) return fail(c, GSJ_ERR_INVALID, "null num_neighbors");
    if (!neighbor_table && cap) return fail(c, GSJ_ERR_INVALID, "null neighbor_table");
    GSJ_TRY(validate(c, *cfg, num_points));
    if (cfg->device != c->device) return fail(c, GSJ_ERR_INVALID, "config device differs from the context's device");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    *total_pairs = 0;
    HostOut ho{num_neighbors, neighbor_table, cap};
    const double t0 = now_ms();
    int r = cfg->dtype == GSJ_FLOAT32 ? run_join<float>(c, data, num_points, eps, *cfg, data_on_device, &ho)
                                      : run_join<double>(c, data, num_points, eps, *cfg, data_on_device, &ho);
    if (r == GSJ_OK || r == GSJ_ERR_OVERFLOW) *total_pairs = c->R;
    if (r == GSJ_OK && c->table_on_device && c->N) {
        // paths without batches: the finished result is copied out
        if (cap < c->R) {
            r = d2h_staged(c, num_neighbors, c->counts.p, c->N * sizeof(uint32_t));
            if (r == GSJ_OK) r = GSJ_ERR_OVERFLOW;
        } else {
            const double t1 = now_ms();
            r = d2h_staged(c, num_neighbors, c->counts.p, c->N * sizeof(uint32_t));
            if (r == GSJ_OK && c->R) r = d2h_staged(c, neighbor_table, c->table.p, c->R * sizeof(uint32_t));
            c->stats.ms_d2h += now_ms() - t1;
        }
    }
    if (r == GSJ_ERR_OVERFLOW) fail(c, r, "neighbor_table holds fewer entries than the result (see total_pairs)");
    c->stats.ms_total = now_ms() - t0;
    if (stats) *stats = c->stats;
    return r;
}

static int tuning_valid(gsj_context* c, const gsj_tuning& t) {
    if (t.threads && (t.threads < 64 || t.threads > 256 || (t.threads & 31u)))
        return fail(c, GSJ_ERR_INVALID, "tuning: threads must be 64..256, a multiple of 32");
    if (t.warps > 8) return fail(c, GSJ_ERR_INVALID, "tuning: warps must be at most 8");
    if (t.streams > (uint32_t)gsj_context::kMaxSeg) return fail(c, GSJ_ERR_INVALID, "tuning: at most 8 streams");
    return GSJ_OK;
}

int gsj_tuning_get(gsj_context* c, uint32_t path, uint32_t dim, uint32_t dlog, gsj_tuning* t) {
    if (!c || !t) return fail(c, GSJ_ERR_INVALID, "null argument");
    auto it = c->tuning.find(std::make_tuple(path, dim, dlog));
    if (it == c->tuning.end()) return fail(c, GSJ_ERR_STATE, "no tuning entry for this key");
    *t = it->second;
    return GSJ_OK;
}

int gsj_tuning_set(gsj_context* c, uint32_t path, uint32_t dim, uint32_t dlog, const gsj_tuning* t) {
    if (!c || !t) return fail(c, GSJ_ERR_INVALID, "null argument");
    GSJ_TRY(tuning_valid(c, *t));
    c->tuning[std::make_tuple(path, dim, dlog)] = *t;
    return GSJ_OK;
}

int gsj_autotune(gsj_context* c, const void* data, uint64_t num_points, double eps, const gsj_config* cfg,
                 int data_on_device, uint32_t repeats, gsj_tuning* best) {
    if (!c || !cfg || !best) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (repeats == 0) repeats = 1;
    gsj_stats st{};
    // the path and density of this join, under the current shape
    GSJ_TRY(gsj_join(c, data, num_points, eps, cfg, data_on_device, &st));
    if (num_points == 0) return fail(c, GSJ_ERR_INVALID, "nothing to tune on an empty input");
    const uint32_t path = (uint32_t)st.join_path, dlog = (uint32_t)st.density_log2;
    gsj_tuning cur{};
    {
        auto it = c->tuning.find(std::make_tuple(path, cfg->dim, dlog));
        if (it != c->tuning.end()) cur = it->second;
    }
    auto timed = [&](const gsj_tuning& t, double* ms) -> int {
        c->forced = &t;
        int r = gsj_join(c, data, num_points, eps, cfg, data_on_device, &st);  // warm-up
        double sum = 0.0;
        for (uint32_t i = 0; r == GSJ_OK && i < repeats; i++) {
            r = gsj_join(c, data, num_points, eps, cfg, data_on_device, &st);
            sum += st.dev_ms_index + st.dev_ms_count + st.dev_ms_fill;
        }
        c->forced = nullptr;
        *ms = sum / repeats;
        return r;
    };
    // the knobs of the path and their candidate values (0 = the default)
    std::vector<std::pair<uint32_t gsj_tuning::*, std::vector<uint32_t>>> knobs;
    if (path == GSJ_PATH_ROWS) knobs.push_back({&gsj_tuning::threads, {0, 128, 192}});
    if (path == GSJ_PATH_WARP) {
        knobs.push_back({&gsj_tuning::warps, {0, 4, 2}});
        knobs.push_back({&gsj_tuning::ctas_per_sm, {0, 4, 2}});
    }
    if (path == GSJ_PATH_TILE) knobs.push_back({&gsj_tuning::ctas_per_sm, {0, 2, 1}});
    if (path == GSJ_PATH_SCREEN) knobs.push_back({&gsj_tuning::ctas_per_sm, {0, 1}});
    double best_ms = 0.0;
    GSJ_TRY(timed(cur, &best_ms));
    for (auto& kv : knobs) {
        for (uint32_t v : kv.second) {
            gsj_tuning cand = cur;
            cand.*(kv.first) = v;
            if (cand.*(kv.first) == cur.*(kv.first)) continue;
            double ms = 0.0;
            GSJ_TRY(timed(cand, &ms));
            if (ms < best_ms) {
                best_ms = ms;
                cur = cand;
            }
        }
    }
    c->tuning[std::make_tuple(path, cfg->dim, dlog)] = cur;
    *best = cur;
    return GSJ_OK;
}

int gsj_bruteforce_count(gsj_context* c, const void* data, uint64_t num_points, double eps, const gsj_config* cfg,
                         int data_on_device, uint32_t* counts, uint64_t* total) {
    if (!c || !cfg || !total) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!data && num_points) return fail(c, GSJ_ERR_INVALID, "null data");
    if (cfg->dim == 0 || cfg->dim > 4096) return fail(c, GSJ_ERR_INVALID, "dim must be in 1..4096");
    if (cfg->dtype != GSJ_FLOAT32 && cfg->dtype != GSJ_FLOAT64) return fail(c, GSJ_ERR_INVALID, "unknown dtype");
    if (num_points >= (1ull << 31)) return fail(c, GSJ_ERR_INVALID, "at most 2^31-1 points");
    if (cfg->device != c->device) return fail(c, GSJ_ERR_INVALID, "config device differs from the context's device");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    *total = 0;
    if (num_points == 0) return GSJ_OK;
    const uint32_t n = cfg->dim, N = (uint32_t)num_points;
    const size_t tsz = cfg->dtype == GSJ_FLOAT32 ? 4 : 8;
    cudaStream_t st = c->st;
    const void* d_pts = data;
    if (!data_on_device) {
        unsigned char* p = nullptr;
        GSJ_TRY(dev_get(c, c->in, (size_t)N * n * tsz, &p));
        GSJ_TRY(h2d_copy(c, p, data, (size_t)N * n * tsz));
        d_pts = p;
    }
    uint32_t* d_counts = nullptr;
    unsigned long long* d_total = nullptr;
    GSJ_TRY(dev_get(c, c->counts, (size_t)N + 1, &d_counts));
    GSJ_TRY(dev_get(c, c->misc, kMiscWords, reinterpret_cast<double**>(&d_total)));
    GSJ_CUDA(c, cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), st));
    if (cfg->dtype == GSJ_FLOAT32) {
        const float e = (float)eps;
        if (!(e >= 0.f)) return fail(c, GSJ_ERR_INVALID, "epsilon must be non-negative");
        GSJ_CUDA(c, launch_bruteforce<float>(static_cast<const float*>(d_pts), N, n, threshold_of<float>(e), d_counts,
                                             d_total, st));
    } else {
        if (!(eps >= 0.0)) return fail(c, GSJ_ERR_INVALID, "epsilon must be non-negative");
        GSJ_CUDA(c, launch_bruteforce<double>(static_cast<const double*>(d_pts), N, n, threshold_of<double>(eps),
                                              d_counts, d_total, st));
    }
    unsigned long long t = 0;
    GSJ_TRY(d2h_small(c, &t, d_total, 1));
    *total = t;
    if (counts) GSJ_TRY(d2h_staged(c, counts, d_counts, (size_t)N * 4));
    c->have_result = false;  // the context's result buffers were reused
    return GSJ_OK;
}

int gsj_result_size(gsj_context* c, uint64_t* total) {
    if (!c || !total) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!c->have_result) return fail(c, GSJ_ERR_STATE, "no join result");
    *total = c->R;
    return GSJ_OK;
}

int gsj_result_counts(gsj_context* c, uint32_t* out, int dst_on_device) {
    if (!c || (!out && c->N)) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!c->have_result) return fail(c, GSJ_ERR_STATE, "no join result");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    if (c->N == 0) return GSJ_OK;
    if (dst_on_device) {
        GSJ_CUDA(c, cudaMemcpyAsync(out, c->counts.p, c->N * 4, cudaMemcpyDeviceToDevice, c->st));
        GSJ_CUDA(c, cudaStreamSynchronize(c->st));
        return GSJ_OK;
    }
    const double t0 = now_ms();
    int r = d2h_staged(c, out, c->counts.p, c->N * 4);
    c->stats.ms_d2h += now_ms() - t0;
    return r;
}

int gsj_result_table(gsj_context* c, uint32_t* out, uint64_t cap, int dst_on_device) {
    if (!c || (!out && c->R)) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (!c->have_result) return fail(c, GSJ_ERR_STATE, "no join result");
    if (!c->table_on_device) return fail(c, GSJ_ERR_STATE, "the last join delivered its table to host memory");
    if (cap < c->R) return fail(c, GSJ_ERR_INVALID, "destination smaller than the result");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    if (c->R == 0) return GSJ_OK;
    if (dst_on_device) {
        GSJ_CUDA(c, cudaMemcpyAsync(out, c->table.p, c->R * 4, cudaMemcpyDeviceToDevice, c->st));
        GSJ_CUDA(c, cudaStreamSynchronize(c->st));
        return GSJ_OK;
    }
    const double t0 = now_ms();
    int r = d2h_staged(c, out, c->table.p, c->R * 4);
    c->stats.ms_d2h += now_ms() - t0;
    return r;
}

int gsj_result_device(gsj_context* c, const uint32_t** counts, const uint64_t** offsets, const uint32_t** table) {
    if (!c) return fail(c, GSJ_ERR_INVALID, "null context");
    if (!c->have_result) return fail(c, GSJ_ERR_STATE, "no join result");
    if (table && !c->table_on_device) return fail(c, GSJ_ERR_STATE, "the last join delivered its table to host memory");
    if (counts) *counts = static_cast<const uint32_t*>(c->counts.p);
    if (offsets) *offsets = static_cast<const uint64_t*>(c->offsets.p);
    if (table) *table = static_cast<const uint32_t*>(c->table.p);
    return GSJ_OK;
}

const char* gsj_last_error(gsj_context* c) {
    if (c) return c->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_err_default.c_str();
}

float gsj_threshold_f32(float eps) { return threshold_of<float>(eps); }
double gsj_threshold_f64(double eps) { return threshold_of<double>(eps); }

// ---------------------------------------------------------------- learned model
static int model_ensure(gsj_context* c) {
    float *w = nullptr, *m1 = nullptr, *m2 = nullptr;
    GSJ_TRY(dev_get(c, c->mw, kModelWeights, &w));
    GSJ_TRY(dev_get(c, c->mm1, kModelWeights, &m1));
    GSJ_TRY(dev_get(c, c->mm2, kModelWeights, &m2));
    if (!c->model_ready) {
        GSJ_CUDA(c, model_init(w, m1, m2, 0x5eed1234u, c->st));
        c->model_ready = true;
        c->model_trained = false;
        c->model_t = 0;
        c->model_unc_ratio = 0.0;
    }
    return GSJ_OK;
}

// Features and targets of the last join's cells into c->mx / c->my.
static int model_dataset(gsj_context* c, uint32_t* M_out) {
    if (!c->have_result || !c->last.valid) return fail(c, GSJ_ERR_STATE, "no indexed join result to learn from");
    const uint32_t M = c->last.M;
    float *X = nullptr, *Y = nullptr;
    GSJ_TRY(dev_get(c, c->mx, (size_t)M * kModelFeatures, &X));
    GSJ_TRY(dev_get(c, c->my, M, &Y));
    GSJ_CUDA(c, model_features(c->last.lookup, M, c->last.log2_eps, c->last.n, X, c->st));
    GSJ_CUDA(c, model_targets(c->last.lookup.cell_start, c->last.lookup.ids, static_cast<const uint32_t*>(c->counts.p),
                              M, Y, c->st));
    *M_out = M;
    return GSJ_OK;
}

int gsj_model_reset(gsj_context* c) {
    if (!c) return fail(c, GSJ_ERR_INVALID, "null context");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    c->model_ready = false;
    GSJ_TRY(model_ensure(c));
    GSJ_CUDA(c, cudaStreamSynchronize(c->st));
    return GSJ_OK;
}

int gsj_model_train(gsj_context* c, uint32_t steps, float* loss) {
    if (!c) return fail(c, GSJ_ERR_INVALID, "null context");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    GSJ_TRY(model_ensure(c));
    uint32_t M = 0;
    GSJ_TRY(model_dataset(c, &M));
    if (M == 0) return fail(c, GSJ_ERR_STATE, "the last join has no cells");
    const uint32_t ntr = std::min<uint32_t>(M, kModelTrainRows);
    float *Xt = nullptr, *Yt = nullptr, *d_loss = nullptr;
    GSJ_TRY(dev_get(c, c->mxt, (size_t)ntr * kModelFeatures, &Xt));
    GSJ_TRY(dev_get(c, c->myt, ntr, &Yt));
    GSJ_TRY(dev_get(c, c->mtmp, 4, reinterpret_cast<double**>(&d_loss)));
    GSJ_CUDA(c, model_subsample(static_cast<const float*>(c->mx.p), static_cast<const float*>(c->my.p), M, ntr, Xt,
                                Yt, c->st));
    GSJ_CUDA(c, model_train(Xt, Yt, ntr, static_cast<float*>(c->mw.p), static_cast<float*>(c->mm1.p),
                            static_cast<float*>(c->mm2.p), c->model_t, steps, 3e-3f, d_loss + 2, c->st));
    c->model_t += steps;
    float l = 0.f;
    GSJ_TRY(d2h_small(c, &l, d_loss + 2, 1));
    if (loss) *loss = l;
    c->model_trained = steps > 0 || c->model_trained;
    if (c->stats.join_path == GSJ_PATH_SCREEN && c->stats.total_pairs)
        c->model_unc_ratio = (double)c->stats.screen_rechecks / (double)c->stats.total_pairs;
    return GSJ_OK;
}

int gsj_model_weights(gsj_context* c, float* weights, uint32_t count, int set) {
    if (!c || !weights) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (count != (uint32_t)kModelWeights)
        return fail(c, GSJ_ERR_INVALID, "the model has " + std::to_string(kModelWeights) + " weights");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    GSJ_TRY(model_ensure(c));
    if (set) {
        GSJ_CUDA(c, cudaMemcpyAsync(c->mw.p, weights, count * sizeof(float), cudaMemcpyHostToDevice, c->st));
        GSJ_CUDA(c, cudaMemsetAsync(c->mm1.p, 0, count * sizeof(float), c->st));
        GSJ_CUDA(c, cudaMemsetAsync(c->mm2.p, 0, count * sizeof(float), c->st));
        GSJ_CUDA(c, cudaStreamSynchronize(c->st));
        c->model_t = 0;
        c->model_trained = true;
        return GSJ_OK;
    }
    return d2h_small(c, weights, static_cast<const float*>(c->mw.p), count);
}

int gsj_model_features(gsj_context* c, float* features, float* targets, uint32_t cap, uint32_t* cells) {
    if (!c || !cells) return fail(c, GSJ_ERR_INVALID, "null argument");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    uint32_t M = 0;
    GSJ_TRY(model_dataset(c, &M));
    *cells = M;
    if (cap < M) {
        GSJ_CUDA(c, cudaStreamSynchronize(c->st));
        return GSJ_OK;
    }
    if (features) GSJ_TRY(d2h_small(c, features, static_cast<const float*>(c->mx.p), (size_t)M * kModelFeatures));
    if (targets) GSJ_TRY(d2h_small(c, targets, static_cast<const float*>(c->my.p), M));
    GSJ_CUDA(c, cudaStreamSynchronize(c->st));
    return GSJ_OK;
}

// Host rows -> device scratch (c->mxt / c->myt).
static int model_upload(gsj_context* c, const float* features, const float* targets, uint32_t n, float** X,
                        float** Y) {
    GSJ_TRY(dev_get(c, c->mxt, (size_t)n * kModelFeatures, X));
    GSJ_TRY(dev_get(c, c->myt, n, Y));
    GSJ_CUDA(c, cudaMemcpyAsync(*X, features, (size_t)n * kModelFeatures * sizeof(float), cudaMemcpyHostToDevice,
                                c->st));
    if (targets) GSJ_CUDA(c, cudaMemcpyAsync(*Y, targets, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, c->st));
    return GSJ_OK;
}

int gsj_model_predict(gsj_context* c, const float* features, uint32_t n, float* out) {
    if (!c || (n && (!features || !out))) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (n == 0) return GSJ_OK;
    GSJ_CUDA(c, cudaSetDevice(c->device));
    GSJ_TRY(model_ensure(c));
    float *X = nullptr, *Y = nullptr;
    GSJ_TRY(model_upload(c, features, nullptr, n, &X, &Y));
    GSJ_CUDA(c, model_predict(X, n, static_cast<const float*>(c->mw.p), Y, nullptr, 0.f, nullptr, c->st));
    return d2h_small(c, out, Y, n);
}

int gsj_model_loss_grad(gsj_context* c, const float* features, const float* targets, uint32_t n, float* loss,
                        float* grad) {
    if (!c || !features || !targets || !loss || !grad) return fail(c, GSJ_ERR_INVALID, "null argument");
    if (n == 0) return fail(c, GSJ_ERR_INVALID, "no rows");
    GSJ_CUDA(c, cudaSetDevice(c->device));
    GSJ_TRY(model_ensure(c));
    float *X = nullptr, *Y = nullptr, *g = nullptr;
    GSJ_TRY(model_upload(c, features, targets, n, &X, &Y));
    GSJ_TRY(dev_get(c, c->mtmp, kModelWeights + 8, reinterpret_cast<double**>(&g)));
    GSJ_CUDA(c, model_grad(X, Y, n, static_cast<const float*>(c->mw.p), g + kModelWeights, g, c->st));
    GSJ_TRY(d2h_small(c, loss, g + kModelWeights, 1));
    return d2h_small(c, grad, g, kModelWeights);
}

// ---------------------------------------------------------------- drop-in
static std::mutex g_py_mu;
static gsj_context* g_py_ctx = nullptr;
static bool g_py_pending = false;

static int py_join(const void* dataset, unsigned int N, double eps, unsigned int NDIM, int dev, uint32_t dtype,
                   unsigned int* outNum) {
    std::lock_guard<std::mutex> lk(g_py_mu);
    gsj_config cfg;
    gsj_default_config(&cfg);
    if (cfg.dim != 0 && NDIM != cfg.dim) {
        std::fprintf(stderr, "\nERROR: GPUNUMDIM=%u of this library differs from NDIM=%u\n", cfg.dim, NDIM);
        return fail(nullptr, GSJ_ERR_INVALID, "NDIM differs from the library's GPUNUMDIM");
    }
    cfg.dim = NDIM;
    cfg.dtype = dtype;
    cfg.device = dev;
    if (cfg.indexed_dims > NDIM) cfg.indexed_dims = NDIM;
    if (g_py_ctx && g_py_ctx->device != dev) {
        gsj_destroy(g_py_ctx);
        g_py_ctx = nullptr;
    }
    if (!g_py_ctx) GSJ_TRY(gsj_create(&g_py_ctx, dev));
    g_py_pending = false;
    GSJ_TRY(gsj_join(g_py_ctx, dataset, N, eps, &cfg, 0, nullptr));
    GSJ_TRY(gsj_result_counts(g_py_ctx, outNum, 0));
    g_py_pending = true;
    return GSJ_OK;
}

int GDSJoinPy_f32(const float* dataset, unsigned int N, float eps, unsigned int NDIM, int dev, unsigned int* out) {
    return py_join(dataset, N, eps, NDIM, dev, GSJ_FLOAT32, out);
}
int GDSJoinPy_f64(const double* dataset, unsigned int N, double eps, unsigned int NDIM, int dev, unsigned int* out) {
    return py_join(dataset, N, eps, NDIM, dev, GSJ_FLOAT64, out);
}

void GDSJoinPy(gsj_dtype_t* dataset, unsigned int NUMPOINTS, gsj_dtype_t epsilon, unsigned int NDIM, int gpuContext,
               unsigned int* outNumNeighborsWithinEps) {
#ifdef GSJ_DTYPE_DOUBLE
    int r = GDSJoinPy_f64(dataset, NUMPOINTS, epsilon, NDIM, gpuContext, outNumNeighborsWithinEps);
#else
    int r = GDSJoinPy_f32(dataset, NUMPOINTS, epsilon, NDIM, gpuContext, outNumNeighborsWithinEps);
#endif
    if (r != GSJ_OK) std::fprintf(stderr, "\nGDSJoinPy: %s\n", gsj_last_error(nullptr));
}

int copyResultIntoPythonArray64(unsigned int* out, uint64_t numResults) {
    std::lock_guard<std::mutex> lk(g_py_mu);
    if (!g_py_ctx || !g_py_pending) return fail(nullptr, GSJ_ERR_STATE, "no pending GDSJoinPy result");
    if (numResults > g_py_ctx->R) return fail(nullptr, GSJ_ERR_INVALID, "numResults exceeds the result size");
    int r = GSJ_OK;
    if (numResults) {
        GSJ_CUDA(g_py_ctx, cudaSetDevice(g_py_ctx->device));
        r = d2h_staged(g_py_ctx, out, g_py_ctx->table.p, numResults * 4);
    }
    g_py_pending = false;
    return r;
}

void copyResultIntoPythonArray(unsigned int* out, unsigned int numResults) {
    int r = copyResultIntoPythonArray64(out, numResults);
    if (r != GSJ_OK) std::fprintf(stderr, "\ncopyResultIntoPythonArray: %s\n", gsj_last_error(nullptr));
}

}  // extern "C"
