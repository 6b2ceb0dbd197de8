// Host-side launchers of the self-join kernels (internal interface between
// gsj_api.cu and the kernel translation units).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"

namespace gsj {

// Resident CTAs per SM for a launch: the larger of the occupancy calculation
// and the same fit computed from the SM's limits (shared memory with the
// per-block reservation, registers in 256-register warp units, threads),
// since the calculation can come out below what the SM holds.  Results are
// cached per (device, kernel, block size, dynamic shared memory).
cudaError_t blocks_per_sm(const void* kern, int threads, size_t smem, int* per_sm);

constexpr unsigned kVarStageBytes = 98304;  // shared staging of sampled rows (REORDER statistic)

template <typename T>
cudaError_t launch_variance(const T* in, uint64_t N, uint32_t n, T denom, T* var_out, cudaStream_t st);
template <typename T>
cudaError_t launch_minmax(const T* in, uint64_t N, uint32_t n, uint32_t k, const uint32_t* perm, T* part,
                          uint32_t nparts, T* out, cudaStream_t st);
// Cell key per point (K = uint32_t when the grid has fewer than 2^32 cells)
// and the point ids 0..N-1.  *bad (zeroed by the caller) is raised when a
// point's cell index reaches its dimension's extent.
template <typename T, typename K>
cudaError_t launch_cell_keys(const T* in, uint64_t N, uint32_t n, const uint32_t* perm, const GridGeom& g,
                             const T* minArr, T eps, K* keys, uint32_t* vals, uint32_t* bad, cudaStream_t st);
template <typename T>
cudaError_t launch_gather_points(const T* in, uint64_t N, uint32_t n, uint32_t npad, const uint32_t* perm,
                                 const uint32_t* ids, T* pts, cudaStream_t st);
// Either the dense per-linear-id point counts (dcnt[key] = size, to be
// scanned into the slot-prefix table) or the hash table of the non-empty cells.
cudaError_t launch_cell_tables(const uint64_t* cell_key, const uint32_t* cell_start, uint32_t M, uint32_t* dcnt,
                               unsigned long long* hkeys, uint32_t* hvals, uint64_t hmask, cudaStream_t st);
cudaError_t launch_cell_plan(const uint64_t* cell_key, uint32_t M, const GridGeom& g, const uint32_t* ds,
                             uint2* plan, uint8_t* par, cudaStream_t st);
cudaError_t launch_item_counts(const uint32_t* cell_start, const uint32_t* order, uint32_t M, uint32_t qchunk,
                               uint32_t* nchunks, uint32_t* sizes, cudaStream_t st);
cudaError_t launch_make_items(const uint32_t* order, const uint32_t* nchunks, const uint32_t* item_off,
                              uint32_t M, uint2* items, cudaStream_t st);
cudaError_t launch_iota(uint32_t* out, uint32_t M, cudaStream_t st);

// The warp-per-item join: appends packed pair keys into `o` (its rechecks
// counter receives the exact number of keys; with o.emit false only that
// count is taken) and visits items 0, o.stride, ..., (nvisit - 1) * o.stride.
// `model` is one of Model; `stamp` selects the unicomp traversal; `rows` the
// dense low-dimensional specialisation (k <= 3, a.ds set).  The launcher picks
// the specialisation.
struct TileOut;
template <typename T>
cudaError_t launch_join_emit(const JoinArgs<T>& a, const TileOut& o, uint32_t nvisit, int model, bool stamp, bool rows,
                             int num_sms, cudaStream_t st);

// ROWS path: dense low-dimensional grids (k <= 3, n <= 4), full neighbourhood.
// slot_cell[s] = cell of slot s; with swords non-null also the bit-mask words
// of slot s's query (ceil(candidates / 32); plan rows nrows per cell).
cudaError_t launch_slot_cell(const uint32_t* cell_start, uint32_t M, const uint2* plan, uint32_t nrows,
                             uint32_t* slot_cell, uint32_t* swords, cudaStream_t st);
template <typename T>
bool tpq_supported(const JoinArgs<T>& a);
// Count pass (a.work_counter zeroed): a.fwd_cnt[s] and counts_by_id[ids[s]]
// receive the list lengths, bits[bitoff[s] ...] the query's hit mask.
template <typename T>
cudaError_t launch_rows_count(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff, uint32_t* bits,
                              uint32_t* counts_by_id, int num_sms, cudaStream_t st);
// Fill pass (a.work_counter zeroed, a.offsets/table/table_cap/err_flag set):
// replays the hit masks of the queries at slots qslots[0 .. nq) (slots
// 0 .. nq-1 when qslots is null) into the point-id-ordered table; the list of
// point id i lands at a.table[offsets[i] - base].
template <typename T>
cudaError_t launch_rows_fill(const JoinArgs<T>& a, const uint32_t* slot_cell, const uint64_t* bitoff,
                             const uint32_t* bits, const uint32_t* qslots, uint32_t nq, uint64_t base, int num_sms,
                             cudaStream_t st);
// Result batches by point-id range: bound[0..nb] (ids) and boff[0..nb] (their
// table offsets), each batch's lists at most `step` + the longest list
// entries; per-slot batch keys (with the slot index as value, for a stable
// sort by batch); the start of each batch in the sorted slot list.
cudaError_t launch_batch_bounds(const uint64_t* offsets, uint32_t N, uint64_t step, uint32_t nb, uint32_t* bound,
                                unsigned long long* boff, cudaStream_t st);
cudaError_t launch_slot_batch(const uint32_t* ids, uint32_t N, const uint32_t* bound, uint32_t nb, uint32_t* bkey,
                              uint32_t* slot, cudaStream_t st);
cudaError_t launch_group_starts(const uint32_t* sorted_bkey, uint32_t N, uint32_t nb, uint32_t* gstart,
                                cudaStream_t st);
// *out = max of in[0 .. n) (*out zeroed by the caller).
cudaError_t launch_max_u32(const uint32_t* in, uint64_t n, uint32_t* out, cudaStream_t st);

// SORT variant (gsj_join_sort.cu): a count pass (fill == false: list lengths
// into counts_by_id, candidates into a.cand_cnt) and a fill pass (a.offsets,
// a.table, a.err_flag set) of the reference's pruned per-cell scans; the
// points of each cell must be in sort-dimension order.  `model` is one of Model.
template <typename T>
cudaError_t launch_sort_join(const JoinArgs<T>& a, const uint32_t* slot_cell, uint32_t* counts_by_id, int model,
                             bool fill, int num_sms, cudaStream_t st);
// out[s] = in[ids[s] * n + col]: the sort dimension's values in slot order.
template <typename T>
cudaError_t launch_sort_values(const T* in, uint64_t N, uint32_t n, uint32_t col, const uint32_t* ids, T* out,
                               cudaStream_t st);

// Tile join of high-dimensional float data (5 <= n <= kTileMaxN, k <= 6):
// a CTA per item of up to kTileQ query slots; hits become packed
// (query id << shift | candidate id) keys in a pair buffer.
constexpr int kTileQ = 64;            // queries per tile-join work item
constexpr uint32_t kTileMaxN = 128;   // dimensions held in shared memory
struct TileOut {
    unsigned long long* pairs;    // [cap] packed pairs
    unsigned long long cap;       // pairs beyond cap are counted, not written
    unsigned long long* cursor;   // pairs found so far (zeroed by the caller)
    uint32_t shift;               // bits of a point id
    uint32_t stride;              // items visited: 0, stride, 2*stride, ...
    bool emit;                    // false: count only (the sampling pass)
    unsigned long long* rechecks; // screened join: pairs sent to the exact check
};
bool tile_supported(uint32_t n, uint32_t npad, uint32_t k, int model, uint32_t ilp);
// Visits items 0, stride, ..., (nvisit-1)*stride; a.work_counter must be zero.
cudaError_t launch_tile_join(const JoinArgs<float>& a, const TileOut& o, bool stamp, int model, uint32_t nvisit,
                             int num_sms, cudaStream_t st);
// Sorted packed pairs -> table (low bits) and counts[query] += pairs (counts zeroed by the caller).
cudaError_t launch_pairs_to_table(const unsigned long long* keys, uint64_t R, uint32_t shift, uint32_t* table,
                                  uint32_t* counts, int num_sms, cudaStream_t st);

// Tensor-core screened tile join (gsj_join_screen.cu): BF16 tcgen05 dot
// products with a proven rejection bound, exact FP32 check of the rest.
constexpr int kScreenQ = 128;         // queries per screened work item (MMA M)
struct ScreenConst {
    float r0;             // >= sqrt(thr) with the reference sum's rounding room
    float ke;             // BF16 rounding bound per unit norm
    float c1;             // FP32 accumulation bound per unit squared norm
    uint32_t kpad;        // dimensions + 2 padded to the MMA K step (16)
    const uint4* rows;    // [N][kpad/8] centred BF16 rows [c^, |c^|^2_hi, |c^|^2_lo, 0...], slot order
    const float* norms;   // [N] |c^|^2 (FP32 sum of the BF16 squares)
};
// Centred BF16 rows and norms of all points (slot order) for the screen:
// centre = per-dimension mean of the finite values (deterministic two-level
// FP64 sum); `partial` holds kScreenPrepBlocks x n x 2 doubles, `centre` n floats.
constexpr uint32_t kScreenPrepBlocks = 256;
cudaError_t launch_screen_prep(const float* pts, uint32_t N, uint32_t n, uint32_t npad, uint32_t kpad,
                               double* partial, float* centre, uint4* rows, float* norms, cudaStream_t st);
bool screen_supported(uint32_t n, uint32_t npad, uint32_t k, int model, uint32_t ilp, float thr);
ScreenConst make_screen_const(uint32_t n, float thr);
// Screen pass: the undecided pairs, packed as (query slot | cross << 31) << 32
// | candidate slot, go to o.pairs in blocks of kScreenBlockSlack entries that
// consumer warps reserve on o.cursor; a warp abandons its block when its next
// chunk (up to 512 pairs) does not fit, padding the tail with kUndecidedPad,
// so up to 511 entries of every block and most of each warp's last block can
// stay unused; o.rechecks receives the exact number of undecided pairs.
constexpr unsigned long long kUndecidedPad = ~0ull;
constexpr uint64_t kScreenBlockSlack = 1024;
cudaError_t launch_tile_screen(const JoinArgs<float>& a, const TileOut& o, const ScreenConst& sc, bool stamp,
                               int model, uint32_t nvisit, int num_sms, cudaStream_t st);
// Exact check of the undecided pairs; hits go to o as packed (query id, candidate id) keys.
cudaError_t launch_screen_recheck(const JoinArgs<float>& a, const unsigned long long* unc, unsigned long long nunc,
                                  const TileOut& o, bool stamp, int model, int num_sms, cudaStream_t st);

// Brute-force neighbour counts over all N^2 pairs (the reference's algorithm
// 1, kernel.cu:486-515) with the sequential model: counts[q] and the total.
template <typename T>
cudaError_t launch_bruteforce(const T* pts, uint32_t N, uint32_t n, T thr, uint32_t* counts,
                              unsigned long long* total, cudaStream_t st);

}  // namespace gsj
