// Shared definitions of the B200 epsilon-grid self-join kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gsj {

constexpr int kMaxK = 10;        // indexed dimensions supported (3^10 neighbour offsets)
constexpr int kMaxIlp = 64;      // ILP register blocks supported
constexpr int kQChunk = 32;      // queries per work item (one per lane)
constexpr uint64_t kEmptyKey = ~0ull;        // hash table empty slot

// Arithmetic order of the squared-distance sum, i.e. the reference's
// ILP/SHORTCIRCUIT switches (kernel.cu:307-377):
//   kSeq    ILP==0                  s = fma(d, d, s) over l = 0..n-1
//   kIlp    ILP>0,  SHORTCIRCUIT=0  r_j = fma(d, d, r_j) for l = j (mod ILP); s = r_0 + r_1 + ...
//   kIlpSc  ILP>0,  SHORTCIRCUIT=1  per ILP block: s = fma(d_l, d_l, s); s += d_{l+j}^2 (j >= 1)
enum Model : int { kSeq = 0, kIlp = 1, kIlpSc = 2 };

// Grid geometry (k <= kMaxK indexed dims).
struct GridGeom {
    uint32_t k;
    uint32_t ncells[kMaxK];
    uint64_t mult[kMaxK];  // linear id stride of dim j (dim 0 fastest, main.cu:867-883)
};

template <typename T>
struct JoinArgs {
    const T* pts;                 // [N][npad] points in cell order, columns reordered
    const uint32_t* ids;          // [N] slot -> original point id
    const uint32_t* cell_start;   // [M+1]
    const uint64_t* cell_key;     // [M]
    const uint32_t* ds;           // [totalCells+1] slot prefix over all linear ids (dense grids), or null
    const uint2* plan;            // [M][3^(k-1)] (slot start, count) of each neighbour row (dense, k <= 3)
    const uint8_t* plan_par;      // [M] parities of the own cell coordinates (bit j = dim j)
    const uint64_t* hkeys;        // [hcap] hash table keys (kEmptyKey = empty), or null
    const uint32_t* hvals;        // [hcap] cell indices
    uint64_t hmask;               // hcap - 1
    const uint2* items;           // [num_items] (cell, chunk)
    const uint4* nbtab;           // [3^k] neighbour offsets: linear-id delta (x lo, y hi), z = moved-down dims
                                  // | moved-up dims << 16, w = highest moved dim (0xff: none)
    uint32_t num_items;
    uint32_t* work_counter;       // dynamic work distribution
    uint32_t n, npad, ilp;
    uint32_t n_points;            // N
    GridGeom g;
    T thr;                        // s <= thr  <=>  sqrt(s) <= eps
    T eps;                        // epsilon in T (cell formula)
    T minv[kMaxK];                // minArr (grid origin per indexed dim)
    // counts (ROWS path; the other paths add to cand_cnt only)
    uint32_t* fwd_cnt;            // [N] list length by slot
    unsigned long long* cand_cnt; // candidate evaluations
    // fill pass (ROWS path)
    const uint64_t* offsets;      // [N+1] by original id
    uint32_t* table;              // [R]
    unsigned long long table_cap; // R: writes at or beyond it are dropped and flagged
    uint32_t* err_flag;           // set to 1 when a write would leave the table
    // launch shape of this join (0 = the launcher's default), from the tuning table
    uint32_t shape_threads;       // ROWS count / fill CTA size (64..256, a multiple of 32)
    uint32_t shape_warps;         // WARP join: warps per CTA (1..8)
    uint32_t shape_per_sm;        // WARP, TILE, SCREEN joins: CTAs per SM at most
};

__host__ __device__ inline uint64_t mix64(uint64_t x) {
    // splitmix64 finaliser: hash of a linear cell id
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Neighbour offset `o` of a cell: usable when it stays inside the grid (no
// moved-down dim at the cell's low edge, no moved-up dim at its high edge) and,
// with unicomp, when the highest moved dim has an odd own coordinate
// (stamploops.h: `nDCellIDs[d] & 1`; the cell itself is always visited).
// Returns the neighbour's linear id in `lin`.
template <typename T, bool STAMP>
__device__ __forceinline__ bool nb_offset(const JoinArgs<T>& a, uint32_t o, uint64_t own_lin, uint32_t lowmask,
                                          uint32_t highmask, uint32_t oddmask, uint64_t& lin) {
    const uint4 e = a.nbtab[o];
    if ((e.z & 0xffffu) & lowmask) return false;
    if ((e.z >> 16) & highmask) return false;
    if (STAMP && e.w != 0xffu && !((oddmask >> e.w) & 1u)) return false;
    lin = own_lin + (((uint64_t)e.y << 32) | e.x);
    return true;
}

// Edge and parity masks of a cell's coordinates for nb_offset.
__device__ __forceinline__ void cell_masks(const uint32_t (&own)[kMaxK], const GridGeom& g, uint32_t& lowmask,
                                           uint32_t& highmask, uint32_t& oddmask) {
    lowmask = highmask = oddmask = 0u;
#pragma unroll
    for (int j = 0; j < kMaxK; j++)
        if (j < (int)g.k) {
            lowmask |= (own[j] == 0u ? 1u : 0u) << j;
            highmask |= (own[j] + 1u >= g.ncells[j] ? 1u : 0u) << j;
            oddmask |= (own[j] & 1u) << j;
        }
}

// Slot range of the cell with linear id `lin`: from the dense slot-prefix
// table (ds[lin] .. ds[lin+1]) or through the hash table of non-empty cells.
template <typename T>
__device__ __forceinline__ bool lookup_range(const JoinArgs<T>& a, uint64_t lin, uint32_t& start, uint32_t& cnt) {
    if (a.ds) {
        start = a.ds[lin];
        cnt = a.ds[lin + 1] - start;
        return cnt != 0;
    }
    uint64_t h = mix64(lin) & a.hmask;
    for (uint64_t p = 0; p <= a.hmask; p++) {
        const uint64_t kk = a.hkeys[h];
        if (kk == lin) {
            const uint32_t c = a.hvals[h];
            start = a.cell_start[c];
            cnt = a.cell_start[c + 1] - start;
            return true;
        }
        if (kk == kEmptyKey) return false;
        h = (h + 1) & a.hmask;
    }
    return false;
}

}  // namespace gsj
