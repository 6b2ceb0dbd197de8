// CPU ORACLE for the epsilon-grid distance self-join (algorithm 3 of
// mgowanlock/gpu_self_join).  TEST INFRASTRUCTURE ONLY: the product path never
// links, loads or calls this file.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py use it, and only as the checker.
//
// It restates, in plain sequential C++ (OpenMP across queries only), the
// reference's algorithm with the reference's own arithmetic:
//   * dataset statistics for REORDER ............ main.cu:981-1075
//   * grid extents ............................... main.cu:891-948
//   * cell coordinates / linear ids / index ...... main.cu:690-883
//   * per-dimension occupancy mask + range filter  kernel.cu:180-253
//   * neighbour-cell enumeration (full / unicomp)  kernel.cu:260-303, stamploops.h
//   * distance arithmetic and the sqrt(s) <= eps test  kernel.cu:307-377
//   * query work ordering (QUERYREORDER) ......... GPU.cu:1491-1525
//   * sampled batch estimator .................... GPU.cu:57-268, kernel.cu:522-694
//
// Arithmetic models (selected with orc_cfg::model):
//   MODEL_DEVICE  - the reference's CUDA code as nvcc emits it: the
//                   `s += (c-p)*(c-p)` statement is contracted into one fused
//                   multiply-add per dimension (s = fma(d, d, s)).  With ILP>0 the
//                   ILP-blocked order of kernel.cu:312-341 is followed; with
//                   ILP>0 and SHORTCIRCUIT=1 the cross-register additions are
//                   plain additions unless orc_cfg::sc_contract asks for them to
//                   be contracted as well (the two candidate code generations;
//                   the tests pin which one the reference build produces).
//   MODEL_HOST    - the reference's host code (CPU brute force main.cu:953-978,
//                   R-tree filter tree_index.cpp:202-233): no contraction.
//   MODEL_FP64    - decision taken in double precision (second oracle).
// The final test is literally sqrt(s) <= eps, as in the reference.
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

enum { MODEL_DEVICE = 0, MODEL_HOST = 1, MODEL_FP64 = 2 };

struct orc_cfg {
    uint32_t k;            // NUMINDEXEDDIM
    uint32_t reorder;      // REORDER
    uint32_t ilp;          // ILP (0 = sequential accumulation)
    uint32_t shortcircuit; // SHORTCIRCUIT
    uint32_t model;        // MODEL_*
    uint32_t sc_contract;  // alias of fold_zero = 1, fuse_left = 0 (kept for callers)
    uint32_t stamp_ref;    // 1: emit the reference's STAMP=1 output (duplicated
                           //    (q,c) pairs, kernel.cu:367-375) instead of the
                           //    symmetric neighbour lists
    uint32_t nthreads;     // OpenMP threads (0 = default)
    uint32_t fold_zero;    // device contraction policy, see DevNode
    uint32_t fuse_left;    // chains acc += d*d
    uint32_t cross_left;   // cross-register sums runningDist[0] += runningDist[j]
    uint32_t sort;         // SORT (params.h:46): per-cell sorted points, pruned scans
};

}  // extern "C"

namespace {

// ---------------------------------------------------------------- distance
template <typename T>
inline T fmaT(T a, T b, T c);
template <>
inline float fmaT<float>(float a, float b, float c) { return fmaf(a, b, c); }
template <>
inline double fmaT<double>(double a, double b, double c) { return fma(a, b, c); }

template <typename T>
inline T sqrtT(T x);
template <>
inline float sqrtT<float>(float x) { return sqrtf(x); }
template <>
inline double sqrtT<double>(double x) { return sqrt(x); }

// A value of the device-side distance expression.  The reference accumulates
// `acc += d*d` from acc = 0; how nvcc turns that source into fused
// multiply-adds depends on the precision, and is pinned against the
// reference's own builds (tests/golden/ref_pins.json):
//   * a product d*d is "pending" until it is added to something;
//   * acc + pending            -> fma(d, d, acc)              (contraction)
//   * 0 + pending              -> fma(d, d, 0) = round(d*d)   (fold_zero = 0)
//                                 or stays pending            (fold_zero = 1)
//   * pending + pending        -> fma(d_l, d_l, round(d_r*d_r)) (left)
//                                 or fma(d_r, d_r, round(d_l*d_l)) (right);
//                                 fuse_left chooses for the acc += d*d chains,
//                                 cross_left for runningDist[0] += runningDist[j]
//   * value + value            -> plain rounded addition.
template <typename T>
struct DevNode {
    T v;         // rounded value
    T d;         // the difference whose square is pending (prod only)
    bool is_prod;  // pending product d*d
    bool is_zero;  // the literal 0 the accumulators start from
    static DevNode make_zero() { return {T(0), T(0), false, true}; }
    static DevNode make_prod(T d) { return {d * d, d, true, false}; }
};

template <typename T>
DevNode<T> dev_add(const DevNode<T>& x, const DevNode<T>& y, bool fold0, bool left) {
    if (y.is_zero) return x;
    if (x.is_zero) {
        if (y.is_prod && !fold0) return {fmaT<T>(y.d, y.d, T(0)), T(0), false, false};
        return y;
    }
    if (x.is_prod && y.is_prod) {
        if (left) return {fmaT<T>(x.d, x.d, y.v), T(0), false, false};
        return {fmaT<T>(y.d, y.d, x.v), T(0), false, false};
    }
    if (y.is_prod) return {fmaT<T>(y.d, y.d, x.v), T(0), false, false};
    if (x.is_prod) return {fmaT<T>(x.d, x.d, y.v), T(0), false, false};
    return {x.v + y.v, T(0), false, false};
}

// Returns true when point c is within eps of point p under the configured model.
// p is the query ("point" in kernel.cu:307), c the candidate ("database[dataIdx]").
template <typename T>
bool within(const T* p, const T* c, uint32_t n, T eps, const orc_cfg& cfg) {
    if (cfg.model == MODEL_FP64) {
        double s = 0.0;
        for (uint32_t l = 0; l < n; l++) {
            double d = (double)c[l] - (double)p[l];
            s = s + d * d;  // -ffp-contract=off keeps this unfused
        }
        return sqrt(s) <= (double)eps;
    }
    if (cfg.model == MODEL_HOST) {
        // main.cu:963-968 / tree_index.cpp:217-224: runningDist += d*d, unfused.
        T s = 0;
        for (uint32_t l = 0; l < n; l++) {
            T d = p[l] - c[l];
            T sq = d * d;
            s = s + sq;
        }
        return sqrtT<T>(s) <= eps;
    }
    // MODEL_DEVICE: the source-level expression of kernel.cu:312-365 evaluated
    // under the compiler's contraction policy (see DevNode).
    const uint32_t ilp = cfg.ilp;
    const bool fold0 = cfg.sc_contract || cfg.fold_zero;
    const bool left = cfg.fuse_left;
    const bool xleft = cfg.cross_left;
    auto P = [&](uint32_t l) { return DevNode<T>::make_prod(c[l] - p[l]); };
    if (ilp == 0) {
        // kernel.cu:346-356: runningTotalDist += d*d
        DevNode<T> s = DevNode<T>::make_zero();
        for (uint32_t l = 0; l < n; l++) {
            s = dev_add(s, P(l), fold0, left);
            if (cfg.shortcircuit && sqrtT<T>(s.v) > eps) return false;  // kernel.cu:350-353
        }
        return sqrtT<T>(s.v) <= eps;
    }
    // kernel.cu:312-341: ILP accumulators runningDist[0..ILP-1]
    DevNode<T> r[64];
    for (uint32_t j = 0; j < ilp; j++) r[j] = DevNode<T>::make_zero();
    for (uint32_t l = 0; l < n; l += ilp) {
        for (uint32_t j = 0; j < ilp && (l + j) < n; j++) r[j] = dev_add(r[j], P(l + j), fold0, left);
        if (cfg.shortcircuit) {
            for (uint32_t j = 1; j < ilp; j++) {
                r[0] = dev_add(r[0], r[j], fold0, xleft);
                r[j] = DevNode<T>::make_zero();
            }
            if (sqrtT<T>(r[0].v) > eps) return false;  // kernel.cu:331-333
        }
    }
    for (uint32_t j = 1; j < ilp; j++) r[0] = dev_add(r[0], r[j], fold0, xleft);  // kernel.cu:337-340
    return sqrtT<T>(r[0].v) <= eps;
}

// ---------------------------------------------------------------- REORDER
// main.cu:981-1075.  Returns perm such that new column j = old column perm[j].
struct DimVar {
    unsigned int dim;
    // variance is stored in T; the struct is templated below
};

template <typename T>
struct dim_reorder_sort_T {
    unsigned int dim;
    T variance;
};

template <typename T>
bool cmp_var_desc(const dim_reorder_sort_T<T>& a, const dim_reorder_sort_T<T>& b) {
    return a.variance > b.variance;
}

template <typename T>
void reorder_perm(const T* pts, uint64_t N, uint32_t n, uint32_t* perm, T* var_out) {
    std::vector<T> sums(n, (T)0), avg(n, (T)0);
    std::vector<dim_reorder_sort_T<T>> dv(n);
    const int sample = 100;
    const T inv_sample = (T)(1.0 / (sample * 1.0));
    const T denom = (T)N * inv_sample;  // size()*inv_sample: size_t -> T, then multiply
    for (uint32_t i = 0; i < n; i++) {
        for (uint64_t j = 0; j < N; j += sample) sums[i] = sums[i] + pts[j * n + i];
        avg[i] = sums[i] / denom;
        sums[i] = 0;
        for (uint64_t j = 0; j < N; j += sample) {
            T d = pts[j * n + i] - avg[i];
            T sq = d * d;
            sums[i] = sums[i] + sq;
        }
        dv[i].variance = sums[i] / denom;
        dv[i].dim = i;
    }
    std::sort(dv.begin(), dv.end(), cmp_var_desc<T>);
    for (uint32_t j = 0; j < n; j++) {
        perm[j] = dv[j].dim;
        if (var_out) var_out[j] = dv[j].variance;
    }
}

// ---------------------------------------------------------------- grid
template <typename T>
struct Grid {
    uint32_t k;
    std::vector<T> minArr, maxArr;
    std::vector<uint32_t> nCells;
    uint64_t totalCells;
    // index (main.cu:690-857)
    std::vector<uint64_t> cellIds;    // sorted unique linear ids (gridCellLookupArr)
    std::vector<uint32_t> cellBegin;  // index[].indexmin
    std::vector<uint32_t> cellEnd;    // index[].indexmax + 1
    std::vector<uint32_t> lookup;     // indexLookupArr
    std::vector<std::vector<uint32_t>> mask;  // gridCellNDMask per dim (sorted unique)
};

template <typename T>
void grid_dims(const T* pts, uint64_t N, uint32_t n, uint32_t k, T eps, Grid<T>& g) {
    g.k = k;
    g.minArr.assign(k, 0);
    g.maxArr.assign(k, 0);
    g.nCells.assign(k, 0);
    for (uint32_t j = 0; j < k; j++) {
        g.minArr[j] = pts[j];
        g.maxArr[j] = pts[j];
    }
    for (uint64_t i = 1; i < N; i++)
        for (uint32_t j = 0; j < k; j++) {
            T v = pts[i * n + j];
            if (v < g.minArr[j]) g.minArr[j] = v;
            if (v > g.maxArr[j]) g.maxArr[j] = v;
        }
    for (uint32_t j = 0; j < k; j++) {
        g.minArr[j] = g.minArr[j] - eps;
        g.maxArr[j] = g.maxArr[j] + eps;
    }
    for (uint32_t j = 0; j < k; j++) {
        T q = (g.maxArr[j] - g.minArr[j]) / eps;
        g.nCells[j] = (uint32_t)std::ceil(q);
    }
    uint64_t t = g.nCells[0];
    for (uint32_t j = 1; j < k; j++) t *= g.nCells[j];
    g.totalCells = t;
}

template <typename T>
inline uint32_t cell_coord(T x, T mn, T eps) {
    T q = (x - mn) / eps;  // main.cu:713, kernel.cu:184
    return (uint32_t)q;
}

inline uint64_t linear_id(const uint32_t* idx, const uint32_t* dimLen, uint32_t k) {
    // main.cu:867-883 (dim 0 fastest)
    uint64_t index = 0, mult = 1;
    for (uint32_t i = 0; i < k; i++) {
        index += (uint64_t)idx[i] * mult;
        mult *= dimLen[i];
    }
    return index;
}

template <typename T>
void build_index(const T* pts, uint64_t N, uint32_t n, T eps, Grid<T>& g) {
    const uint32_t k = g.k;
    std::vector<std::pair<uint64_t, uint32_t>> kv(N);
    g.mask.assign(k, {});
    std::vector<std::vector<char>> seen(k);
    for (uint32_t j = 0; j < k; j++) seen[j].assign((size_t)g.nCells[j] + 2, 0);
    uint32_t c[64];
    for (uint64_t i = 0; i < N; i++) {
        for (uint32_t j = 0; j < k; j++) {
            c[j] = cell_coord<T>(pts[i * n + j], g.minArr[j], eps);
            if (c[j] < seen[j].size()) seen[j][c[j]] = 1;
            else g.mask[j].push_back(c[j]);  // out-of-range coordinate (degenerate input)
        }
        kv[i] = {linear_id(c, g.nCells.data(), k), (uint32_t)i};
    }
    for (uint32_t j = 0; j < k; j++) {
        for (size_t v = 0; v < seen[j].size(); v++)
            if (seen[j][v]) g.mask[j].push_back((uint32_t)v);
        std::sort(g.mask[j].begin(), g.mask[j].end());
        g.mask[j].erase(std::unique(g.mask[j].begin(), g.mask[j].end()), g.mask[j].end());
    }
    // per cell: ascending point ids (main.cu:741-763)
    std::sort(kv.begin(), kv.end());
    g.lookup.resize(N);
    g.cellIds.clear();
    g.cellBegin.clear();
    g.cellEnd.clear();
    for (uint64_t i = 0; i < N; i++) {
        g.lookup[i] = kv[i].second;
        if (i == 0 || kv[i].first != kv[i - 1].first) {
            if (i) g.cellEnd.push_back((uint32_t)i);
            g.cellIds.push_back(kv[i].first);
            g.cellBegin.push_back((uint32_t)i);
        }
    }
    if (N) g.cellEnd.push_back((uint32_t)N);
}

inline bool mask_has(const std::vector<uint32_t>& m, uint32_t v) {
    return std::binary_search(m.begin(), m.end(), v);
}

// kernel.cu:180-253: own cell coordinates and the range-filtered cell ranges.
template <typename T>
void query_ranges(const T* p, T eps, const Grid<T>& g, uint32_t* own, uint32_t* rmin, uint32_t* rmax) {
    for (uint32_t i = 0; i < g.k; i++) {
        own[i] = cell_coord<T>(p[i], g.minArr[i], eps);
        // max(0, own-1) on unsigned operands: own==0 wraps to UINT_MAX
        uint32_t lo = own[i] - 1u;
        uint32_t hi = std::min(g.nCells[i] - 1u, own[i] + 1u);
        bool fmin = mask_has(g.mask[i], lo);
        bool fmax = mask_has(g.mask[i], hi);
        if (fmin && fmax) { rmin[i] = lo; rmax[i] = hi; }
        else if (fmin) { rmin[i] = lo; rmax[i] = lo + 1u; }
        else if (fmax) { rmin[i] = lo + 1u; rmax[i] = hi; }
        else { rmin[i] = lo + 1u; rmax[i] = lo + 1u; }
    }
}

inline int64_t find_cell(const std::vector<uint64_t>& ids, uint64_t id) {
    auto it = std::lower_bound(ids.begin(), ids.end(), id);
    if (it == ids.end() || *it != id) return -1;
    return it - ids.begin();
}

// Visits every (cell, differentCell) the reference visits for one query.
// Full enumeration: kernel.cu:292-302.  Unicomp: kernel.cu:263-270 + stamploops.h.
template <typename F>
void for_each_cell(uint32_t k, const uint32_t* own, const uint32_t* rmin, const uint32_t* rmax,
                   bool stamp, F&& f) {
    uint32_t idx[64];
    if (!stamp) {
        for (uint32_t i = 0; i < k; i++) idx[i] = rmin[i];
        while (true) {
            f(idx, false);
            uint32_t d = k;  // odometer, dim k-1 innermost as in the nested loops
            while (d > 0) {
                d--;
                if (idx[d] < rmax[d]) { idx[d]++; break; }
                idx[d] = rmin[d];
                if (d == 0) return;
            }
            if (k == 0) return;
        }
    }
    for (uint32_t i = 0; i < k; i++) idx[i] = own[i];
    f(idx, false);
    for (uint32_t d = 0; d < k; d++) {
        if (!(own[d] & 1u)) continue;
        // dims 0..d range over [rmin, rmax], dim d != own, dims > d fixed at own
        for (uint32_t i = 0; i <= d; i++) idx[i] = rmin[i];
        for (uint32_t i = d + 1; i < k; i++) idx[i] = own[i];
        while (true) {
            if (idx[d] != own[d]) f(idx, true);
            uint32_t e = d + 1;
            bool done = false;
            while (true) {
                e--;
                if (idx[e] < rmax[e]) { idx[e]++; break; }
                idx[e] = rmin[e];
                if (e == 0) { done = true; break; }
            }
            if (done) break;
        }
    }
}

template <typename T>
struct Prepared {
    std::vector<T> data;  // reordered copy when REORDER, else a copy
    Grid<T> g;
};

// SORT (GPU.cu:351-395): each cell's points, in the index's order, sorted by
// their value in the sort dimension (the first non-indexed dimension, dim 0
// when every dimension is indexed) with std::sort and the reference's
// comparator (GPU.cu:51-54); the tie order is std::sort's.
template <typename T>
struct key_val_sort {
    unsigned int pid;
    T value_at_dim;
};
template <typename T>
bool compareByPointValue(const key_val_sort<T>& a, const key_val_sort<T>& b) {
    return a.value_at_dim < b.value_at_dim;
}

inline uint32_t sort_dim_of(uint32_t n, uint32_t k) { return n > k ? k : 0u; }

template <typename T>
void sort_cells(const T* D, uint32_t n, Grid<T>& g) {
    const uint32_t sd = sort_dim_of(n, g.k);
    std::vector<key_val_sort<T>> tmp;
    for (size_t c = 0; c < g.cellIds.size(); c++) {
        tmp.clear();
        for (uint32_t s = g.cellBegin[c]; s < g.cellEnd[c]; s++)
            tmp.push_back({g.lookup[s], D[(uint64_t)g.lookup[s] * n + sd]});
        std::sort(tmp.begin(), tmp.end(), compareByPointValue<T>);
        for (size_t x = 0; x < tmp.size(); x++) g.lookup[g.cellBegin[c] + x] = tmp[x].pid;
    }
}

template <typename T>
void prepare(const T* pts, uint64_t N, uint32_t n, T eps, const orc_cfg& cfg, Prepared<T>& P) {
    P.data.assign(pts, pts + N * n);
    if (cfg.reorder && N > 0) {
        std::vector<uint32_t> perm(n);
        reorder_perm<T>(pts, N, n, perm.data(), nullptr);
        for (uint64_t i = 0; i < N; i++)
            for (uint32_t j = 0; j < n; j++) P.data[i * n + j] = pts[i * n + perm[j]];
    }
    grid_dims<T>(P.data.data(), N, n, cfg.k, eps, P.g);
    build_index<T>(P.data.data(), N, n, eps, P.g);
    if (cfg.sort) sort_cells<T>(P.data.data(), n, P.g);
}

// The candidate positions of one neighbour cell under SORT (kernel.cu:400-467):
// calls f(position in the cell's sorted points) for each point the reference
// evaluates.  own0 / nb0: the query's and the cell's coordinate in dim 0.
template <typename T, typename F>
void sort_scan(const T* D, uint32_t n, uint32_t k, const std::vector<uint32_t>& lookup, uint32_t begin,
               uint32_t end, const T* p, T eps, uint32_t own0, uint32_t nb0, F&& f) {
    if (n == k) {
        // sortedDim = 0, an indexed dimension: from the side nearer the query,
        // stop at the first point farther than eps in dim 0
        const bool mid = own0 == nb0, left = own0 > nb0;
        const uint32_t len = end - begin;
        for (uint32_t kk = 0; kk < len; kk++) {
            const uint32_t pos = left ? len - 1 - kk : kk;
            const T dv = D[(uint64_t)lookup[begin + pos] * n] - p[0];
            if (std::abs(dv) > eps && !mid) break;
            f(pos);
        }
        return;
    }
    // sortedDim = NUMINDEXEDDIM: the stepping search, then the window
    const uint32_t sd = k;
    const int offset = (int)begin;
    const int length = (int)(end - begin) - 1;
    auto db = [&](int pos) { return D[(uint64_t)lookup[pos + offset] * n + sd]; };
    int searchIdx = length / 2;
    bool lessThan;
    for (int step = (length + 3) / 4; step > 1; step = (step + 1) / 2) {
        lessThan = ((p[sd] - db(searchIdx)) >= eps);
        if (lessThan) {
            searchIdx += step;
            if (searchIdx > length) searchIdx = length;
        } else {
            searchIdx -= step;
            if (searchIdx < 0) {
                searchIdx = 0;
                step = 0;
            }
        }
    }
    if (searchIdx > 0 && ((p[sd] - db(searchIdx - 1)) <= eps)) searchIdx--;
    if (searchIdx > 0 && ((p[sd] - db(searchIdx - 1)) <= eps)) searchIdx--;
    while (searchIdx <= length && ((db(searchIdx) - p[sd]) < eps)) {
        f((uint32_t)searchIdx);
        searchIdx++;
    }
}

// Runs the join.  When lists == nullptr only counts are produced.  Symmetric
// mode (stamp_ref == 0) produces, per query, the set {c : within(q, c)} over the
// cells the full enumeration visits; stamp_ref == 1 reproduces the reference's
// STAMP=1 output multiset for query q (own cell once, unicomp cells twice).
template <typename T>
int join(const T* pts, uint64_t N, uint32_t n, T eps, const orc_cfg& cfg, uint32_t* counts,
         uint64_t* total, uint64_t* cand, const uint64_t* offsets, uint32_t* lists) {
    if (cfg.k == 0 || cfg.k > n || cfg.k > 64 || cfg.ilp > 64) return -1;
    Prepared<T> P;
    if (N == 0) {
        if (total) *total = 0;
        if (cand) *cand = 0;
        return 0;
    }
    prepare<T>(pts, N, n, eps, cfg, P);
    const Grid<T>& g = P.g;
    const T* D = P.data.data();
    uint64_t tot = 0, cc = 0;
    int nth = cfg.nthreads ? (int)cfg.nthreads : 0;
#ifdef _OPENMP
    if (nth <= 0) nth = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : tot, cc) num_threads(nth)
#endif
    for (int64_t qi = 0; qi < (int64_t)N; qi++) {
        const T* p = D + (uint64_t)qi * n;
        uint32_t own[64], rmin[64], rmax[64];
        query_ranges<T>(p, eps, g, own, rmin, rmax);
        uint32_t cnt = 0;
        uint64_t lc = 0;
        uint64_t base = lists ? offsets[qi] : 0;
        auto visit = [&](const uint32_t* idx, bool diff) {
            uint64_t lid = linear_id(idx, g.nCells.data(), g.k);
            int64_t ci = find_cell(g.cellIds, lid);
            if (ci < 0) return;
            auto eval = [&](uint32_t s) {
                uint32_t c = g.lookup[s];
                lc++;
                if (within<T>(p, D + (uint64_t)c * n, n, eps, cfg)) {
                    uint32_t rep = (cfg.stamp_ref && diff) ? 2u : 1u;
                    for (uint32_t r = 0; r < rep; r++) {
                        if (lists) lists[base + cnt] = c;
                        cnt++;
                    }
                }
            };
            if (cfg.sort) {
                sort_scan<T>(D, n, g.k, g.lookup, g.cellBegin[ci], g.cellEnd[ci], p, eps, own[0], idx[0],
                             [&](uint32_t pos) { eval(g.cellBegin[ci] + pos); });
            } else {
                for (uint32_t s = g.cellBegin[ci]; s < g.cellEnd[ci]; s++) eval(s);
            }
        };
        for_each_cell(g.k, own, rmin, rmax, cfg.stamp_ref != 0, visit);
        if (counts) counts[qi] = cnt;
        if (lists) std::sort(lists + base, lists + base + cnt);
        tot += cnt;
        cc += lc;
    }
    if (total) *total = tot;
    if (cand) *cand = cc;
    return 0;
}

template <typename T>
int bruteforce(const T* pts, uint64_t N, uint32_t n, T eps, const orc_cfg& cfg, uint32_t* counts,
               uint64_t* total) {
    std::vector<T> data(pts, pts + N * n);
    if (cfg.reorder && N > 0) {
        std::vector<uint32_t> perm(n);
        reorder_perm<T>(pts, N, n, perm.data(), nullptr);
        for (uint64_t i = 0; i < N; i++)
            for (uint32_t j = 0; j < n; j++) data[i * n + j] = pts[i * n + perm[j]];
    }
    uint64_t tot = 0;
    int nth = cfg.nthreads ? (int)cfg.nthreads : 0;
#ifdef _OPENMP
    if (nth <= 0) nth = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tot) num_threads(nth)
#endif
    for (int64_t i = 0; i < (int64_t)N; i++) {
        uint32_t cnt = 0;
        for (uint64_t j = 0; j < N; j++)
            if (within<T>(&data[i * n], &data[j * n], n, eps, cfg)) cnt++;
        if (counts) counts[i] = cnt;
        tot += cnt;
    }
    if (total) *total = tot;
    return 0;
}

// ---------------------------------------------------------------- QUERYREORDER
// GPU.cu:1491-1525
struct workArray {
    unsigned int queryPntID;
    unsigned long int pntsInCell;
};
bool cmp_work_desc(const workArray& a, const workArray& b) { return a.pntsInCell > b.pntsInCell; }

template <typename T>
void query_order(const Grid<T>& g, std::vector<uint32_t>& out) {
    std::vector<workArray> w;
    w.reserve(g.lookup.size());
    for (size_t i = 0; i < g.cellIds.size(); i++) {
        unsigned long np = g.cellEnd[i] - g.cellBegin[i];
        for (uint32_t j = g.cellBegin[i]; j < g.cellEnd[i]; j++) w.push_back({g.lookup[j], np});
    }
    std::sort(w.begin(), w.end(), cmp_work_desc);
    out.resize(w.size());
    for (size_t i = 0; i < w.size(); i++) out[i] = w[i].queryPntID;
}

}  // namespace

extern "C" {

int orc_reorder_perm_f32(const float* p, uint64_t N, uint32_t n, uint32_t* perm, float* var) {
    reorder_perm<float>(p, N, n, perm, var);
    return 0;
}
int orc_reorder_perm_f64(const double* p, uint64_t N, uint32_t n, uint32_t* perm, double* var) {
    reorder_perm<double>(p, N, n, perm, var);
    return 0;
}

int orc_grid_dims_f32(const float* p, uint64_t N, uint32_t n, uint32_t k, float eps, float* mn,
                      float* mx, uint32_t* nc, uint64_t* tot) {
    Grid<float> g;
    grid_dims<float>(p, N, n, k, eps, g);
    for (uint32_t j = 0; j < k; j++) { mn[j] = g.minArr[j]; mx[j] = g.maxArr[j]; nc[j] = g.nCells[j]; }
    *tot = g.totalCells;
    return 0;
}
int orc_grid_dims_f64(const double* p, uint64_t N, uint32_t n, uint32_t k, double eps, double* mn,
                      double* mx, uint32_t* nc, uint64_t* tot) {
    Grid<double> g;
    grid_dims<double>(p, N, n, k, eps, g);
    for (uint32_t j = 0; j < k; j++) { mn[j] = g.minArr[j]; mx[j] = g.maxArr[j]; nc[j] = g.nCells[j]; }
    *tot = g.totalCells;
    return 0;
}

int orc_join_counts_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                        uint32_t* counts, uint64_t* total, uint64_t* cand) {
    return join<float>(p, N, n, eps, *cfg, counts, total, cand, nullptr, nullptr);
}
int orc_join_counts_f64(const double* p, uint64_t N, uint32_t n, double eps, const orc_cfg* cfg,
                        uint32_t* counts, uint64_t* total, uint64_t* cand) {
    return join<double>(p, N, n, eps, *cfg, counts, total, cand, nullptr, nullptr);
}
// offsets: N+1 exclusive prefix of the counts from orc_join_counts_*; lists
// receives each point's neighbour ids sorted ascending.
int orc_join_lists_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                       const uint64_t* offsets, uint32_t* lists) {
    return join<float>(p, N, n, eps, *cfg, nullptr, nullptr, nullptr, offsets, lists);
}
int orc_join_lists_f64(const double* p, uint64_t N, uint32_t n, double eps, const orc_cfg* cfg,
                       const uint64_t* offsets, uint32_t* lists) {
    return join<double>(p, N, n, eps, *cfg, nullptr, nullptr, nullptr, offsets, lists);
}

int orc_bruteforce_counts_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                              uint32_t* counts, uint64_t* total) {
    return bruteforce<float>(p, N, n, eps, *cfg, counts, total);
}
int orc_bruteforce_counts_f64(const double* p, uint64_t N, uint32_t n, double eps,
                              const orc_cfg* cfg, uint32_t* counts, uint64_t* total) {
    return bruteforce<double>(p, N, n, eps, *cfg, counts, total);
}

// Distance decision for one pair (test helper).
int orc_within_f32(const float* p, const float* c, uint32_t n, float eps, const orc_cfg* cfg) {
    return within<float>(p, c, n, eps, *cfg) ? 1 : 0;
}
int orc_within_f64(const double* p, const double* c, uint32_t n, double eps, const orc_cfg* cfg) {
    return within<double>(p, c, n, eps, *cfg) ? 1 : 0;
}

// The reference's sampled batch plan (GPU.cu:57-268) for the given per-query
// output counts (the reference's own per-query counts: with STAMP=1 these are
// the duplicated-multiset counts).  Reports the estimate, number of batches,
// per-stream buffer size and the largest per-batch result count, so that a
// caller can check that the reference's unguarded result buffers
// (kernel.cu:367-375) cannot overflow before it runs the reference build.
// query_reorder selects QUERYREORDER; alpha is 0.05 (CLI) or 0.10 (library).
int orc_ref_batch_plan_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                           const uint32_t* ref_counts, const uint32_t* sample_counts,
                           uint32_t query_reorder, double alpha, uint64_t* est_out,
                           uint32_t* num_batches, uint32_t* buffer_size, uint64_t* max_batch) {
    Prepared<float> P;
    prepare<float>(p, N, n, eps, *cfg, P);
    std::vector<uint32_t> order;
    if (query_reorder) query_order<float>(P.g, order);
    else { order.resize(N); for (uint64_t i = 0; i < N; i++) order[i] = (uint32_t)i; }
    const double sampleRate = 0.015;
    const int offsetRate = (int)(1.0 / sampleRate);
    uint32_t nSample = (uint32_t)(N * sampleRate);
    uint64_t sampleCnt = 0;
    for (uint32_t t = 0; t < nSample; t++) sampleCnt += sample_counts[order[(uint64_t)t * offsetRate]];
    uint64_t est = (uint64_t)(uint32_t)sampleCnt * (uint64_t)offsetRate;
    unsigned int GPUBufferSize = 100000000u;
    const unsigned GPUSTREAMS = 3, MINBATCHES = 3;
    if (est < (uint64_t)GPUBufferSize * GPUSTREAMS)
        GPUBufferSize = (unsigned int)(est * (1.0 + (alpha * 3.0)) / (GPUSTREAMS));
    unsigned int numBatches = (unsigned int)ceil(((1.0 + alpha) * est * 1.0) / ((uint64_t)GPUBufferSize * 1.0));
    if (numBatches < MINBATCHES) {
        GPUBufferSize = (unsigned int)(GPUBufferSize * ((numBatches * 1.0) / (MINBATCHES * 1.0)));
        numBatches = MINBATCHES;
    }
    uint64_t mx = 0;
    uint32_t batchSize = (uint32_t)(N / numBatches);
    uint32_t extra = (uint32_t)(N - (uint64_t)batchSize * numBatches);
    for (uint32_t b = 0; b < numBatches; b++) {
        uint32_t nb = b < extra ? batchSize + 1 : batchSize;
        uint64_t s = 0;
        for (uint32_t t = 0; t < nb; t++) s += ref_counts[order[(uint64_t)t * numBatches + b]];
        mx = std::max(mx, s);
    }
    *est_out = est;
    *num_batches = numBatches;
    *buffer_size = GPUBufferSize;
    *max_batch = mx;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- import
// import_dataset.cpp:49-95: split on ',' then stream-extract values; the flat
// vector is cut into n-tuples (a trailing partial tuple is dropped).
#include <fstream>
#include <sstream>
#include <string>
namespace {
template <typename T>
int64_t import_text(const char* fname, uint32_t n, T* out, uint64_t cap) {
    std::vector<T> all;
    std::ifstream in(fname);
    if (!in) return -1;
    for (std::string f; std::getline(in, f, ',');) {
        T v;
        std::stringstream ss(f);
        while (ss >> v) {
            all.push_back(v);
            if (ss.peek() == ',') ss.ignore();
        }
    }
    uint64_t pts = n ? all.size() / n : 0;
    if (out) {
        if (pts * n > cap) return -2;
        std::copy(all.begin(), all.begin() + pts * n, out);
    }
    return (int64_t)pts;
}
}  // namespace
extern "C" {
// Returns the number of points (or <0 on error); out may be null to query size.
int64_t orc_import_text_f32(const char* f, uint32_t n, float* out, uint64_t cap) { return import_text<float>(f, n, out, cap); }
int64_t orc_import_text_f64(const char* f, uint32_t n, double* out, uint64_t cap) { return import_text<double>(f, n, out, cap); }
}

// ---------------------------------------------------------------- CPU timing
// The oracle's grid join on a query sample (the cpu_baseline leg of bench.py):
// index over all N points, then the listed queries only.  Returns the pair
// count of the sample and the wall times of both phases.
#include <chrono>
namespace {
template <typename T>
int join_sample(const T* pts, uint64_t N, uint32_t n, T eps, const orc_cfg& cfg, const uint32_t* q, uint64_t nq,
                uint64_t* total, double* sec_index, double* sec_query) {
    using clk = std::chrono::steady_clock;
    auto t0 = clk::now();
    Prepared<T> P;
    prepare<T>(pts, N, n, eps, cfg, P);
    auto t1 = clk::now();
    const Grid<T>& g = P.g;
    const T* D = P.data.data();
    uint64_t tot = 0;
    int nth = cfg.nthreads ? (int)cfg.nthreads : 0;
#ifdef _OPENMP
    if (nth <= 0) nth = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tot) num_threads(nth)
#endif
    for (int64_t i = 0; i < (int64_t)nq; i++) {
        const T* p = D + (uint64_t)q[i] * n;
        uint32_t own[64], rmin[64], rmax[64];
        query_ranges<T>(p, eps, g, own, rmin, rmax);
        uint64_t cnt = 0;
        auto visit = [&](const uint32_t* idx, bool) {
            int64_t ci = find_cell(g.cellIds, linear_id(idx, g.nCells.data(), g.k));
            if (ci < 0) return;
            for (uint32_t s = g.cellBegin[ci]; s < g.cellEnd[ci]; s++)
                if (within<T>(p, D + (uint64_t)g.lookup[s] * n, n, eps, cfg)) cnt++;
        };
        for_each_cell(g.k, own, rmin, rmax, false, visit);
        tot += cnt;
    }
    auto t2 = clk::now();
    *total = tot;
    *sec_index = std::chrono::duration<double>(t1 - t0).count();
    *sec_query = std::chrono::duration<double>(t2 - t1).count();
    return 0;
}
}  // namespace
extern "C" int orc_join_sample_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                                   const uint32_t* q, uint64_t nq, uint64_t* total, double* si, double* sq) {
    return join_sample<float>(p, N, n, eps, *cfg, q, nq, total, si, sq);
}

// ---------------------------------------------------------------- sample lists
// Sorted neighbour lists of a query sample (the full-size workloads' parity
// tests): the index over all N points, then the full enumeration of `join`
// (kernel.cu:292-302) for the listed queries only.  counts[i] receives query
// q[i]'s list length and *total their sum; when *total <= cap the lists are
// written to `lists`, query after query, each ascending.  The model may be
// any of the decision models (MODEL_FP64 for the double-precision decision).
namespace {
template <typename T>
int sample_lists(const T* pts, uint64_t N, uint32_t n, T eps, const orc_cfg& cfg, const uint32_t* q, uint64_t nq,
                 uint32_t* counts, uint32_t* lists, uint64_t cap, uint64_t* total) {
    if (cfg.k == 0 || cfg.k > n || cfg.k > 64 || cfg.ilp > 64) return -1;
    for (uint64_t i = 0; i < nq; i++)
        if (q[i] >= N) return -2;
    Prepared<T> P;
    prepare<T>(pts, N, n, eps, cfg, P);
    const Grid<T>& g = P.g;
    const T* D = P.data.data();
    std::vector<std::vector<uint32_t>> out(nq);
    int nth = cfg.nthreads ? (int)cfg.nthreads : 0;
#ifdef _OPENMP
    if (nth <= 0) nth = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
#endif
    for (int64_t i = 0; i < (int64_t)nq; i++) {
        const T* p = D + (uint64_t)q[i] * n;
        uint32_t own[64], rmin[64], rmax[64];
        query_ranges<T>(p, eps, g, own, rmin, rmax);
        std::vector<uint32_t>& v = out[i];
        auto visit = [&](const uint32_t* idx, bool) {
            int64_t ci = find_cell(g.cellIds, linear_id(idx, g.nCells.data(), g.k));
            if (ci < 0) return;
            auto eval = [&](uint32_t s) {
                if (within<T>(p, D + (uint64_t)g.lookup[s] * n, n, eps, cfg)) v.push_back(g.lookup[s]);
            };
            if (cfg.sort)
                sort_scan<T>(D, n, g.k, g.lookup, g.cellBegin[ci], g.cellEnd[ci], p, eps, own[0], idx[0],
                             [&](uint32_t pos) { eval(g.cellBegin[ci] + pos); });
            else
                for (uint32_t s = g.cellBegin[ci]; s < g.cellEnd[ci]; s++) eval(s);
        };
        for_each_cell(g.k, own, rmin, rmax, false, visit);
        std::sort(v.begin(), v.end());
    }
    uint64_t tot = 0;
    for (uint64_t i = 0; i < nq; i++) {
        counts[i] = (uint32_t)out[i].size();
        tot += out[i].size();
    }
    *total = tot;
    if (lists && tot <= cap) {
        uint64_t o = 0;
        for (uint64_t i = 0; i < nq; i++) {
            std::copy(out[i].begin(), out[i].end(), lists + o);
            o += out[i].size();
        }
    }
    return 0;
}
}  // namespace
extern "C" int orc_sample_lists_f32(const float* p, uint64_t N, uint32_t n, float eps, const orc_cfg* cfg,
                                    const uint32_t* q, uint64_t nq, uint32_t* counts, uint32_t* lists, uint64_t cap,
                                    uint64_t* total) {
    return sample_lists<float>(p, N, n, eps, *cfg, q, nq, counts, lists, cap, total);
}
extern "C" int orc_sample_lists_f64(const double* p, uint64_t N, uint32_t n, double eps, const orc_cfg* cfg,
                                    const uint32_t* q, uint64_t nq, uint32_t* counts, uint32_t* lists, uint64_t cap,
                                    uint64_t* total) {
    return sample_lists<double>(p, N, n, eps, *cfg, q, nq, counts, lists, cap, total);
}
