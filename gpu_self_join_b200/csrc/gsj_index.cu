// Grid index construction on the device (subsystem (a)).
//
// Replaces the reference's host-side index build, which is restated here with
// the same arithmetic so that every point lands in the same cell:
//   ReorderByDimension        main.cu:981-1075   (variance statistic: k_variance)
//   generateNDGridDimensions  main.cu:891-948    (k_minmax_*; the scalar tail runs on the host)
//   populateNDGridIndexAndLookupArray + getLinearID_nDimensions
//                             main.cu:690-883    (k_cell_keys -> radix sort -> runs -> lookup)
//   computeWorkDifficulty     GPU.cu:1491-1525   (k_item_* work items, heavy cells first)
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

#include "gsj_common.cuh"
#include "gsj_fp.cuh"
#include "gsj_kernels.h"

namespace gsj {

// ------------------------------------------------------------ REORDER statistic
// One block.  Thread i owns dimension i and adds the sampled values in the
// reference's sequential order (rows 0, 100, 200, ...), unfused, in T.  The
// sampled rows are staged through shared memory in chunks by the whole block
// (up to 1024 threads, many loads in flight) so that the sequential chains run
// on on-chip data.
template <typename T>
__global__ void k_variance(const T* __restrict__ in, uint64_t N, uint32_t n, T denom,
                           T* __restrict__ var_out) {
    extern __shared__ unsigned char smem_raw[];
    T* stage = reinterpret_cast<T*>(smem_raw);
    const uint32_t chunk = (uint32_t)(kVarStageBytes / sizeof(T)) / n;  // samples per chunk
    const uint64_t nsamp = (N + 99) / 100;
    for (uint32_t d0 = 0; d0 < n; d0 += blockDim.x) {
        const uint32_t d = d0 + threadIdx.x;
        T sum = 0, avg = 0, ssq = 0;
        for (int pass = 0; pass < 2; pass++) {
            for (uint64_t s0 = 0; s0 < nsamp; s0 += chunk) {
                const uint32_t cs = (uint32_t)((nsamp - s0) < chunk ? (nsamp - s0) : chunk);
                __syncthreads();
                for (uint32_t e = threadIdx.x; e < cs * n; e += blockDim.x) {
                    const uint32_t s = e / n, c = e - s * n;
                    stage[e] = in[(s0 + s) * 100ull * n + c];
                }
                __syncthreads();
                if (d < n) {
                    if (pass == 0) {
                        for (uint32_t s = 0; s < cs; s++) sum = FP<T>::add(sum, stage[s * n + d]);
                    } else {
                        for (uint32_t s = 0; s < cs; s++) {
                            const T dv = FP<T>::sub(stage[s * n + d], avg);
                            ssq = FP<T>::add(ssq, FP<T>::mul(dv, dv));
                        }
                    }
                }
            }
            if (pass == 0) avg = FP<T>::div(sum, denom);
        }
        if (d < n) var_out[d] = FP<T>::div(ssq, denom);
    }
}

// ------------------------------------------------------------ grid extents
// Per indexed dim j (input column perm[j]): min/max with the reference's
// sequential semantics (start from point 0, replace on strict < / >), so NaN
// values other than point 0's are skipped exactly as main.cu:906-916 skips them.
template <typename T>
__global__ void k_minmax_partial(const T* __restrict__ in, uint64_t N, uint32_t n, uint32_t k,
                                 const uint32_t* __restrict__ perm, T* __restrict__ part) {
    __shared__ T smin[kMaxK][32], smax[kMaxK][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T mn[kMaxK], mx[kMaxK];
    uint32_t col[kMaxK];
#pragma unroll
    for (int j = 0; j < kMaxK; j++)
        if (j < (int)k) {
            col[j] = perm[j];
            mn[j] = mx[j] = in[col[j]];
        }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    // four points per round, their loads issued together
    for (; i + 3u * stride < N; i += 4u * stride) {
#pragma unroll
        for (int j = 0; j < kMaxK; j++)
            if (j < (int)k) {
                T v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) v[u] = in[(i + (uint64_t)u * stride) * n + col[j]];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (v[u] < mn[j]) mn[j] = v[u];
                    if (v[u] > mx[j]) mx[j] = v[u];
                }
            }
    }
    for (; i < N; i += stride) {
#pragma unroll
        for (int j = 0; j < kMaxK; j++)
            if (j < (int)k) {
                const T v = in[i * n + col[j]];
                if (v < mn[j]) mn[j] = v;
                if (v > mx[j]) mx[j] = v;
            }
    }
#pragma unroll
    for (int j = 0; j < kMaxK; j++)
        if (j < (int)k) {
            for (int o = 16; o > 0; o >>= 1) {
                const T a = __shfl_down_sync(0xffffffffu, mn[j], o);
                const T b = __shfl_down_sync(0xffffffffu, mx[j], o);
                if (a < mn[j]) mn[j] = a;
                if (b > mx[j]) mx[j] = b;
            }
            if (lane == 0) { smin[j][warp] = mn[j]; smax[j][warp] = mx[j]; }
        }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        for (int j = 0; j < (int)k; j++) {
            T a = lane < nw ? smin[j][lane] : smin[j][0];
            T b = lane < nw ? smax[j][lane] : smax[j][0];
            for (int o = 16; o > 0; o >>= 1) {
                const T a2 = __shfl_down_sync(0xffffffffu, a, o);
                const T b2 = __shfl_down_sync(0xffffffffu, b, o);
                if (a2 < a) a = a2;
                if (b2 > b) b = b2;
            }
            if (lane == 0) {
                part[(size_t)blockIdx.x * 2 * k + j] = a;
                part[(size_t)blockIdx.x * 2 * k + k + j] = b;
            }
        }
    }
}

// Warp j reduces dim j's partials (every partial starts from point 0's value,
// so the strict comparisons keep the sequential semantics in any order).
template <typename T>
__global__ void k_minmax_final(const T* __restrict__ part, uint32_t nparts, uint32_t k,
                               T* __restrict__ out) {
    const uint32_t j = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (j >= k) return;
    T a = part[j], b = part[k + j];
    for (uint32_t p = lane; p < nparts; p += 32u) {
        const T a2 = part[(size_t)p * 2 * k + j], b2 = part[(size_t)p * 2 * k + k + j];
        if (a2 < a) a = a2;
        if (b2 > b) b = b2;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const T a2 = __shfl_down_sync(0xffffffffu, a, o);
        const T b2 = __shfl_down_sync(0xffffffffu, b, o);
        if (a2 < a) a = a2;
        if (b2 > b) b = b2;
    }
    if (lane == 0) {
        out[j] = a;
        out[k + j] = b;
    }
}

// ------------------------------------------------------------ cell keys
// Cell coordinate (x - minArr)/eps truncated to unsigned (main.cu:713,744 and
// kernel.cu:184 compute it identically), linear id with dim 0 fastest.
// Linear cell id of point i (dim 0 fastest); a coordinate whose index
// reaches the grid's extent (eps below the data's resolution, so that the
// rounded max + eps equals max) raises *bad and counts as cell 0.
template <typename T>
__device__ __forceinline__ uint64_t cell_key_of(const T* __restrict__ in, uint64_t i, uint32_t n,
                                                const uint32_t* __restrict__ perm, const GridGeom& g,
                                                const T* __restrict__ minArr, T eps, uint32_t* bad) {
    uint64_t key = 0;
    bool out = false;
#pragma unroll
    for (int j = 0; j < kMaxK; j++)
        if (j < (int)g.k) {
            const T x = in[i * n + perm[j]];
            const uint32_t c = FP<T>::to_uint_rz(FP<T>::div(FP<T>::sub(x, minArr[j]), eps));
            out |= c >= g.ncells[j];
            key += (uint64_t)c * g.mult[j];
        }
    if (out) {
        *bad = 1u;
        key = 0;
    }
    return key;
}

template <typename T, typename K>
__global__ void k_cell_keys(const T* __restrict__ in, uint64_t N, uint32_t n, const uint32_t* __restrict__ perm,
                            GridGeom g, const T* __restrict__ minArr, T eps,
                            K* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* __restrict__ bad) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    keys[i] = (K)cell_key_of<T>(in, i, n, perm, g, minArr, eps, bad);
    vals[i] = (uint32_t)i;
}

// Points in cell order with reordered, zero-padded columns: pts[s][j] = in[ids[s]][perm[j]].
template <typename T>
__global__ void k_gather_points(const T* __restrict__ in, uint64_t N, uint32_t n, uint32_t npad,
                                const uint32_t* __restrict__ perm, const uint32_t* __restrict__ ids,
                                T* __restrict__ pts) {
    const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (e >= N * npad) return;
    const uint64_t s = e / npad;
    const uint32_t j = (uint32_t)(e - s * npad);
    pts[e] = j < n ? in[(uint64_t)ids[s] * n + perm[j]] : T(0);
}

// The same for rows of npad = NP <= 4 entries: a thread per point, one id
// load and the row stored as one vector.
template <typename T, int NP>
__global__ void k_gather_rows(const T* __restrict__ in, uint64_t N, uint32_t n, const uint32_t* __restrict__ perm,
                              const uint32_t* __restrict__ ids, T* __restrict__ pts) {
    const uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= N) return;
    const T* src = in + (uint64_t)ids[s] * n;
    T v[NP];
#pragma unroll
    for (int j = 0; j < NP; j++) v[j] = (uint32_t)j < n ? src[perm[j]] : T(0);
    T* dst = pts + s * NP;
    if constexpr (std::is_same<T, float>::value && NP == 2) {
        *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
    } else if constexpr (std::is_same<T, float>::value && NP == 4) {
        *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (std::is_same<T, double>::value && NP >= 2) {
#pragma unroll
        for (int j = 0; j < NP; j += 2) *reinterpret_cast<double2*>(dst + j) = make_double2(v[j], v[j + 1]);
    } else {
#pragma unroll
        for (int j = 0; j < NP; j++) dst[j] = v[j];
    }
}

// ------------------------------------------------------------ cell lookup
// Points per linear cell id (zero elsewhere); its exclusive scan is the
// slot-prefix table ds: cell L holds slots [ds[L], ds[L+1]).
__global__ void k_dense_counts(const uint64_t* __restrict__ cell_key, const uint32_t* __restrict__ cell_start,
                               uint32_t M, uint32_t* __restrict__ dcnt) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < M) dcnt[cell_key[c]] = cell_start[c + 1] - cell_start[c];
}

__global__ void k_hash_insert(const uint64_t* __restrict__ cell_key, uint32_t M, unsigned long long* hkeys,
                              uint32_t* hvals, uint64_t hmask) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const unsigned long long key = cell_key[c];
    uint64_t h = mix64(key) & hmask;
    for (uint64_t probe = 0; probe <= hmask; probe++) {
        const unsigned long long prev = atomicCAS(&hkeys[h], (unsigned long long)kEmptyKey, key);
        if (prev == kEmptyKey || prev == key) {
            hvals[h] = c;
            return;
        }
        h = (h + 1) & hmask;
    }
}

// Cell plan of dense low-dimensional grids (k <= 3): for every non-empty
// cell and each of its 3^(k-1) neighbour rows, the slot range of the row's
// cells x-1..x+1, clipped to the grid (kernel.cu:180-188 clamp the same way).
// These cells have consecutive linear ids (dim 0 is fastest), so the range is
// [ds[row + xlo], ds[row + xhi + 1]).  par holds the parity bit of each own
// coordinate for the unicomp traversal.
__global__ void k_cell_plan(const uint64_t* __restrict__ cell_key, uint32_t M, GridGeom g,
                            const uint32_t* __restrict__ ds, uint2* __restrict__ plan, uint8_t* __restrict__ par) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const uint32_t k = g.k;
    const uint32_t key = (uint32_t)cell_key[c];
    const uint32_t n0 = g.ncells[0];
    const uint32_t o0 = key % n0, rest = key / n0;
    const uint32_t o1 = k >= 2 ? rest % g.ncells[1] : 0u;
    const uint32_t o2 = k >= 3 ? rest / g.ncells[1] : 0u;
    const uint32_t nrows = k == 1 ? 1u : (k == 2 ? 3u : 9u);
    const uint32_t xlo = o0 > 0 ? o0 - 1u : 0u;
    const uint32_t xhi = o0 + 1u < n0 ? o0 + 1u : n0 - 1u;
    for (uint32_t r = 0; r < nrows; r++) {
        const long long r1 = (long long)o1 + (k >= 2 ? (long long)(r % 3) - 1 : 0);
        const long long r2 = (long long)o2 + (k >= 3 ? (long long)(r / 3) - 1 : 0);
        uint2 e = make_uint2(0u, 0u);
        const bool ok = (k < 2 || (r1 >= 0 && r1 < (long long)g.ncells[1])) &&
                        (k < 3 || (r2 >= 0 && r2 < (long long)g.ncells[2]));
        if (ok) {
            const uint32_t rowbase = (uint32_t)r1 * n0 + (k >= 3 ? (uint32_t)r2 * (uint32_t)g.mult[2] : 0u);
            const uint32_t lo = ds[rowbase + xlo];
            e = make_uint2(lo, ds[rowbase + xhi + 1u] - lo);
        }
        plan[(size_t)c * nrows + r] = e;
    }
    par[c] = (uint8_t)((o0 & 1u) | ((o1 & 1u) << 1) | ((o2 & 1u) << 2));
}

// ------------------------------------------------------------ work items
// A work item is one chunk of up to `qchunk` consecutive query slots of one cell.
__global__ void k_item_counts(const uint32_t* __restrict__ cell_start, const uint32_t* __restrict__ order,
                              uint32_t M, uint32_t qchunk, uint32_t* __restrict__ nchunks,
                              uint32_t* __restrict__ sizes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const uint32_t c = order ? order[i] : i;
    const uint32_t sz = cell_start[c + 1] - cell_start[c];
    nchunks[i] = (sz + qchunk - 1) / qchunk;
    if (sizes) sizes[i] = ~sz;  // complemented: an ascending sort gives the descending order
}

__global__ void k_make_items(const uint32_t* __restrict__ order, const uint32_t* __restrict__ nchunks,
                             const uint32_t* __restrict__ item_off, uint32_t M, uint2* __restrict__ items) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const uint32_t c = order ? order[i] : i;
    const uint32_t off = item_off[i], nc = nchunks[i];
    for (uint32_t q = 0; q < nc; q++) items[off + q] = make_uint2(c, q);
}

__global__ void k_iota(uint32_t* __restrict__ out, uint32_t M) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) out[i] = i;
}



// ------------------------------------------------------------ launchers
static inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

template <typename T>
cudaError_t launch_variance(const T* in, uint64_t N, uint32_t n, T denom, T* var_out, cudaStream_t st) {
    // the staging uses every thread; the sums use the first n (d0 loop above 1024)
    const unsigned threads = 1024;
    cudaError_t e = cudaFuncSetAttribute(k_variance<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kVarStageBytes);
    if (e != cudaSuccess) return e;
    k_variance<T><<<1, threads, kVarStageBytes, st>>>(in, N, n, denom, var_out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_minmax(const T* in, uint64_t N, uint32_t n, uint32_t k, const uint32_t* perm, T* part,
                          uint32_t nparts, T* out, cudaStream_t st) {
    k_minmax_partial<T><<<nparts, 256, 0, st>>>(in, N, n, k, perm, part);
    k_minmax_final<T><<<1, 32u * k, 0, st>>>(part, nparts, k, out);
    return cudaGetLastError();
}

template <typename T, typename K>
cudaError_t launch_cell_keys(const T* in, uint64_t N, uint32_t n, const uint32_t* perm, const GridGeom& g,
                             const T* minArr, T eps, K* keys, uint32_t* vals, uint32_t* bad, cudaStream_t st) {
    k_cell_keys<T, K><<<blocks_for(N, 256), 256, 0, st>>>(in, N, n, perm, g, minArr, eps, keys, vals, bad);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gather_points(const T* in, uint64_t N, uint32_t n, uint32_t npad, const uint32_t* perm,
                                 const uint32_t* ids, T* pts, cudaStream_t st) {
    if (npad == 1) k_gather_rows<T, 1><<<blocks_for(N, 256), 256, 0, st>>>(in, N, n, perm, ids, pts);
    else if (npad == 2) k_gather_rows<T, 2><<<blocks_for(N, 256), 256, 0, st>>>(in, N, n, perm, ids, pts);
    else if (npad == 4) k_gather_rows<T, 4><<<blocks_for(N, 256), 256, 0, st>>>(in, N, n, perm, ids, pts);
    else k_gather_points<T><<<blocks_for(N * npad, 256), 256, 0, st>>>(in, N, n, npad, perm, ids, pts);
    return cudaGetLastError();
}


cudaError_t launch_cell_tables(const uint64_t* cell_key, const uint32_t* cell_start, uint32_t M, uint32_t* dcnt,
                               unsigned long long* hkeys, uint32_t* hvals, uint64_t hmask, cudaStream_t st) {
    if (dcnt) k_dense_counts<<<blocks_for(M, 256), 256, 0, st>>>(cell_key, cell_start, M, dcnt);
    if (hkeys) k_hash_insert<<<blocks_for(M, 256), 256, 0, st>>>(cell_key, M, hkeys, hvals, hmask);
    return cudaGetLastError();
}

cudaError_t launch_cell_plan(const uint64_t* cell_key, uint32_t M, const GridGeom& g, const uint32_t* ds,
                             uint2* plan, uint8_t* par, cudaStream_t st) {
    k_cell_plan<<<blocks_for(M, 256), 256, 0, st>>>(cell_key, M, g, ds, plan, par);
    return cudaGetLastError();
}

cudaError_t launch_item_counts(const uint32_t* cell_start, const uint32_t* order, uint32_t M, uint32_t qchunk,
                               uint32_t* nchunks, uint32_t* sizes, cudaStream_t st) {
    k_item_counts<<<blocks_for(M, 256), 256, 0, st>>>(cell_start, order, M, qchunk, nchunks, sizes);
    return cudaGetLastError();
}

cudaError_t launch_make_items(const uint32_t* order, const uint32_t* nchunks, const uint32_t* item_off,
                              uint32_t M, uint2* items, cudaStream_t st) {
    k_make_items<<<blocks_for(M, 256), 256, 0, st>>>(order, nchunks, item_off, M, items);
    return cudaGetLastError();
}

cudaError_t launch_iota(uint32_t* out, uint32_t M, cudaStream_t st) {
    k_iota<<<blocks_for(M, 256), 256, 0, st>>>(out, M);
    return cudaGetLastError();
}


#define GSJ_INST_INDEX(T)                                                                                  \
    template cudaError_t launch_variance<T>(const T*, uint64_t, uint32_t, T, T*, cudaStream_t);           \
    template cudaError_t launch_minmax<T>(const T*, uint64_t, uint32_t, uint32_t, const uint32_t*, T*,     \
                                          uint32_t, T*, cudaStream_t);                                     \
    template cudaError_t launch_cell_keys<T, uint64_t>(const T*, uint64_t, uint32_t, const uint32_t*,      \
                                                       const GridGeom&, const T*, T, uint64_t*, uint32_t*, \
                                                       uint32_t*, cudaStream_t);                           \
    template cudaError_t launch_cell_keys<T, uint32_t>(const T*, uint64_t, uint32_t, const uint32_t*,      \
                                                       const GridGeom&, const T*, T, uint32_t*, uint32_t*, \
                                                       uint32_t*, cudaStream_t);                           \
    template cudaError_t launch_gather_points<T>(const T*, uint64_t, uint32_t, uint32_t, const uint32_t*,  \
                                                 const uint32_t*, T*, cudaStream_t);
GSJ_INST_INDEX(float)
GSJ_INST_INDEX(double)

}  // namespace gsj
