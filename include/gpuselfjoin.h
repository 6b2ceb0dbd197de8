/*
 * gpuselfjoin.h - C ABI of the B200 (sm_100a) epsilon-grid distance self-join.
 *
 * Drop-in for algorithm 3 of mgowanlock/gpu_self_join: every pair (q, c) of
 * the N input points with sqrt(sum_l (c_l - q_l)^2) <= eps is reported (self
 * pairs included), in the reference's own floating-point arithmetic, as one
 * neighbour list per point:
 *     numNeighbors[N]   (uint32)        - list length of point i
 *     neighborTable[R]  (uint32)        - the lists, concatenated in point-id order
 *
 * The params.h switches of the reference become run-time fields of gsj_config
 * (same names, same meaning).  All entry points return a status code (GSJ_OK
 * == 0, negative on error) and never terminate the process; gsj_last_error()
 * describes the most recent failure of the calling thread's default context.
 *
 * Plain C types only; no CUDA or PyTorch types appear in these signatures.
 * Device pointers are passed as void* / uint32_t* and are marked as such.
 */
#ifndef GPUSELFJOIN_H
#define GPUSELFJOIN_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GSJ_API __attribute__((visibility("default")))
#else
#define GSJ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define GSJ_OK 0
#define GSJ_ERR_INVALID (-1)    /* bad argument / configuration            */
#define GSJ_ERR_CUDA (-2)       /* a CUDA runtime call failed              */
#define GSJ_ERR_NOMEM (-3)      /* device or pinned host allocation failed */
#define GSJ_ERR_STATE (-4)      /* call order violated (no result, ...)    */
#define GSJ_ERR_OVERFLOW (-5)   /* a result count exceeds the ABI's range  */

/* ---------------------------------------------------------------- dtype */
#define GSJ_FLOAT32 0
#define GSJ_FLOAT64 1

/* flags */
#define GSJ_FLAG_SORT_LISTS 0x1u  /* sort every neighbour list ascending (an
                                     on-device segmented sort after the fill; the
                                     tile and screen paths' lists are ascending
                                     anyway); below 2^31 result pairs per join   */
#define GSJ_FLAG_QUIET      0x2u  /* no progress output on stdout              */
#define GSJ_FLAG_NO_UNICOMP 0x4u  /* full neighbourhood traversal even with STAMP
                                     (same pair set, different work split)   */
#define GSJ_FLAG_PLAIN      0x8u  /* no tensor-core screen: every candidate pair
                                     is evaluated with the exact FP32 arithmetic */
#define GSJ_FLAG_EXACT_SIZE 0x10u /* size the pair buffers of the warp, tile and
                                     screen paths without an estimate: the first
                                     pass only counts, the pass is repeated into a
                                     buffer of the counted size (the re-run path
                                     that a short estimate takes)              */

/*
 * Run-time configuration.  Field names follow params.h of the reference
 * (params.h:17-93); the values have the same meaning.
 */
typedef struct gsj_config {
    uint32_t dim;           /* GPUNUMDIM      number of dimensions n            */
    uint32_t indexed_dims;  /* NUMINDEXEDDIM  grid dimensions k, 1 <= k <= n     */
    uint32_t dtype;         /* DTYPE          GSJ_FLOAT32 or GSJ_FLOAT64         */
    uint32_t reorder;       /* REORDER        permute dims by sampled variance   */
    uint32_t shortcircuit;  /* SHORTCIRCUIT   early exit of the distance sum     */
    uint32_t ilp;           /* ILP            accumulation order (0 = sequential)*/
    uint32_t stamp;         /* STAMP          unidirectional cell comparison     */
    uint32_t query_reorder; /* QUERYREORDER   schedule heavy query cells first   */
    int32_t device;         /* gpuContext     CUDA device ordinal                */
    uint32_t flags;         /* GSJ_FLAG_*                                        */
    /* Batching scheme (params.h:78-93), used when results go to host memory
     * (gsj_join_host): the table is produced in batches of point ids whose
     * lists fit one device result segment, each copied to the host while the
     * next is computed. */
    uint64_t buffer_pairs;  /* GPUBUFFERSIZE  result entries per device segment
                                              (0: 100,000,000)                   */
    uint32_t streams;       /* GPUSTREAMS     segments in flight (0: 3)          */
    uint32_t min_batches;   /* MINBATCHES     fewest batches (0: 3)              */
    uint32_t estimator;     /* GSJ_EST_*      result-size estimate of the pair
                                              paths (SAMPLERATE's role)         */
    uint32_t sort;          /* SORT           points of each cell ordered by one
                                              dimension, neighbour scans pruned
                                              by it (params.h:46); the reference's
                                              pairs (GSJ_PATH_SORT)               */
} gsj_config;

/* Result-size estimators (gsj_config.estimator): how the warp, tile and screen
 * paths size their pair buffers before the exact pass (a short buffer is
 * re-sized and the pass repeated, so the output never depends on it). */
#define GSJ_EST_SAMPLED 0u /* an exact pass over every 64th work item         */
#define GSJ_EST_LEARNED 1u /* the context's result-count model (gsj_model_*),
                              trained on the counts of earlier joins; the sampled
                              estimate while the model is untrained          */

/* Statistics of the most recent join of a context. */
typedef struct gsj_stats {
    uint64_t num_points;      /* N                                              */
    uint64_t total_pairs;     /* R = sum(numNeighbors)                          */
    uint64_t candidates;      /* distance evaluations (reference COUNTMETRICS
                                 workCounts[0] semantics for the traversal used)*/
    uint64_t total_cells;     /* product of cells per indexed dim (main.cu:941) */
    uint64_t nonempty_cells;  /* non-empty grid cells                           */
    uint64_t work_items;      /* scheduled (query cell chunk) work items        */
    double ms_h2d;            /* host->device copy of the dataset               */
    double ms_index;          /* REORDER + grid extents + on-device index build */
    double ms_join;           /* join: count + offsets + fill (ROWS), or pair
                                 emission + pair sort + table (other paths)     */
    double ms_d2h;            /* result copies to the host                      */
    double ms_total;          /* whole call                                     */
    /* device time (CUDA events on the context's stream) */
    double dev_ms_index;      /* index build: keys, sort, cells, lookup, items  */
    double dev_ms_count;      /* count pass (other paths: the distance pass)    */
    double dev_ms_fill;       /* fill pass (other paths: pair sort + table)     */
    uint64_t kernel_launches; /* launches of this library's own kernels         */
    uint64_t join_path;       /* GSJ_PATH_* taken by the last join              */
    uint64_t screen_rechecks; /* GSJ_PATH_SCREEN: pairs the BF16 screen could not
                                 reject, evaluated exactly (0 on other paths)   */
    uint64_t reruns;          /* passes repeated because a buffer sized from the
                                 estimate was short (the output is unchanged)  */
    uint64_t batches;         /* result batches of gsj_join_host (1 otherwise)  */
    uint64_t tuned;           /* 1 when a tuning-table entry shaped the launches */
    uint64_t density_log2;    /* floor(log2(points per non-empty cell)): the
                                 tuning table's density key                    */
    uint64_t estimate;        /* pairs (or undecided pairs) the estimator
                                 predicted for the exact pass                  */
    double dev_ms_estimate;   /* device time of the estimate                    */
} gsj_stats;

/* Join paths (gsj_stats.join_path). */
#define GSJ_PATH_WARP 0u  /* warp per (cell, 32 queries): pair keys + on-device sort */
#define GSJ_PATH_ROWS 1u  /* dense k <= 3, n <= 4: thread-per-query count + fill   */
#define GSJ_PATH_TILE 2u  /* float, 5 <= n <= 128, k <= 6, >= 8 points per cell:
                             64 x 64 register tiles, pair buffer, on-device sort */
#define GSJ_PATH_SCREEN 3u /* float, 16 <= n <= 128, k <= 6, >= 8 points per cell:
                             BF16 tcgen05 screen with a proven bound, exact FP32
                             check of the rest, pair buffer, on-device sort   */
#define GSJ_PATH_SORT 4u  /* cfg.sort: thread per query, the reference's pruned
                             scans of sorted cells, count + fill              */

typedef struct gsj_context gsj_context;

/* Fills *cfg with the build-time defaults (the GPUNUMDIM ... QUERYREORDER
 * macros given when the library was built). */
GSJ_API void gsj_default_config(gsj_config* cfg);

/* Replaces the defaults used by GDSJoinPy (the run-time counterpart of
 * rebuilding the reference with another params.h).  dim may be 0 (take NDIM). */
GSJ_API int gsj_set_default_config(const gsj_config* cfg);

/* Context: owns a CUDA stream and a device memory pool reused across joins. */
GSJ_API int gsj_create(gsj_context** ctx, int device);
GSJ_API int gsj_destroy(gsj_context* ctx);

/*
 * Runs the self-join.  `data` is a row-major N x cfg->dim array of cfg->dtype,
 * in host memory (data_on_device == 0) or device memory of cfg->device
 * (data_on_device == 1).  eps is converted to cfg->dtype first, as the
 * reference stores epsilon as DTYPE (main.cu:98).  Results stay on the device
 * until fetched with the gsj_result_* calls.  Replaces the mode-3 body of
 * main.cu:178-262 and distanceTableNDGridBatches (GPU.cu:270-1088).
 */
GSJ_API int gsj_join(gsj_context* ctx, const void* data, uint64_t num_points, double eps,
             const gsj_config* cfg, int data_on_device, gsj_stats* stats);

/*
 * Runs the self-join and delivers the result to host memory: numNeighbors into
 * num_neighbors[N] (host) and neighborTable into neighbor_table (host, `cap`
 * entries).  Replaces distanceTableNDGridBatches' batch loop (GPU.cu:765-994)
 * with a pipeline: on the dense low-dimensional path the table is produced in
 * batches of point ids whose lists fit one device segment of
 * cfg->buffer_pairs entries, and each batch is copied to the host (directly
 * into pinned destinations, through pinned staging otherwise) while the next
 * one is computed, cfg->streams segments in flight; the other paths copy the
 * finished table.  When cap < R, *total_pairs receives R, num_neighbors is
 * filled, no table entry is written and GSJ_ERR_OVERFLOW is returned.  The
 * device keeps numNeighbors and the offsets (gsj_result_device) but not
 * necessarily the table afterwards.
 */
GSJ_API int gsj_join_host(gsj_context* ctx, const void* data, uint64_t num_points, double eps,
                          const gsj_config* cfg, int data_on_device, uint32_t* num_neighbors,
                          uint32_t* neighbor_table, uint64_t cap, uint64_t* total_pairs, gsj_stats* stats);

/* Number of result pairs R of the last join. */
GSJ_API int gsj_result_size(gsj_context* ctx, uint64_t* total_pairs);

/* numNeighbors[N] of the last join, into host (dst_on_device == 0) or device
 * memory.  storeNumberOfNeighborsForPython, main.cu:630-636. */
GSJ_API int gsj_result_counts(gsj_context* ctx, uint32_t* num_neighbors, int dst_on_device);

/* neighborTable[R] (capacity `cap` entries) into host or device memory; lists
 * are concatenated in point-id order.  storeNeighborTableContiguousPython,
 * main.cu:514-542.  Host destinations are filled through pinned staging
 * buffers on two streams, overlapping the copy-out with the PCIe transfer. */
GSJ_API int gsj_result_table(gsj_context* ctx, uint32_t* neighbor_table, uint64_t cap, int dst_on_device);

/* Device pointers of the last result (valid until the next join or destroy):
 * counts[N], offsets[N+1] (uint64 exclusive prefix), table[R]. */
GSJ_API int gsj_result_device(gsj_context* ctx, const uint32_t** counts, const uint64_t** offsets,
                      const uint32_t** table);

/* Error text of the last failing call on ctx (or of the default context when
 * ctx is NULL). */
GSJ_API const char* gsj_last_error(gsj_context* ctx);

/* The largest s with sqrt(s) <= eps in the given precision: the distance test
 * sqrt(s) <= eps of kernel.cu:361/364 is evaluated as s <= threshold. */
GSJ_API float gsj_threshold_f32(float eps);
GSJ_API double gsj_threshold_f64(double eps);

/* Brute-force neighbour counts over all N^2 pairs, self pairs included: the
 * reference's GPU algorithm 1 (kernelBruteForce, kernel.cu:486-515, via
 * makeDistanceTableGPUBruteForce, GPU.cu:1285-1440), with its arithmetic
 * (`runningDist += (c-q)*(c-q)` over the dimensions in order, sqrt <= eps).
 * cfg supplies dim and dtype (the index switches do not apply).  counts
 * (optional, host, uint32[N]) receives each point's count, total the sum.
 * O(N^2 n) work: an exact-count check of the grid join on small inputs. */
GSJ_API int gsj_bruteforce_count(gsj_context* ctx, const void* data, uint64_t num_points, double eps,
                                 const gsj_config* cfg, int data_on_device, uint32_t* counts,
                                 uint64_t* total);

/*
 * List offsets without allocating: d_offsets[i] = d_counts[0] + ... +
 * d_counts[i-1] for i in [0, n], so d_offsets[n] is the total (the layout of
 * neighborTable for the numNeighbors in d_counts).  No counterpart in the
 * reference; it is the scan the join itself uses to lay out its table, made
 * callable by code that must not allocate device memory: a host framework
 * whose allocator already reserves (nearly) all device memory for its own
 * pool, where a cudaMalloc fails or forces the pool to give memory back, and
 * code on a latency-critical path, where cudaMalloc and cudaFree would
 * synchronise the device.  The call uses no cudaMalloc, cudaFree or
 * allocating library routine: its scratch (64 KiB of per-tile sums) is a
 * fixed array inside the library that every device loading the library keeps
 * until the process exits.  Limits: n <= 33,550,336; larger n returns
 * GSJ_ERR_INVALID.  d_counts and d_offsets (n + 1 entries) are device memory of
 * the calling thread's current device; the work is queued on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) and the call returns
 * without waiting for it.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and caches it; make that first call
 * before any stream capture.  The cached address belongs to the device's
 * context of that first call: after a cudaDeviceReset of the device, use the
 * entry point only from a new process.  All calls share the one array, which keeps the
 * last call's contents (nothing in it needs to start at zero): calls that
 * overlap on the GPU, e.g. on two streams at once, race and must be ordered by
 * the caller.
 */
GSJ_API int gsj_list_offsets_noalloc(const uint32_t* d_counts, uint64_t n, uint64_t* d_offsets, void* stream);

/* ---------------------------------------------------------------- autotuning
 * Launch shapes chosen per (join path, dimensionality, density).  The
 * reference fixes them at compile time (BLOCKSIZE, params.h:17; GPUSTREAMS,
 * params.h:85).  A context keeps a table of tuned shapes; a join whose
 * (path, dim, density_log2) has an entry launches with it (gsj_stats.tuned).
 * Shapes never change results, only speed. */
typedef struct gsj_tuning {
    uint32_t threads;     /* ROWS path: CTA size of the count and fill passes
                             (64..256, a multiple of 32; 0: 256)              */
    uint32_t warps;       /* WARP path: warps per CTA (1..8; 0: as many as the
                             shared memory allows, up to 8)                   */
    uint32_t ctas_per_sm; /* WARP, TILE, SCREEN paths: resident CTAs per SM at
                             most (0: all that fit)                           */
    uint32_t streams;     /* gsj_join_host: segments in flight (0: the config's) */
} gsj_tuning;

/* Times the join of `data` under candidate shapes of the path it takes
 * (coordinate descent, each candidate the mean device time of `repeats`
 * joins after one warm-up), stores the fastest in the context's table for the
 * join's (path, dim, density_log2) and returns it in *best. */
GSJ_API int gsj_autotune(gsj_context* ctx, const void* data, uint64_t num_points, double eps, const gsj_config* cfg,
                         int data_on_device, uint32_t repeats, gsj_tuning* best);
/* Reads (GSJ_ERR_STATE when absent) or writes one table entry, e.g. to keep
 * tuned shapes across processes. */
GSJ_API int gsj_tuning_get(gsj_context* ctx, uint32_t path, uint32_t dim, uint32_t density_log2, gsj_tuning* t);
GSJ_API int gsj_tuning_set(gsj_context* ctx, uint32_t path, uint32_t dim, uint32_t density_log2,
                           const gsj_tuning* t);

/* ---------------------------------------------------------------- learned
 * The context's result-count model (GSJ_EST_LEARNED): a 16-64-32-1 MLP
 * (GSJ_MODEL_WEIGHTS weights) that predicts the mean neighbour count of a
 * cell's queries from the sizes of the cell and its face-adjacent cells, eps
 * and the dimensionality.  It replaces the reference's sampled estimator
 * (callGPUBatchEst, GPU.cu:57-268; SAMPLERATE, params.h:93) for sizing the
 * pair buffers; the exact count still checks every buffer.  Training and
 * inference run on the device with this library's own kernels. */
#define GSJ_MODEL_WEIGHTS 3201
#define GSJ_MODEL_FEATURES 16

/* Trains the model for `steps` Adam steps on the exact per-cell counts of the
 * last join of ctx (up to 65,536 of its cells); *loss (optional) receives the
 * last minibatch's mean squared error of log2(1 + count). */
GSJ_API int gsj_model_train(gsj_context* ctx, uint32_t steps, float* loss);
/* Back to the initial (untrained) weights. */
GSJ_API int gsj_model_reset(gsj_context* ctx);
/* Copies the weights out (set == 0) or in (set != 0; marks the model
 * trained); count must be GSJ_MODEL_WEIGHTS. */
GSJ_API int gsj_model_weights(gsj_context* ctx, float* weights, uint32_t count, int set);
/* The last join's per-cell features [cells][GSJ_MODEL_FEATURES] and targets
 * [cells] (host arrays of capacity `cap` rows; only *cells is written when
 * cap is smaller). */
GSJ_API int gsj_model_features(gsj_context* ctx, float* features, float* targets, uint32_t cap, uint32_t* cells);
/* Network outputs (log2(1 + count)) of n host feature rows. */
GSJ_API int gsj_model_predict(gsj_context* ctx, const float* features, uint32_t n, float* out);
/* Mean squared error over n host rows and its gradient (GSJ_MODEL_WEIGHTS
 * floats), computed by the training kernels' forward and backward code. */
GSJ_API int gsj_model_loss_grad(gsj_context* ctx, const float* features, const float* targets, uint32_t n,
                                float* loss, float* grad);

/* ---------------------------------------------------------------- drop-in
 * The reference's shared-library ABI (built with -DPYTHON, Makefile:58-77).
 *
 * GDSJoinPy replaces main.cu:360 (`extern "C" void GDSJoinPy(DTYPE* dataset,
 * unsigned int NUMPOINTS, DTYPE epsilon, unsigned int NDIM, int gpuContext,
 * unsigned int* outNumNeighborsWithinEps)`).  DTYPE is float in the default
 * build (define GSJ_DTYPE_DOUBLE at build time for double, as params.h:26
 * does); the typed variants below take either precision.  The configuration is
 * the build-time default (gsj_default_config) with dim = NDIM; when the library
 * was built with a non-zero GPUNUMDIM, NDIM must equal it (main.cu:372-375).
 * Unlike the reference, STAMP=1 is accepted and produces the same symmetric
 * lists as STAMP=0, and nothing ever calls exit().
 *
 * copyResultIntoPythonArray replaces main.cu:507: it copies the first
 * numResults entries of the table produced by the preceding GDSJoinPy and
 * releases it.  The two calls are paired as in the reference; the pair is
 * not re-entrant across threads.
 */
#ifdef GSJ_DTYPE_DOUBLE
typedef double gsj_dtype_t;
#else
typedef float gsj_dtype_t;
#endif
GSJ_API void GDSJoinPy(gsj_dtype_t* dataset, unsigned int NUMPOINTS, gsj_dtype_t epsilon, unsigned int NDIM,
               int gpuContext, unsigned int* outNumNeighborsWithinEps);
GSJ_API void copyResultIntoPythonArray(unsigned int* outPythonNeighborTable, unsigned int numResults);

/* Typed, status-returning forms of the same two calls.  The 64-bit count
 * variant lifts the reference's 2^32 limit on the table size (main.cu:507). */
GSJ_API int GDSJoinPy_f32(const float* dataset, unsigned int NUMPOINTS, float epsilon, unsigned int NDIM,
                  int gpuContext, unsigned int* outNumNeighborsWithinEps);
GSJ_API int GDSJoinPy_f64(const double* dataset, unsigned int NUMPOINTS, double epsilon, unsigned int NDIM,
                  int gpuContext, unsigned int* outNumNeighborsWithinEps);
GSJ_API int copyResultIntoPythonArray64(unsigned int* outPythonNeighborTable, uint64_t numResults);

#ifdef __cplusplus
}
#endif

#endif /* GPUSELFJOIN_H */
