// Learned result-count model: a small MLP that predicts how many neighbours
// the queries of a grid cell have, from the occupancy of the cell and of its
// adjacent cells, eps and the dimensionality.  It takes the place of the
// reference's sampled estimator (callGPUBatchEst + kernelNDGridIndexBatch-
// Estimator, GPU.cu:57-268, kernel.cu:522-694; SAMPLERATE, params.h:93) in
// sizing the pair buffers of the warp, tile and screen paths; the buffers are
// still checked against the exact count, and a short one is re-sized and the
// pass repeated, so the output never depends on the model.
//
// Network: kF = 16 features -> 64 ReLU -> 32 ReLU -> 1 (3,201 weights), output
// log2(1 + mean neighbours per query of the cell).  Training data are the
// exact per-cell counts a finished join emitted; the loss is the mean squared
// error of the log2 output; Adam updates.
//
// Kernels (all written here):
//   k_model_features  per cell: own size, a histogram of the sizes of the 2k
//                     face-adjacent cells (log2 bins), their sum and maximum,
//                     k, n, eps, N
//   k_model_targets   per cell: log2(1 + mean list length of its points)
//   k_model_predict   per cell: the network's output, and the estimated pairs
//                     (cell size x predicted list length, summed)
//   k_model_train     one CTA runs S Adam steps on minibatches of 128 cells;
//                     every gradient is a sum over the minibatch in a fixed
//                     order (no atomics), so training is deterministic
//   k_model_grad      the full-batch loss and gradient (the gradient check)
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"
#include "gsj_model.h"

namespace gsj {

namespace {

constexpr int kF = kModelFeatures;
constexpr int kH1 = 64;
constexpr int kH2 = 32;
constexpr int kOffB1 = kH1 * kF;
constexpr int kOffW2 = kOffB1 + kH1;
constexpr int kOffB2 = kOffW2 + kH2 * kH1;
constexpr int kOffW3 = kOffB2 + kH2;
constexpr int kOffB3 = kOffW3 + kH2;
static_assert(kOffB3 + 1 == kModelWeights, "weight layout");
constexpr int kMB = 128;           // minibatch
constexpr int kTT = 256;           // training CTA threads
constexpr int kWPT = (kModelWeights + kTT - 1) / kTT;  // weights per thread

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// Shared-memory work area of the training and gradient kernels.
struct TrainSmem {
    float w[kModelWeights];
    float x[kMB][kF];
    float y[kMB];
    float h1[kMB][kH1];
    float h2[kMB][kH2];
    float g[kMB];      // d loss / d output
    float d2[kMB][kH2];
    float d1[kMB][kH1];
    float red[kTT / 32];
};

// Forward and backward of the minibatch held in sm.x / sm.y (nb <= kMB
// valid rows; the others contribute nothing).  gscale: 2 / (samples in the
// loss).  Returns this thread's share of the squared error.
__device__ float fwd_bwd(TrainSmem& sm, int nb, float gscale) {
    const int tid = threadIdx.x;
    for (int e = tid; e < kMB * kH1; e += kTT) {
        const int b = e / kH1, j = e % kH1;
        float acc = sm.w[kOffB1 + j];
#pragma unroll
        for (int f = 0; f < kF; f++) acc = fmaf(sm.w[j * kF + f], sm.x[b][f], acc);
        sm.h1[b][j] = relu(acc);
    }
    __syncthreads();
    for (int e = tid; e < kMB * kH2; e += kTT) {
        const int b = e / kH2, j = e % kH2;
        float acc = sm.w[kOffB2 + j];
        for (int i = 0; i < kH1; i++) acc = fmaf(sm.w[kOffW2 + j * kH1 + i], sm.h1[b][i], acc);
        sm.h2[b][j] = relu(acc);
    }
    __syncthreads();
    float se = 0.f;
    for (int b = tid; b < kMB; b += kTT) {
        float o = sm.w[kOffB3];
        for (int j = 0; j < kH2; j++) o = fmaf(sm.w[kOffW3 + j], sm.h2[b][j], o);
        const float r = b < nb ? o - sm.y[b] : 0.f;
        sm.g[b] = gscale * r;
        se += r * r;
    }
    __syncthreads();
    for (int e = tid; e < kMB * kH2; e += kTT) {
        const int b = e / kH2, j = e % kH2;
        sm.d2[b][j] = sm.h2[b][j] > 0.f ? sm.g[b] * sm.w[kOffW3 + j] : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < kMB * kH1; e += kTT) {
        const int b = e / kH1, i = e % kH1;
        float acc = 0.f;
        if (sm.h1[b][i] > 0.f)
            for (int j = 0; j < kH2; j++) acc = fmaf(sm.d2[b][j], sm.w[kOffW2 + j * kH1 + i], acc);
        sm.d1[b][i] = acc;
    }
    __syncthreads();
    return se;
}

// Gradient of weight w over the minibatch rows [0, kMB) (sums in row order).
__device__ float weight_grad(const TrainSmem& sm, int w) {
    float acc = 0.f;
    if (w < kOffB1) {
        const int j = w / kF, f = w % kF;
        for (int b = 0; b < kMB; b++) acc = fmaf(sm.d1[b][j], sm.x[b][f], acc);
    } else if (w < kOffW2) {
        const int j = w - kOffB1;
        for (int b = 0; b < kMB; b++) acc += sm.d1[b][j];
    } else if (w < kOffB2) {
        const int j = (w - kOffW2) / kH1, i = (w - kOffW2) % kH1;
        for (int b = 0; b < kMB; b++) acc = fmaf(sm.d2[b][j], sm.h1[b][i], acc);
    } else if (w < kOffW3) {
        const int j = w - kOffB2;
        for (int b = 0; b < kMB; b++) acc += sm.d2[b][j];
    } else if (w < kOffB3) {
        const int j = w - kOffW3;
        for (int b = 0; b < kMB; b++) acc = fmaf(sm.g[b], sm.h2[b][j], acc);
    } else {
        for (int b = 0; b < kMB; b++) acc += sm.g[b];
    }
    return acc;
}

__device__ float block_sum(float v, float* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < kTT / 32; w++) t += red[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(kTT) k_model_train(const float* __restrict__ X, const float* __restrict__ Y,
                                                     uint32_t ntr, float* __restrict__ W, float* __restrict__ M1,
                                                     float* __restrict__ M2, uint32_t t0, uint32_t steps, float lr,
                                                     float* __restrict__ loss_out) {
    extern __shared__ __align__(16) unsigned char model_smem[];
    TrainSmem& sm = *reinterpret_cast<TrainSmem*>(model_smem);
    const int tid = threadIdx.x;
    for (int w = tid; w < kModelWeights; w += kTT) sm.w[w] = W[w];
    float m1[kWPT], m2[kWPT];
#pragma unroll
    for (int r = 0; r < kWPT; r++) {
        const int w = tid + r * kTT;
        m1[r] = w < kModelWeights ? M1[w] : 0.f;
        m2[r] = w < kModelWeights ? M2[w] : 0.f;
    }
    __syncthreads();
    const float b1 = 0.9f, b2 = 0.999f;
    float last = 0.f;
    for (uint32_t s = 0; s < steps; s++) {
        const uint32_t t = t0 + s + 1;
        for (int e = tid; e < kMB * kF; e += kTT) {
            const int b = e / kF, f = e % kF;
            const uint32_t idx = hash32(t * 0x9e3779b9u + (uint32_t)b) % ntr;
            sm.x[b][f] = X[(size_t)idx * kF + f];
            if (f == 0) sm.y[b] = Y[idx];
        }
        __syncthreads();
        const float se = fwd_bwd(sm, kMB, 2.f / (float)kMB);
        const float tot = block_sum(se, sm.red);
        if (tid == 0) last = tot / (float)kMB;
        float gr[kWPT];
#pragma unroll
        for (int r = 0; r < kWPT; r++) {
            const int w = tid + r * kTT;
            gr[r] = w < kModelWeights ? weight_grad(sm, w) : 0.f;
        }
        __syncthreads();  // every read of the weights of this step is done
        const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
#pragma unroll
        for (int r = 0; r < kWPT; r++) {
            const int w = tid + r * kTT;
            if (w < kModelWeights) {
                m1[r] = b1 * m1[r] + (1.f - b1) * gr[r];
                m2[r] = b2 * m2[r] + (1.f - b2) * gr[r] * gr[r];
                sm.w[w] -= lr * (m1[r] / c1) / (sqrtf(m2[r] / c2) + 1e-8f);
            }
        }
        __syncthreads();
    }
    for (int w = tid; w < kModelWeights; w += kTT) W[w] = sm.w[w];
#pragma unroll
    for (int r = 0; r < kWPT; r++) {
        const int w = tid + r * kTT;
        if (w < kModelWeights) {
            M1[w] = m1[r];
            M2[w] = m2[r];
        }
    }
    if (tid == 0 && loss_out) *loss_out = last;
}

// Full-batch mean squared error and its gradient over n samples (chunks of
// kMB rows, gradients summed chunk after chunk in order).
__global__ void __launch_bounds__(kTT) k_model_grad(const float* __restrict__ X, const float* __restrict__ Y,
                                                    uint32_t n, const float* __restrict__ W,
                                                    float* __restrict__ loss, float* __restrict__ grad) {
    extern __shared__ __align__(16) unsigned char model_smem[];
    TrainSmem& sm = *reinterpret_cast<TrainSmem*>(model_smem);
    const int tid = threadIdx.x;
    for (int w = tid; w < kModelWeights; w += kTT) sm.w[w] = W[w];
    float gr[kWPT];
#pragma unroll
    for (int r = 0; r < kWPT; r++) gr[r] = 0.f;
    float se_all = 0.f;
    for (uint32_t c0 = 0; c0 < n; c0 += kMB) {
        const int nb = (int)min((uint32_t)kMB, n - c0);
        for (int e = tid; e < kMB * kF; e += kTT) {
            const int b = e / kF, f = e % kF;
            sm.x[b][f] = b < nb ? X[(size_t)(c0 + b) * kF + f] : 0.f;
            if (f == 0) sm.y[b] = b < nb ? Y[c0 + b] : 0.f;
        }
        __syncthreads();
        const float se = fwd_bwd(sm, nb, 2.f / (float)n);
        se_all += block_sum(se, sm.red);
#pragma unroll
        for (int r = 0; r < kWPT; r++) {
            const int w = tid + r * kTT;
            if (w < kModelWeights) gr[r] += weight_grad(sm, w);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < kWPT; r++) {
        const int w = tid + r * kTT;
        if (w < kModelWeights) grad[w] = gr[r];
    }
    if (tid == 0) *loss = se_all / (float)n;
}

// Network output for one feature row (weights in shared memory).
__device__ float mlp_out(const float* __restrict__ w, const float* x) {
    float h1[kH1];
#pragma unroll 4
    for (int j = 0; j < kH1; j++) {
        float acc = w[kOffB1 + j];
#pragma unroll
        for (int f = 0; f < kF; f++) acc = fmaf(w[j * kF + f], x[f], acc);
        h1[j] = relu(acc);
    }
    float o = w[kOffB3];
    for (int j = 0; j < kH2; j++) {
        float acc = w[kOffB2 + j];
#pragma unroll 8
        for (int i = 0; i < kH1; i++) acc = fmaf(w[kOffW2 + j * kH1 + i], h1[i], acc);
        o = fmaf(w[kOffW3 + j], relu(acc), o);
    }
    return o;
}

// out[c] = network output of row c; with cell_start, *est += size_c x
// predicted list length (2^out - 1, clamped to [0, N]).
__global__ void __launch_bounds__(256) k_model_predict(const float* __restrict__ X, uint32_t m,
                                                       const float* __restrict__ W, float* __restrict__ out,
                                                       const uint32_t* __restrict__ cell_start, float nmax,
                                                       double* __restrict__ est) {
    __shared__ float w[kModelWeights];
    __shared__ double red[8];
    for (int i = threadIdx.x; i < kModelWeights; i += blockDim.x) w[i] = W[i];
    __syncthreads();
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (c < m) {
        float x[kF];
#pragma unroll
        for (int f = 0; f < kF; f++) x[f] = X[(size_t)c * kF + f];
        const float o = mlp_out(w, x);
        if (out) out[c] = o;
        if (cell_start) {
            const float per = fminf(fmaxf(exp2f(fminf(o, 40.f)) - 1.f, 0.f), nmax);
            part = (double)(cell_start[c + 1] - cell_start[c]) * (double)per;
        }
    }
    if (est) {
        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
            atomicAdd(est, t);
        }
    }
}

__device__ __forceinline__ float log2p1(float v) { return log2f(1.f + v); }

__global__ void __launch_bounds__(256) k_model_features(const JoinArgs<float> a, uint32_t M, float log2_eps,
                                                        uint32_t n, float* __restrict__ X) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const uint32_t k = a.g.k;
    const uint64_t key = a.cell_key[c];
    const uint32_t size = a.cell_start[c + 1] - a.cell_start[c];
    float hist[8];
#pragma unroll
    for (int i = 0; i < 8; i++) hist[i] = 0.f;
    float sum = 0.f, mx = 0.f;
    for (uint32_t j = 0; j < k; j++) {
        const uint32_t own = (uint32_t)((key / a.g.mult[j]) % a.g.ncells[j]);
        for (int dir = -1; dir <= 1; dir += 2) {
            uint32_t cnt = 0;
            const bool inside = dir < 0 ? own > 0u : own + 1u < a.g.ncells[j];
            if (inside) {
                const uint64_t lin = dir < 0 ? key - a.g.mult[j] : key + a.g.mult[j];
                uint32_t st = 0;
                if (!lookup_range(a, lin, st, cnt)) cnt = 0;
            }
            const int bin = cnt == 0u ? 0 : min(7, 1 + (31 - __clz(cnt)));
            hist[bin] += 1.f;
            sum += (float)cnt;
            mx = fmaxf(mx, (float)cnt);
        }
    }
    const float inv = k ? 1.f / (2.f * (float)k) : 0.f;
    float* x = X + (size_t)c * kF;
    x[0] = log2p1((float)size) / 8.f;
#pragma unroll
    for (int i = 0; i < 8; i++) x[1 + i] = hist[i] * inv;
    x[9] = log2p1(sum) / 8.f;
    x[10] = log2p1(mx) / 8.f;
    x[11] = (float)k / 8.f;
    x[12] = (float)n / 128.f;
    x[13] = log2_eps / 16.f;
    x[14] = log2p1((float)a.n_points) / 32.f;
    x[15] = n ? (float)(n - k) / (float)n : 0.f;
}

__global__ void k_model_targets(const uint32_t* __restrict__ cell_start, const uint32_t* __restrict__ ids,
                                const uint32_t* __restrict__ counts, uint32_t M, float* __restrict__ Y) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M) return;
    const uint32_t s0 = cell_start[c], s1 = cell_start[c + 1];
    double sum = 0.0;
    for (uint32_t s = s0; s < s1; s++) sum += counts[ids[s]];
    Y[c] = log2p1((float)(sum / (double)(s1 - s0)));
}

// Rows of the training set: every stride-th cell.
__global__ void k_model_subsample(const float* __restrict__ X, const float* __restrict__ Y, uint32_t M,
                                  uint32_t stride, uint32_t ntr, float* __restrict__ Xt, float* __restrict__ Yt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntr) return;
    const uint32_t c = (uint32_t)(((uint64_t)i * stride) % M);
    for (int f = 0; f < kF; f++) Xt[(size_t)i * kF + f] = X[(size_t)c * kF + f];
    Yt[i] = Y[c];
}

__global__ void k_model_init(float* __restrict__ W, float* __restrict__ M1, float* __restrict__ M2, uint32_t seed) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= kModelWeights) return;
    float fan_in = kF, fan_out = kH1;
    bool bias = false;
    if (w >= kOffB1 && w < kOffW2) bias = true;
    else if (w >= kOffW2 && w < kOffB2) { fan_in = kH1; fan_out = kH2; }
    else if (w >= kOffB2 && w < kOffW3) bias = true;
    else if (w >= kOffW3 && w < kOffB3) { fan_in = kH2; fan_out = 1; }
    else if (w == kOffB3) bias = true;
    const float lim = sqrtf(6.f / (fan_in + fan_out));
    const float u = (float)(hash32((uint32_t)w * 0x85ebca6bu + seed) >> 8) * (1.f / 16777216.f);
    W[w] = bias ? (w >= kOffB1 && w < kOffW2 ? 0.01f : 0.f) : (2.f * u - 1.f) * lim;
    M1[w] = 0.f;
    M2[w] = 0.f;
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t model_init(float* W, float* M1, float* M2, uint32_t seed, cudaStream_t st) {
    k_model_init<<<blocks_for(kModelWeights, 256), 256, 0, st>>>(W, M1, M2, seed);
    return cudaGetLastError();
}

cudaError_t model_features(const JoinArgs<float>& lookup, uint32_t M, float log2_eps, uint32_t n, float* X,
                           cudaStream_t st) {
    if (M == 0) return cudaSuccess;
    k_model_features<<<blocks_for(M, 256), 256, 0, st>>>(lookup, M, log2_eps, n, X);
    return cudaGetLastError();
}

cudaError_t model_targets(const uint32_t* cell_start, const uint32_t* ids, const uint32_t* counts, uint32_t M,
                          float* Y, cudaStream_t st) {
    if (M == 0) return cudaSuccess;
    k_model_targets<<<blocks_for(M, 256), 256, 0, st>>>(cell_start, ids, counts, M, Y);
    return cudaGetLastError();
}

cudaError_t model_subsample(const float* X, const float* Y, uint32_t M, uint32_t ntr, float* Xt, float* Yt,
                            cudaStream_t st) {
    if (ntr == 0) return cudaSuccess;
    uint32_t stride = M / ntr;
    if (stride == 0) stride = 1;
    k_model_subsample<<<blocks_for(ntr, 256), 256, 0, st>>>(X, Y, M, stride, ntr, Xt, Yt);
    return cudaGetLastError();
}

cudaError_t model_predict(const float* X, uint32_t m, const float* W, float* out, const uint32_t* cell_start,
                          float nmax, double* est, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    k_model_predict<<<blocks_for(m, 256), 256, 0, st>>>(X, m, W, out, cell_start, nmax, est);
    return cudaGetLastError();
}

cudaError_t model_train(const float* X, const float* Y, uint32_t ntr, float* W, float* M1, float* M2, uint32_t t0,
                        uint32_t steps, float lr, float* loss, cudaStream_t st) {
    if (ntr == 0 || steps == 0) return cudaSuccess;
    const size_t smem = sizeof(TrainSmem);
    cudaError_t e = cudaFuncSetAttribute(k_model_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_model_train<<<1, kTT, smem, st>>>(X, Y, ntr, W, M1, M2, t0, steps, lr, loss);
    return cudaGetLastError();
}

cudaError_t model_grad(const float* X, const float* Y, uint32_t n, const float* W, float* loss, float* grad,
                       cudaStream_t st) {
    if (n == 0) return cudaErrorInvalidValue;
    const size_t smem = sizeof(TrainSmem);
    cudaError_t e = cudaFuncSetAttribute(k_model_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_model_grad<<<1, kTT, smem, st>>>(X, Y, n, W, loss, grad);
    return cudaGetLastError();
}

}  // namespace gsj
