// Learned result-count model (gsj_model.cu): launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gsj_common.cuh"

namespace gsj {

constexpr int kModelFeatures = 16;
constexpr int kModelWeights = 16 * 64 + 64 + 64 * 32 + 32 + 32 + 1;  // 3201
constexpr uint32_t kModelTrainRows = 65536;  // cells sampled for training

// Deterministic initial weights (uniform Glorot), Adam moments zeroed.
cudaError_t model_init(float* W, float* M1, float* M2, uint32_t seed, cudaStream_t st);
// Per-cell features X[M][16]: `lookup` supplies the cell table (cell_key,
// cell_start, dense table or hash table, grid geometry, n_points).
cudaError_t model_features(const JoinArgs<float>& lookup, uint32_t M, float log2_eps, uint32_t n, float* X,
                           cudaStream_t st);
// Per-cell targets: log2(1 + mean list length of the cell's points).
cudaError_t model_targets(const uint32_t* cell_start, const uint32_t* ids, const uint32_t* counts, uint32_t M,
                          float* Y, cudaStream_t st);
// ntr rows spread over the M cells.
cudaError_t model_subsample(const float* X, const float* Y, uint32_t M, uint32_t ntr, float* Xt, float* Yt,
                            cudaStream_t st);
// out[c] (optional) = network output of row c; with cell_start and est
// (zeroed by the caller), *est += size_c * clamp(2^out - 1, 0, nmax).
cudaError_t model_predict(const float* X, uint32_t m, const float* W, float* out, const uint32_t* cell_start,
                          float nmax, double* est, cudaStream_t st);
// `steps` Adam steps (learning rate lr) on minibatches of the ntr rows, step
// numbers t0 + 1 ...; *loss (optional) receives the last minibatch's mean
// squared error.
cudaError_t model_train(const float* X, const float* Y, uint32_t ntr, float* W, float* M1, float* M2, uint32_t t0,
                        uint32_t steps, float lr, float* loss, cudaStream_t st);
// Mean squared error over n rows and its gradient (kModelWeights floats).
cudaError_t model_grad(const float* X, const float* Y, uint32_t n, const float* W, float* loss, float* grad,
                       cudaStream_t st);

}  // namespace gsj
