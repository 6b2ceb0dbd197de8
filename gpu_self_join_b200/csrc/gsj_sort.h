// Project-written stable LSD radix sort and run-length encoding (gsj_sort.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gsj {

// Temporary bytes of radix_sort for n keys.
size_t radix_sort_temp_bytes(uint64_t n);

// Stable sort of n < 2^32 keys (K = uint32_t or uint64_t) on bits
// [begin_bit, end_bit) in 8-bit digit passes, carrying 32-bit values when
// `vals` is non-null.  The passes alternate between the two buffers; on return
// *in_alt tells whether the sorted keys (and values) are in keys_alt/vals_alt.
// *launches (optional) is increased by the kernels launched.
template <typename K>
cudaError_t radix_sort(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int begin_bit,
                       int end_bit, void* temp, bool* in_alt, int* launches, cudaStream_t st);

// Temporary bytes of run_length for n keys.
size_t runs_temp_bytes(uint64_t n);

// Runs of equal keys in a sorted array: run_key[r] (as uint64), run_start[r]
// for r < M and run_start[M] = n, with M written to *d_nruns (device).
// run_key and run_start need n and n + 1 entries.
template <typename K>
cudaError_t run_length(const K* keys, uint64_t n, uint64_t* run_key, uint32_t* run_start, uint32_t* d_nruns,
                       void* temp, cudaStream_t st);

}  // namespace gsj
