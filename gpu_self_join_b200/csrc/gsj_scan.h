// Project-written prefix sums used to lay out the neighbour table.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gsj {
// Temporary bytes needed by scan_u32_u64 for n inputs.
size_t scan_u32_u64_temp_bytes(uint64_t n);
// out[i] = sum_{j<i} in[j] for i in [0, n]; out[n] is the total.
cudaError_t scan_u32_u64(const uint32_t* in, uint64_t* out, uint64_t n, void* temp, cudaStream_t st);
// The same with 32-bit outputs (the caller guarantees that the total fits);
// temp as for scan_u32_u64.
cudaError_t scan_u32_u32(const uint32_t* in, uint32_t* out, uint64_t n, void* temp, cudaStream_t st);
}  // namespace gsj
