// Pair keys -> neighbour table without a global sort, and per-list sorting
// (gsj_place.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gsj {

// Temporary bytes of place_pairs / find_long_lists for nlists lists.
size_t place_temp_bytes(uint64_t nlists);

// Lists of the packed keys (query id << shift | neighbour id; entries equal
// to ~0 are skipped): counts[q] (nlists + 1 entries), offsets (exclusive
// prefix, nlists + 1 entries), and each neighbour id at a free place of its
// query's list in table (capacity cap).  cursor: nlists scratch counters.
// *err (device, zeroed by the caller) is set when a key falls outside its
// list.  The order within a list is arbitrary until the lists are sorted.
cudaError_t place_pairs(const unsigned long long* keys, uint64_t nkeys, uint32_t shift, uint32_t nlists,
                        uint32_t* counts, uint64_t* offsets, uint32_t* table, uint64_t cap, uint32_t* cursor,
                        uint32_t* err, void* temp, int num_sms, int* launches, cudaStream_t st);

// Sorts every list of min_len+1 .. 256 entries ascending (a warp per list;
// shorter lists are left as they are) and gathers the indices of the longer
// lists into temp: *h_nlong receives their number, *h_nvery the number above
// 4096 entries (synchronises the stream).  List l is table[offsets[l] ..
// offsets[l+1]) (OffT = uint64_t or uint32_t).  d_nlong: two device words.
template <typename OffT>
cudaError_t sort_short_lists(uint32_t* table, const OffT* offsets, uint32_t nlists, uint32_t min_len, void* temp,
                             uint32_t* d_nlong, uint32_t* h_nlong, uint32_t* h_nvery, int num_sms, int* launches,
                             cudaStream_t st);
// Sorts the lists gathered by sort_short_lists (ids below 2^id_bits): a CTA
// bitonic network up to 4096 entries; above that LSD radix passes using the
// same ranges of `scratch` (as large as the table; needed only when nvery > 0)
// as a second buffer.
template <typename OffT>
cudaError_t sort_long_lists(uint32_t* table, uint32_t* scratch, const OffT* offsets, const void* temp,
                            uint32_t nlong, uint32_t nvery, uint32_t id_bits, int num_sms, int* launches,
                            cudaStream_t st);

}  // namespace gsj
