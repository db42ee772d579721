// radix_sort.h -- the library's own device radix sort (replaces a library
// sort on the per-frame path of the prefix-endpoint structure).
//
// Sorts 64-bit keys stably by their high 32 bits: least-significant-digit
// first, four passes of 8 bits, each pass a per-tile histogram, a scan of the
// (digit, tile) counts and a stable scatter.  For the endpoint keys
// (Morton code << 32 | entry index, all ones for an absent entry) this is the
// order of sorting all 64 bits: entries are given in index order, equal codes
// keep it, and absent entries are identical keys.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace crisb {
namespace rsort {

// scratch bytes for sorting n keys
size_t temp_bytes(uint32_t n);

// keys_out = keys_in stably sorted by bits [32, 64); keys_in is left
// unchanged.  `temp` holds temp_bytes(n) bytes.  Enqueued on `st` (kLaunches
// launches, no host synchronisation).
cudaError_t sort_high32(const uint64_t* keys_in, uint64_t* keys_out, void* temp, size_t temp_size, uint32_t n,
                        cudaStream_t st);

// launches one sort_high32 enqueues
constexpr uint32_t kLaunches = 20;

// Exclusive prefix sum of n uint32 values (in and out may alias); the grand
// total to *total (device memory) when total is not null.  `temp` holds
// scan_temp_bytes(n) bytes.  Enqueued on `st` (3 launches).
size_t scan_temp_bytes(uint32_t n);
cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, void* temp,
                           cudaStream_t st);

}  // namespace rsort
}  // namespace crisb
