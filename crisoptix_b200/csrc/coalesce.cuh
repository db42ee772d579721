// coalesce.cuh -- a warp's records of consecutive indices moved through
// shared memory, so that every memory instruction covers 512 contiguous bytes
// instead of 32 records' 16-byte pieces at the record stride.
//
// Every lane of the warp calls these with its own record index i, the warp's
// indices consecutive (i = the warp's first index + lane, as in pixel-parallel
// kernels whose block size is a multiple of 32).  Lanes with `valid` false
// neither read nor write their record: the memory behind them is never
// touched, so indices past the end of the array are safe to pass.  `stage`
// is kStage 16-byte words of shared memory for the calling warp alone; a
// padding word per record keeps both the lane-major and the row-major
// accesses free of bank conflicts.
#pragma once

#include <cstdint>

namespace crisb {

template <int kW>
struct WarpRows {
    static constexpr int kStage = 32 * (kW + 1);
};

template <int kW>
__device__ inline void warp_store_rows(uint4* base, uint32_t i, const uint4 (&w)[kW], bool valid, uint4* stage) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (vmask == 0u) return;
#pragma unroll
    for (int k = 0; k < kW; ++k) stage[lane * (kW + 1) + k] = w[k];
    __syncwarp();
    const size_t first = static_cast<size_t>(i - lane) * kW;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
        const uint32_t c = lane + 32u * static_cast<uint32_t>(k);
        const uint32_t r = c / kW, q = c % kW;
        if ((vmask >> r) & 1u) base[first + c] = stage[r * (kW + 1) + q];
    }
    __syncwarp();
}

template <int kW>
__device__ inline void warp_load_rows(const uint4* base, uint32_t i, uint4 (&w)[kW], bool valid, uint4* stage) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (vmask == 0u) return;
    const size_t first = static_cast<size_t>(i - lane) * kW;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
        const uint32_t c = lane + 32u * static_cast<uint32_t>(k);
        const uint32_t r = c / kW, q = c % kW;
        if ((vmask >> r) & 1u) stage[r * (kW + 1) + q] = base[first + c];
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kW; ++k) w[k] = stage[lane * (kW + 1) + k];
    __syncwarp();
}

}  // namespace crisb
