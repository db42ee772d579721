// radix_sort.cu -- rsort::sort_high32 (radix_sort.h).
#include "radix_sort.h"

#include <algorithm>

namespace crisb {
namespace rsort {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr uint32_t kTile = kThreads * kPerThread;  // keys per tile (one block)
constexpr int kBins = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kScanThreads = 1024;

inline uint32_t tiles_for(uint32_t n) { return (n + kTile - 1) / kTile; }
inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// counts of each digit in the block's tile, stored digit-major:
// hist[digit * tiles + tile]
__global__ void __launch_bounds__(kThreads) k_hist(const uint64_t* __restrict__ keys, uint32_t n, int shift,
                                                   uint32_t* __restrict__ hist, uint32_t tiles) {
    __shared__ uint32_t h[kBins];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kTile;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const uint32_t i = base + k * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[static_cast<uint32_t>(keys[i] >> shift) & (kBins - 1)], 1u);
    }
    __syncthreads();
    hist[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

// ---- exclusive scan: tile scans, a one-block scan of the tile sums, an add ----
constexpr uint32_t kScanTile = 2 * kScanThreads;

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* out,
                                                             uint32_t n, uint32_t* tile_sums) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const uint32_t base = blockIdx.x * kScanTile + 2 * threadIdx.x;
    const uint32_t a = base < n ? in[base] : 0u, b = base + 1 < n ? in[base + 1] : 0u;
    const uint32_t pair = a + b;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = pair;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_tot[lane];
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += v;
        }
        warp_tot[lane] = w;  // inclusive over the warps
    }
    __syncthreads();
    const uint32_t excl = incl - pair + (warp > 0 ? warp_tot[warp - 1] : 0u);
    if (base < n) out[base] = excl;
    if (base + 1 < n) out[base + 1] = excl + a;
    if (threadIdx.x == kScanThreads - 1) tile_sums[blockIdx.x] = warp_tot[31];
}

// exclusive scan of m tile sums in place (m is small: one per 2048 values);
// the grand total to *total when total is not null
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* sums, uint32_t m, uint32_t* total) {
    __shared__ uint32_t s[kScanThreads];
    const uint32_t per = (m + kScanThreads - 1) / kScanThreads;
    const uint32_t b = threadIdx.x * per, e = min(b + per, m);
    uint32_t sum = 0;
    for (uint32_t i = b; i < e; ++i) sum += sums[i];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const uint32_t v = threadIdx.x >= static_cast<uint32_t>(off) ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = s[threadIdx.x] - sum;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t v = sums[i];
        sums[i] = run;
        run += v;
    }
    if (total && threadIdx.x == kScanThreads - 1) *total = s[kScanThreads - 1];
}

__global__ void k_scan_add(uint32_t* out, uint32_t n, const uint32_t* __restrict__ tile_sums) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_sums[i / kScanTile];
}

inline uint32_t scan_tiles(uint32_t n) { return (std::max<uint32_t>(n, 1) + kScanTile - 1) / kScanTile; }

// Stable scatter of the block's tile: keys go in rounds of kThreads
// consecutive keys; within a round a key's rank among equal digits is its
// rank in its warp (__match_any_sync) plus the counts of the lower warps, and
// each digit's running position advances by the round's count.
__global__ void __launch_bounds__(kThreads) k_scatter(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst,
                                                      uint32_t n, int shift, const uint32_t* __restrict__ offs,
                                                      uint32_t tiles) {
    __shared__ uint32_t run[kBins];
    __shared__ uint32_t wcnt[kWarps][kBins];
    run[threadIdx.x] = offs[static_cast<size_t>(threadIdx.x) * tiles + blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lower = (1u << lane) - 1u;
    const uint32_t base = blockIdx.x * kTile;
    for (int k = 0; k < kPerThread; ++k) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        const uint32_t i = base + k * kThreads + threadIdx.x;
        const bool have = i < n;
        const uint64_t key = have ? src[i] : 0ull;
        const uint32_t d = have ? (static_cast<uint32_t>(key >> shift) & (kBins - 1)) : static_cast<uint32_t>(kBins);
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lower);
        if (have && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (have) {
            uint32_t pos = run[d] + rank;
            for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
            dst[pos] = key;
        }
        __syncthreads();
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) tot += wcnt[w][threadIdx.x];
        run[threadIdx.x] += tot;
        __syncthreads();
    }
}

}  // namespace

size_t scan_temp_bytes(uint32_t n) { return align256(static_cast<size_t>(scan_tiles(n)) * sizeof(uint32_t)); }

cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, void* temp,
                           cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t* sums = static_cast<uint32_t*>(temp);
    const uint32_t tiles = scan_tiles(n);
    k_scan_tiles<<<tiles, kScanThreads, 0, st>>>(in, out, n, sums);
    k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, tiles, total);
    k_scan_add<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(out, n, sums);
    return cudaGetLastError();
}

size_t temp_bytes(uint32_t n) {
    const size_t m = n > 0 ? n : 1;
    const uint32_t hist = kBins * tiles_for(static_cast<uint32_t>(m));
    return align256(m * sizeof(uint64_t)) + align256(static_cast<size_t>(hist) * sizeof(uint32_t)) +
           scan_temp_bytes(hist);
}

cudaError_t sort_high32(const uint64_t* keys_in, uint64_t* keys_out, void* temp, size_t temp_size, uint32_t n,
                        cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    if (temp_size < temp_bytes(n)) return cudaErrorInvalidValue;
    const uint32_t tiles = tiles_for(n);
    const uint32_t nh = kBins * tiles;
    uint64_t* alt = static_cast<uint64_t*>(temp);
    uint32_t* hist = reinterpret_cast<uint32_t*>(static_cast<char*>(temp) + align256(static_cast<size_t>(n) * 8));
    void* scan_temp = reinterpret_cast<char*>(hist) + align256(static_cast<size_t>(nh) * sizeof(uint32_t));
    // passes: in -> alt -> out -> alt -> out (keys_in untouched)
    const uint64_t* src = keys_in;
    for (int pass = 0; pass < 4; ++pass) {
        uint64_t* dst = (pass & 1) ? keys_out : alt;
        const int shift = 32 + 8 * pass;
        k_hist<<<tiles, kThreads, 0, st>>>(src, n, shift, hist, tiles);
        const cudaError_t e = exclusive_scan(hist, hist, nh, nullptr, scan_temp, st);
        if (e != cudaSuccess) return e;
        k_scatter<<<tiles, kThreads, 0, st>>>(src, dst, n, shift, hist, tiles);
        src = dst;
    }
    return cudaGetLastError();
}

}  // namespace rsort
}  // namespace crisb
