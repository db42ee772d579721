// tonemap.cu -- ToneMapping (src/kernel/tonemap.cu:23-39, called once per
// frame from src/main.cpp:127): linear float RGB to sRGB bytes.
//
// The byte of one channel is srgb8(c) (rt_common.cuh): the reference's curve
// in the reference's own arithmetic.  It is 0 for NaN, for negative c and for
// c above c_max (where 12.92 c overflows and the blend turns NaN), and on
// [0, c_max] a non-decreasing step function of c with 255 steps: every float
// operation in it rounds monotonically, and the power is the correctly
// rounded one except within 1e-14 of a rounding midpoint, far below the 5e-8
// relative gap between the powers of neighbouring floats.  So the kernel does
// not evaluate the curve, which costs about ninety double-precision
// operations per channel and would make this copy-shaped kernel FP64-bound.
// The host finds, once, the smallest float T[k] with srgb8(T[k]) >= k for
// k = 1..255 by bisection over float bit patterns, checks both sides of every
// step, and files the steps into 1665 buckets of float bit patterns (one
// exponent and 7 leading mantissa bits each) so that no bucket holds more
// than one step.  A bucket stores the byte at its start and the bit pattern of
// its step; the kernel copies the buckets to shared memory and finds a
// channel's byte with one bucket load and one integer compare
// (srgb8_lookup).  The bytes are the formula's by construction.
//
// Memory: 12 bytes read and 3 written per pixel.  Each thread takes four
// pixels (three 16-byte loads, three 4-byte stores) when both pointers are
// aligned for that, and the ragged tail pixel by pixel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <utility>
#include <vector>

#include "context.h"
#include "passes.cuh"

namespace crisb {
namespace {

constexpr int kToneBlock = 512;

// Buckets of float bit patterns: bucket i (1 <= i < kBuckets) holds the
// patterns [kBucketBase + (i << kBucketShift), kBucketBase + ((i + 1) <<
// kBucketShift)), i.e. one exponent and 7 leading mantissa bits between
// 2^-12 and 2; bucket 0 also holds everything below, bucket kBuckets
// everything from 2 up to c_max.
constexpr uint32_t kBucketShift = 16;                  // 23 - 7 mantissa bits
constexpr uint32_t kBucketBase = (127u - 12u) << 23;   // 2^-12
constexpr uint32_t kBuckets = 13u << (23 - kBucketShift);  // 2^-12 .. 2

struct SrgbTable {
    float t[256];  // t[0] = 0; t[k] smallest float c >= 0 with srgb8(c) >= k
    float c_max;   // largest float c with 12.92f * c finite
    // per bucket: the byte at its first pattern and the bit pattern of the
    // next step above it (0xffffffff for byte 255)
    uint2 bucket[kBuckets + 1];
};

float bits_to_float(uint32_t b) {
    float f;
    memcpy(&f, &b, sizeof f);
    return f;
}
uint32_t float_bits(float f) {
    uint32_t b;
    memcpy(&b, &f, sizeof b);
    return b;
}

SrgbTable build_srgb_table() {
    SrgbTable tab{};
    // c_max: largest float with a finite 12.92f * c (positive floats order as
    // their bit patterns)
    uint32_t lo = 0, hi = 0x7f7fffffu;  // 12.92 * 0 finite; FLT_MAX * 12.92 not
    while (hi - lo > 1) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (std::isinf(12.92f * bits_to_float(mid)))
            hi = mid;
        else
            lo = mid;
    }
    tab.c_max = bits_to_float(lo);
    const uint32_t max_bits = lo;
    if (srgb8(tab.c_max) != 255) throw std::runtime_error("sRGB table: byte below c_max is not 255");
    if (srgb8(0.0f) != 0) throw std::runtime_error("sRGB table: byte of 0 is not 0");
    tab.t[0] = 0.0f;
    uint32_t tb[257];
    tb[0] = 0;
    for (uint32_t k = 1; k < 256; ++k) {
        uint32_t a = 0, b = max_bits;  // srgb8(a) < k <= srgb8(b)
        while (b - a > 1) {
            const uint32_t mid = a + (b - a) / 2;
            if (srgb8(bits_to_float(mid)) >= k)
                b = mid;
            else
                a = mid;
        }
        tab.t[k] = bits_to_float(b);
        tb[k] = b;
        if (srgb8(tab.t[k]) < k || srgb8(bits_to_float(b - 1)) >= k || tab.t[k] < tab.t[k - 1])
            throw std::runtime_error("sRGB table: step check failed");
    }
    tb[256] = 0xffffffffu;
    // byte of pattern x (0 <= x <= max_bits): steps at or below x
    auto count = [&](uint32_t x) {
        uint32_t k = 0;
        while (k < 255 && tb[k + 1] <= x) ++k;
        return k;
    };
    if (tb[1] < kBucketBase + (1u << kBucketShift) || tb[255] >= kBucketBase + (kBuckets << kBucketShift))
        throw std::runtime_error("sRGB table: steps outside the bucketed range");
    for (uint32_t i = 0; i <= kBuckets; ++i) {
        const uint32_t first = i == 0 ? 0u : kBucketBase + (i << kBucketShift);
        const uint32_t last = i == kBuckets ? max_bits : kBucketBase + ((i + 1) << kBucketShift) - 1;
        const uint32_t b0 = count(first);
        if (count(last) > b0 + 1) throw std::runtime_error("sRGB table: two steps in one bucket");
        tab.bucket[i] = make_uint2(b0, tb[b0 + 1]);
    }
    return tab;
}

const SrgbTable& srgb_table() {
    static const SrgbTable tab = build_srgb_table();
    return tab;
}

// Byte of a channel from its bit pattern: 0 for negative (sign bit set), NaN
// and values above c_max (patterns above c_max's); otherwise the byte at the
// start of the bucket, plus one if the bucket's single step is at or below it.
RT_D uint32_t srgb8_lookup(const uint2* bucket, float c, uint32_t max_bits) {
    const uint32_t x = __float_as_uint(c);
    if (x > max_bits) return 0u;
    const uint32_t i = x < kBucketBase ? 0u : min((x - kBucketBase) >> kBucketShift, kBuckets);
    const uint2 e = bucket[i];
    return e.x + (x >= e.y ? 1u : 0u);
}

// Pixels [0, 4 * quads) four per thread with vector accesses (rgb 16-byte and
// out 4-byte aligned), pixels [4 * quads, n) one per thread.
__global__ void __launch_bounds__(kToneBlock) k_tonemap_srgb8(const float* __restrict__ rgb,
                                                             uint8_t* __restrict__ out, uint32_t n, uint32_t quads,
                                                             const uint2* __restrict__ table, uint32_t max_bits) {
    __shared__ uint2 t[kBuckets + 1];
    for (uint32_t i = threadIdx.x; i <= kBuckets; i += blockDim.x) t[i] = table[i];
    __syncthreads();
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const float4* in4 = reinterpret_cast<const float4*>(rgb);
    uint32_t* out4 = reinterpret_cast<uint32_t*>(out);
    for (uint64_t q = tid; q < quads; q += stride) {
        const float4 a = __ldcs(in4 + 3 * q);
        const float4 b = __ldcs(in4 + 3 * q + 1);
        const float4 c = __ldcs(in4 + 3 * q + 2);
        const uint32_t w0 = srgb8_lookup(t, a.x, max_bits) | srgb8_lookup(t, a.y, max_bits) << 8 |
                            srgb8_lookup(t, a.z, max_bits) << 16 | srgb8_lookup(t, a.w, max_bits) << 24;
        const uint32_t w1 = srgb8_lookup(t, b.x, max_bits) | srgb8_lookup(t, b.y, max_bits) << 8 |
                            srgb8_lookup(t, b.z, max_bits) << 16 | srgb8_lookup(t, b.w, max_bits) << 24;
        const uint32_t w2 = srgb8_lookup(t, c.x, max_bits) | srgb8_lookup(t, c.y, max_bits) << 8 |
                            srgb8_lookup(t, c.z, max_bits) << 16 | srgb8_lookup(t, c.w, max_bits) << 24;
        __stcs(out4 + 3 * q, w0);
        __stcs(out4 + 3 * q + 1, w1);
        __stcs(out4 + 3 * q + 2, w2);
    }
    for (uint64_t i = 4 * static_cast<uint64_t>(quads) + tid; i < n; i += stride) {
        const uint64_t o = 3 * i;
        out[o] = static_cast<uint8_t>(srgb8_lookup(t, rgb[o], max_bits));
        out[o + 1] = static_cast<uint8_t>(srgb8_lookup(t, rgb[o + 1], max_bits));
        out[o + 2] = static_cast<uint8_t>(srgb8_lookup(t, rgb[o + 2], max_bits));
    }
}

// the bucket table in device memory, uploaded once per CUDA context (13 KB)
// and kept for the life of that context: no handle owns it, and a table freed
// while a caller's stream still runs a tone-mapping kernel would be read after
// free.  Keyed by context id (context.h), so a context created after a
// cudaDeviceReset, or a caller's own context, gets a table of its own.
const uint2* device_table() {
    static std::mutex mu;
    static std::vector<std::pair<unsigned long long, const uint2*>> tables;
    unsigned long long ctx = 0;
    if (current_context_id(&ctx) != cudaSuccess) throw std::runtime_error("no current CUDA context");
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& t : tables)
        if (t.first == ctx) return t.second;
    void* p = nullptr;
    const SrgbTable& tab = srgb_table();
    if (cudaMalloc(&p, sizeof tab.bucket) != cudaSuccess) throw std::runtime_error("sRGB table allocation");
    if (cudaMemcpy(p, tab.bucket, sizeof tab.bucket, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p);
        throw std::runtime_error("sRGB table upload");
    }
    tables.emplace_back(ctx, static_cast<const uint2*>(p));
    return tables.back().second;
}

// blocks of the kernel resident on the whole device at once
unsigned tone_grid_cap() {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tonemap_srgb8, kToneBlock, 0) == cudaSuccess &&
        sms > 0 && per_sm > 0)
        return static_cast<unsigned>(sms * per_sm);
    return 148u * 8u;
}

}  // namespace

void srgb8_thresholds(float* t256, float* c_max) {
    const SrgbTable& tab = srgb_table();
    memcpy(t256, tab.t, sizeof tab.t);
    *c_max = tab.c_max;
}

cudaError_t launch_tonemap_srgb8(const float* rgb, uint8_t* out, uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const bool vec = (reinterpret_cast<uintptr_t>(rgb) % 16 == 0) && (reinterpret_cast<uintptr_t>(out) % 4 == 0);
    const uint32_t quads = vec ? n / 4 : 0;
    const uint32_t work = quads + (n - 4 * quads);
    static const unsigned cap = tone_grid_cap();
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((work + kToneBlock - 1) / kToneBlock, cap));
    k_tonemap_srgb8<<<grid, kToneBlock, 0, st>>>(rgb, out, n, quads, device_table(),
                                                 float_bits(srgb_table().c_max));
    return cudaGetLastError();
}

}  // namespace crisb
