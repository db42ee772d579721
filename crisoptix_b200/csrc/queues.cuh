// queues.cuh -- ray queues shared by the path machines (wavefront.cu) and the
// shift machines (reuse_passes.cu): warp-aggregated append, and the closest /
// shadow traversal kernels over a queue of record indices.
//
// A record type R provides closest_ray / set_hit for closest-hit rays and
// shadow_ray / set_occluded for visibility rays; the kernels only move rays
// and results, so one traversal kernel serves every kind of machine.
#pragma once

#include <algorithm>

#include "passes.cuh"

namespace crisb {
namespace {

// Warp-aggregated append of `val` to queue q (count cnt) for the lanes with
// `take` set.  Every lane of the warp must call this.
RT_D void q_append(uint32_t* q, uint32_t* cnt, bool take, uint32_t val) {
    const unsigned mask = __ballot_sync(0xffffffffu, take);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cnt, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (take) q[base + __popc(mask & ((1u << lane) - 1u))] = val;
}

// path machine records: next closest-hit ray in ray_o / ray_d, the NEE shadow
// ray from it_pos along nee_dir (w = light distance)
RT_D void closest_ray(const WfPath& w, V3& o, V3& d) {
    const float4 a = w.ray_o, b = w.ray_d;
    o = V3{a.x, a.y, a.z};
    d = V3{b.x, b.y, b.z};
}
RT_D void set_hit(WfPath& w, float4 h) { w.hit = h; }
RT_D void shadow_ray(const WfPath& w, V3& o, V3& d, float& tmax) {
    const float4 a = w.it_pos, b = w.nee_dir;
    o = V3{a.x, a.y, a.z};
    d = V3{b.x, b.y, b.z};
    tmax = b.w;
}
RT_D void set_occluded(WfPath& w, uint32_t v) { w.occluded = v; }

// shift machine records: one ray in flight in o / d
RT_D void closest_ray(const ShiftJob& j, V3& o, V3& d) {
    const float4 a = j.o, b = j.d;
    o = V3{a.x, a.y, a.z};
    d = V3{b.x, b.y, b.z};
}
RT_D void set_hit(ShiftJob& j, float4 h) { j.hit = h; }
RT_D void shadow_ray(const ShiftJob& j, V3& o, V3& d, float& tmax) {
    const float4 a = j.o, b = j.d;
    o = V3{a.x, a.y, a.z};
    d = V3{b.x, b.y, b.z};
    tmax = a.w;
}
RT_D void set_occluded(ShiftJob& j, uint32_t v) { j.hit.x = __uint_as_float(v); }

// Grid-stride loops over the queue, each lane walking its ray to the end.
// Warps lose most of their lanes to that (a warp runs 2.4x the node visits
// its rays need on the 1080p workload), but refilling finished lanes measured
// slower every time: with 4-wide nodes (per-warp batches, 31 ms against 20 ms
// of trace per frame: the per-step convergence removes the latency hiding
// between diverged inner-node and leaf lanes) and with compressed nodes
// (per-warp chunks of the queue, every idle lane refilled at once when at most
// 8-31 lanes are busy: 19.1-19.8 against 12.1 ms: lanes on different rays and
// depths no longer load the same nodes in the same instruction).
// One launch per round over both queues: entries [0, nc) of the closest-hit
// queue, then [nc, nc + ns) of the shadow queue, so the two queues' tails
// (the last, slowest rays) overlap instead of running back to back.
// Block sizes of the traversal kernel (crisb_set_trace_block, tuned by
// crisb_autotune): resident blocks per SM chosen so every size keeps the
// register budget of 9 x 128 threads (56 registers; 64 at 256 threads).
// 9 resident 128-thread blocks per SM: 13.40 -> 13.25 ms of traversal per
// 1080p frame against 8 blocks (64 registers), despite a few more spills.
template <int kB>
struct TraceShape;
template <>
struct TraceShape<64> {
    static constexpr int kMinBlocks = 18;
};
template <>
struct TraceShape<128> {
    static constexpr int kMinBlocks = 9;
};
template <>
struct TraceShape<256> {
    static constexpr int kMinBlocks = 4;
};

template <class R, int kB, int kFmt>
__global__ void __launch_bounds__(kB, TraceShape<kB>::kMinBlocks) k_q_trace(SceneView s, const uint32_t* qc,
                                                                          const uint32_t* ccnt, const uint32_t* qs,
                                                                          const uint32_t* scnt, R* rec) {
    const uint32_t nc = *ccnt, ns = *scnt;
    const uint32_t n = nc + ns;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        V3 o, d;
        if (t < nc) {
            const uint32_t i = qc[t];
            closest_ray(rec[i], o, d);
            count_ray(s, 0);
            const TraceResult h = traverse_fmt<kFmt, false>(s, make_ray(o, d), 1e-3f, 1e16f);
            set_hit(rec[i], make_float4(__uint_as_float(h.prim), h.t, h.u, h.v));
        } else {
            const uint32_t i = qs[t - nc];
            float tmax;
            shadow_ray(rec[i], o, d, tmax);
            count_ray(s, 1);
            const bool occ = traverse_fmt<kFmt, true>(s, make_ray(o, d), 1e-3f, tmax).prim != CRISB_INVALID_PRIM;
            set_occluded(rec[i], occ ? 1u : 0u);
        }
    }
}

// all blocks of `kernel` that are resident on the device at once
inline unsigned persistent_grid(const void* kernel) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPassBlock, 0) == cudaSuccess && sms > 0 &&
        per_sm > 0)
        return static_cast<unsigned>(sms * per_sm);
    return 148u * 4u;
}

inline unsigned grid_for(uint32_t n) { return (n + kPassBlock - 1) / kPassBlock; }

// all blocks of `kernel` at `block` threads resident on the device at once
inline unsigned persistent_grid_at(const void* kernel, int block) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) == cudaSuccess && sms > 0 &&
        per_sm > 0)
        return static_cast<unsigned>(sms * per_sm);
    return 148u * 4u;
}

template <class R, int kB, int kFmt>
unsigned trace_grid_of() {
    static const unsigned g = persistent_grid_at(reinterpret_cast<const void*>(k_q_trace<R, kB, kFmt>), kB);
    return g;
}

template <class R, int kFmt>
void launch_trace_fmt(uint32_t block, uint32_t m, cudaStream_t st, const SceneView& s, const uint32_t* qc,
                      const uint32_t* ccnt, const uint32_t* qs, const uint32_t* scnt, R* rec) {
    if (block == 64)
        k_q_trace<R, 64, kFmt><<<trace_grid_of<R, 64, kFmt>() * m, 64, 0, st>>>(s, qc, ccnt, qs, scnt, rec);
    else if (block == 256)
        k_q_trace<R, 256, kFmt><<<trace_grid_of<R, 256, kFmt>() * m, 256, 0, st>>>(s, qc, ccnt, qs, scnt, rec);
    else
        k_q_trace<R, 128, kFmt><<<trace_grid_of<R, 128, kFmt>() * m, 128, 0, st>>>(s, qc, ccnt, qs, scnt, rec);
}

// one traversal launch over a closest-hit and a shadow queue: `block`
// threads (64, 128 or 256) and `mult` x the blocks resident at once, the
// kernel instance of the scene tree's node format
template <class R>
void launch_trace(uint32_t block, uint32_t mult, cudaStream_t st, const SceneView& s, const uint32_t* qc,
                  const uint32_t* ccnt, const uint32_t* qs, const uint32_t* scnt, R* rec) {
    const uint32_t m = std::max(mult, 1u);
    if (s.qnodes) launch_trace_fmt<R, kFmtCompressed8>(block, m, st, s, qc, ccnt, qs, scnt, rec);
    else launch_trace_fmt<R, kFmtWide4>(block, m, st, s, qc, ccnt, qs, scnt, rec);
}

}  // namespace
}  // namespace crisb
