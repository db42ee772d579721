// passes.cuh -- declarations shared by the pass kernels and the host side.
#pragma once

#include <cuda_runtime.h>

#include "knn.cuh"
#include "rt_restir.cuh"
#include "wavefront.cuh"

namespace crisb {

// State of one shift job between its rays (80 bytes).  A job replays the
// source path's bounces from the destination vertex (closest-hit rays) and
// then tests the reconnection edge (one shadow ray); everything that does not
// depend on visibility is evaluated before that ray is queued.
struct ShiftJob {
    float4 o;      // ray origin xyz; w = shadow ray length
    float4 d;      // ray direction xyz
    float4 hit;    // closest-hit result (triangle bits, t, u, v); x = occluded flag after a shadow ray
    float4 acc;    // during replays: throughput xyz; before the shadow ray: shifted f xyz, Jacobian w
    uint64_t rng;  // replay RNG of the source path
    uint32_t code; // job code: pixel << 6 | slot
    uint32_t ctr;  // replays left after the ray in flight
};

// A reservoir buffer in one of the two storage layouts: crisb_*_res_rec
// (FP32) or crisb_*_res16_rec (FP16, f16 != 0).
struct PresBuf {
    void* p;
    uint32_t f16;
};
struct SresBuf {
    void* p;
    uint32_t f16;
};

// Device buffers of one renderer.  Prefix reservoirs keep the reference's
// front/back pair; suffix reservoirs live in two physical buffers where
// `sres_cur` holds the state every logical copy front -> back has made equal
// and the temporal pass and each spatial round write `sres_next` (then the
// roles swap), so every read sees the pass-start state.
// bits of the per-pixel byte beside each suffix reservoir buffer
constexpr uint8_t kNvalNeighbor = 1;  // usable as a spatial neighbour: valid primary hit and sample
constexpr uint8_t kNvalSpatial = 2;   // takes part in the next spatial round: valid prefix (not NEE),
                                      // canonical suffix and sample
constexpr uint8_t kNvalSample = 4;    // valid reservoir sample

struct Bufs {
    PresBuf pres[2];
    crisb_prefix_rec* canon_prefix;
    SresBuf sres_cur;
    SresBuf sres_next;
    // per pixel, beside each suffix reservoir buffer, written with the
    // reservoir: kNval* bits, so that the spatial selection and the gather
    // query test one dense byte instead of flag words of large records
    uint8_t* nval_cur;
    uint8_t* nval_next;
    crisb_suffix_res_rec* canon_suffix;  // 112-byte slots, w_sum/confidence unused
    crisb_gbuffer_rec* gbuf;
    crisb_neighbor_rec* neighbors;  // P * k
    uint32_t* neigh_count;          // P
    float4* entries;                // P: endpoint xyz + radius (w < 0: no entry)
    // prefix-endpoint search structure (rebuilt every frame)
    const BvhNode* knn_nodes;
    const float4* knn_leaf;  // leaf order: endpoint xyz + radius
    const uint32_t* knn_pixel;  // leaf order -> pixel index
    const uint32_t* knn_n;
    // split suffix passes: per-pixel status / valid-neighbour flags, spatial
    // neighbour pixels, the compacted shift-job list and the shift results
    uint32_t* pass_status;  // P
    uint32_t* pass_flags;   // P
    uint32_t* spatial_nbr;  // P * slots / 2
    uint32_t* job_items;    // P * slots
    uint32_t* job_count;    // 1
    float4* shift_out;      // P * slots: shifted f (xyz) and Jacobian (w)
    crisb_suffix_res_rec* gather_cs;  // P: canonical suffix of the final gather
    // gatherN > 1 only (else null): per pixel the camera ray direction (xyz, w
    // = 1 when the gather ran), the radiance accumulated over the gathers, and
    // the current extra prefix's throughput and pdf; its last vertex
    float4* gather_ext;     // P * 3
    crisb_hit_rec* gather_last;  // P
    float4* gather_state;   // P * 3: prefix f / p, canonical contribution, direct result
    uint32_t slots;         // job slots per pixel (>= 2 * max(k, spatial count, 1))
    // capacity of the shift machines' job records and queues; list entries
    // beyond it run in k_shift_overflow, tracing their rays in place
    uint32_t job_cap;
    // statistics level 2 only (else null): bytes read and written by each
    // resampling kernel for the work present in the frame (kTally*)
    unsigned long long* tally;
    // wavefront path tracing: one path state per pixel, ray queues of two
    // rounds (closest, shadow) x 2 and their counts
    WfPath* wf;
    uint32_t* wf_queue[4];
    uint32_t* wf_count;          // 4
    crisb_prefix_rec* gather_cp; // canonical prefix of the final gather
    // shift machines: one record per job of the list, ray queues of two
    // rounds (closest, shadow) x 2 and their counts
    ShiftJob* jobs;         // P * slots
    uint32_t* job_queue[4]; // P * slots each
    uint32_t* job_qcount;   // 4

    RT_HD KnnView knn() const { return KnnView{knn_nodes, knn_leaf, knn_pixel, knn_n}; }
};

constexpr int kPassBlock = 128;

// kernel classes of the per-kernel timing
enum KernelClass : int {
    kClsTrace = 0,     // closest-hit / shadow traversal of the path queues
    kClsShift = 1,     // shift jobs
    kClsResample = 2,  // MIS + reservoir streaming, neighbour selection
    kClsSearch = 3,    // prefix-endpoint entries, structure build, queries
    kClsOther = 4,
    kClsShade = 5,     // path-machine shading steps and per-pass finish kernels
};

// pass_status of a pixel after a wavefront init kernel
constexpr uint32_t kWfIdle = 0;  // no path ran for the pixel
constexpr uint32_t kWfPath = 4;  // a path ran for the pixel

// called after each kernel launch when per-kernel timing is on
struct Marker {
    virtual void mark(int cls, cudaStream_t st) = 0;
};
constexpr int kKnnLeafMax = 8;
constexpr int kTriLeafMax = 4;
// binary levels of SAH splits before the scene builder switches to median splits
constexpr int kMedianDepth = 40;

void launch_prefix_spatial(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out, int round,
                           cudaStream_t st, Marker* m);
void launch_prefix_copy_front_back(const FrameParams& fp, const Bufs& b, cudaStream_t st);
// reuse passes as per-pixel kernel -> compacted shift jobs -> per-pixel combine
void launch_prefix_gen_temp_split(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out,
                                  cudaStream_t st, Marker* m);
void launch_suffix_gen_temp(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m);
void launch_suffix_spatial(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m);
void launch_final_gather_split(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out,
                               cudaStream_t st, Marker* m);
// wavefront path tracing (wavefront.cu): init + rounds of trace / shade
void launch_wf_prefix(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m);
void launch_wf_suffix(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m);
void launch_wf_gather(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m);
// kernels of one wavefront pass of `flow` (0 prefix, 1 suffix, 2 gather)
uint32_t wf_launches_per_pass(const FrameParams& fp, int flow);
// kernels of one shift-job phase (begin + rounds of closest / shadow / step)
uint32_t shift_launches_per_phase();
// kernels the prefix pass adds after its combine (the reprojection back copy)
uint32_t prefix_pass_extra_launches(const FrameParams& fp);
// prefix entries, endpoint bounds/count and Morton keys (w.keys_in); the
// caller then sorts w.keys_in into w.keys and calls launch_knn_finish
void launch_store_entries(const SceneView& s, const FrameParams& fp, const Bufs& b, const lbvh::Work& w,
                          unsigned int* bounds, cudaStream_t st);
void launch_knn_finish(const FrameParams& fp, const Bufs& b, const lbvh::Work& w, float4* leaf_entries,
                       cudaStream_t st);

// path-replay adjoint of the frozen-sampling path tracer (adjoint.cu)
void adjoint_forward(const SceneView& eval, const crisb_material* sample_mats, uint32_t num_mats,
                     const FrameParams& fp, float* out, cudaStream_t st);
void adjoint_backward(const SceneView& eval, const crisb_material* sample_mats, uint32_t num_mats,
                      const FrameParams& fp, const float* d_img, float* g_mat, float* g_em, cudaStream_t st);
// path-replay adjoint of the final gather's resampled estimator of the last
// frame (restir_adjoint.cu): `b` holds that frame's state, frame_mats and
// frame_emitters the tables it was rendered with; `pairs` is scratch of
// width * height * k float4 (one per pixel and final-gather neighbour)
void restir_adjoint_forward(const SceneView& eval, const crisb_material* frame_mats,
                            const crisb_emitter* frame_emitters, uint32_t num_mats, const FrameParams& fp,
                            const Bufs& b, float4* pairs, float* out, cudaStream_t st);
void restir_adjoint_backward(const SceneView& eval, const crisb_material* frame_mats,
                             const crisb_emitter* frame_emitters, uint32_t num_mats, const FrameParams& fp,
                             const Bufs& b, float4* pairs, const float* d_img, float* g_mat, float* g_em,
                             cudaStream_t st);
// sRGB tone mapping of n float RGB pixels to bytes (tonemap.cu)
cudaError_t launch_tonemap_srgb8(const float* rgb, uint8_t* out, uint32_t n, cudaStream_t st);
// the kernel's step table: t256[k] smallest float with byte >= k, and c_max
void srgb8_thresholds(float* t256, float* c_max);
// generic LBVH stages over `cap` primitives (count in w.n)
void launch_lbvh_hierarchy(const lbvh::Work& w, uint32_t cap, int leaf_max, cudaStream_t st);

}  // namespace crisb
