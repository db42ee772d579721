// passes.cu -- the per-frame pass kernels of Conditional ReSTIR PT.
//
// The prefix-endpoint entries and search structure and the front -> back
// prefix copy: one thread per pixel.  (The reuse passes and the final gather
// are split into shift jobs in reuse_passes.cu.)
#define CRISB_LBVH_KERNELS 1
#include "coalesce.cuh"
#include "records.cuh"

namespace crisb {

namespace {

__global__ void k_prefix_copy(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    copy_pres(b.pres[fp.back], b.pres[fp.front], i);
}

__global__ void k_bounds_init(unsigned int* ob, uint32_t* n) {
    if (threadIdx.x < 3) ob[threadIdx.x] = float_to_ordered(INFINITY);
    else if (threadIdx.x < 6) ob[threadIdx.x] = float_to_ordered(-INFINITY);
    if (threadIdx.x == 0) *n = 0;
}

// __raygen__prefix_store_entries, shader/prefix_store_entries.cu:9-53: the
// endpoint of the front prefix and the radius the search tests against,
// (aabb.maxX - aabb.minX) / 2 (shader/prefix_search_hit.cu:42).
// kStage: the front prefix reservoirs of a warp's 32 pixels are one
// contiguous run, loaded through shared memory (coalesce.cuh; 20 KB per
// block), and the flags, last vertex and path length taken from the words.
// Otherwise each thread reads its own reservoir's three fields: the instance
// for views rendering at once, whose kernels stay clear of large shared
// memory blocks.
template <bool kStage>
__global__ void k_store_entries(FrameParams fp, Bufs b, const SceneView s, unsigned int* ob, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t P = pixel_count(fp);
    float4 e = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    bool valid = false;
    uint32_t pflags = 0;
    Hit plast{};
    float plen = 0.0f;
    if constexpr (!kStage) {
        if (i < P) {
            pflags = pres_flags(b.pres[fp.front], i);
            plast = pres_last(b.pres[fp.front], i);
            plen = pres_path_len(b.pres[fp.front], i);
        }
    } else {
        __shared__ uint4 stage[kPassBlock / 32][WarpRows<9>::kStage];
        if (b.pres[fp.front].f16) {
            static_assert(sizeof(crisb_prefix_res16_rec) == 5 * 16, "FP16 prefix reservoir size");
            uint4 w[5];
            warp_load_rows<5>(static_cast<const uint4*>(b.pres[fp.front].p), i, w, i < P, stage[threadIdx.x >> 5]);
            crisb_prefix_res16_rec o;
            memcpy(&o, w, sizeof(o));
            pflags = o.flags;
            plast = unpack_hit16(o.last);
            plen = o.path_len;
        } else {
            static_assert(sizeof(crisb_prefix_res_rec) == 9 * 16, "FP32 prefix reservoir size");
            uint4 w[9];
            warp_load_rows<9>(static_cast<const uint4*>(b.pres[fp.front].p), i, w, i < P, stage[threadIdx.x >> 5]);
            const Prefix pr = prefix_of_words(reinterpret_cast<const uint4 (&)[8]>(w));
            pflags = pr.flags;
            plast = pr.last;
            plen = pr.path_len;
        }
    }
    if (i < P) {
        const uint32_t sflags = sres_flags(b.sres_cur, i);
        const Isect last = unpack(s, plast);
        if (fl_valid(pflags) && fl_valid(sflags) && last.valid) {
            float radius = fp.p.gather_radius;
            if (fp.p.gather_radius_type == CRISB_RADIUS_PATH_LENGTH) radius *= plen / 4.5f;
            const float minx = last.pos.x - radius, maxx = last.pos.x + radius;
            e = make_float4(last.pos.x, last.pos.y, last.pos.z, (maxx - minx) / 2.0f);
            valid = true;
        }
        b.entries[i] = e;
    }
    // block-level bounds of valid endpoints, then one atomic per block
    __shared__ float smin[3][kPassBlock], smax[3][kPassBlock];
    __shared__ uint32_t scount[kPassBlock];
    smin[0][threadIdx.x] = valid ? e.x : INFINITY;
    smin[1][threadIdx.x] = valid ? e.y : INFINITY;
    smin[2][threadIdx.x] = valid ? e.z : INFINITY;
    smax[0][threadIdx.x] = valid ? e.x : -INFINITY;
    smax[1][threadIdx.x] = valid ? e.y : -INFINITY;
    smax[2][threadIdx.x] = valid ? e.z : -INFINITY;
    scount[threadIdx.x] = valid ? 1u : 0u;
    __syncthreads();
    for (int off = kPassBlock / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int a = 0; a < 3; ++a) {
                smin[a][threadIdx.x] = fminf(smin[a][threadIdx.x], smin[a][threadIdx.x + off]);
                smax[a][threadIdx.x] = fmaxf(smax[a][threadIdx.x], smax[a][threadIdx.x + off]);
            }
            scount[threadIdx.x] += scount[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && scount[0] > 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&ob[a], float_to_ordered(smin[a][0]));
            atomicMax(&ob[3 + a], float_to_ordered(smax[a][0]));
        }
        atomicAdd(count, scount[0]);
    }
}

__global__ void k_knn_keys(FrameParams fp, Bufs b, lbvh::Work w, const unsigned int* ob) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const float4 e = b.entries[i];
    uint64_t key = ~0ull;
    if (e.w >= 0.0f) {
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = ordered_to_float(ob[a]);
            hi[a] = ordered_to_float(ob[3 + a]);
        }
        key = lbvh::morton_key(lo, hi, e.x, e.y, e.z, i);
    }
    w.keys_in[i] = key;
}

__global__ void k_knn_leaves(FrameParams fp, Bufs b, lbvh::Work w, float4* leaf_entries) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *w.n) return;
    const uint32_t pix = static_cast<uint32_t>(w.keys[i] & 0xFFFFFFFFull);
    w.order[i] = pix;
    const float4 e = b.entries[pix];
    leaf_entries[i] = e;
    w.leaf_box[i] = entry_box(e);
}

inline unsigned grid_for(uint32_t n) { return (n + kPassBlock - 1) / kPassBlock; }

}  // namespace

void launch_prefix_copy_front_back(const FrameParams& fp, const Bufs& b, cudaStream_t st) {
    k_prefix_copy<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
}
void launch_store_entries(const SceneView& s, const FrameParams& fp, const Bufs& b, const lbvh::Work& w,
                          unsigned int* bounds, cudaStream_t st) {
    k_bounds_init<<<1, 32, 0, st>>>(bounds, w.n);
    if (fp.shared_stage) k_store_entries<true><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, s, bounds, w.n);
    else k_store_entries<false><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, s, bounds, w.n);
    k_knn_keys<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, w, bounds);
}
void launch_knn_finish(const FrameParams& fp, const Bufs& b, const lbvh::Work& w, float4* leaf_entries,
                       cudaStream_t st) {
    const uint32_t P = fp.width * fp.height;
    k_knn_leaves<<<grid_for(P), kPassBlock, 0, st>>>(fp, b, w, leaf_entries);
    launch_lbvh_hierarchy(w, P, kKnnLeafMax, st);
}
void launch_lbvh_hierarchy(const lbvh::Work& w, uint32_t cap, int leaf_max, cudaStream_t st) {
    const unsigned g = grid_for(cap > 1 ? cap : 1);
    lbvh::k_karras<<<g, kPassBlock, 0, st>>>(w);
    lbvh::k_refit<<<g, kPassBlock, 0, st>>>(w);
    lbvh::k_emit<<<g, kPassBlock, 0, st>>>(w, leaf_max);
}

}  // namespace crisb
