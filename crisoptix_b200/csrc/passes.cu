// passes.cu -- the per-frame pass kernels of Conditional ReSTIR PT.
//
// The prefix-endpoint entries and search structure, the front -> back prefix
// copy, and the final gather for gatherN > 1: one thread per pixel, records
// loaded whole, updated with the reference's in-place field semantics, stored
// whole.  (Prefix temporal and spatial, suffix temporal and spatial, and the
// gatherN == 1 final gather are split into shift jobs in reuse_passes.cu.)
#define CRISB_LBVH_KERNELS 1
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
__global__ void k_store_entries(FrameParams fp, Bufs b, const SceneView s, unsigned int* ob, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t P = pixel_count(fp);
    float4 e = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    bool valid = false;
    if (i < P) {
        const uint32_t pflags = pres_flags(b.pres[fp.front], i);
        const uint32_t sflags = sres_flags(b.sres_cur, i);
        const Isect last = unpack(s, pres_last(b.pres[fp.front], i));
        if (fl_valid(pflags) && fl_valid(sflags) && last.valid) {
            float radius = fp.p.gather_radius;
            if (fp.p.gather_radius_type == CRISB_RADIUS_PATH_LENGTH) radius *= pres_path_len(b.pres[fp.front], i) / 4.5f;
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

// ---- final gather -----------------------------------------------------------------------
RT_D void write_neighbors(const FrameParams& fp, const Bufs& b, uint32_t i, const NeighborList& nl) {
    const uint32_t k = fp.k;
    for (uint32_t n = 0; n < k; ++n) {
        crisb_neighbor_rec r;
        r.pixel = n < nl.count ? nl.pix[n] : 0u;
        r.dist = n < nl.count ? nl.dist[n] : 0.0f;
        b.neighbors[static_cast<size_t>(i) * k + n] = r;
    }
    b.neigh_count[i] = nl.count;
}

// FinalGatherCanon, shader/final_gather.cu:69-188
RT_D V3 final_gather_canon(const SceneView& s, const FrameParams& fp, const Bufs& b, uint32_t i, V3 origin, V3 dir,
                           Rng& rng, NeighborList& nl, bool& queried) {
    Prefix cp;
    cp.rng = 0;
    cp.primary = cp.recon = cp.last = Hit{CRISB_INVALID_PRIM, 0.0f, 0.0f, splat(0.0f)};
    cp.flags = 0;
    cp.f = cp.prf = cp.rod = splat(0.0f);
    cp.p = cp.path_len = 0.0f;
    trace_prefix(s, fp, cp, origin, dir, rng);
    if (!fl_valid(cp.flags)) return splat(0.0f);
    if (fl_nee(cp.flags)) return cp.f / cp.p;
    Suffix cs;
    cs.rng = 0;
    cs.recon = cs.last_prefix = Hit{CRISB_INVALID_PRIM, 0.0f, 0.0f, splat(0.0f)};
    cs.flags = 0;
    cs.f = cs.prf = cs.rod = splat(0.0f);
    cs.p = 0.0f;
    trace_suffix(s, fp, cs, cp, rng);
    if (!fl_valid(cs.flags)) return splat(0.0f);
    const V3 canon_contrib = cp.f * cs.f / (cp.p * cs.p);
    const uint32_t k = fp.k;
    if (k == 0) return canon_contrib;
    const Isect last = unpack(s, cs.last_prefix);
    knn_query(b.knn(), s.err, last.pos, k, nl);
    queried = true;
    uint32_t nvalid = 0, vflags = 0;
    for (uint32_t n = 0; n < nl.count; ++n) {
        if (!fl_valid(sres_flags(b.sres_cur, nl.pix[n]))) continue;
        ++nvalid;
        vflags |= 1u << n;
    }
    V3 suffix_contrib = splat(0.0f);
    const float K = static_cast<float>(nvalid);
    float canon_mis = 1.0f;
    for (uint32_t n = 0; n < nl.count; ++n) {
        if (!(vflags & (1u << n))) continue;
        const Res<Suffix> nr = ld_sres(b.sres_cur, nl.pix[n]);
        float jac_n2c = 0.0f, jac_c2n = 0.0f;
        const V3 f_c_of_n = shift_suffix(s, nr.s, cs, jac_n2c);
        const V3 f_n_of_c = shift_suffix(s, cs, nr.s, jac_c2n);
        float nmis = mis_neighbor(f_c_of_n, nr.s.f, jac_n2c, K, 1.0f, nr.conf);
        if (nonfinite(nmis)) nmis = 0.0f;
        const V3 contrib = nmis * f_c_of_n * nr.w_sum * jac_n2c;
        if (!nonfinite(contrib)) suffix_contrib = suffix_contrib + contrib;
        canon_mis += mis_canonical(cs.f, f_n_of_c, jac_c2n, K, 1.0f, nr.conf);
    }
    V3 gather = suffix_contrib * cp.f / cp.p;
    gather = gather / static_cast<float>(nvalid + 1);
    V3 result = gather + (canon_contrib * canon_mis);
    result = result / (K + 1.0f);
    if (nonfinite(result)) return splat(0.0f);
    return result;
}

// FinalGatherNotCanon, shader/final_gather.cu:190-288
RT_D V3 final_gather_not_canon(const SceneView& s, const FrameParams& fp, const Bufs& b, V3 origin, V3 dir, Rng& rng,
                               NeighborList& nl, bool& queried) {
    const uint32_t k = fp.k;
    if (k == 0) return splat(0.0f);
    Isect last;
    last.valid = false;
    V3 tp;
    float pp;
    if (!trace_prefix_for_gather(s, tp, pp, last, origin, dir, static_cast<uint32_t>(fp.p.prefix_len), rng))
        return splat(0.0f);
    knn_query(b.knn(), s.err, last.pos, k, nl);
    queried = true;
    uint32_t nvalid = 0, vflags = 0;
    for (uint32_t n = 0; n < nl.count; ++n) {
        if (!fl_valid(sres_flags(b.sres_cur, nl.pix[n]))) continue;
        ++nvalid;
        vflags |= 1u << n;
    }
    V3 suffix_contrib = splat(0.0f);
    const float K = static_cast<float>(nvalid);
    for (uint32_t n = 0; n < nl.count; ++n) {
        if (!(vflags & (1u << n))) continue;
        const Res<Suffix> nr = ld_sres(b.sres_cur, nl.pix[n]);
        float jac_n2c = 0.0f;
        const V3 f_c_of_n = shift_suffix(s, nr.s, last, jac_n2c);
        float nmis = mis_neighbor(f_c_of_n, nr.s.f, jac_n2c, K, 1.0f, nr.conf);
        if (nonfinite(nmis)) nmis = 0.0f;
        const V3 contrib = nmis * f_c_of_n * nr.w_sum * jac_n2c;
        if (!nonfinite(contrib)) suffix_contrib = suffix_contrib + contrib;
    }
    V3 result = suffix_contrib * tp / pp;
    result = result / static_cast<float>(fp.p.gather_n);
    result = result / (K + 1.0f);
    if (nonfinite(result)) return splat(0.0f);
    return result;
}

// GetRadiance + __raygen__final_gather, shader/final_gather.cu:290-356
__global__ void __launch_bounds__(kPassBlock) k_final_gather(SceneView s, FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const uint32_t x = i % fp.width, y = i / fp.width;
    NeighborList nl;
    nl.count = 0;
    bool queried = false;
    V3 L = splat(0.0f);
    if (b.canon_prefix[i].primary.prim != CRISB_INVALID_PRIM) {
        Rng rng{b.gbuf[i].rng};
        const V3 dir = camera_dir(fp, x, y, rng);
        const V3 origin = ld3(fp.cam.pos);
        L = L + final_gather_canon(s, fp, b, i, origin, dir, rng, nl, queried);
        for (int g = 1; g < fp.p.gather_n; ++g) L = L + final_gather_not_canon(s, fp, b, origin, dir, rng, nl, queried);
        if (nonfinite(L)) L = splat(0.0f);
        b.gbuf[i].rng = rng.state;
    }
    if (!queried) nl.count = 0;
    if (fp.k > 0) write_neighbors(fp, b, i, nl);
    else b.neigh_count[i] = 0;
    store_output(fp, out, i, L);
}

inline unsigned grid_for(uint32_t n) { return (n + kPassBlock - 1) / kPassBlock; }

}  // namespace

void launch_prefix_copy_front_back(const FrameParams& fp, const Bufs& b, cudaStream_t st) {
    k_prefix_copy<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
}
void launch_store_entries(const SceneView& s, const FrameParams& fp, const Bufs& b, const lbvh::Work& w,
                          unsigned int* bounds, cudaStream_t st) {
    k_bounds_init<<<1, 32, 0, st>>>(bounds, w.n);
    k_store_entries<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, s, bounds, w.n);
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
void launch_final_gather(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out, cudaStream_t st) {
    k_final_gather<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b, out);
}

}  // namespace crisb
