// wavefront.cu -- the wavefront engine that runs the path machines of
// wavefront.cuh for one pass: an init kernel starts one path per pixel, then
// each round traces the queued closest-hit rays and shadow rays in two
// dedicated traversal kernels and resumes every path whose ray finished in a
// shading kernel, which queues the path's next ray for the following round.
//
// Flows (which records a path writes):
//   prefix: TracePrefix into the canonical prefix record (prefix pass);
//   suffix: TraceSuffix into the canonical suffix record from the pixel's
//           reservoir prefix (suffix temporal pass);
//   gather: TracePrefix, then TraceSuffix when the prefix ends without NEE,
//           into fresh records (final gather, FinalGatherCanon).
#include <algorithm>
#include <cstddef>
#include <mutex>

#include "coalesce.cuh"
#include "queues.cuh"
#include "records.cuh"

namespace crisb {

namespace {

RT_D void wf_push(const Bufs& b, int round, int req, uint32_t i) {
    q_append(b.wf_queue[2 * round], &b.wf_count[2 * round], req == kReqClosest, i);
    q_append(b.wf_queue[2 * round + 1], &b.wf_count[2 * round + 1], req == kReqShadow, i);
}

RT_D WfPath wf_blank() {
    WfPath w;
    w.rng = 0;
    w.phase = kPhDone;
    w.ctr = 0;
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.ray_o = w.ray_d = w.it_pos = w.it_nrm = w.it_dir = w.nee_dir = w.nee_col = w.nee_brdf = w.hit = z;
    w.occluded = 0;
    w.pad[0] = w.pad[1] = w.pad[2] = 0;
    return w;
}

RT_D Suffix fresh_suffix() {
    Suffix cs;
    cs.rng = 0;
    cs.recon = cs.last_prefix = Hit{CRISB_INVALID_PRIM, 0.0f, 0.0f, splat(0.0f)};
    cs.flags = 0;
    cs.f = cs.prf = cs.rod = splat(0.0f);
    cs.p = 0.0f;
    return cs;
}

RT_D Prefix fresh_prefix() {
    Prefix cp;
    cp.rng = 0;
    cp.primary = cp.recon = cp.last = Hit{CRISB_INVALID_PRIM, 0.0f, 0.0f, splat(0.0f)};
    cp.flags = 0;
    cp.f = cp.prf = cp.rod = splat(0.0f);
    cp.p = cp.path_len = 0.0f;
    return cp;
}

// A machine step's record: the running values (flags, f, postReconF, p, path
// length, reconOutDir) move every step, the vertex fields only when the step
// set them (kSet*); the rng and first-vertex fields are written when the
// record is started, by a whole-record store.
RT_D Prefix ld_prefix_run(const crisb_prefix_rec& r) {
    Prefix p;
    ld_prefix_tail_v(r, p);
    return p;
}
RT_D void st_prefix_step(crisb_prefix_rec& r, const Prefix& p, uint32_t set) {
    if (set & kSetPrimary) st_hit(r.primary, p.primary);
    if (set & kSetRecon) st_hit(r.recon, p.recon);
    if (set & kSetLast) st_hit(r.last, p.last);
    st_prefix_tail_v(r, p);
}
RT_D Suffix ld_suffix_run(const crisb_suffix_rec& r) {
    Suffix s;
    s.flags = r.flags;
    s.f = ld3(r.f);
    s.prf = ld3(r.post_recon_f);
    s.p = r.p;
    s.rod = ld3(r.recon_out_dir);
    return s;
}
RT_D void st_suffix_step(crisb_suffix_rec& r, const Suffix& s, uint32_t set) {
    if (set & kSetRecon) st_hit(r.recon, s.recon);
    r.flags = s.flags;
    st3(r.f, s.f);
    st3(r.post_recon_f, s.prf);
    r.p = s.p;
    st3(r.recon_out_dir, s.rod);
}

// a whole reservoir slot (112 bytes) as seven 16-byte stores
RT_D void st_suffix_slot(crisb_suffix_res_rec& slot, const Suffix& sfx) {
    crisb_suffix_res_rec o;
    st_suffix(o.sample, sfx);
    o.sample.pad = 0u;
    o.w_sum = 0.0f;
    o.confidence = 0.0f;
    st_rec(&slot, 0, o);
}

// Path records move between rounds field group by field group.  A step after
// a closest hit reads the header (rng, phase, ctr), the ray and the hit; a
// shadow or reconnection step reads the whole record.  A step writes the
// header and the groups of the phase it leaves the path in: the next ray
// (hit phases), the interaction and light (shadow phases), the ray and the
// NEE BRDF (reconnection); a finished path only its header.  Fields a later
// step reads are therefore always current in memory, and the hit / occluded
// words written by the traversal kernels are never overwritten.
static_assert(offsetof(WfPath, ray_o) == 16, "WfPath header is one 16-byte chunk");

RT_D WfPath wf_load(const WfPath* rec, uint32_t i) {
    const WfPath* r = rec + i;
    const uint4 h = *reinterpret_cast<const uint4*>(r);
    const uint32_t phase = h.z;
    if (phase != kPhPreHit && phase != kPhSufHit) return *r;
    WfPath w;
    w.rng = static_cast<uint64_t>(h.x) | (static_cast<uint64_t>(h.y) << 32);
    w.phase = h.z;
    w.ctr = h.w;
    w.ray_o = r->ray_o;
    w.ray_d = r->ray_d;
    w.hit = r->hit;
    w.occluded = 0u;
    return w;
}

RT_D void wf_store(WfPath* rec, uint32_t i, const WfPath& w) {
    WfPath* r = rec + i;
    *reinterpret_cast<uint4*>(r) =
        make_uint4(static_cast<uint32_t>(w.rng), static_cast<uint32_t>(w.rng >> 32), w.phase, w.ctr);
    if (w.phase == kPhPreHit || w.phase == kPhSufHit) {
        r->ray_o = w.ray_o;
        r->ray_d = w.ray_d;
    } else if (w.phase == kPhPreShadow || w.phase == kPhSufShadow) {
        r->it_pos = w.it_pos;
        r->it_nrm = w.it_nrm;
        r->it_dir = w.it_dir;
        r->nee_dir = w.nee_dir;
        r->nee_col = w.nee_col;
    } else if (w.phase == kPhSufRecon) {
        r->ray_o = w.ray_o;
        r->ray_d = w.ray_d;
        r->nee_brdf = w.nee_brdf;
    }
}

// ---- init kernels (round 0 requests) ----------------------------------------------
// The canonical prefix records of a warp's 32 pixels are one contiguous 4 KB
// run.  kStage: they move through shared memory (warp_load_rows /
// warp_store_rows; 18 KB per block).  Otherwise each thread moves its own
// record's eight 16-byte words and the kernel uses no shared memory, which is
// the instance for views rendering at once (the staged one slowed a 16-view
// batch by 5%).  Every lane calls both; lanes with `valid` false are untouched.
template <bool kStage>
struct PrefixRows {
    uint4* stage = nullptr;
    RT_D PrefixRows() {
        if constexpr (kStage) {
            __shared__ uint4 rows[kPassBlock / 32][WarpRows<8>::kStage];
            stage = rows[threadIdx.x >> 5];
        }
    }
    RT_D void load(const crisb_prefix_rec* base, uint32_t i, uint4 (&w)[8], bool valid) const {
        if constexpr (kStage) {
            warp_load_rows<8>(reinterpret_cast<const uint4*>(base), i, w, valid, stage);
        } else if (valid) {
            const uint4* s = reinterpret_cast<const uint4*>(base + i);
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = s[k];
        }
    }
    RT_D void store(crisb_prefix_rec* base, uint32_t i, const uint4 (&w)[8], bool valid) const {
        if constexpr (kStage) {
            warp_store_rows<8>(reinterpret_cast<uint4*>(base), i, w, valid, stage);
        } else if (valid) {
            uint4* d = reinterpret_cast<uint4*>(base + i);
#pragma unroll
            for (int k = 0; k < 8; ++k) d[k] = w[k];
        }
    }
};

template <bool kStage>
__global__ void __launch_bounds__(kPassBlock) k_wf_init_prefix(FrameParams fp, Bufs b) {
    const PrefixRows<kStage> rows;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < pixel_count(fp);
    uint4 rec[8];
    rows.load(b.canon_prefix, i, rec, in);
    int req = kReqDone;
    if (in) {
        const uint32_t x = i % fp.width, y = i / fp.width;
        Rng rng = rng_seeded(tea64(i, fp.random));
        const V3 dir = camera_dir(fp, x, y, rng);
        Prefix pre = prefix_of_words(rec);
        WfPath w = wf_blank();
        req = pre_begin(fp, pre, w, ld3(fp.cam.pos), dir, rng);
        words_of_prefix(pre, rec);
        w.rng = rng.state;
        wf_store(b.wf, i, w);
        b.pass_status[i] = kWfPath;
    }
    rows.store(b.canon_prefix, i, rec, in);
    wf_push(b, 0, req, i);
}

template <bool kTex>
__global__ void __launch_bounds__(kPassBlock) k_wf_init_suffix(SceneView s, FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int req = kReqDone;
    if (i < pixel_count(fp)) {
        const uint32_t pflags = pres_flags(b.pres[fp.front], i);
        if (!fl_valid(pflags) || fl_nee(pflags)) {
            Res<Suffix> cur = ld_sres(b.sres_cur, i);
            invalidate(cur);
            st_sres(b.sres_next, i, cur);  // the temporal pass writes sres_next
            b.nval_next[i] = 0;
            b.pass_status[i] = kWfIdle;
        } else {
            Rng rng{b.gbuf[i].rng};
            Suffix suf = ld_suffix(ld_rec<crisb_suffix_res_rec>(b.canon_suffix, i).sample);
            WfPath w = wf_blank();
            req = suf_begin<kTex>(s, fp, suf, w, pflags, pres_last(b.pres[fp.front], i), rng);
            st_suffix_slot(b.canon_suffix[i], suf);
            w.rng = rng.state;
            wf_store(b.wf, i, w);
            b.pass_status[i] = kWfPath;
        }
    }
    wf_push(b, 0, req, i);
}

template <bool kStage>
__global__ void __launch_bounds__(kPassBlock) k_wf_init_gather(FrameParams fp, Bufs b) {
    const PrefixRows<kStage> rows;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int req = kReqDone;
    uint4 rec[8];
    bool started = false;
    if (i < pixel_count(fp)) {
        if (b.canon_prefix[i].primary.prim == CRISB_INVALID_PRIM) {
            b.pass_status[i] = kWfIdle;
            if (b.gather_ext) b.gather_ext[3 * static_cast<size_t>(i)] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            const uint32_t x = i % fp.width, y = i / fp.width;
            Rng rng{b.gbuf[i].rng};
            const V3 dir = camera_dir(fp, x, y, rng);
            // gatherN > 1: the extra prefixes start along the same ray
            if (b.gather_ext) b.gather_ext[3 * static_cast<size_t>(i)] = make_float4(dir.x, dir.y, dir.z, 1.0f);
            Prefix cp = fresh_prefix();
            WfPath w = wf_blank();
            req = pre_begin(fp, cp, w, ld3(fp.cam.pos), dir, rng);
            words_of_prefix(cp, rec);
            started = true;
            w.rng = rng.state;
            wf_store(b.wf, i, w);
            b.pass_status[i] = kWfPath;
        }
    }
    rows.store(b.gather_cp, i, rec, started);
    wf_push(b, 0, req, i);
}

// ---- shading: resume every path whose ray of round `cur` finished ---------------------
template <bool kTex>
RT_D int wf_step(const SceneView& s, const FrameParams& fp, const Bufs& b, int flow, uint32_t i, WfPath& w,
                 Rng& rng) {
    if (w.phase == kPhPreHit || w.phase == kPhPreShadow) {
        crisb_prefix_rec& rec = flow == 0 ? b.canon_prefix[i] : b.gather_cp[i];
        Prefix pre = ld_prefix_run(rec);
        uint32_t set = 0;
        int req = w.phase == kPhPreHit ? pre_on_hit<kTex>(s, fp, pre, w, rng, set) : pre_on_shadow<kTex>(s, pre, w, set);
        st_prefix_step(rec, pre, set);
        if (req == kReqDone && flow == 2 && fl_valid(pre.flags) && !fl_nee(pre.flags)) {
            // FinalGatherCanon: the canonical suffix continues the canonical prefix
            Suffix cs = fresh_suffix();
            req = suf_begin<kTex>(s, fp, cs, w, pre.flags, pre.last, rng);
            st_suffix_slot(b.gather_cs[i], cs);
        }
        return req;
    }
    crisb_suffix_res_rec& slot = flow == 1 ? b.canon_suffix[i] : b.gather_cs[i];
    Suffix suf = ld_suffix_run(slot.sample);
    uint32_t set = 0;
    int req = kReqDone;
    if (w.phase == kPhSufHit) req = suf_on_hit<kTex>(s, fp, suf, w, rng, set);
    else if (w.phase == kPhSufShadow) req = suf_on_shadow<kTex>(s, suf, w);
    else if (w.phase == kPhSufRecon) req = suf_on_recon(s, suf, w, set);
    st_suffix_step(slot.sample, suf, set);
    return req;
}

// the ray a path asked for, traced in place (the queue kernels' semantics)
RT_D void wf_trace_inline(const SceneView& s, WfPath& w, int req) {
    V3 o, d;
    if (req == kReqClosest) {
        closest_ray(w, o, d);
        count_ray(s, 0);
        const TraceResult h = traverse<false>(s, make_ray(o, d), 1e-3f, 1e16f);
        set_hit(w, make_float4(__uint_as_float(h.prim), h.t, h.u, h.v));
    } else {
        float tmax;
        shadow_ray(w, o, d, tmax);
        set_occluded(w, occluded(s, o, d, 1e-3f, tmax) ? 1u : 0u);
    }
}

// Resume every path whose ray of round `cur` finished and queue its next ray;
// with kInline (the last wavefront round) trace the path's remaining rays in
// place until it ends, so the few long paths left do not cost a trace and a
// shade launch per bounce.  One launch over both queues: a separate instance
// for the shadow-ray results (94 against 126 registers) cost more in launches
// than it gained in occupancy (shading 3.85 -> 3.98 ms per 1080p frame).
// kTex: the scene has textured materials.  The untextured step kernel runs
// at 5 resident blocks per SM (96 registers; shading 3.86 -> 3.78 ms per
// 1080p frame against one kernel for both), the textured one at 4.
template <bool kInline, bool kTex>
__global__ void __launch_bounds__(kPassBlock, kInline ? 1 : (kTex ? 4 : 5)) k_wf_shade(SceneView s, FrameParams fp, Bufs b, int flow, int cur) {
    const uint32_t nc = b.wf_count[2 * cur], ns = b.wf_count[2 * cur + 1];
    const uint32_t total = nc + ns;
    const uint32_t* qc = b.wf_queue[2 * cur];
    const uint32_t* qs = b.wf_queue[2 * cur + 1];
    const int nxt = cur ^ 1;
    // a path traces at most a prefix, a suffix and one shadow ray per vertex
    const int max_steps = 4 * (fp.p.max_path_len + 2);
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        int req = kReqDone;
        uint32_t i = 0;
        if (t < total) {
            i = t < nc ? qc[t] : qs[t - nc];
            WfPath w = wf_load(b.wf, i);
            Rng rng{w.rng};
            req = wf_step<kTex>(s, fp, b, flow, i, w, rng);
            if (kInline) {
                for (int k = 0; req != kReqDone; ++k) {
                    if (k >= max_steps) {
                        dev_error(s, kDevErrIterations);
                        break;
                    }
                    wf_trace_inline(s, w, req);
                    req = wf_step<kTex>(s, fp, b, flow, i, w, rng);
                }
                req = kReqDone;
            }
            w.rng = rng.state;
            wf_store(b.wf, i, w);
        }
        if (!kInline) wf_push(b, nxt, req, i);
    }
}

struct WfGrids {
    unsigned shade, shade_inline;
};

template <bool kTex>
const WfGrids& wf_grids() {
    static std::once_flag once;
    static WfGrids g{};
    std::call_once(once, [] {
        g.shade = persistent_grid(reinterpret_cast<const void*>(k_wf_shade<false, kTex>));
        g.shade_inline = persistent_grid(reinterpret_cast<const void*>(k_wf_shade<true, kTex>));
    });
    return g;
}

// Wavefront rounds of a pass: a path traces at most max_path_len + 1 rays
// after its first; the shading kernel of the last round finishes any path
// still running in place.  Finishing in place from an earlier round (3 to 6)
// saved traversal launches but cost as much in the in-place kernel on the
// 1080p workload (24.2 ms/frame either way).
// (the ConditionalRestir prefix flow stops after prefix_len vertices: at most
// prefix_len closest-hit rays and one shadow ray per path)
int wf_round_count(const FrameParams& fp, int flow) {
    if (flow == 0 && fp.p.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR)
        return std::min(fp.p.prefix_len + 2, fp.p.max_path_len + 2);
    return fp.p.max_path_len + 2;
}

// rounds after the init kernel
template <bool kTex>
void wf_rounds_t(const SceneView& s, const FrameParams& fp, const Bufs& b, int flow, cudaStream_t st, Marker* m) {
    const WfGrids& g = wf_grids<kTex>();
    const int rounds = wf_round_count(fp, flow);
    for (int r = 0; r < rounds; ++r) {
        const int cur = r & 1, nxt = cur ^ 1;
        launch_trace<WfPath>(fp.trace_block, fp.trace_grid, st, s, b.wf_queue[2 * cur], b.wf_count + 2 * cur,
                             b.wf_queue[2 * cur + 1], b.wf_count + 2 * cur + 1, b.wf);
        if (m) m->mark(kClsTrace, st);
        if (r + 1 < rounds) {
            cudaMemsetAsync(b.wf_count + 2 * nxt, 0, 2 * sizeof(uint32_t), st);
            k_wf_shade<false, kTex><<<g.shade, kPassBlock, 0, st>>>(s, fp, b, flow, cur);
        } else {
            k_wf_shade<true, kTex><<<g.shade_inline, kPassBlock, 0, st>>>(s, fp, b, flow, cur);
        }
        if (m) m->mark(kClsShade, st);
    }
}

void wf_rounds(const SceneView& s, const FrameParams& fp, const Bufs& b, int flow, cudaStream_t st, Marker* m) {
    if (s.mat_tex) wf_rounds_t<true>(s, fp, b, flow, st, m);
    else wf_rounds_t<false>(s, fp, b, flow, st, m);
}

}  // namespace

uint32_t wf_launches_per_pass(const FrameParams& fp, int flow) {
    return 1 + 2 * static_cast<uint32_t>(wf_round_count(fp, flow));
}

void launch_wf_prefix(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m) {
    cudaMemsetAsync(b.wf_count, 0, 2 * sizeof(uint32_t), st);
    if (fp.shared_stage) k_wf_init_prefix<true><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    else k_wf_init_prefix<false><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    if (m) m->mark(kClsShade, st);
    wf_rounds(s, fp, b, 0, st, m);
}

void launch_wf_suffix(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m) {
    cudaMemsetAsync(b.wf_count, 0, 2 * sizeof(uint32_t), st);
    if (s.mat_tex) k_wf_init_suffix<true><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b);
    else k_wf_init_suffix<false><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b);
    if (m) m->mark(kClsShade, st);
    wf_rounds(s, fp, b, 1, st, m);
}

void launch_wf_gather(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m) {
    cudaMemsetAsync(b.wf_count, 0, 2 * sizeof(uint32_t), st);
    if (fp.shared_stage) k_wf_init_gather<true><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    else k_wf_init_gather<false><<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    if (m) m->mark(kClsShade, st);
    wf_rounds(s, fp, b, 2, st, m);
}

}  // namespace crisb
