// wavefront.cuh -- TracePrefix and TraceSuffix as resumable state machines.
//
// The per-pixel loops of include/graph/restir/path_gen.h:74-387 are cut at
// every ray they trace: a machine step runs the shading logic of one vertex
// up to its next closest-hit ray (extension, reconnection-vertex trace) or
// shadow ray (NEE visibility), stores its state, and queues the ray.  Trace
// kernels then run whole queues of rays, and the next shading step resumes
// every path whose ray is done.  The arithmetic of each step is the loop body
// of the reference function, in the same order, so a path ends with the same
// record bits as the per-pixel loop.
#pragma once

#include "rt_restir.cuh"

namespace crisb {

enum WfPhase : uint32_t {
    kPhDone = 0,
    kPhPreHit = 1,     // prefix: extension ray done
    kPhPreShadow = 2,  // prefix: NEE shadow ray done
    kPhSufHit = 3,     // suffix: extension ray done
    kPhSufShadow = 4,  // suffix: NEE shadow ray done
    kPhSufRecon = 5,   // suffix: reconnection-vertex ray done
};

enum WfReq : int { kReqDone = 0, kReqClosest = 1, kReqShadow = 2 };

// Path state between machine steps (176 bytes).
struct WfPath {
    uint64_t rng;
    uint32_t phase;
    uint32_t ctr;    // bits 0-7 loop index, bit 8 postRecon, bits 16-23 max length, 24-31 prefix length
    float4 ray_o;    // next closest-hit ray: origin (also lastPos of the suffix loop)
    float4 ray_d;    // next closest-hit ray: direction (currentDir / lastDir)
    float4 it_pos;   // current interaction: position, w = bary u
    float4 it_nrm;   // normal, w = bary v
    float4 it_dir;   // incoming direction, w = triangle index bits
    float4 nee_dir;  // NEE light direction, w = light distance
    float4 nee_col;  // NEE emitter colour
    float4 nee_brdf; // suffix: brdf * cos at the NEE vertex, kept across the reconnection trace
    float4 hit;      // closest-hit result: triangle bits, t, u, v
    uint32_t occluded;
    uint32_t pad[3];
};

RT_D V3 f3(float4 v) { return V3{v.x, v.y, v.z}; }
RT_D float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

RT_D uint32_t wf_idx(const WfPath& w) { return w.ctr & 0xFFu; }
RT_D bool wf_post(const WfPath& w) { return ((w.ctr >> 8) & 1u) != 0; }
RT_D uint32_t wf_maxlen(const WfPath& w) { return (w.ctr >> 16) & 0xFFu; }
RT_D uint32_t wf_prelen(const WfPath& w) { return (w.ctr >> 24) & 0xFFu; }
RT_D void wf_set(WfPath& w, uint32_t idx, bool post, uint32_t max_len, uint32_t pre_len) {
    w.ctr = (idx & 0xFFu) | (post ? (1u << 8) : 0u) | ((max_len & 0xFFu) << 16) | ((pre_len & 0xFFu) << 24);
}

RT_D Isect wf_it(const WfPath& w) {
    Isect it;
    it.valid = true;
    it.prim = __float_as_uint(w.it_dir.w);
    it.bu = w.it_pos.w;
    it.bv = w.it_nrm.w;
    it.pos = f3(w.it_pos);
    it.nrm = f3(w.it_nrm);
    it.dir = f3(w.it_dir);
    return it;
}
RT_D void wf_keep_it(WfPath& w, const Isect& it) {
    w.it_pos = f4(it.pos, it.bu);
    w.it_nrm = f4(it.nrm, it.bv);
    w.it_dir = f4(it.dir, __uint_as_float(it.prim));
}

// interaction of the finished closest-hit ray (trace_closest semantics)
RT_D bool wf_hit_isect(const SceneView& s, const WfPath& w, Isect& it) {
    const uint32_t prim = __float_as_uint(w.hit.x);
    it.dir = f3(w.ray_d);
    if (prim == CRISB_INVALID_PRIM) {
        it.valid = false;
        return false;
    }
    it.valid = true;
    it.prim = prim;
    it.bu = w.hit.z;
    it.bv = w.hit.w;
    const ShadeTri t = load_shade(s, prim);
    it.pos = interp(it.bu, it.bv, t.p0, t.p1, t.p2);
    it.nrm = normalize(interp(it.bu, it.bv, t.n0, t.n1, t.n2));
    return true;
}

RT_D int wf_done(WfPath& w) {
    w.phase = kPhDone;
    return kReqDone;
}

// ---- TracePrefix (path_gen.h:74-250) ----------------------------------------------
RT_D int pre_begin(const FrameParams& fp, Prefix& pre, WfPath& w, V3 origin, V3 dir, const Rng& rng) {
    pre.flags = 0u;
    pre.path_len = 0.0f;
    pre.rng = rng.state;
    pre.p = 1.0f;
    pre.f = splat(1.0f);
    pre.prf = splat(1.0f);
    pre.flags = fl_set_valid(pre.flags, true);
    const uint32_t max_len = fp.p.renderer_type == CRISB_RENDERER_RESTIR_PT ? static_cast<uint32_t>(fp.p.max_path_len)
                                                                            : static_cast<uint32_t>(fp.p.prefix_len);
    wf_set(w, 0, false, max_len, 0);
    w.ray_o = f4(origin, 0.0f);
    w.ray_d = f4(dir, 0.0f);
    w.phase = kPhPreHit;
    return kReqClosest;
}

// Vertex fields a machine step wrote (the steps never read them: a step's
// record moves as its running values plus the vertex fields it set)
enum : uint32_t { kSetPrimary = 1u, kSetRecon = 2u, kSetLast = 4u };

RT_D int pre_invalid(Prefix& pre, WfPath& w) {
    pre.flags = fl_set_valid(pre.flags, false);
    return wf_done(w);
}

template <bool kTex>
RT_D int pre_on_hit(const SceneView& s, const FrameParams& fp, Prefix& pre, WfPath& w, Rng& rng, uint32_t& set) {
    Isect it;
    if (!wf_hit_isect(s, w, it)) return pre_invalid(pre, w);
    const V3 cur_pos = f3(w.ray_o);
    const uint32_t ti = wf_idx(w), max_len = wf_maxlen(w);
    bool post = wf_post(w);
    const int type = fp.p.renderer_type;
    const float nee = fp.p.nee_prob;
    pre.path_len += distance(cur_pos, it.pos);
    pre.flags = fl_set_len(pre.flags, fl_len(pre.flags) + 1);
    if (fl_len(pre.flags) == 1) {
        pre.primary = it.pack();
        set |= kSetPrimary;
    }
    if (type == CRISB_RENDERER_CONDITIONAL_RESTIR && ti == max_len - 1) {
        if (!post) {
            pre.recon = it.pack();
            pre.flags = fl_set_recon(pre.flags, fl_len(pre.flags));
            pre.rod = splat(0.0f);
            set |= kSetRecon;
        }
        pre.flags = fl_set_valid(pre.flags, true);
        pre.last = it.pack();
        set |= kSetLast;
        return wf_done(w);
    }
    const bool force_nee = type == CRISB_RENDERER_RESTIR_PT && ti == max_len - 1;
    if (rng.next_float() < nee || force_nee) {
        pre.p *= nee;
        const EmitterSample es = sample_emitter(s, rng);
        const V3 light_dir = normalize(es.pos - it.pos);
        const float dist = length(es.pos - it.pos);
        wf_keep_it(w, it);
        w.nee_dir = f4(light_dir, dist);
        w.nee_col = f4(es.color, 0.0f);
        w.phase = kPhPreShadow;
        return kReqShadow;
    }
    const BrdfSample bs = brdf_sample<kTex>(s, it, rng);
    if (bs.pdf <= 0.0f) return pre_invalid(pre, w);
    const float recon_dist = distance(cur_pos, it.pos);
    const bool can_recon = recon_dist > fp.p.recon_min_distance && bs.roughness > fp.p.recon_min_roughness &&
                           fl_len(pre.flags) >= 2;
    if (!post && can_recon) {
        pre.recon = it.pack();
        pre.flags = fl_set_recon(pre.flags, fl_len(pre.flags));
        pre.rod = bs.dir;
        post = true;
        set |= kSetRecon;
    }
    pre.f = pre.f * bs.brdf;
    pre.p *= bs.pdf * (1.0f - nee);
    if (post) pre.prf = pre.prf * bs.brdf;
    if (ti + 1 < max_len) {
        w.ray_o = f4(it.pos, 0.0f);
        w.ray_d = f4(bs.dir, 0.0f);
        wf_set(w, ti + 1, post, max_len, 0);
        w.phase = kPhPreHit;
        return kReqClosest;
    }
    pre.last = it.pack();
    set |= kSetLast;
    return wf_done(w);
}

template <bool kTex>
RT_D int pre_on_shadow(const SceneView& s, Prefix& pre, WfPath& w, uint32_t& set) {
    if (w.occluded) return pre_invalid(pre, w);
    const Isect it = wf_it(w);
    if (!wf_post(w)) {
        // the reference re-traces the same ray here; the result is `it`
        pre.recon = it.pack();
        pre.flags = fl_set_recon(pre.flags, fl_len(pre.flags));
        pre.rod = f3(w.ray_d);
        set |= kSetRecon;
    }
    const bool post = true;
    const V3 light_dir = f3(w.nee_dir), color = f3(w.nee_col);
    const float dist = w.nee_dir.w;
    const BrdfEval be = brdf_eval<kTex>(s, it, light_dir);
    if (be.pdf <= 0.0f) return pre_invalid(pre, w);
    const float dist_factor = 1.0f / (dist * dist);
    pre.f = pre.f * (be.brdf * color * dist_factor);
    if (post) pre.prf = pre.prf * (be.brdf * color * dist_factor);
    if (fl_len(pre.flags) == 1) pre.f = pre.f + be.emission * dist_factor;
    pre.flags = fl_set_nee(pre.flags, true);
    pre.flags = fl_set_valid(pre.flags, true);
    pre.last = it.pack();
    set |= kSetLast;
    return wf_done(w);
}

// ---- TraceSuffix (path_gen.h:252-387) ----------------------------------------------
RT_D int suf_finish_nee(Suffix& suf, WfPath& w, V3 brdf) {
    const float light_len = w.nee_dir.w;
    const V3 color = f3(w.nee_col);
    const float dist_factor = 1.0f / (light_len * light_len);
    suf.f = suf.f * (brdf * color * dist_factor);
    suf.prf = suf.prf * (color * dist_factor);
    if (fl_recon(suf.flags) < fl_len(suf.flags)) suf.prf = suf.prf * brdf;
    suf.flags = fl_set_valid(suf.flags, true);
    return wf_done(w);
}

// loop body at vertex index wf_idx(w) with interaction `it`; last_pos is the
// position the vertex was traced from (lastPos)
template <bool kTex>
RT_D int suf_vertex(const SceneView& s, const FrameParams& fp, Suffix& suf, WfPath& w, const Isect& it, V3 last_pos,
                    Rng& rng, uint32_t& set) {
    const uint32_t vi = wf_idx(w), max_len = wf_maxlen(w), pre_len = wf_prelen(w);
    bool post = wf_post(w);
    const float nee = fp.p.nee_prob;
    const bool force_nee = vi == max_len - 1;
    if (rng.next_float() < nee || force_nee) {
        if (!force_nee) suf.p *= nee;
        const EmitterSample es = sample_emitter(s, rng);
        const V3 light_vec = es.pos - it.pos;
        const float light_len = length(light_vec);
        const V3 light_dir = normalize(light_vec);
        if (nonfinite(light_dir)) return wf_done(w);
        wf_keep_it(w, it);
        w.nee_dir = f4(light_dir, light_len);
        w.nee_col = f4(es.color, 0.0f);
        w.phase = kPhSufShadow;
        return kReqShadow;
    }
    const BrdfSample bs = brdf_sample<kTex>(s, it, rng);
    if (bs.pdf <= 0.0f) return wf_done(w);
    suf.p *= bs.pdf * (1.0f - nee);
    suf.f = suf.f * bs.brdf;
    if (post) suf.prf = suf.prf * bs.brdf;
    const float recon_dist = distance(last_pos, it.pos);
    const bool can_recon =
        recon_dist > fp.p.recon_min_distance && bs.roughness > fp.p.recon_min_roughness && pre_len >= 1;
    if (!post && can_recon) {
        suf.recon = it.pack();
        suf.flags = fl_set_recon(suf.flags, pre_len);
        suf.flags = fl_set_recon_vert(suf.flags, fl_len(suf.flags));  // the loop index vi
        suf.rod = bs.dir;
        post = true;
        set |= kSetRecon;
    }
    suf.flags = fl_set_len(suf.flags, fl_len(suf.flags) + 1);
    if (vi + 1 < max_len) {
        w.ray_o = f4(it.pos, 0.0f);
        w.ray_d = f4(bs.dir, 0.0f);
        wf_set(w, vi + 1, post, max_len, pre_len);
        w.phase = kPhSufHit;
        return kReqClosest;
    }
    return wf_done(w);
}

// suffix from the prefix with flags `pre_flags` ending at `pre_last`; `suf`
// holds the previous record content
template <bool kTex>
RT_D int suf_begin(const SceneView& s, const FrameParams& fp, Suffix& suf, WfPath& w, uint32_t pre_flags,
                   const Hit& pre_last, Rng& rng) {
    suf.f = splat(1.0f);
    suf.p = 1.0f;
    suf.prf = splat(1.0f);
    suf.rng = rng.state;
    suf.last_prefix = pre_last;
    suf.flags = 0u;
    if (!fl_valid(pre_flags) || fl_nee(pre_flags)) return wf_done(w);
    const uint32_t max_len = static_cast<uint32_t>(fp.p.max_path_len) - fl_len(pre_flags);
    const Isect it = unpack(s, pre_last);
    if (!it.valid || max_len == 0) return wf_done(w);
    wf_set(w, 0, false, max_len, fl_len(pre_flags));
    uint32_t set = 0;  // suf_begin's callers store the whole record
    return suf_vertex<kTex>(s, fp, suf, w, it, it.pos, rng, set);
}

template <bool kTex>
RT_D int suf_on_hit(const SceneView& s, const FrameParams& fp, Suffix& suf, WfPath& w, Rng& rng, uint32_t& set) {
    Isect it;
    if (!wf_hit_isect(s, w, it)) return wf_done(w);
    return suf_vertex<kTex>(s, fp, suf, w, it, f3(w.ray_o), rng, set);
}

template <bool kTex>
RT_D int suf_on_shadow(const SceneView& s, Suffix& suf, WfPath& w) {
    if (w.occluded) return wf_done(w);
    const Isect it = wf_it(w);
    const V3 light_dir = f3(w.nee_dir);
    const BrdfEval be = brdf_eval<kTex>(s, it, light_dir);
    if (be.pdf <= 0.0f) return wf_done(w);
    suf.flags = fl_set_len(suf.flags, fl_len(suf.flags) + 1);
    if (!wf_post(w)) {
        w.ray_o = f4(it.pos, 0.0f);
        w.ray_d = f4(light_dir, 0.0f);
        w.nee_brdf = f4(be.brdf, 0.0f);
        w.phase = kPhSufRecon;
        return kReqClosest;
    }
    return suf_finish_nee(suf, w, be.brdf);
}

RT_D int suf_on_recon(const SceneView& s, Suffix& suf, WfPath& w, uint32_t& set) {
    Isect rc;
    if (!wf_hit_isect(s, w, rc)) return wf_done(w);
    set |= kSetRecon;
    suf.recon = rc.pack();
    suf.flags = fl_set_recon(suf.flags, fl_len(suf.flags));
    suf.flags = fl_set_recon_vert(suf.flags, fl_len(suf.flags) - 1);  // the NEE vertex
    suf.rod = splat(0.0f);
    return suf_finish_nee(suf, w, f3(w.nee_brdf));
}

}  // namespace crisb
