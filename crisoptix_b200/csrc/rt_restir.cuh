// rt_restir.cuh -- path generation, hybrid shift mappings, pairwise MIS and
// reservoir streaming of Conditional ReSTIR PT.
//
// Device restatement of include/graph/restir/path_gen.h, prefix_reuse.h,
// suffix_reuse.h and Reservoir.h.  Records are modified in place with the
// reference's field-by-field semantics (fields a function does not write keep
// their previous value).
#pragma once

#include "rt_scene.cuh"

namespace crisb {

// Frame-constant parameters (LaunchParams + RestirParams knobs)
struct FrameParams {
    crisb_params p;
    crisb_camera_data cam;
    uint32_t width, height;
    uint32_t random;
    uint32_t frame_idx;  // for the accumulation blend factor
    int front, back;     // 0/1 buffer selection
    uint32_t k;          // gatherM - 1
    uint32_t trace_grid; // traversal launches: blocks per resident block (host side only)
    uint32_t trace_block; // traversal launches: threads per block, 64 / 128 / 256 (host side only)
    uint32_t shared_stage = 1;  // init kernels stage record runs in shared memory (host side only)
    const float2* motion = nullptr;  // CRISB_MOTION_VECTORS: per-pixel motion vectors
    crisb_camera_data prev_cam{};    // CRISB_MOTION_REPROJECT: the previous frame's camera
    uint32_t has_prev_cam = 0;
};

// ---- temporal reprojection (prevPixelCoord) ---------------------------------------
// G-buffer prev_xy: x | y << 16, or kPrevNone when the pixel has no previous
// pixel (IsPixelValid false); resolutions stay below 65535 so no valid pixel
// packs to it.
constexpr uint32_t kPrevNone = 0xffffffffu;

RT_HD uint32_t pack_prev(uint32_t px, uint32_t py, uint32_t w, uint32_t h) {
    return (px < w && py < h) ? (px | (py << 16)) : kPrevNone;
}

// glm::uvec2(vec2) as it compiles on the GPU (cvt.rzi.u32.f32): truncation
// toward zero, saturating at 0 and 2^32 - 1, NaN to 0
RT_HD uint32_t f2u_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return static_cast<uint32_t>(v);
}

// prevPixelCoord = uvec2(vec2(pixelCoord) + vec2(0.5) + motionVector)
// (prefix_gen_temp_reuse.cu:136, the commented-out form)
RT_HD uint32_t prev_from_motion(uint32_t x, uint32_t y, float mx, float my, uint32_t w, uint32_t h) {
    const float fx = (static_cast<float>(x) + 0.5f) + mx;
    const float fy = (static_cast<float>(y) + 0.5f) + my;
    return pack_prev(f2u_sat(fx), f2u_sat(fy), w, h);
}

// The pixel of camera `c` whose footprint holds world point p: the inverse of
// camera_dir (d = U ux + V uy + W with U, V, W orthogonal), ux = 2 x / width -
// 1 over the pixel's footprint [x, x + 1).  None behind the camera or off
// screen.
RT_HD uint32_t reproject(const crisb_camera_data& c, V3 p, uint32_t w, uint32_t h) {
    const V3 U = ld3(c.u), V = ld3(c.v), W = ld3(c.w);
    const V3 d = p - ld3(c.pos);
    const float t = dot(d, W) / dot(W, W);
    if (!(t > 0.0f)) return kPrevNone;
    const float ux = dot(d, U) / (t * dot(U, U));
    const float uy = dot(d, V) / (t * dot(V, V));
    const float xc = (ux + 1.0f) * 0.5f * static_cast<float>(w);
    const float yc = (uy + 1.0f) * 0.5f * static_cast<float>(h);
    if (!(xc >= 0.0f && xc < static_cast<float>(w) && yc >= 0.0f && yc < static_cast<float>(h))) return kPrevNone;
    return pack_prev(static_cast<uint32_t>(xc), static_cast<uint32_t>(yc), w, h);
}

RT_HD uint32_t prev_index(uint32_t prev_xy, uint32_t w) { return (prev_xy & 0xffffu) + (prev_xy >> 16) * w; }

// ---- reservoir (include/graph/restir/Reservoir.h:28-50) ------------------------
template <typename T>
RT_D bool res_update(Res<T>& r, const T& s, float w, Rng& rng, float in_conf) {
    if (isnan(w) || isinf(w)) w = 0.0f;
    r.w_sum += w;
    r.conf += in_conf;
    r.conf = gmin(r.conf, CRISB_CONFIDENCE_MAX);
    if (rng.next_float() < w / r.w_sum) {
        r.s = s;
        return true;
    }
    return false;
}
// res_update without the sample: the same weight and confidence arithmetic and
// the same random draw; true when the candidate replaces the current sample
RT_D bool res_choose(float& w_sum, float& conf, float w, Rng& rng, float in_conf) {
    if (isnan(w) || isinf(w)) w = 0.0f;
    w_sum += w;
    conf += in_conf;
    conf = gmin(conf, CRISB_CONFIDENCE_MAX);
    return rng.next_float() < w / w_sum;
}

template <typename T>
RT_D void res_finalize(Res<T>& r) {
    const float phat = luminance(r.s.f);
    if (phat == 0.0f) r.w_sum = 0.0f;
    else r.w_sum /= phat;
}

// ---- pairwise MIS (include/graph/restir/path_gen.h:15-48) ----------------------
RT_D float mis_canonical(V3 b_at_b, V3 b_at_n, float jac, float K, float cM, float nM) {
    float w = 1.f;
    if (luminance(b_at_b) > 0.f) {
        const float at_basis = luminance(b_at_b) * cM;
        w = at_basis / (at_basis + luminance(b_at_n) * jac * nM * K);
    }
    return w;
}
RT_D float mis_neighbor(V3 n_at_b, V3 n_at_n, float jac, float K, float cM, float nM) {
    float w = 0.f;
    if (luminance(n_at_n) > 0.f) {
        w = luminance(n_at_n) * nM / (luminance(n_at_n) * nM + luminance(n_at_b) * jac * cM / K);
    }
    return w;
}

// SelectSpatialNeighbor (path_gen.h:50-57) with a configurable window radius
RT_D void select_spatial_neighbor(uint32_t px, uint32_t py, uint32_t radius, Rng& rng, uint32_t& nx, uint32_t& ny) {
    const uint32_t ws = 2 * radius + 1;
    const uint32_t x = (px + radius) - (rng.next_u32() % ws);
    const uint32_t y = (py + radius) - (rng.next_u32() % ws);
    if (x == px && y == py) {
        nx = px + 1;
        ny = py + 1;
        return;
    }
    nx = x;
    ny = y;
}

// CalcReconnectionJacobian (path_gen.h:59-72)
RT_D float recon_jacobian(V3 old_xi, V3 new_xi, V3 target, V3 target_n) {
    const float term1 =
        fabsf(dot(normalize(new_xi - target), target_n) / dot(normalize(old_xi - target), target_n));
    const float term2 = dot(target - old_xi, target - old_xi);
    const float term3 = dot(target - new_xi, target - new_xi);
    const float result = term1 * term2 / term3;
    if (isinf(result) || isnan(result)) return 0.0f;
    return gmax(0.0f, result);
}

// ---- path generation -----------------------------------------------------------------
// TracePrefix (path_gen.h:74-250); `prefix` holds the previous record content.
RT_D void trace_prefix(const SceneView& s, const FrameParams& fp, Prefix& prefix, V3 origin, V3 dir, Rng& rng) {
    V3 cur_pos = origin, cur_dir = dir;
    prefix.flags = 0u;
    prefix.path_len = 0.0f;
    prefix.rng = rng.state;
    prefix.p = 1.0f;
    prefix.f = splat(1.0f);
    prefix.prf = splat(1.0f);
    prefix.flags = fl_set_valid(prefix.flags, true);
    const int type = fp.p.renderer_type;
    const uint32_t max_len = type == CRISB_RENDERER_RESTIR_PT ? static_cast<uint32_t>(fp.p.max_path_len)
                                                              : static_cast<uint32_t>(fp.p.prefix_len);
    const float nee = fp.p.nee_prob;
    Isect it;
    it.valid = false;
    bool post = false;
    for (uint32_t ti = 0; ti < max_len; ++ti) {
        trace_closest(s, cur_pos, cur_dir, 1e-3f, 1e16f, it);
        if (!it.valid) {
            prefix.flags = fl_set_valid(prefix.flags, false);
            return;
        }
        prefix.path_len += distance(cur_pos, it.pos);
        prefix.flags = fl_set_len(prefix.flags, fl_len(prefix.flags) + 1);
        if (fl_len(prefix.flags) == 1) prefix.primary = it.pack();
        if (type == CRISB_RENDERER_CONDITIONAL_RESTIR && ti == max_len - 1) {
            if (!post) {
                prefix.recon = it.pack();
                prefix.flags = fl_set_recon(prefix.flags, fl_len(prefix.flags));
                prefix.rod = splat(0.0f);
            }
            prefix.flags = fl_set_valid(prefix.flags, true);
            prefix.last = it.pack();
            return;
        }
        const bool force_nee = type == CRISB_RENDERER_RESTIR_PT && ti == max_len - 1;
        if (rng.next_float() < nee || force_nee) {
            prefix.p *= nee;
            const EmitterSample es = sample_emitter(s, rng);
            const V3 light_dir = normalize(es.pos - it.pos);
            const float dist = length(es.pos - it.pos);
            if (occluded(s, it.pos, light_dir, 1e-3f, dist)) {
                prefix.flags = fl_set_valid(prefix.flags, false);
                return;
            }
            if (!post) {
                // the reference re-traces the same ray here; the result is `it`
                prefix.recon = it.pack();
                prefix.flags = fl_set_recon(prefix.flags, fl_len(prefix.flags));
                prefix.rod = cur_dir;
                post = true;
            }
            const BrdfEval be = brdf_eval(s, it, light_dir);
            if (be.pdf <= 0.0f) {
                prefix.flags = fl_set_valid(prefix.flags, false);
                return;
            }
            const float dist_factor = 1.0f / (dist * dist);
            prefix.f = prefix.f * (be.brdf * es.color * dist_factor);
            if (post) prefix.prf = prefix.prf * (be.brdf * es.color * dist_factor);
            if (fl_len(prefix.flags) == 1) prefix.f = prefix.f + be.emission * dist_factor;
            prefix.flags = fl_set_nee(prefix.flags, true);
            prefix.flags = fl_set_valid(prefix.flags, true);
            prefix.last = it.pack();
            return;
        }
        const BrdfSample bs = brdf_sample(s, it, rng);
        if (bs.pdf <= 0.0f) {
            prefix.flags = fl_set_valid(prefix.flags, false);
            return;
        }
        const float recon_dist = distance(cur_pos, it.pos);
        const bool can_recon = recon_dist > fp.p.recon_min_distance && bs.roughness > fp.p.recon_min_roughness &&
                               fl_len(prefix.flags) >= 2;
        if (!post && can_recon) {
            prefix.recon = it.pack();
            prefix.flags = fl_set_recon(prefix.flags, fl_len(prefix.flags));
            prefix.rod = bs.dir;
            post = true;
        }
        cur_pos = it.pos;
        cur_dir = bs.dir;
        prefix.f = prefix.f * bs.brdf;
        prefix.p *= bs.pdf * (1.0f - nee);
        if (post) prefix.prf = prefix.prf * bs.brdf;
    }
    prefix.last = it.pack();
}

// TraceSuffix (path_gen.h:252-387); `suffix` holds the previous record content.
RT_D void trace_suffix(const SceneView& s, const FrameParams& fp, Suffix& suffix, const Prefix& prefix, Rng& rng) {
    suffix.f = splat(1.0f);
    suffix.p = 1.0f;
    suffix.prf = splat(1.0f);
    suffix.rng = rng.state;
    suffix.last_prefix = prefix.last;
    suffix.flags = 0u;
    if (!fl_valid(prefix.flags) || fl_nee(prefix.flags)) return;
    const uint32_t max_len = static_cast<uint32_t>(fp.p.max_path_len) - fl_len(prefix.flags);
    Isect it = unpack(s, prefix.last);
    if (!it.valid) return;
    const float nee = fp.p.nee_prob;
    bool post = false;
    V3 last_dir = splat(0.0f);
    for (uint32_t vi = 0; vi < max_len; ++vi) {
        const V3 last_pos = it.pos;
        if (fl_len(suffix.flags) > 0) {
            trace_closest(s, last_pos, last_dir, 1e-3f, 1e16f, it);
            if (!it.valid) return;
        }
        const bool force_nee = vi == max_len - 1;
        if (rng.next_float() < nee || force_nee) {
            if (!force_nee) suffix.p *= nee;
            const EmitterSample es = sample_emitter(s, rng);
            const V3 light_vec = es.pos - it.pos;
            const float light_len = length(light_vec);
            const V3 light_dir = normalize(light_vec);
            if (nonfinite(light_dir)) return;
            if (occluded(s, it.pos, light_dir, 1e-3f, light_len)) return;
            const BrdfEval be = brdf_eval(s, it, light_dir);
            if (be.pdf <= 0.0f) return;
            suffix.flags = fl_set_len(suffix.flags, fl_len(suffix.flags) + 1);
            if (!post) {
                Isect rc;
                rc.valid = false;
                trace_closest(s, it.pos, light_dir, 1e-3f, 1e16f, rc);
                if (!rc.valid) return;
                suffix.recon = rc.pack();
                suffix.flags = fl_set_recon(suffix.flags, fl_len(suffix.flags));
                suffix.flags = fl_set_recon_vert(suffix.flags, vi);
                suffix.rod = splat(0.0f);
                post = true;
            }
            const float dist_factor = 1.0f / (light_len * light_len);
            suffix.f = suffix.f * (be.brdf * es.color * dist_factor);
            suffix.prf = suffix.prf * (es.color * dist_factor);
            if (fl_recon(suffix.flags) < fl_len(suffix.flags)) suffix.prf = suffix.prf * be.brdf;
            suffix.flags = fl_set_valid(suffix.flags, true);
            return;
        }
        const BrdfSample bs = brdf_sample(s, it, rng);
        if (bs.pdf <= 0.0f) return;
        suffix.p *= bs.pdf * (1.0f - nee);
        suffix.f = suffix.f * bs.brdf;
        if (post) suffix.prf = suffix.prf * bs.brdf;
        const float recon_dist = distance(last_pos, it.pos);
        const bool can_recon = recon_dist > fp.p.recon_min_distance && bs.roughness > fp.p.recon_min_roughness &&
                               fl_len(prefix.flags) >= 1;
        if (!post && can_recon) {
            suffix.recon = it.pack();
            suffix.flags = fl_set_recon(suffix.flags, fl_len(prefix.flags));
            suffix.flags = fl_set_recon_vert(suffix.flags, vi);
            suffix.rod = bs.dir;
            post = true;
        }
        last_dir = bs.dir;
        suffix.flags = fl_set_len(suffix.flags, fl_len(suffix.flags) + 1);
    }
}

// TraceCompletePath (path_gen.h:389-472)
RT_D V3 trace_complete_path(const SceneView& s, const FrameParams& fp, V3 origin, V3 dir, Rng& rng) {
    V3 cur_pos = origin, cur_dir = dir;
    uint32_t depth = 0;
    V3 radiance = splat(0.0f), tp = splat(1.0f);
    const float nee = fp.p.nee_prob;
    for (int ti = 0; ti < fp.p.max_path_len; ++ti) {
        Isect it;
        it.valid = false;
        trace_closest(s, cur_pos, cur_dir, 1e-3f, 1e16f, it);
        if (!it.valid) break;
        ++depth;
        if (rng.next_float() < nee) {
            tp = tp / nee;
            const EmitterSample es = sample_emitter(s, rng);
            const V3 light_dir = normalize(es.pos - it.pos);
            const float dist = length(es.pos - it.pos);
            if (occluded(s, it.pos, light_dir, 1e-3f, dist)) return splat(0.0f);
            const BrdfEval be = brdf_eval(s, it, light_dir);
            const float dist_factor = 1.0f / (dist * dist);
            radiance = tp * be.brdf * es.color * dist_factor;
            if (depth == 1) radiance = radiance + be.emission;
            break;
        }
        const BrdfSample bs = brdf_sample(s, it, rng);
        if (bs.pdf <= 0.0f) break;
        cur_pos = it.pos;
        cur_dir = bs.dir;
        tp = tp * (bs.brdf / bs.pdf);
        tp = tp / (1.0f - nee);
    }
    return radiance;
}

// TracePrefixForFinalGather (path_gen.h:474-531)
RT_D bool trace_prefix_for_gather(const SceneView& s, V3& tp, float& p, Isect& last, V3 origin, V3 dir,
                                  uint32_t max_len, Rng& rng) {
    V3 cur_pos = origin, cur_dir = dir;
    tp = splat(1.0f);
    p = 1.0f;
    last.valid = false;
    for (uint32_t ti = 0; ti < max_len; ++ti) {
        trace_closest(s, cur_pos, cur_dir, 1e-3f, 1e16f, last);
        if (!last.valid) return false;
        const BrdfSample bs = brdf_sample(s, last, rng);
        if (bs.pdf <= 0.0f) return false;
        cur_pos = last.pos;
        cur_dir = bs.dir;
        tp = tp * bs.brdf;
        p *= bs.pdf;
    }
    return true;
}

// ---- shift mappings ------------------------------------------------------------------
// prefix CalcCurrContribInOtherDomain (include/graph/restir/prefix_reuse.h:10-99)
RT_D V3 shift_prefix(const SceneView& s, const Prefix& src, const Prefix& dst, float& jac) {
    jac = 0.0f;
    if (!fl_valid(src.flags) || fl_recon(src.flags) < 2) return splat(0.0f);
    const Isect src_primary = unpack(s, src.primary);
    if (!src_primary.valid) return splat(0.0f);
    Isect cur = unpack(s, dst.primary);
    if (!cur.valid) return splat(0.0f);
    Isect src_recon = unpack(s, src.recon);
    if (!src_recon.valid) return splat(0.0f);
    const int nrep = max(static_cast<int>(fl_recon(src.flags) - 2u), 0);
    Rng srng{src.rng};
    V3 tp = splat(1.0f);
    for (int i = 0; i < nrep; ++i) {
        srng.next_float();
        const BrdfSample bs = brdf_sample(s, cur, srng);
        if (bs.pdf <= 0.0f) return splat(0.0f);
        tp = tp * bs.brdf;
        const V3 pos = cur.pos;
        trace_closest(s, pos, bs.dir, 1e-3f, 1e16f, cur);
        if (!cur.valid) return splat(0.0f);
    }
    const V3 rv = src_recon.pos - cur.pos;
    const float rlen = length(rv);
    const V3 rdir = normalize(rv);
    if (isinf(rlen) || nonfinite(rdir)) return splat(0.0f);
    if (occluded(s, cur.pos, rdir, 1e-3f, rlen)) return splat(0.0f);
    const BrdfEval b1 = brdf_eval(s, cur, rdir);
    if (b1.pdf <= 0.0f) return splat(0.0f);
    tp = tp * b1.brdf;
    src_recon.dir = rdir;
    const BrdfEval b2 = brdf_eval(s, src_recon, src.rod);
    if (b2.pdf <= 0.0f) return splat(0.0f);
    tp = tp * b2.brdf;
    jac = recon_jacobian(src_primary.pos, cur.pos, src_recon.pos, src_recon.nrm);
    return gmax(splat(0.0f), tp * src.prf);
}

// suffix CalcCurrContribInOtherDomain (include/graph/restir/suffix_reuse.h:10-108)
RT_D V3 shift_suffix(const SceneView& s, const Suffix& src, const Isect& dst_last, float& jac) {
    jac = 0.0f;
    if (!fl_valid(src.flags)) return splat(0.0f);
    if (!dst_last.valid) return splat(0.0f);
    const Isect src_last = unpack(s, src.last_prefix);
    if (!src_last.valid) return splat(0.0f);
    Isect src_recon = unpack(s, src.recon);
    if (!src_recon.valid) return splat(0.0f);
    const int nrep = max(static_cast<int>(fl_recon(src.flags) - 1u), 0);
    Isect cur = dst_last;
    Rng srng{src.rng};
    V3 tp = splat(1.0f);
    for (int i = 0; i < nrep; ++i) {
        srng.next_float();
        const BrdfSample bs = brdf_sample(s, cur, srng);
        if (bs.pdf <= 0.0f) return splat(0.0f);
        tp = tp * bs.brdf;
        const V3 pos = cur.pos;
        trace_closest(s, pos, bs.dir, 1e-3f, 1e16f, cur);
        if (!cur.valid) return splat(0.0f);
    }
    const V3 rv = src_recon.pos - cur.pos;
    const float rlen = length(rv);
    const V3 rdir = normalize(rv);
    if (nonfinite(rdir)) return splat(0.0f);
    if (occluded(s, cur.pos, rdir, 1e-3f, rlen)) return splat(0.0f);
    const BrdfEval b1 = brdf_eval(s, cur, rdir);
    if (b1.pdf <= 0.0f) return splat(0.0f);
    tp = tp * b1.brdf;
    if (fl_recon(src.flags) < fl_len(src.flags)) {
        src_recon.dir = rdir;
        if (is_zero(src.rod)) return splat(0.0f);
        const BrdfEval b2 = brdf_eval(s, src_recon, src.rod);
        if (b2.pdf <= 0.0f) return splat(0.0f);
        tp = tp * b2.brdf;
    }
    jac = recon_jacobian(src_last.pos, cur.pos, src_recon.pos, src_recon.nrm);
    return tp * src.prf;
}

// suffix_reuse.h:111-123
RT_D V3 shift_suffix(const SceneView& s, const Suffix& src, const Suffix& dst, float& jac) {
    const Isect dst_last = unpack(s, dst.last_prefix);
    if (!dst_last.valid) return splat(0.0f);
    return shift_suffix(s, src, dst_last, jac);
}

// SpawnCameraRay's direction (include/graph/Camera.h:14-22) at viewport
// coordinates (ux, uy)
RT_D V3 spawn_camera_dir(V3 U, V3 V, V3 W, float ux, float uy) { return normalize(U * ux + V * uy + W); }

// jittered camera ray of the pixel (prefix_gen_temp_reuse.cu:124-126); the x
// jitter is drawn before the y jitter.
RT_D V3 camera_dir(const FrameParams& fp, uint32_t x, uint32_t y, Rng& rng) {
    const float jx = rng.next_float();
    const float jy = rng.next_float();
    float ux = (static_cast<float>(x) + jx) / static_cast<float>(fp.width);
    float uy = (static_cast<float>(y) + jy) / static_cast<float>(fp.height);
    ux = 2.0f * ux - 1.0f;
    uy = 2.0f * uy - 1.0f;
    return spawn_camera_dir(ld3(fp.cam.u), ld3(fp.cam.v), ld3(fp.cam.w), ux, uy);
}

}  // namespace crisb
