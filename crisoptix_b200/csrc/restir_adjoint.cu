// restir_adjoint.cu -- path-replay adjoint of the final gather's resampled
// estimator (Conditional ReSTIR PT).
//
// The estimator differentiated is a pixel's FinalGatherCanon
// (shader/final_gather.cu:69-188; k_gather_finish and k_gather_combine here)
// in the frame a renderer rendered last:
//
//   L = ( (S (.) Fp / Pp) / (K + 1) + (Fp (.) Fs / (Pp Ps)) cm ) / (K + 1),
//   S = sum_n A_n fshift_n,  A_n = m_n W_n J_n,  fshift_n = T_n (.) R_n
//
// ((.) per channel; K valid neighbours).  Fp and Fs are the throughputs of the
// gather's canonical prefix and suffix, T_n the throughput of the shift of
// neighbour n's suffix onto the canonical prefix (random-replay vertices and
// the two reconnection BRDFs), R_n that suffix's throughput after its
// reconnection vertex (postReconF).  Frozen at the materials and emitter
// colours the frame was rendered with (theta0): every random decision,
// sampled direction and sampling pdf (Pp, Ps), the validity of paths and
// shifts, the neighbour lists, the MIS weights m_n and cm, the neighbours'
// unbiased contribution weights W_n and the Jacobians J_n.  At the scene's
// current tables (theta): every BRDF value along the paths, the emitter
// colours and the emission.  At theta = theta0 the estimator is the frame's
// gather value (before accumulation); for any theta it is the resampling
// estimator with a fixed proposal applied to the integrand at theta, so its
// expectation's gradient is the expectation of its gradient (W_n are unbiased
// contribution weights and the MIS weights sum to one whatever the integrand).
//
// Nothing is taped: each factor is re-traced.  The canonical prefix from the
// camera along its stored primary direction with its stored random state, the
// canonical suffix from the prefix's last vertex with its stored state, the
// shift from the stored neighbour sample, and R_n from the neighbour sample's
// own seed: its random state advanced four draws per suffix vertex (one NEE
// decision, three for BRDF sampling) to the vertex after its reconnection
// vertex, whose loop index the suffix flags carry (bits 24-31).  Forward mode
// carries d(throughput)/d(diffuse, roughness) per material met, d/d(colour) of
// the emitter sampled and d/d(emission); the backward kernel weighs each
// factor's derivatives with dLoss/dL times the other factors (chain rule at
// theta0) and adds them through the warp-aggregated gradient sink.
#include "adjoint_common.cuh"
#include "records.cuh"

namespace crisb {
namespace {

RT_D V3 xyz(float4 v) { return V3{v.x, v.y, v.z}; }

struct RAdjView {
    SceneView eval;  // current tables (theta): BRDF values, emitter colours, emission
    SceneView samp;  // the frame's materials and emitters (theta0): sampling and validity
    uint32_t num_mats;
};

// a path segment's throughput at theta with its derivatives (kGrad)
template <bool kGrad>
struct Seg {
    V3 val;
    Touched tl[kGrad ? kMaxTouched : 1];
    int nt;
    int em;    // emitter whose colour entered val, or -1
    V3 d_em;   // d val / d colour (channel-diagonal)
    int emm;   // material whose emission entered val, or -1
    V3 d_emm;  // d val / d emission (channel-diagonal)

    RT_D void init() {
        val = splat(1.0f);
        nt = 0;
        em = emm = -1;
        d_em = d_emm = splat(0.0f);
    }
    // val *= c; c's derivatives: dc_diff / dc_rough for material mi (>= 0),
    // dc_col for emitter e (>= 0)
    RT_D void mul(V3 c, int mi, V3 dc_diff, V3 dc_rough, int e, V3 dc_col) {
        if (kGrad) {
            for (int t = 0; t < nt; ++t) {
                tl[t].d_diff = tl[t].d_diff * c;
                tl[t].d_rough = tl[t].d_rough * c;
            }
            d_em = d_em * c;
            d_emm = d_emm * c;
            if (mi >= 0) {
                int slot = -1;
                for (int t = 0; t < nt; ++t)
                    if (tl[t].mat == static_cast<uint32_t>(mi)) slot = t;
                if (slot < 0 && nt < kMaxTouched) {
                    slot = nt++;
                    tl[slot].mat = static_cast<uint32_t>(mi);
                    tl[slot].d_diff = tl[slot].d_rough = splat(0.0f);
                }
                if (slot >= 0) {
                    tl[slot].d_diff = tl[slot].d_diff + val * dc_diff;
                    tl[slot].d_rough = tl[slot].d_rough + val * dc_rough;
                }
            }
            if (e >= 0) {
                em = e;
                d_em = d_em + val * dc_col;
            }
        }
        val = val * c;
    }
    RT_D void mul_brdf(const BrdfGrad& g, uint32_t mi) {
        mul(g.brdf, static_cast<int>(mi), g.d_diff, g.d_rough, -1, splat(0.0f));
    }
    // val += emission * dist_factor of material mi
    RT_D void add_emission(V3 emission, float dist_factor, uint32_t mi) {
        if (kGrad) {
            emm = static_cast<int>(mi);
            d_emm = splat(dist_factor);
        }
        val = val + emission * dist_factor;
    }
    // w . d val / d theta into the sink
    RT_D void emit(V3 w, GradSink* sink) const {
        if (!kGrad) return;
        for (int t = 0; t < nt; ++t) {
            const V3 c_diff = w * tl[t].d_diff;
            sink->add_mat(tl[t].mat, 0, c_diff.x);
            sink->add_mat(tl[t].mat, 1, c_diff.y);
            sink->add_mat(tl[t].mat, 2, c_diff.z);
            const V3 c_r = w * tl[t].d_rough;
            sink->add_mat(tl[t].mat, 3, (c_r.x + c_r.y) + c_r.z);
        }
        if (em >= 0) {
            const V3 c = w * d_em;
            sink->add_em(static_cast<uint32_t>(em), 0, c.x);
            sink->add_em(static_cast<uint32_t>(em), 1, c.y);
            sink->add_em(static_cast<uint32_t>(em), 2, c.z);
        }
        if (emm >= 0) {
            const V3 c = w * d_emm;
            sink->add_mat(static_cast<uint32_t>(emm), 4, c.x);
            sink->add_mat(static_cast<uint32_t>(emm), 5, c.y);
            sink->add_mat(static_cast<uint32_t>(emm), 6, c.z);
        }
    }
};

// the BRDF * cos at theta of the material at `it` toward `out`, with its derivatives
RT_D BrdfGrad grad_at(const RAdjView& a, const Isect& it, V3 out, uint32_t& mi) {
    mi = material_of(a.eval, it.prim);
    return brdf_grad(a.eval.mats[mi], it.nrm, -it.dir, out);
}

// (brdf (.) colour) * dist_factor of an NEE connection, with its derivatives
template <bool kGrad>
RT_D void mul_nee(Seg<kGrad>& sg, const BrdfGrad& g, uint32_t mi, const EmitterSample& es, float dist_factor) {
    sg.mul(g.brdf * es.color * dist_factor, static_cast<int>(mi), g.d_diff * es.color * dist_factor,
           g.d_rough * es.color * dist_factor, static_cast<int>(es.index), g.brdf * dist_factor);
}

// Fp: TracePrefix of a valid gather prefix (path_gen.h:74-250, Conditional
// ReSTIR), from the camera along its primary direction
template <bool kGrad>
RT_D void seg_prefix(const RAdjView& a, const FrameParams& fp, const Prefix& cp, Seg<kGrad>& sg) {
    sg.init();
    Rng rng{cp.rng};
    const float nee = fp.p.nee_prob;
    const uint32_t max_len = static_cast<uint32_t>(fp.p.prefix_len);
    V3 cur_pos = ld3(fp.cam.pos), cur_dir = cp.primary.dir;
    Isect it;
    for (uint32_t ti = 0; ti < max_len; ++ti) {
        trace_closest(a.eval, cur_pos, cur_dir, 1e-3f, 1e16f, it);
        if (!it.valid || ti == max_len - 1) return;
        if (rng.next_float() < nee) {
            const EmitterSample es = sample_emitter(a.eval, rng);
            const V3 light_dir = normalize(es.pos - it.pos);
            const float dist = length(es.pos - it.pos);
            uint32_t mi;
            const BrdfGrad g = grad_at(a, it, light_dir, mi);
            const float dist_factor = 1.0f / (dist * dist);
            mul_nee(sg, g, mi, es, dist_factor);
            if (ti == 0) sg.add_emission(mat_vals(a.eval.mats[mi]).emission, dist_factor, mi);
            return;
        }
        const BrdfSample bs = brdf_sample(a.samp, it, rng);
        uint32_t mi;
        sg.mul_brdf(grad_at(a, it, bs.dir, mi), mi);
        cur_pos = it.pos;
        cur_dir = bs.dir;
    }
}

// Fs: TraceSuffix of a valid gather suffix (path_gen.h:252-387)
template <bool kGrad>
RT_D void seg_suffix(const RAdjView& a, const FrameParams& fp, const Suffix& cs, Seg<kGrad>& sg) {
    sg.init();
    Rng rng{cs.rng};
    const float nee = fp.p.nee_prob;
    const uint32_t max_len = static_cast<uint32_t>(fp.p.max_path_len - fp.p.prefix_len);
    Isect it = unpack(a.eval, cs.last_prefix);
    V3 last_dir = splat(0.0f);
    for (uint32_t vi = 0; vi < max_len; ++vi) {
        if (vi > 0) {
            const V3 last_pos = it.pos;
            trace_closest(a.eval, last_pos, last_dir, 1e-3f, 1e16f, it);
            if (!it.valid) return;
        }
        const bool force_nee = vi == max_len - 1;
        if (rng.next_float() < nee || force_nee) {
            const EmitterSample es = sample_emitter(a.eval, rng);
            const V3 light_vec = es.pos - it.pos;
            const float light_len = length(light_vec);
            const V3 light_dir = normalize(light_vec);
            uint32_t mi;
            const BrdfGrad g = grad_at(a, it, light_dir, mi);
            mul_nee(sg, g, mi, es, 1.0f / (light_len * light_len));
            return;
        }
        const BrdfSample bs = brdf_sample(a.samp, it, rng);
        uint32_t mi;
        sg.mul_brdf(grad_at(a, it, bs.dir, mi), mi);
        last_dir = bs.dir;
    }
}

// T_n: the throughput of the shift of `src` onto the vertex `dst_last`
// (suffix CalcCurrContribInOtherDomain, suffix_reuse.h:10-108) before its
// postReconF; false where the frame's shift failed (its value was zero).
// Validity uses the frozen tables, as the frame did; `passed`: the frame's
// shift value was nonzero, so its occlusion and pdf checks passed and are not
// repeated (a zero value may be a failure: those shifts run every check).
template <bool kGrad>
RT_D bool seg_shift(const RAdjView& a, const Suffix& src, const Isect& dst_last, bool passed, Seg<kGrad>& sg) {
    sg.init();
    if (!fl_valid(src.flags) || !dst_last.valid) return false;
    if (!unpack(a.eval, src.last_prefix).valid) return false;
    Isect src_recon = unpack(a.eval, src.recon);
    if (!src_recon.valid) return false;
    const int nrep = max(static_cast<int>(fl_recon(src.flags)) - 1, 0);
    Isect cur = dst_last;
    Rng srng{src.rng};
    for (int i = 0; i < nrep; ++i) {
        srng.next_float();
        const BrdfSample bs = brdf_sample(a.samp, cur, srng);
        if (!passed && bs.pdf <= 0.0f) return false;
        uint32_t mi;
        sg.mul_brdf(grad_at(a, cur, bs.dir, mi), mi);
        const V3 pos = cur.pos;
        trace_closest(a.eval, pos, bs.dir, 1e-3f, 1e16f, cur);
        if (!cur.valid) return false;
    }
    const V3 rv = src_recon.pos - cur.pos;
    const float rlen = length(rv);
    const V3 rdir = normalize(rv);
    if (!passed) {
        if (nonfinite(rdir)) return false;
        if (occluded(a.eval, cur.pos, rdir, 1e-3f, rlen)) return false;
        if (brdf_eval(a.samp, cur, rdir).pdf <= 0.0f) return false;
    }
    uint32_t m1;
    sg.mul_brdf(grad_at(a, cur, rdir, m1), m1);
    if (fl_recon(src.flags) < fl_len(src.flags)) {
        src_recon.dir = rdir;
        if (!passed && (is_zero(src.rod) || brdf_eval(a.samp, src_recon, src.rod).pdf <= 0.0f)) return false;
        uint32_t m2;
        sg.mul_brdf(grad_at(a, src_recon, src.rod, m2), m2);
    }
    return true;
}

// R_n: the postReconF of the valid suffix sample `src` at theta, re-traced
// from its seed past its reconnection vertex
template <bool kGrad>
RT_D void seg_post(const RAdjView& a, const FrameParams& fp, const Suffix& src, Seg<kGrad>& sg) {
    sg.init();
    const uint32_t len = fl_len(src.flags), r = fl_recon_vert(src.flags);
    const uint32_t max_len = static_cast<uint32_t>(fp.p.max_path_len - fp.p.prefix_len);
    const float nee = fp.p.nee_prob;
    Rng rng{src.rng};
    if (r + 1 >= len) {
        // reconnected at the NEE vertex (the light ray's hit): postReconF =
        // colour * dist_factor of the emitter sampled there; the NEE vertex
        // is not stored, so dist_factor comes from the frozen colour:
        // R = postReconF (.) colour / colour0
        for (uint32_t k = 0; k < 4 * r + 1; ++k) rng.next_u32();
        const EmitterSample es = sample_emitter(a.eval, rng);
        const crisb_emitter& e0 = a.samp.emitters[es.index];
        const V3 c0 = V3{e0.color[0], e0.color[1], e0.color[2]};
        const float cmax = gmax(gmax(c0.x, c0.y), c0.z);
        const float df = cmax > 0.0f ? (cmax == c0.x ? src.prf.x / c0.x : cmax == c0.y ? src.prf.y / c0.y
                                                                                        : src.prf.z / c0.z)
                                     : 0.0f;
        const V3 d = V3{c0.x > 0.0f ? src.prf.x / c0.x : df, c0.y > 0.0f ? src.prf.y / c0.y : df,
                        c0.z > 0.0f ? src.prf.z / c0.z : df};
        sg.val = V3{c0.x > 0.0f ? src.prf.x * (es.color.x / c0.x) : es.color.x * df,
                    c0.y > 0.0f ? src.prf.y * (es.color.y / c0.y) : es.color.y * df,
                    c0.z > 0.0f ? src.prf.z * (es.color.z / c0.z) : es.color.z * df};
        if (kGrad) {
            sg.em = static_cast<int>(es.index);
            sg.d_em = d;
        }
        return;
    }
    for (uint32_t k = 0; k < 4 * (r + 1); ++k) rng.next_u32();
    V3 cur_pos = unpack(a.eval, src.recon).pos, cur_dir = src.rod;
    Isect it;
    for (uint32_t vi = r + 1; vi < max_len; ++vi) {
        trace_closest(a.eval, cur_pos, cur_dir, 1e-3f, 1e16f, it);
        if (!it.valid) return;
        const bool force_nee = vi == max_len - 1;
        if (rng.next_float() < nee || force_nee) {
            const EmitterSample es = sample_emitter(a.eval, rng);
            const V3 light_vec = es.pos - it.pos;
            const float light_len = length(light_vec);
            const V3 light_dir = normalize(light_vec);
            const float dist_factor = 1.0f / (light_len * light_len);
            sg.mul(es.color * dist_factor, -1, splat(0.0f), splat(0.0f), static_cast<int>(es.index),
                   splat(dist_factor));
            if (fl_recon(src.flags) < len) {
                uint32_t mi;
                sg.mul_brdf(grad_at(a, it, light_dir, mi), mi);
            }
            return;
        }
        const BrdfSample bs = brdf_sample(a.samp, it, rng);
        uint32_t mi;
        sg.mul_brdf(grad_at(a, it, bs.dir, mi), mi);
        cur_pos = it.pos;
        cur_dir = bs.dir;
    }
}

// Neighbour terms run as threads of their own, one per (pixel, neighbour
// slot), neighbour-major (thread t = n * P + i): a warp replays the n-th
// neighbours of 32 adjacent pixels instead of one thread replaying all of a
// pixel's neighbours in turn (3 of 32 lanes busy).  The pair buffer holds per
// (pixel, neighbour) the term's value at theta (forward: the pair kernel runs
// first, the pixel kernel adds the terms in the frame's order) or its weight
// dLoss/d(shifted throughput) (backward: the pixel kernel runs first), with
// w = 1 where the frame added the term and 0 elsewhere.

// what the frame's gather read for neighbour n of pixel i (K valid neighbours)
struct NeighTerm {
    uint32_t np;
    float nmis, nwsum, jac;
    V3 f0;      // the shifted value at theta0
    bool used;  // the frame added the term (finite)
};

RT_D NeighTerm neigh_term(const FrameParams& fp, const Bufs& b, uint32_t i, uint32_t n, float K) {
    NeighTerm t;
    t.np = b.neighbors[static_cast<size_t>(i) * fp.k + n].pixel;
    const float4 o0 = b.shift_out[static_cast<size_t>(i) * b.slots + 2 * n];
    t.f0 = xyz(o0);
    t.jac = o0.w;
    t.nwsum = sres_wsum(b.sres_cur, t.np);
    float nmis = mis_neighbor(t.f0, sres_f(b.sres_cur, t.np), t.jac, K, 1.0f, sres_conf(b.sres_cur, t.np));
    if (nonfinite(nmis)) nmis = 0.0f;
    t.nmis = nmis;
    t.used = !nonfinite(nmis * t.f0 * t.nwsum * t.jac);
    return t;
}

// One pixel: kGrad false returns the frozen estimator's value at theta, its
// neighbour terms read from `pairs`; kGrad true adds dl . dL/dtheta of the
// canonical factors at theta0 to the sink, writes the neighbour terms'
// weights into `pairs` and returns zero.
template <bool kGrad>
RT_D V3 gather_pixel(const RAdjView& a, const FrameParams& fp, const Bufs& b, uint32_t i, V3 dl, GradSink* sink,
                     float4* pairs) {
    if (b.canon_prefix[i].primary.prim == CRISB_INVALID_PRIM) return splat(0.0f);  // no gather ran
    const Prefix cp = ld_prefix_v(b.gather_cp[i]);
    if (!fl_valid(cp.flags)) return splat(0.0f);
    Seg<kGrad> sg;
    if (fl_nee(cp.flags)) {  // the gather prefix ended in NEE: Fp / Pp
        if (kGrad && nonfinite(cp.f / cp.p)) return splat(0.0f);
        seg_prefix(a, fp, cp, sg);
        sg.emit(dl / cp.p, sink);
        return sg.val / cp.p;
    }
    const Suffix cs = ld_suffix(b.gather_cs[i].sample);
    if (!fl_valid(cs.flags)) return splat(0.0f);
    const float pp = cp.p, ps = cs.p;
    if (fp.k == 0) {  // canonical contribution alone: Fp Fs / (Pp Ps)
        if (kGrad) {
            if (nonfinite(cp.f * cs.f / (pp * ps))) return splat(0.0f);
            seg_prefix(a, fp, cp, sg);
            sg.emit(dl * cs.f / (pp * ps), sink);
            seg_suffix(a, fp, cs, sg);
            sg.emit(dl * cp.f / (pp * ps), sink);
            return splat(0.0f);
        }
        seg_prefix(a, fp, cp, sg);
        const V3 fpv = sg.val;
        seg_suffix(a, fp, cs, sg);
        return fpv * sg.val / (pp * ps);
    }
    // the frozen weights, from what k_gather_combine read
    const uint32_t P = pixel_count(fp);
    const uint32_t count = b.neigh_count[i];
    const uint32_t vflags = b.pass_flags[i];
    const uint32_t nvalid = __popc(vflags);
    const float K = static_cast<float>(nvalid);
    const float E = static_cast<float>(nvalid + 1), D = K + 1.0f;
    const float4* sh = b.shift_out + static_cast<size_t>(i) * b.slots;
    V3 s0 = splat(0.0f);
    float canon_mis = 1.0f;
    for (uint32_t n = 0; n < count; ++n) {
        if (!(vflags & (1u << n))) continue;
        const NeighTerm t = neigh_term(fp, b, i, n, K);
        if (t.used) s0 = s0 + t.nmis * t.f0 * t.nwsum * t.jac;
        const float4 o1 = sh[2 * n + 1];
        canon_mis += mis_canonical(cs.f, xyz(o1), o1.w, K, 1.0f, sres_conf(b.sres_cur, t.np));
    }
    {
        V3 g0 = s0 * cp.f / pp;
        g0 = g0 / E;
        const V3 r0 = (g0 + (cp.f * cs.f / (pp * ps)) * canon_mis) / D;
        if (nonfinite(r0)) return splat(0.0f);  // the frame stored zero
    }
    if (kGrad) {
        seg_prefix(a, fp, cp, sg);
        sg.emit(dl * ((s0 / pp) / E + (cs.f / (pp * ps)) * canon_mis) / D, sink);
        seg_suffix(a, fp, cs, sg);
        sg.emit(dl * (cp.f / (pp * ps)) * canon_mis / D, sink);
        for (uint32_t n = 0; n < count; ++n) {
            if (!(vflags & (1u << n))) continue;
            const NeighTerm t = neigh_term(fp, b, i, n, K);
            const float wa = t.nmis * t.nwsum * t.jac;
            if (!t.used || wa == 0.0f) continue;  // no term, or no weight: no gradient
            const V3 wn = dl * cp.f * (wa / (pp * E * D));
            pairs[static_cast<size_t>(n) * P + i] = make_float4(wn.x, wn.y, wn.z, 1.0f);
        }
        return splat(0.0f);
    }
    seg_prefix(a, fp, cp, sg);
    const V3 fpv = sg.val;
    seg_suffix(a, fp, cs, sg);
    const V3 canon = fpv * sg.val / (pp * ps);
    V3 suffix_contrib = splat(0.0f);
    for (uint32_t n = 0; n < count; ++n) {
        const float4 c = pairs[static_cast<size_t>(n) * P + i];
        if (c.w != 0.0f) suffix_contrib = suffix_contrib + xyz(c);
    }
    V3 gather = suffix_contrib * fpv / pp;
    gather = gather / E;
    V3 result = gather + (canon * canon_mis);
    return result / D;
}

// the gradient sink of a block: all parameters in shared memory when they fit
struct BlockSink {
    GradSink sink;
    float* sh;
    uint32_t n_sh;
    RT_D void begin() {
        if (sh) {
            for (uint32_t k = threadIdx.x; k < n_sh; k += blockDim.x) sh[k] = 0.0f;
            __syncthreads();
        }
    }
    RT_D void end() {
        if (sh) {
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < n_sh; k += blockDim.x) {
                const float v = sh[k];
                if (v == 0.0f) continue;
                if (k < sink.num_mats * kMatGrad) atomicAdd(&sink.g_mat[k], v);
                else atomicAdd(&sink.g_em[k - sink.num_mats * kMatGrad], v);
            }
        }
    }
};

template <bool kGrad>
__global__ void __launch_bounds__(kPassBlock) k_restir_adjoint(RAdjView a, FrameParams fp, Bufs b, const float* d_img,
                                                               float* out, float4* pairs, float* g_mat, float* g_em,
                                                               int use_shared) {
    extern __shared__ float shm[];
    BlockSink bs{GradSink{kGrad && use_shared ? shm : nullptr, g_mat, g_em, a.num_mats},
                 kGrad && use_shared ? shm : nullptr, a.num_mats * kMatGrad + a.eval.num_emitters * kEmGrad};
    bs.begin();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t P = pixel_count(fp);
    if (i < P) {
        if (kGrad) {
            for (uint32_t n = 0; n < fp.k; ++n) pairs[static_cast<size_t>(n) * P + i] = make_float4(0.f, 0.f, 0.f, 0.f);
            const V3 dl = V3{d_img[3 * i], d_img[3 * i + 1], d_img[3 * i + 2]};
            if (!nonfinite(dl) && !is_zero(dl)) gather_pixel<true>(a, fp, b, i, dl, &bs.sink, pairs);
        } else {
            V3 L = splat(0.0f) + gather_pixel<false>(a, fp, b, i, splat(0.0f), nullptr, pairs);
            if (nonfinite(L)) L = splat(0.0f);
            out[3 * i] = L.x;
            out[3 * i + 1] = L.y;
            out[3 * i + 2] = L.z;
        }
    }
    bs.end();
}

// one neighbour term per thread: forward, its value at theta; backward, the
// gradient of its shifted throughput T_n (.) R_n under the weight the pixel
// kernel wrote.  Only slots below the pixel's neighbour count (written by the
// frame's query for every pixel) are read.
template <bool kGrad>
__global__ void __launch_bounds__(kPassBlock) k_restir_pairs(RAdjView a, FrameParams fp, Bufs b, float4* pairs,
                                                             float* g_mat, float* g_em, int use_shared) {
    extern __shared__ float shm[];
    BlockSink bs{GradSink{kGrad && use_shared ? shm : nullptr, g_mat, g_em, a.num_mats},
                 kGrad && use_shared ? shm : nullptr, a.num_mats * kMatGrad + a.eval.num_emitters * kEmGrad};
    bs.begin();
    const uint32_t P = pixel_count(fp);
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < P * fp.k) {
        const uint32_t n = t / P, i = t - n * P;
        Seg<kGrad> sg;
        if (kGrad) {
            const float4 w4 = pairs[t];
            if (w4.w != 0.0f) {
                const V3 wn = xyz(w4);
                const uint32_t np_ = b.neighbors[static_cast<size_t>(i) * fp.k + n].pixel;
                const Suffix ns = ld_sres(b.sres_cur, np_).s;
                const float4 o0 = b.shift_out[static_cast<size_t>(i) * b.slots + 2 * n];
                const Isect dst_last = unpack(a.eval, ld_hit(b.gather_cs[i].sample.last_prefix));
                if (seg_shift(a, ns, dst_last, !is_zero(xyz(o0)), sg)) {
                    sg.emit(wn * ns.prf, &bs.sink);
                    const V3 tn = sg.val;
                    seg_post(a, fp, ns, sg);
                    sg.emit(wn * tn, &bs.sink);
                }
            }
        } else {
            float4 res = make_float4(0.f, 0.f, 0.f, 0.f);
            const uint32_t vflags = b.pass_flags[i];
            if (n < b.neigh_count[i] && ((vflags >> n) & 1u)) {
                const NeighTerm tm = neigh_term(fp, b, i, n, static_cast<float>(__popc(vflags)));
                if (tm.used) {
                    const Suffix ns = ld_sres(b.sres_cur, tm.np).s;
                    const Isect dst_last = unpack(a.eval, ld_hit(b.gather_cs[i].sample.last_prefix));
                    V3 fshift = splat(0.0f);
                    if (seg_shift(a, ns, dst_last, !is_zero(tm.f0), sg)) {
                        const V3 tn = sg.val;
                        seg_post(a, fp, ns, sg);
                        fshift = tn * sg.val;
                    }
                    const V3 c = tm.nmis * fshift * tm.nwsum * tm.jac;
                    res = make_float4(c.x, c.y, c.z, 1.0f);
                }
            }
            pairs[t] = res;
        }
    }
    bs.end();
}

RAdjView make_view(const SceneView& eval, const crisb_material* frame_mats, const crisb_emitter* frame_emitters,
                   uint32_t num_mats) {
    RAdjView a;
    a.eval = eval;
    a.samp = eval;
    a.samp.mats = frame_mats;
    a.samp.emitters = frame_emitters;
    a.num_mats = num_mats;
    return a;
}

}  // namespace

void restir_adjoint_forward(const SceneView& eval, const crisb_material* frame_mats,
                            const crisb_emitter* frame_emitters, uint32_t num_mats, const FrameParams& fp,
                            const Bufs& b, float4* pairs, float* out, cudaStream_t st) {
    const RAdjView a = make_view(eval, frame_mats, frame_emitters, num_mats);
    const uint32_t P = fp.width * fp.height;
    if (fp.k > 0)
        k_restir_pairs<false><<<(P * fp.k + kPassBlock - 1) / kPassBlock, kPassBlock, 0, st>>>(a, fp, b, pairs, nullptr,
                                                                                              nullptr, 0);
    k_restir_adjoint<false><<<(P + kPassBlock - 1) / kPassBlock, kPassBlock, 0, st>>>(a, fp, b, nullptr, out, pairs,
                                                                                       nullptr, nullptr, 0);
}

void restir_adjoint_backward(const SceneView& eval, const crisb_material* frame_mats,
                             const crisb_emitter* frame_emitters, uint32_t num_mats, const FrameParams& fp,
                             const Bufs& b, float4* pairs, const float* d_img, float* g_mat, float* g_em,
                             cudaStream_t st) {
    const RAdjView a = make_view(eval, frame_mats, frame_emitters, num_mats);
    const uint32_t P = fp.width * fp.height;
    const size_t sh_bytes = (static_cast<size_t>(num_mats) * kMatGrad + eval.num_emitters * kEmGrad) * sizeof(float);
    const int use_shared = sh_bytes <= 48u * 1024u ? 1 : 0;
    const size_t shb = use_shared ? sh_bytes : 0;
    k_restir_adjoint<true><<<(P + kPassBlock - 1) / kPassBlock, kPassBlock, shb, st>>>(a, fp, b, d_img, nullptr, pairs,
                                                                                       g_mat, g_em, use_shared);
    if (fp.k > 0)
        k_restir_pairs<true><<<(P * fp.k + kPassBlock - 1) / kPassBlock, kPassBlock, shb, st>>>(a, fp, b, pairs, g_mat,
                                                                                               g_em, use_shared);
}

}  // namespace crisb
