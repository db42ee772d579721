// reuse_passes.cu -- prefix generation + temporal reuse, suffix temporal
// reuse, suffix spatial reuse and the final gather, each split into three
// kernels:
//
//   1. a per-pixel kernel that does everything sequential in the pixel's RNG
//      stream (canonical path tracing, neighbour selection, the endpoint
//      query) and appends one job per needed shift to a compacted list;
//   2. one kernel over that list evaluating the hybrid shifts (the expensive,
//      traversal-heavy part) as independent, uniform work items;
//   3. a per-pixel kernel that streams the shifted candidates through pairwise
//      MIS and the reservoir in the reference's order.
//
// Shifts are pure functions of their two records, so the split evaluates the
// same operations as the per-pixel formulation (shader/suffix_gen_temp_reuse.cu,
// shader/suffix_spatial_reuse.cu, shader/final_gather.cu:69-188,
// shader/prefix_gen_temp_reuse.cu) and gives
// the same bits; only the SIMD utilisation changes.
#include <algorithm>
#include <mutex>

#include "queues.cuh"
#include "records.cuh"

namespace crisb {
namespace {

constexpr uint32_t kStFinal = 0;      // nothing left to do in the combine kernel
constexpr uint32_t kStCanonOnly = 1;  // temporal: stream the canonical sample only
constexpr uint32_t kStReuse = 2;      // reuse with the shift results

enum ShiftMode : int { kModeTemporal = 0, kModeSpatial = 1, kModeGather = 2 };

constexpr uint32_t kSlotBits = 6;  // job code = pixel << 6 | slot

// Append the job slots set in `mask` for pixel i to the list.  Every thread of
// the warp must call this (warp-aggregated reservation of list space).
RT_D void push_jobs(const Bufs& b, uint32_t i, uint64_t mask) {
    const uint32_t n = static_cast<uint32_t>(__popcll(mask));
    const int lane = threadIdx.x & 31;
    uint32_t incl = n;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && total) base = atomicAdd(b.job_count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    uint32_t pos = base + incl - n;
    while (mask) {
        const int bit = __ffsll(static_cast<long long>(mask)) - 1;
        mask &= mask - 1;
        b.job_items[pos++] = (i << kSlotBits) | static_cast<uint32_t>(bit);
    }
}

RT_D V3 xyz(float4 v) { return V3{v.x, v.y, v.z}; }

// ---- 2. the shift jobs ------------------------------------------------------------
// Slot 2n: neighbour / previous sample shifted onto the pixel's own path;
// slot 2n+1: the pixel's own sample shifted onto the neighbour's.
// statistics view of the shift kernels: rays and jobs in their own counters
SceneView shift_view(const SceneView& s) {
    SceneView v = s;
    if (v.ray_count) v.ray_count += 2;
    return v;
}

RT_D void count_jobs(const SceneView& s, uint32_t total) {
    if (s.ray_count && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&s.ray_count[2], static_cast<unsigned long long>(total));
}

// ---- shift machines ---------------------------------------------------------------
// A shift job is CalcCurrContribInOtherDomain of the reference
// (include/graph/restir/suffix_reuse.h:10-123 for suffixes,
// include/graph/restir/prefix_reuse.h for prefixes) cut at its rays: the
// replayed bounces are closest-hit rays traced by the queue kernels, and the
// reconnection edge is one shadow ray.  The BRDF terms, the Jacobian and the
// shifted contribution do not depend on the visibility result, so they are
// evaluated before the shadow ray is queued and the ray only selects between
// them and zero -- the value the per-job function returns when the edge is
// occluded.  Jobs that still need a replay in the last round finish inline.
// Three rounds: 4 / 5 / 6 rounds cut the shift steps from 1.46 to 1.40 / 1.27
// / 1.20 ms per 1080p frame but added more in traversal launches (frame 17.04
// -> 17.20 / 17.32 / 17.35 ms).
constexpr int kShiftRounds = 3;
constexpr int kModePrefix = 3;  // prefix temporal reuse (slot 0: previous onto canonical)
// prefix spatial reuse (slot 2n: neighbour n onto the pixel's prefix; 2n + 1:
// the pixel's prefix onto neighbour n's)
constexpr int kModePrefixSpatial = 4;
// the final gather's extra prefixes (slot 2n: neighbour n's suffix onto the
// extra prefix's last vertex)
constexpr int kModeGatherExtra = 5;

RT_HD bool prefix_mode(int mode) { return mode == kModePrefix || mode == kModePrefixSpatial; }

// source path of a job
struct ShiftSrc {
    uint64_t rng;
    uint32_t flags;
    Hit anchor;  // suffix: the source's last prefix vertex; prefix: its primary hit
    Hit recon;
    V3 prf, rod;
};

RT_D ShiftSrc shift_src(const Suffix& S) { return ShiftSrc{S.rng, S.flags, S.last_prefix, S.recon, S.prf, S.rod}; }
RT_D ShiftSrc shift_src(const Prefix& P) { return ShiftSrc{P.rng, P.flags, P.primary, P.recon, P.prf, P.rod}; }

// the previous pixel of pixel i (its G-buffer entry; i itself without
// reprojection); only called for pixels whose previous pixel exists
RT_D uint32_t prev_pixel(const FrameParams& fp, const Bufs& b, uint32_t i) {
    return fp.p.motion_mode == CRISB_MOTION_NONE ? i : prev_index(b.gbuf[i].prev_xy, fp.width);
}

// the job's source path and, when `dst` is given, its destination vertex
RT_D ShiftSrc resolve_job(const FrameParams& fp, const Bufs& b, int mode, uint32_t code, Hit* dst) {
    const uint32_t i = code >> kSlotBits, slot = code & ((1u << kSlotBits) - 1), n = slot >> 1;
    if (mode == kModePrefixSpatial) {
        // neighbours from the back buffer (equal to the front at pass start),
        // the pixel's own prefix from the front buffer
        const uint32_t ni = b.spatial_nbr[static_cast<size_t>(i) * (b.slots >> 1) + n];
        if ((slot & 1u) == 0) {
            if (dst) *dst = pres_primary(b.pres[fp.front], i);
            return shift_src(ld_pres(b.pres[fp.back], ni).s);
        }
        if (dst) *dst = pres_primary(b.pres[fp.back], ni);
        return shift_src(ld_pres(b.pres[fp.front], i).s);
    }
    if (mode == kModePrefix) {
        // slot 0: the previous prefix onto the canonical one; slot 1: back
        const uint32_t pi = prev_pixel(fp, b, i);
        if (slot == 0) {
            if (dst) *dst = ld_hit(b.canon_prefix[i].primary);
            return shift_src(ld_pres(b.pres[fp.back], pi).s);
        }
        if (dst) *dst = pres_primary(b.pres[fp.back], pi);
        return shift_src(ld_prefix_v(b.canon_prefix[i]));
    }
    if (mode == kModeGatherExtra) {
        if (dst) *dst = ld_hit(b.gather_last[i]);
        return shift_src(ld_sres(b.sres_cur, b.neighbors[static_cast<size_t>(i) * fp.k + n].pixel).s);
    }
    const bool onto_own = (slot & 1u) == 0;
    SufRef own, other;
    if (mode == kModeTemporal) {
        own = SufRef{b.canon_suffix, b.sres_cur, i};  // canonical; "other" is the previous sample
        other = SufRef{nullptr, b.sres_cur, prev_pixel(fp, b, i)};
    } else if (mode == kModeSpatial) {
        own = SufRef{nullptr, b.sres_cur, i};
        other = SufRef{nullptr, b.sres_cur, b.spatial_nbr[static_cast<size_t>(i) * (b.slots >> 1) + n]};
    } else {
        own = SufRef{b.gather_cs, b.sres_cur, i};
        other = SufRef{nullptr, b.sres_cur, b.neighbors[static_cast<size_t>(i) * fp.k + n].pixel};
    }
    if (dst) *dst = ld_suf_last(onto_own ? own : other);
    return shift_src(ld_suf(onto_own ? other : own));
}

// the job's destination vertex as an interaction: a stored hit re-derived as
// the reference unpacks it (interpolated, unnormalised normal), except the
// extra gather prefix's last vertex, which the reference hands over straight
// from the trace (normalised normal, trace_closest)
RT_D Isect job_dst(const SceneView& s, int mode, const Hit& h) {
    Isect it = unpack(s, h);
    if (mode == kModeGatherExtra && it.valid) it.nrm = normalize(it.nrm);
    return it;
}

RT_D void job_out(const Bufs& b, uint32_t code, float4 v) {
    const uint32_t i = code >> kSlotBits, slot = code & ((1u << kSlotBits) - 1);
    b.shift_out[static_cast<size_t>(i) * b.slots + slot] = v;
}

// Runs the job from vertex `cur` with `left` replays to go: queues its next
// ray (returned request) or, when `inline_rays`, traces the remaining rays in
// place; a finished job writes its result.
template <bool kTex>
RT_D int shift_advance(const SceneView& s, const Bufs& b, bool prefix, const ShiftSrc& src, ShiftJob& j, Isect cur,
                       Rng& srng, V3 tp, uint32_t left, bool inline_rays) {
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    while (left > 0) {
        srng.next_float();
        const BrdfSample bs = brdf_sample<kTex>(s, cur, srng);
        if (bs.pdf <= 0.0f) {
            job_out(b, j.code, zero);
            return kReqDone;
        }
        tp = tp * bs.brdf;
        --left;
        if (!inline_rays) {
            j.o = f4(cur.pos, 0.0f);
            j.d = f4(bs.dir, 0.0f);
            j.acc = f4(tp, 0.0f);
            j.rng = srng.state;
            j.ctr = left;
            return kReqClosest;
        }
        const V3 pos = cur.pos;
        trace_closest(s, pos, bs.dir, 1e-3f, 1e16f, cur);
        if (!cur.valid) {
            job_out(b, j.code, zero);
            return kReqDone;
        }
    }
    // the reconnection edge
    const Isect src_anchor = unpack(s, src.anchor);
    Isect src_recon = unpack(s, src.recon);
    const V3 rv = src_recon.pos - cur.pos;
    const float rlen = length(rv);
    const V3 rdir = normalize(rv);
    if ((prefix && isinf(rlen)) || nonfinite(rdir)) {
        job_out(b, j.code, zero);
        return kReqDone;
    }
    const BrdfEval b1 = brdf_eval<kTex>(s, cur, rdir);
    float4 res = zero;
    if (b1.pdf > 0.0f) {
        tp = tp * b1.brdf;
        bool ok = true;
        if (prefix || fl_recon(src.flags) < fl_len(src.flags)) {
            src_recon.dir = rdir;
            if (!prefix && is_zero(src.rod)) ok = false;
            if (ok) {
                const BrdfEval b2 = brdf_eval<kTex>(s, src_recon, src.rod);
                if (b2.pdf <= 0.0f) ok = false;
                else tp = tp * b2.brdf;
            }
        }
        if (ok) {
            const float jac = recon_jacobian(src_anchor.pos, cur.pos, src_recon.pos, src_recon.nrm);
            const V3 f = prefix ? gmax(splat(0.0f), tp * src.prf) : tp * src.prf;
            res = f4(f, jac);
        }
    }
    if ((__float_as_uint(res.x) | __float_as_uint(res.y) | __float_as_uint(res.z) | __float_as_uint(res.w)) == 0u) {
        job_out(b, j.code, zero);  // +0 whether or not the edge is visible
        return kReqDone;
    }
    if (inline_rays) {
        job_out(b, j.code, occluded(s, cur.pos, rdir, 1e-3f, rlen) ? zero : res);
        return kReqDone;
    }
    j.o = f4(cur.pos, rlen);
    j.d = f4(rdir, 0.0f);
    j.acc = res;
    return kReqShadow;
}

// a job waiting for its ray: everything but the hit word, which the traversal
// kernels write
RT_D void job_store(ShiftJob* r, const ShiftJob& j) {
    r->o = j.o;
    r->d = j.d;
    r->acc = j.acc;
    r->rng = j.rng;
    r->code = j.code;
    r->ctr = j.ctr;
}

RT_D void job_push(const Bufs& b, int round, int req, uint32_t t) {
    q_append(b.job_queue[2 * round], &b.job_qcount[2 * round], req == kReqClosest, t);
    q_append(b.job_queue[2 * round + 1], &b.job_qcount[2 * round + 1], req == kReqShadow, t);
}

// first step of every job of the list: the checks of the reference function,
// then the first ray
// kTex: the scene has textured materials
template <bool kTex>
__global__ void __launch_bounds__(kPassBlock) k_shift_begin(SceneView s, FrameParams fp, Bufs b, int mode) {
    const uint32_t all = *b.job_count;
    count_jobs(s, all);
    const uint32_t total = min(all, b.job_cap);
    const bool prefix = prefix_mode(mode);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        int req = kReqDone;
        if (t < total) {
            ShiftJob j;
            j.code = b.job_items[t];
            Hit dh;
            const ShiftSrc src = resolve_job(fp, b, mode, j.code, &dh);
            const Isect cur = job_dst(s, mode, dh);
            bool ok = fl_valid(src.flags) && cur.valid;
            if (prefix) ok = ok && fl_recon(src.flags) >= 2;
            ok = ok && unpack(s, src.anchor).valid && unpack(s, src.recon).valid;
            if (!ok) {
                job_out(b, j.code, zero);
            } else {
                const int skip = prefix ? 2 : 1;
                const uint32_t left = static_cast<uint32_t>(max(static_cast<int>(fl_recon(src.flags)) - skip, 0));
                Rng srng{src.rng};
                req = shift_advance<kTex>(s, b, prefix, src, j, cur, srng, splat(1.0f), left, false);
                if (req != kReqDone) job_store(b.jobs + t, j);
            }
        }
        job_push(b, 0, req, t);
    }
}

// list entries beyond the machines' capacity: the same job, every ray traced
// in place (shift_advance with inline rays is the machine's own step)
template <bool kTex>
__global__ void __launch_bounds__(kPassBlock) k_shift_overflow(SceneView s, FrameParams fp, Bufs b, int mode) {
    const uint32_t total = *b.job_count;
    const bool prefix = prefix_mode(mode);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t t = b.job_cap + blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        ShiftJob j;
        j.code = b.job_items[t];
        Hit dh;
        const ShiftSrc src = resolve_job(fp, b, mode, j.code, &dh);
        const Isect cur = job_dst(s, mode, dh);
        bool ok = fl_valid(src.flags) && cur.valid;
        if (prefix) ok = ok && fl_recon(src.flags) >= 2;
        ok = ok && unpack(s, src.anchor).valid && unpack(s, src.recon).valid;
        if (!ok) {
            job_out(b, j.code, zero);
            continue;
        }
        const int skip = prefix ? 2 : 1;
        const uint32_t left = static_cast<uint32_t>(max(static_cast<int>(fl_recon(src.flags)) - skip, 0));
        Rng srng{src.rng};
        shift_advance<kTex>(s, b, prefix, src, j, cur, srng, splat(1.0f), left, true);
    }
}

// resume every job whose ray of round `cur` finished; in the last round jobs
// with replays left finish inline
template <bool kLast, bool kTex>
__global__ void __launch_bounds__(kPassBlock) k_shift_step(SceneView s, FrameParams fp, Bufs b, int mode, int cur) {
    const uint32_t nc = b.job_qcount[2 * cur], ns = b.job_qcount[2 * cur + 1];
    const uint32_t total = nc + ns;
    const uint32_t* qc = b.job_queue[2 * cur];
    const uint32_t* qs = b.job_queue[2 * cur + 1];
    const bool prefix = prefix_mode(mode);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        const uint32_t u = base + threadIdx.x;
        int req = kReqDone;
        uint32_t t = 0;
        if (u < total) {
            t = u < nc ? qc[u] : qs[u - nc];
            const ShiftJob* jr = b.jobs + t;
            if (u >= nc) {
                // the shadow ray's result: occluded flag, prepared value, job code
                job_out(b, jr->code, __float_as_uint(jr->hit.x) ? zero : jr->acc);
            } else {
                ShiftJob j;  // o is written before it is read
                j.d = jr->d;
                j.hit = jr->hit;
                j.acc = jr->acc;
                j.rng = jr->rng;
                j.code = jr->code;
                j.ctr = jr->ctr;
                // trace_closest semantics: interpolated, normalised normal
                Isect it;
                const uint32_t prim = __float_as_uint(j.hit.x);
                it.dir = f3(j.d);
                it.valid = prim != CRISB_INVALID_PRIM;
                if (!it.valid) {
                    job_out(b, j.code, zero);
                } else {
                    it.prim = prim;
                    it.bu = j.hit.z;
                    it.bv = j.hit.w;
                    const ShadeTri tri = load_shade(s, prim);
                    it.pos = interp(it.bu, it.bv, tri.p0, tri.p1, tri.p2);
                    it.nrm = normalize(interp(it.bu, it.bv, tri.n0, tri.n1, tri.n2));
                    const ShiftSrc src = resolve_job(fp, b, mode, j.code, nullptr);
                    Rng srng{j.rng};
                    req = shift_advance<kTex>(s, b, prefix, src, j, it, srng, f3(j.acc), j.ctr, kLast);
                    if (req != kReqDone) job_store(b.jobs + t, j);
                }
            }
        }
        if (!kLast) job_push(b, cur ^ 1, req, t);
    }
}

// ---- suffix generation + temporal reuse (shader/suffix_gen_temp_reuse.cu) --------
// per pixel after the suffix paths (wavefront.cu, suffix flow) finished:
// the temporal-reuse decision and its shift jobs
__global__ void __launch_bounds__(kPassBlock) k_suffix_temp_finish(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp)) {
        uint32_t st = kStFinal;
        if (b.pass_status[i] == kWfPath) {  // else the init kernel invalidated the reservoir
            b.gbuf[i].rng = b.wf[i].rng;
            const uint32_t prev_xy = b.gbuf[i].prev_xy;
            if (!fl_valid(b.canon_suffix[i].sample.flags)) {
                Res<Suffix> cur = ld_sres(b.sres_cur, i);
                invalidate(cur);
                st_sres(b.sres_next, i, cur);
                b.nval_next[i] = 0;
            } else if (!fp.p.suffix_enable_temporal || prev_xy == kPrevNone) {
                st = kStCanonOnly;
            } else {
                const uint32_t pi = prev_pixel(fp, b, i);
                if (sres_wsum(b.sres_cur, pi) <= 0.0f || !fl_valid(sres_flags(b.sres_cur, pi))) {
                    st = kStCanonOnly;
                } else {
                    st = kStReuse;
                    mask = 3;
                }
            }
        }
        b.pass_status[i] = st;
    }
    push_jobs(b, i, mask);
}

// resampling kernels (selection and combines) at 10 resident 128-thread
// blocks per SM (48 registers, a few spills): their candidate chains are
// latency-bound, and more warps in flight beat the spills (0.935 -> 0.902 ms
// per 1080p frame; 12 and 16 blocks spill more: 0.995 and 1.23 ms).  Their
// reservoir stores stay per thread: storing a warp's records as one run
// through shared memory (as the path-machine init kernels do) took 0.895 ->
// 1.09 ms, the kernels having to reach the store with every lane.
constexpr int kResampleMinBlocks = 10;

__global__ void __launch_bounds__(kPassBlock, kResampleMinBlocks) k_suffix_temp_combine(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    ByteTally bt(b, kTallyTemporalCombine);
    const uint32_t st = b.pass_status[i];
    bt.add(4);
    if (st == kStFinal) return;
    // Reservoir::Update's arithmetic with the chosen sample tracked by index
    // (0: the sample the reset reservoir still holds, 1: the canonical suffix,
    // 2: the previous sample shifted onto it); the candidates contribute their
    // weight fields and the chosen record is read once at the end.
    const crisb_suffix_rec& cs = b.canon_suffix[i].sample;
    const V3 canon_f = ld3(cs.f);
    const float canon_p = cs.p;
    Rng rng{b.gbuf[i].rng};
    bt.add(12 + 4 + 8);  // canonical f and p, RNG
    const float canon_phat = luminance(canon_f);
    float w_sum = 0.0f, conf = 0.0f;
    int sel = 0;
    V3 f_canon_of_prev = splat(0.0f);
    // suffixReservoirs[back][prevPixelIdx]: the previous frame's reservoirs are
    // the pass-start state sres_cur; this pass writes sres_next
    uint32_t pi = i;
    const float K = 1.0f;
    if (st == kStCanonOnly) {
        if (res_choose(w_sum, conf, canon_phat / canon_p, rng, 1.0f)) sel = 1;
    } else {
        pi = prev_pixel(fp, b, i);
        const V3 prev_f = sres_f(b.sres_cur, pi);
        const float prev_conf = sres_conf(b.sres_cur, pi), prev_wsum = sres_wsum(b.sres_cur, pi);
        const float4 o0 = b.shift_out[static_cast<size_t>(i) * b.slots];
        const float4 o1 = b.shift_out[static_cast<size_t>(i) * b.slots + 1];
        bt.add(weight_bytes(b.sres_cur.f16) + 32);
        f_canon_of_prev = xyz(o0);
        const V3 f_prev_of_canon = xyz(o1);
        const float jac_prev_to_canon = o0.w, jac_canon_to_prev = o1.w;
        const float p_canon_of_prev = luminance(f_canon_of_prev) * jac_prev_to_canon;
        const float prev_mis = mis_neighbor(f_canon_of_prev, prev_f, jac_prev_to_canon, K, 1.0f, prev_conf);
        const float canon_mis =
            1.0f + mis_canonical(canon_f, f_prev_of_canon, jac_canon_to_prev, K, 1.0f, prev_conf);
        if (res_choose(w_sum, conf, canon_mis * canon_phat / canon_p, rng, 1.0f)) sel = 1;
        if (res_choose(w_sum, conf, prev_mis * p_canon_of_prev * prev_wsum, rng, prev_conf)) sel = 2;
    }
    Res<Suffix> cur;
    if (sel == 0) {
        cur.s = ld_sres(b.sres_cur, i).s;
        bt.add(sres_bytes(b.sres_cur));
    } else if (sel == 1) {
        cur.s = ld_suffix(cs);
        bt.add(sizeof(crisb_suffix_rec));
    } else {
        // SuffixPath(prev, canon.lastPrefixInt, fFromCanonOfPrev)
        cur.s = ld_sres(b.sres_cur, pi).s;
        cur.s.last_prefix = ld_hit(cs.last_prefix);
        cur.s.f = f_canon_of_prev;
        bt.add(sres_bytes(b.sres_cur) + sizeof(crisb_hit_rec));
    }
    cur.w_sum = w_sum;
    cur.conf = conf;
    if (st == kStCanonOnly) {
        res_finalize(cur);
    } else if (cur.w_sum > 0.0f) {
        cur.w_sum /= K + 1.0f;
        res_finalize(cur);
    }
    b.gbuf[i].rng = rng.state;
    st_sres(b.sres_next, i, cur);
    // this combine runs only for a valid prefix (not NEE) and canonical suffix
    b.nval_next[i] = nval_bits(b.gbuf[i].flags & 1u, true, fl_valid(cur.s.flags));
    bt.add(8 + sres_bytes(b.sres_next) + 1 + 4);  // RNG, reservoir and byte out, primary-valid flag
}

// ---- suffix spatial reuse (shader/suffix_spatial_reuse.cu:16-167) -----------------
// Reads the pass-start state sres_cur (own and neighbours), writes sres_next.
__global__ void __launch_bounds__(kPassBlock, kResampleMinBlocks) k_suffix_spatial_select(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp)) {
        ByteTally bt(b, kTallySpatialSelect);
        // the pixel's byte in, the status word out
        bt.add(1 + 4);
        const uint32_t x = i % fp.width, y = i / fp.width;
        uint32_t st = kStFinal;
        // valid prefix (not NEE), valid reservoir sample and canonical suffix
        // (suffix_spatial_reuse.cu:18-35), as recorded by the previous combine
        if (b.nval_cur[i] & kNvalSpatial) {
            st = kStReuse;
            Rng rng{b.gbuf[i].rng};
            uint32_t vflags = 0;
            uint32_t* nbr = b.spatial_nbr + static_cast<size_t>(i) * (b.slots >> 1);
            for (int n = 0; n < fp.p.suffix_spatial_count; ++n) {
                uint32_t nx, ny;
                select_spatial_neighbor(x, y, static_cast<uint32_t>(fp.p.window_radius), rng, nx, ny);
                if (!(nx < fp.width && ny < fp.height)) continue;
                const uint32_t ni = ny * fp.width + nx;
                bt.add(1);
                if (!(b.nval_cur[ni] & kNvalNeighbor)) continue;  // primary valid && reservoir sample valid
                nbr[n] = ni;
                bt.add(4);
                vflags |= 1u << n;
                mask |= 3ull << (2 * n);
            }
            b.gbuf[i].rng = rng.state;
            b.pass_flags[i] = vflags;
            bt.add(8 + 8 + 4);
        }
        b.pass_status[i] = st;
    }
    push_jobs(b, i, mask);
}

__global__ void __launch_bounds__(kPassBlock, kResampleMinBlocks) k_suffix_spatial_combine(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    ByteTally bt(b, kTallySpatialCombine);
    bt.add(4);
    if (b.pass_status[i] == kStFinal) {
        Res<Suffix> cur = ld_sres(b.sres_cur, i);
        invalidate(cur);
        st_sres(b.sres_next, i, cur);
        b.nval_next[i] = 0;
        bt.add(sres_bytes(b.sres_cur) + sres_bytes(b.sres_next) + 1);
        return;
    }
    Rng rng{b.gbuf[i].rng};
    // the pixel's own sample: its weight fields now, its record at the end
    const V3 own_f = sres_f(b.sres_cur, i);
    const float cur_wsum = sres_wsum(b.sres_cur, i), cur_conf = sres_conf(b.sres_cur, i);
    const uint32_t vflags = b.pass_flags[i];
    bt.add(8 + weight_bytes(b.sres_cur.f16) + 4);  // RNG, own weight fields, neighbour flags
    float w_sum = 0.0f, conf = 0.0f;
    const float K = static_cast<float>(__popc(vflags));
    const uint32_t* nbr = b.spatial_nbr + static_cast<size_t>(i) * (b.slots >> 1);
    const float4* sh = b.shift_out + static_cast<size_t>(i) * b.slots;
    // The reservoir's choices depend on the candidates' weights only, so the
    // neighbours contribute f, confidence and weight here and the record of
    // the chosen one is read once at the end (Reservoir::Update's arithmetic,
    // with the chosen sample tracked by index: -1 is the pixel's own sample,
    // which the reset reservoir also still holds).
    int sel = -1;
    V3 sel_f = own_f;
    float canon_mis = 1.0f;
    for (int n = 0; n < fp.p.suffix_spatial_count; ++n) {
        if (!((vflags >> n) & 1u)) continue;
        const uint32_t ni = nbr[n];
        const V3 nf = sres_f(b.sres_cur, ni);
        const float nconf = sres_conf(b.sres_cur, ni), nwsum = sres_wsum(b.sres_cur, ni);
        const float4 o0 = sh[2 * n], o1 = sh[2 * n + 1];
        bt.add(4 + weight_bytes(b.sres_cur.f16) + 32);  // index, weight fields, two shift results
        const V3 f_c_of_n = xyz(o0), f_n_of_c = xyz(o1);
        const float jac_n2c = o0.w, jac_c2n = o1.w;
        const float p_c_of_n = luminance(f_c_of_n) * jac_n2c;
        float nmis = mis_neighbor(f_c_of_n, nf, jac_n2c, K, cur_conf, nconf);
        if (nonfinite(nmis)) nmis = 0.0f;
        if (res_choose(w_sum, conf, nmis * p_c_of_n * nwsum, rng, nconf)) {
            sel = n;
            sel_f = f_c_of_n;
        }
        canon_mis += mis_canonical(own_f, f_n_of_c, jac_c2n, K, cur_conf, nconf);
    }
    if (nonfinite(canon_mis)) canon_mis = 0.0f;
    if (res_choose(w_sum, conf, canon_mis * cur_wsum * luminance(own_f), rng, cur_conf)) {
        sel = -1;
        sel_f = own_f;
    }
    Res<Suffix> cur;
    if (sel >= 0) {
        // SuffixPath(neighbour, currSuffix.lastPrefixInt, fFromCanonOfNeigh)
        cur.s = ld_sres(b.sres_cur, nbr[sel]).s;
        cur.s.last_prefix = sres_last_prefix(b.sres_cur, i);
        cur.s.f = sel_f;
        bt.add(sres_bytes(b.sres_cur) + (b.sres_cur.f16 ? sizeof(crisb_hit16_rec) : sizeof(crisb_hit_rec)));
    } else {
        cur.s = ld_sres(b.sres_cur, i).s;
        bt.add(sres_bytes(b.sres_cur));
    }
    cur.w_sum = w_sum;
    cur.conf = conf;
    if (cur.w_sum > 0.0f) {
        cur.w_sum /= K + 1.0f;
        res_finalize(cur);
    }
    b.gbuf[i].rng = rng.state;
    st_sres(b.sres_next, i, cur);
    // the pixel took part in this round: its prefix and canonical suffix are valid
    b.nval_next[i] = nval_bits(b.gbuf[i].flags & 1u, true, fl_valid(cur.s.flags));
    bt.add(8 + sres_bytes(b.sres_next) + 1 + 4);  // RNG, reservoir and byte out, primary-valid flag
}

// ---- final gather with gatherN == 1 (shader/final_gather.cu:69-188, 290-356) -----
// The gather flow of wavefront.cu traces the canonical prefix + suffix;
// k_gather_finish forms the canonical contribution; k_gather_query runs the
// endpoint search for the pixels that need it and emits their shift jobs.
constexpr uint32_t kStQuery = 3;

// per pixel after the canonical paths (wavefront.cu, gather flow) finished
__global__ void __launch_bounds__(kPassBlock) k_gather_finish(FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    uint32_t st = kStFinal;
    V3 direct = splat(0.0f);
    if (b.pass_status[i] == kWfPath) {
        b.gbuf[i].rng = b.wf[i].rng;
        const Prefix cp = ld_prefix_v(b.gather_cp[i]);
        if (fl_valid(cp.flags)) {
            if (fl_nee(cp.flags)) {
                direct = cp.f / cp.p;
            } else {
                const crisb_suffix_rec& csr = b.gather_cs[i].sample;
                if (fl_valid(csr.flags)) {
                    const V3 cs_f = ld3(csr.f);
                    const V3 canon_contrib = cp.f * cs_f / (cp.p * csr.p);
                    if (fp.k == 0) {
                        direct = canon_contrib;
                    } else {
                        b.gather_state[2 * i] = make_float4(cp.f.x, cp.f.y, cp.f.z, cp.p);
                        b.gather_state[2 * i + 1] = make_float4(canon_contrib.x, canon_contrib.y, canon_contrib.z, 0.0f);
                        st = kStQuery;
                    }
                }
            }
        }
    }
    if (st == kStFinal) {
        V3 L = splat(0.0f) + direct;
        if (b.gather_ext) {
            // gatherN > 1: the canonical gather's share; the extra gathers add
            // theirs and k_gather_output stores the sum
            b.gather_ext[3 * static_cast<size_t>(i) + 1] = make_float4(L.x, L.y, L.z, 0.0f);
        } else {
            if (nonfinite(L)) L = splat(0.0f);
            store_output(fp, out, i, L);
        }
    }
    b.pass_status[i] = st;
}

__global__ void __launch_bounds__(kPassBlock) k_gather_query(SceneView s, FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp)) {
        const uint32_t k = fp.k;
        NeighborList nl;
        nl.count = 0;
        if (b.pass_status[i] == kStQuery) {
            const Isect last = unpack(s, ld_hit(b.gather_cs[i].sample.last_prefix));
            knn_query(b.knn(), s.err, last.pos, k, nl);
            uint32_t vflags = 0;
            for (uint32_t n = 0; n < nl.count; ++n) {
                if (!(b.nval_cur[nl.pix[n]] & kNvalSample)) continue;
                vflags |= 1u << n;
                mask |= 3ull << (2 * n);
            }
            b.pass_flags[i] = vflags;
            b.pass_status[i] = kStReuse;
        }
        if (k > 0 && (k & 1u) == 0u) {
            // an even count: the pixel's list starts 16-byte aligned, two records a store
            uint4* d = reinterpret_cast<uint4*>(b.neighbors + static_cast<size_t>(i) * k);
            for (uint32_t n = 0; n < k; n += 2) {
                const bool a0 = n < nl.count, a1 = n + 1 < nl.count;
                d[n >> 1] = make_uint4(a0 ? nl.pix[n] : 0u, __float_as_uint(a0 ? nl.dist[n] : 0.0f),
                                       a1 ? nl.pix[n + 1] : 0u, __float_as_uint(a1 ? nl.dist[n + 1] : 0.0f));
            }
        } else if (k > 0) {
            for (uint32_t n = 0; n < k; ++n) {
                crisb_neighbor_rec r;
                r.pixel = n < nl.count ? nl.pix[n] : 0u;
                r.dist = n < nl.count ? nl.dist[n] : 0.0f;
                b.neighbors[static_cast<size_t>(i) * k + n] = r;
            }
        }
        b.neigh_count[i] = nl.count;
    }
    push_jobs(b, i, mask);
}

__global__ void __launch_bounds__(kPassBlock, kResampleMinBlocks) k_gather_combine(FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    ByteTally bt(b, kTallyGatherCombine);
    bt.add(4);
    if (b.pass_status[i] != kStReuse) return;
    // count, flags, canonical suffix f, gather state, the output RGB
    bt.add(4 + 4 + 12 + 32 + (fp.p.enable_accum ? 24 : 12));
    const uint32_t k = fp.k;
    const uint32_t count = b.neigh_count[i];
    const uint32_t vflags = b.pass_flags[i];
    const V3 cs_f = ld3(b.gather_cs[i].sample.f);
    const float4 g0 = b.gather_state[2 * i], g1 = b.gather_state[2 * i + 1];
    const V3 cp_f = xyz(g0), canon_contrib = xyz(g1);
    const float cp_p = g0.w;
    const uint32_t nvalid = __popc(vflags);
    const float K = static_cast<float>(nvalid);
    const float4* sh = b.shift_out + static_cast<size_t>(i) * b.slots;
    V3 suffix_contrib = splat(0.0f);
    float canon_mis = 1.0f;
    for (uint32_t n = 0; n < count; ++n) {
        if (!(vflags & (1u << n))) continue;
        const uint32_t np_ = b.neighbors[static_cast<size_t>(i) * k + n].pixel;
        bt.add(4 + weight_bytes(b.sres_cur.f16) + 32);  // neighbour pixel, weight fields, two shift results
        const V3 nf = sres_f(b.sres_cur, np_);
        const float nconf = sres_conf(b.sres_cur, np_), nwsum = sres_wsum(b.sres_cur, np_);
        const float4 o0 = sh[2 * n], o1 = sh[2 * n + 1];
        const V3 f_c_of_n = xyz(o0), f_n_of_c = xyz(o1);
        const float jac_n2c = o0.w, jac_c2n = o1.w;
        float nmis = mis_neighbor(f_c_of_n, nf, jac_n2c, K, 1.0f, nconf);
        if (nonfinite(nmis)) nmis = 0.0f;
        const V3 contrib = nmis * f_c_of_n * nwsum * jac_n2c;
        if (!nonfinite(contrib)) suffix_contrib = suffix_contrib + contrib;
        canon_mis += mis_canonical(cs_f, f_n_of_c, jac_c2n, K, 1.0f, nconf);
    }
    V3 gather = suffix_contrib * cp_f / cp_p;
    gather = gather / static_cast<float>(nvalid + 1);
    V3 result = gather + (canon_contrib * canon_mis);
    result = result / (K + 1.0f);
    if (nonfinite(result)) result = splat(0.0f);
    V3 L = splat(0.0f) + result;
    if (b.gather_ext) {
        b.gather_ext[3 * static_cast<size_t>(i) + 1] = make_float4(L.x, L.y, L.z, 0.0f);
        return;
    }
    if (nonfinite(L)) L = splat(0.0f);
    store_output(fp, out, i, L);
}

// ---- the final gather's extra prefixes, gatherN > 1 (shader/final_gather.cu:190-288,
// FinalGatherNotCanon, summed by GetRadiance, :290-321) ------------------------------------
constexpr uint32_t kStNoGather = 6;  // the pixel ran no gather (invalid primary hit)

// TracePrefixForFinalGather along the gather's camera ray, continuing the
// pixel's random stream; at most prefix_len closest-hit rays, traced in place
__global__ void __launch_bounds__(kPassBlock) k_gather_extra_prefix(SceneView s, FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const float4 e = b.gather_ext[3 * static_cast<size_t>(i)];
    uint32_t st = kStFinal;  // contributes zero
    if (e.w == 0.0f) {
        st = kStNoGather;
    } else if (fp.k > 0) {
        Rng rng{b.gbuf[i].rng};
        V3 tp;
        float pp;
        Isect last;
        if (trace_prefix_for_gather(s, tp, pp, last, ld3(fp.cam.pos), V3{e.x, e.y, e.z},
                                    static_cast<uint32_t>(fp.p.prefix_len), rng)) {
            b.gather_ext[3 * static_cast<size_t>(i) + 2] = make_float4(tp.x, tp.y, tp.z, pp);
            st_hit(b.gather_last[i], last.pack());
            st = kStQuery;
        }
        b.gbuf[i].rng = rng.state;
    }
    b.pass_status[i] = st;
}

// neighbour search at the extra prefix's last vertex; one job per valid
// neighbour (slot 2n: its suffix shifted onto that vertex)
__global__ void __launch_bounds__(kPassBlock) k_gather_extra_query(SceneView s, FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp) && b.pass_status[i] == kStQuery) {
        const uint32_t k = fp.k;
        NeighborList nl;
        const Isect last = unpack(s, ld_hit(b.gather_last[i]));
        knn_query(b.knn(), s.err, last.pos, k, nl);
        uint32_t vflags = 0;
        for (uint32_t n = 0; n < nl.count; ++n) {
            if (!(b.nval_cur[nl.pix[n]] & kNvalSample)) continue;
            vflags |= 1u << n;
            mask |= 1ull << (2 * n);
        }
        for (uint32_t n = 0; n < k; ++n) {
            crisb_neighbor_rec r;
            r.pixel = n < nl.count ? nl.pix[n] : 0u;
            r.dist = n < nl.count ? nl.dist[n] : 0.0f;
            b.neighbors[static_cast<size_t>(i) * k + n] = r;
        }
        b.neigh_count[i] = nl.count;
        b.pass_flags[i] = vflags;
        b.pass_status[i] = kStReuse;
    }
    push_jobs(b, i, mask);
}

__global__ void __launch_bounds__(kPassBlock) k_gather_extra_combine(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const uint32_t st = b.pass_status[i];
    if (st == kStNoGather) return;
    V3 result = splat(0.0f);
    if (st == kStReuse) {
        const uint32_t k = fp.k;
        const uint32_t vflags = b.pass_flags[i];
        const float K = static_cast<float>(__popc(vflags));
        const uint32_t count = b.neigh_count[i];
        const float4* sh = b.shift_out + static_cast<size_t>(i) * b.slots;
        V3 suffix_contrib = splat(0.0f);
        for (uint32_t n = 0; n < count; ++n) {
            if (!(vflags & (1u << n))) continue;
            const uint32_t np_ = b.neighbors[static_cast<size_t>(i) * k + n].pixel;
            const V3 nf = sres_f(b.sres_cur, np_);
            const float nconf = sres_conf(b.sres_cur, np_), nwsum = sres_wsum(b.sres_cur, np_);
            const float4 o0 = sh[2 * n];
            const V3 f_c_of_n = xyz(o0);
            const float jac_n2c = o0.w;
            float nmis = mis_neighbor(f_c_of_n, nf, jac_n2c, K, 1.0f, nconf);
            if (nonfinite(nmis)) nmis = 0.0f;
            const V3 contrib = nmis * f_c_of_n * nwsum * jac_n2c;
            if (!nonfinite(contrib)) suffix_contrib = suffix_contrib + contrib;
        }
        const float4 t = b.gather_ext[3 * static_cast<size_t>(i) + 2];
        const V3 tp = V3{t.x, t.y, t.z};
        result = suffix_contrib * tp / t.w;
        result = result / static_cast<float>(fp.p.gather_n);
        result = result / (K + 1.0f);
        if (nonfinite(result)) result = splat(0.0f);
    }
    float4& acc = b.gather_ext[3 * static_cast<size_t>(i) + 1];
    const V3 sum = V3{acc.x, acc.y, acc.z} + result;
    acc = make_float4(sum.x, sum.y, sum.z, 0.0f);
}

// GetRadiance's sum over the gathers, stored
__global__ void __launch_bounds__(kPassBlock) k_gather_output(FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const float4 a = b.gather_ext[3 * static_cast<size_t>(i) + 1];
    V3 L = V3{a.x, a.y, a.z};
    if (nonfinite(L)) L = splat(0.0f);
    store_output(fp, out, i, L);
}


// ---- prefix spatial reuse (shader/prefix_spatial_reuse.cu:11-134) -----------------
// Neighbours are read from the back buffer, which equals the front buffer at
// pass start (the front -> back copy follows every round); the pass writes the
// front buffer.  Split like the suffix spatial pass: selection, shift jobs,
// combine.
__global__ void __launch_bounds__(kPassBlock) k_prefix_spatial_select(FrameParams fp, Bufs b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp)) {
        const uint32_t x = i % fp.width, y = i / fp.width;
        const crisb_prefix_rec& canon = b.canon_prefix[i];
        uint32_t st = kStFinal;
        if (fl_valid(pres_flags(b.pres[fp.front], i)) && fl_valid(canon.flags) &&
            canon.primary.prim != CRISB_INVALID_PRIM) {
            st = kStReuse;
            Rng rng{b.gbuf[i].rng};
            uint32_t vflags = 0;
            uint32_t* nbr = b.spatial_nbr + static_cast<size_t>(i) * (b.slots >> 1);
            for (int n = 0; n < fp.p.prefix_spatial_count; ++n) {
                uint32_t nx, ny;
                select_spatial_neighbor(x, y, static_cast<uint32_t>(fp.p.window_radius), rng, nx, ny);
                if (!(nx < fp.width && ny < fp.height)) continue;
                const uint32_t ni = ny * fp.width + nx;
                if (!(b.gbuf[ni].flags & 1u)) continue;
                const uint32_t nflags = pres_flags(b.pres[fp.back], ni);
                const bool skip_nee = fp.p.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR && fl_nee(nflags);
                if (!fl_valid(nflags) || skip_nee) continue;
                nbr[n] = ni;
                vflags |= 1u << n;
                mask |= 3ull << (2 * n);
            }
            b.gbuf[i].rng = rng.state;
            b.pass_flags[i] = vflags;
        }
        b.pass_status[i] = st;
    }
    push_jobs(b, i, mask);
}

__global__ void __launch_bounds__(kPassBlock) k_prefix_spatial_combine(FrameParams fp, Bufs b, float* out,
                                                                      int round) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    const bool output = fp.p.renderer_type == CRISB_RENDERER_RESTIR_PT && round == fp.p.prefix_spatial_rounds - 1;
    if (b.pass_status[i] == kStFinal) {
        if (output) store_output(fp, out, i, splat(0.0f));
        return;
    }
    Rng rng{b.gbuf[i].rng};
    const V3 own_f = pres_f(b.pres[fp.front], i);
    const float cur_wsum = pres_wsum(b.pres[fp.front], i), cur_conf = pres_conf(b.pres[fp.front], i);
    const uint32_t vflags = b.pass_flags[i];
    const float K = static_cast<float>(__popc(vflags));
    const uint32_t* nbr = b.spatial_nbr + static_cast<size_t>(i) * (b.slots >> 1);
    const float4* sh = b.shift_out + static_cast<size_t>(i) * b.slots;
    // Reservoir::Update's arithmetic with the chosen sample tracked by index
    // (-1: the pixel's own prefix, which the reset reservoir still holds)
    float w_sum = 0.0f, conf = 0.0f;
    int sel = -1;
    V3 sel_f = own_f;
    float canon_mis = 1.0f;
    for (int n = 0; n < fp.p.prefix_spatial_count; ++n) {
        if (!((vflags >> n) & 1u)) continue;
        const uint32_t ni = nbr[n];
        const V3 nf = pres_f(b.pres[fp.back], ni);
        const float nconf = pres_conf(b.pres[fp.back], ni), nwsum = pres_wsum(b.pres[fp.back], ni);
        const float4 o0 = sh[2 * n], o1 = sh[2 * n + 1];
        const V3 f_c_of_n = xyz(o0), f_n_of_c = xyz(o1);
        const float jac_n2c = o0.w, jac_c2n = o1.w;
        const float p_c_of_n = luminance(f_c_of_n) * jac_n2c;
        float nmis = mis_neighbor(f_c_of_n, nf, jac_n2c, K, cur_conf, nconf);
        if (nonfinite(nmis)) nmis = 0.0f;
        if (res_choose(w_sum, conf, nmis * p_c_of_n * nwsum, rng, nconf)) {
            sel = n;
            sel_f = f_c_of_n;
        }
        canon_mis += mis_canonical(own_f, f_n_of_c, jac_c2n, K, cur_conf, nconf);
    }
    if (nonfinite(canon_mis)) canon_mis = 0.0f;
    if (res_choose(w_sum, conf, canon_mis * cur_wsum * luminance(own_f), rng, cur_conf)) {
        sel = -1;
        sel_f = own_f;
    }
    Res<Prefix> cur;
    if (sel >= 0) {
        // the neighbour's prefix with f shifted onto this pixel and its primary hit
        cur.s = ld_pres(b.pres[fp.back], nbr[sel]).s;
        cur.s.f = sel_f;
        cur.s.primary = pres_primary(b.pres[fp.front], i);
    } else {
        cur.s = ld_pres(b.pres[fp.front], i).s;
    }
    cur.w_sum = w_sum;
    cur.conf = conf;
    if (cur.w_sum > 0.0f) {
        cur.w_sum /= K + 1.0f;
        res_finalize(cur);
    }
    b.gbuf[i].rng = rng.state;
    st_pres(b.pres[fp.front], i, cur);
    if (output) store_output(fp, out, i, cur.w_sum * cur.s.f);
}

// ---- prefix generation + temporal reuse (shader/prefix_gen_temp_reuse.cu) -----------
// the pass leaves back = front (prefix_gen_temp_reuse.cu:159-164)
RT_HD bool prefix_back_copy(const FrameParams& fp) {
    const int type = fp.p.renderer_type;
    return (type == CRISB_RENDERER_RESTIR_PT && fp.p.prefix_enable_spatial) ||
           (type == CRISB_RENDERER_CONDITIONAL_RESTIR && fp.p.suffix_enable_spatial);
}

RT_D void prefix_tail(const FrameParams& fp, const Bufs& b, float* out, uint32_t i, const Res<Prefix>& cur,
                      bool valid) {
    const int type = fp.p.renderer_type;
    if (type == CRISB_RENDERER_RESTIR_PT && !fp.p.prefix_enable_spatial)
        store_output(fp, out, i, valid ? cur.w_sum * cur.s.f : splat(0.0f));
    // front -> back copy for the spatial passes; with reprojection other
    // pixels still read back[prevPixelIdx] in this pass, so the copy runs as a
    // kernel of its own after it (prefix_back_copy)
    if (prefix_back_copy(fp) && fp.p.motion_mode == CRISB_MOTION_NONE) st_pres(b.pres[fp.back], i, cur);
}

// PathTracer mode: TraceCompletePath per pixel (prefix_gen_temp_reuse.cu:175-192)
__global__ void __launch_bounds__(kPassBlock) k_path_tracer(SceneView s, FrameParams fp, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp)) return;
    Rng rng = rng_seeded(tea64(i, fp.random));
    const V3 dir = camera_dir(fp, i % fp.width, i / fp.width, rng);
    V3 L = trace_complete_path(s, fp, ld3(fp.cam.pos), dir, rng);
    if (nonfinite(L)) L = splat(0.0f);
    store_output(fp, out, i, L);
}

// per pixel after the canonical prefixes (wavefront.cu, prefix flow) finished:
// the temporal-reuse decision, its shift jobs and the G-buffer
__global__ void __launch_bounds__(kPassBlock) k_prefix_finish(SceneView s, FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t mask = 0;
    if (i < pixel_count(fp)) {
        const uint32_t x = i % fp.width, y = i / fp.width;
        const bool valid = fl_valid(b.canon_prefix[i].flags);
        // prevPixelCoord (prefix_gen_temp_reuse.cu:130-136)
        uint32_t prev_xy = x | (y << 16);
        if (fp.p.motion_mode == CRISB_MOTION_VECTORS) {
            const float2 mv = fp.motion[i];
            prev_xy = prev_from_motion(x, y, mv.x, mv.y, fp.width, fp.height);
        } else if (fp.p.motion_mode == CRISB_MOTION_REPROJECT) {
            prev_xy = kPrevNone;
            if (valid && fp.has_prev_cam) {
                const Isect it = unpack(s, ld_hit(b.canon_prefix[i].primary));
                if (it.valid) prev_xy = reproject(fp.prev_cam, it.pos, fp.width, fp.height);
            }
        }
        uint32_t st = kStFinal;
        if (!valid) {
            prefix_tail(fp, b, out, i, ld_pres(b.pres[fp.front], i), false);
        } else if (!fp.p.prefix_enable_temporal || prev_xy == kPrevNone) {
            st = kStCanonOnly;
        } else {
            const uint32_t pi = fp.p.motion_mode == CRISB_MOTION_NONE ? i : prev_index(prev_xy, fp.width);
            const uint32_t pf = pres_flags(b.pres[fp.back], pi);
            const bool skip_nee = fp.p.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR && fl_nee(pf);
            if (pres_wsum(b.pres[fp.back], pi) <= 0.0f || !fl_valid(pf) || skip_nee) {
                st = kStCanonOnly;
            } else {
                st = kStReuse;
                mask = 3;
            }
        }
        crisb_gbuffer_rec g;
        g.rng = b.wf[i].rng;
        g.prev_xy = prev_xy;
        g.flags = valid ? 1u : 0u;
        b.gbuf[i] = g;
        b.pass_status[i] = st;
    }
    push_jobs(b, i, mask);
}

// slot 0: previous prefix shifted onto the canonical one; slot 1: the reverse
__global__ void __launch_bounds__(kPassBlock, kResampleMinBlocks) k_prefix_combine(FrameParams fp, Bufs b, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixel_count(fp) || fp.p.renderer_type == CRISB_RENDERER_PATH_TRACER) return;
    ByteTally bt(b, kTallyPrefixCombine);
    const uint32_t st = b.pass_status[i];
    bt.add(4);
    if (st == kStFinal) return;
    const crisb_prefix_rec& cp = b.canon_prefix[i];
    const V3 canon_f = ld3(cp.f);
    const float canon_p = cp.p;
    Rng rng{b.gbuf[i].rng};
    // canonical f and p, RNG in and out, the front reservoir out (and its back
    // copy for the spatial passes)
    bt.add(12 + 4 + 8 + 8 + pres_bytes(b.pres[fp.front]) +
           (prefix_back_copy(fp) && fp.p.motion_mode == CRISB_MOTION_NONE ? pres_bytes(b.pres[fp.back]) : 0));
    const float canon_phat = luminance(canon_f);
    // Reservoir::Update's arithmetic with the chosen sample tracked by index
    // (0: the sample the reset front reservoir still holds, 1: canonical,
    // 2: the shifted previous sample); the chosen record is read at the end.
    Res<Prefix> cur;
    cur.w_sum = 0.0f;
    cur.conf = 0.0f;
    int sel = 0;
    V3 f_canon_of_prev = splat(0.0f);
    const uint32_t pi = prev_pixel(fp, b, i);
    if (st == kStCanonOnly) {
        if (res_choose(cur.w_sum, cur.conf, canon_phat / canon_p, rng, 1.0f)) sel = 1;
    } else {
        bt.add(weight_bytes(b.pres[fp.back].f16) + 32);  // previous weight fields, two shift results
        const V3 prev_f = pres_f(b.pres[fp.back], pi);
        const float prev_conf = pres_conf(b.pres[fp.back], pi), prev_wsum = pres_wsum(b.pres[fp.back], pi);
        const float4 o0 = b.shift_out[static_cast<size_t>(i) * b.slots];
        const float4 o1 = b.shift_out[static_cast<size_t>(i) * b.slots + 1];
        f_canon_of_prev = xyz(o0);
        const V3 f_prev_of_canon = xyz(o1);
        const float jac_prev_to_canon = o0.w, jac_canon_to_prev = o1.w;
        const float p_canon_of_prev = luminance(f_canon_of_prev) * jac_prev_to_canon;
        const float K = 1.0f;
        const float prev_mis = mis_neighbor(f_canon_of_prev, prev_f, jac_prev_to_canon, K, 1.0f, prev_conf);
        const float canon_mis =
            1.0f + mis_canonical(canon_f, f_prev_of_canon, jac_canon_to_prev, K, 1.0f, prev_conf);
        if (res_choose(cur.w_sum, cur.conf, canon_mis * canon_phat / canon_p, rng, 1.0f)) sel = 1;
        if (res_choose(cur.w_sum, cur.conf, prev_mis * p_canon_of_prev * prev_wsum, rng, prev_conf)) sel = 2;
    }
    if (sel == 0) {
        bt.add(pres_bytes(b.pres[fp.front]));
        cur.s = ld_pres(b.pres[fp.front], i).s;
    } else if (sel == 1) {
        bt.add(sizeof(crisb_prefix_rec));
        cur.s = ld_prefix_v(cp);
    } else {
        bt.add(pres_bytes(b.pres[fp.back]) + sizeof(crisb_hit_rec));
        cur.s = ld_pres(b.pres[fp.back], pi).s;  // PrefixPath(prev, f, canon.primaryInt)
        cur.s.f = f_canon_of_prev;
        cur.s.primary = ld_hit(cp.primary);
    }
    if (st == kStCanonOnly) {
        res_finalize(cur);
    } else if (cur.w_sum > 0.0f) {
        cur.w_sum /= 1.0f + 1.0f;
        res_finalize(cur);
    }
    b.gbuf[i].rng = rng.state;
    st_pres(b.pres[fp.front], i, cur);
    prefix_tail(fp, b, out, i, cur, true);
}

struct ShiftGrids {
    unsigned begin, step, step_last, overflow;
};

template <bool kTex>
const ShiftGrids& shift_grids() {
    static std::once_flag once;
    static ShiftGrids g{};
    std::call_once(once, [] {
        g.begin = persistent_grid(reinterpret_cast<const void*>(k_shift_begin<kTex>));
        g.step = persistent_grid(reinterpret_cast<const void*>(k_shift_step<false, kTex>));
        g.step_last = persistent_grid(reinterpret_cast<const void*>(k_shift_step<true, kTex>));
        g.overflow = persistent_grid(reinterpret_cast<const void*>(k_shift_overflow<kTex>));
    });
    return g;
}


#define MARK(cls)          \
    do {                   \
        if (m) m->mark(cls, st); \
    } while (0)

// the shift jobs of the list: begin, then rounds of trace / step
template <bool kTex>
void run_shift_jobs_as(const SceneView& s, const FrameParams& fp, const Bufs& b, int mode, cudaStream_t st,
                       Marker* m) {
    const ShiftGrids& g = shift_grids<kTex>();
    cudaMemsetAsync(b.job_qcount, 0, 2 * sizeof(uint32_t), st);
    k_shift_begin<kTex><<<g.begin, kPassBlock, 0, st>>>(s, fp, b, mode);
    MARK(kClsShift);
    k_shift_overflow<kTex><<<g.overflow, kPassBlock, 0, st>>>(s, fp, b, mode);
    MARK(kClsShift);
    for (int r = 0; r < kShiftRounds; ++r) {
        const int cur = r & 1, nxt = cur ^ 1;
        launch_trace<ShiftJob>(fp.trace_block, fp.trace_grid, st, s, b.job_queue[2 * cur], b.job_qcount + 2 * cur,
                               b.job_queue[2 * cur + 1], b.job_qcount + 2 * cur + 1, b.jobs);
        MARK(kClsTrace);
        if (r + 1 < kShiftRounds) {
            cudaMemsetAsync(b.job_qcount + 2 * nxt, 0, 2 * sizeof(uint32_t), st);
            k_shift_step<false, kTex><<<g.step, kPassBlock, 0, st>>>(s, fp, b, mode, cur);
        } else {
            k_shift_step<true, kTex><<<g.step_last, kPassBlock, 0, st>>>(s, fp, b, mode, cur);
        }
        MARK(kClsShift);
    }
}

// the shift kernels come in two builds: with the texture lookup, for scenes
// with textured materials, and without it (20 registers fewer, 7 instead of
// 5 resident blocks per SM)
void run_shift_jobs(const SceneView& s0, const FrameParams& fp, const Bufs& b, int mode, cudaStream_t st, Marker* m) {
    const SceneView s = shift_view(s0);
    if (s.mat_tex)
        run_shift_jobs_as<true>(s, fp, b, mode, st, m);
    else
        run_shift_jobs_as<false>(s, fp, b, mode, st, m);
}

}  // namespace

uint32_t shift_launches_per_phase() { return 2 + 2 * kShiftRounds; }

void launch_prefix_gen_temp_split(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out,
                                  cudaStream_t st, Marker* m) {
    if (fp.p.renderer_type == CRISB_RENDERER_PATH_TRACER) {
        k_path_tracer<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, out);
        MARK(kClsOther);
        return;
    }
    launch_wf_prefix(s, fp, b, st, m);
    cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
    k_prefix_finish<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b, out);
    MARK(kClsShade);
    run_shift_jobs(s, fp, b, kModePrefix, st, m);
    k_prefix_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, out);
    MARK(kClsResample);
    if (prefix_back_copy(fp) && fp.p.motion_mode != CRISB_MOTION_NONE) {
        launch_prefix_copy_front_back(fp, b, st);
        MARK(kClsOther);
    }
}

uint32_t prefix_pass_extra_launches(const FrameParams& fp) {
    return prefix_back_copy(fp) && fp.p.motion_mode != CRISB_MOTION_NONE ? 1u : 0u;
}

void launch_prefix_spatial(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out, int round,
                           cudaStream_t st, Marker* m) {
    cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
    k_prefix_spatial_select<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    MARK(kClsResample);
    run_shift_jobs(s, fp, b, kModePrefixSpatial, st, m);
    k_prefix_spatial_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, out, round);
    MARK(kClsResample);
}

void launch_suffix_gen_temp(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m) {
    launch_wf_suffix(s, fp, b, st, m);
    cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
    k_suffix_temp_finish<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    MARK(kClsShade);
    run_shift_jobs(s, fp, b, kModeTemporal, st, m);
    k_suffix_temp_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    MARK(kClsResample);
}

void launch_suffix_spatial(const SceneView& s, const FrameParams& fp, const Bufs& b, cudaStream_t st, Marker* m) {
    cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
    k_suffix_spatial_select<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    MARK(kClsResample);
    run_shift_jobs(s, fp, b, kModeSpatial, st, m);
    k_suffix_spatial_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
    MARK(kClsResample);
}

void launch_final_gather_split(const SceneView& s, const FrameParams& fp, const Bufs& b, float* out,
                               cudaStream_t st, Marker* m) {
    launch_wf_gather(s, fp, b, st, m);
    k_gather_finish<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, out);
    MARK(kClsShade);
    cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
    k_gather_query<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b);
    MARK(kClsSearch);
    run_shift_jobs(s, fp, b, kModeGather, st, m);
    k_gather_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, out);
    MARK(kClsResample);
    if (fp.p.gather_n > 1) {
        for (int g = 1; g < fp.p.gather_n; ++g) {
            cudaMemsetAsync(b.job_count, 0, sizeof(uint32_t), st);
            k_gather_extra_prefix<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b);
            MARK(kClsShade);
            k_gather_extra_query<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(s, fp, b);
            MARK(kClsSearch);
            run_shift_jobs(s, fp, b, kModeGatherExtra, st, m);
            k_gather_extra_combine<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b);
            MARK(kClsResample);
        }
        k_gather_output<<<grid_for(fp.width * fp.height), kPassBlock, 0, st>>>(fp, b, out);
        MARK(kClsOther);
    }
}

#undef MARK

}  // namespace crisb
