// adjoint.cu -- path-replay adjoint of the unidirectional path tracer.
//
// The estimator differentiated is TraceCompletePath
// (include/graph/restir/path_gen.h:389-472; trace_complete_path here) with its
// sampling frozen: every random decision, BRDF-sampled direction and sampling
// pdf comes from a fixed copy of the materials (theta0, taken when the adjoint
// context is made), while the BRDF values, emissions and emitter colours come
// from the scene's current tables (theta).  At theta = theta0 it is the path
// tracer sample for sample; for any theta it is an unbiased estimator of the
// rendering integral at theta (importance sampling with a fixed proposal), and
// it is a smooth function of theta, so its gradient is what central
// differences of the same estimator measure.
//
// The estimator has one term per path: at the vertex j where NEE is chosen,
//   L = T_j * brdf_j(light) * Le / d^2 (+ emission_j when j is the first hit),
//   T_j = prod_{i<j} brdf_i(dir_i) / (pdf0_i (1 - neeProb)) / neeProb.
// The backward kernel replays each pixel's path from its seed (no tape) and
// carries d T / d(diffuse rgb, roughness) for every material met so far
// (forward mode), then turns dLoss/dL into gradients of the diffuse albedo,
// roughness and emission of each material and the colour of each emitter.
// Gradients gather in shared memory per block and reach global memory with one
// atomic per touched parameter per block.
#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "adjoint_common.cuh"

namespace crisb {
namespace {

struct AdjView {
    SceneView eval;           // current materials / emitters (theta)
    const crisb_material* sample_mats;  // theta0
    uint32_t num_mats, num_emitters;
};

// One path of the frozen-sampling estimator; with `sink` also its gradient for
// the pixel adjoint `dl`.  Returns the pixel's radiance.
template <bool kGrad>
RT_D V3 frozen_path(const AdjView& a, const FrameParams& fp, V3 origin, V3 dir, Rng& rng, V3 dl, GradSink* sink) {
    SceneView ss = a.eval;  // sampling view: theta0 materials
    ss.mats = a.sample_mats;
    V3 cur_pos = origin, cur_dir = dir;
    uint32_t depth = 0;
    V3 tp = splat(1.0f);
    Touched tl[kMaxTouched];
    int nt = 0;
    const float nee = fp.p.nee_prob;
    for (int ti = 0; ti < fp.p.max_path_len; ++ti) {
        Isect it;
        it.valid = false;
        trace_closest(a.eval, cur_pos, cur_dir, 1e-3f, 1e16f, it);
        if (!it.valid) break;
        ++depth;
        const uint32_t mi = material_of(a.eval, it.prim);
        const crisb_material mat = a.eval.mats[mi];
        if (rng.next_float() < nee) {
            tp = tp / nee;
            if (kGrad)
                for (int t = 0; t < nt; ++t) {
                    tl[t].d_diff = tl[t].d_diff / nee;
                    tl[t].d_rough = tl[t].d_rough / nee;
                }
            const EmitterSample es = sample_emitter(a.eval, rng);
            const uint32_t ei = es.index;
            const V3 light_dir = normalize(es.pos - it.pos);
            const float dist = length(es.pos - it.pos);
            if (occluded(a.eval, it.pos, light_dir, 1e-3f, dist)) return splat(0.0f);
            const BrdfGrad bg = brdf_grad(mat, it.nrm, -it.dir, light_dir);
            const float dist_factor = 1.0f / (dist * dist);
            V3 radiance = tp * bg.brdf * es.color * dist_factor;
            // brdf_eval reports the emission only past its facing checks
            const bool emit = depth == 1 && dot(it.nrm, -it.dir) > 0.0f && dot(it.nrm, light_dir) >= 0.0f;
            if (emit) radiance = radiance + mat_vals(mat).emission;
            if (kGrad) {
                const V3 lw = es.color * dist_factor;  // light weight
                for (int t = 0; t < nt; ++t) {
                    const V3 c_diff = dl * tl[t].d_diff * bg.brdf * lw;
                    sink->add_mat(tl[t].mat, 0, c_diff.x);
                    sink->add_mat(tl[t].mat, 1, c_diff.y);
                    sink->add_mat(tl[t].mat, 2, c_diff.z);
                    const V3 c_r = dl * tl[t].d_rough * bg.brdf * lw;
                    sink->add_mat(tl[t].mat, 3, (c_r.x + c_r.y) + c_r.z);
                }
                const V3 c_diff = dl * tp * bg.d_diff * lw;
                sink->add_mat(mi, 0, c_diff.x);
                sink->add_mat(mi, 1, c_diff.y);
                sink->add_mat(mi, 2, c_diff.z);
                const V3 c_r = dl * tp * bg.d_rough * lw;
                sink->add_mat(mi, 3, (c_r.x + c_r.y) + c_r.z);
                const V3 c_e = dl * tp * bg.brdf * dist_factor;
                sink->add_em(ei, 0, c_e.x);
                sink->add_em(ei, 1, c_e.y);
                sink->add_em(ei, 2, c_e.z);
                if (emit) {
                    sink->add_mat(mi, 4, dl.x);
                    sink->add_mat(mi, 5, dl.y);
                    sink->add_mat(mi, 6, dl.z);
                }
            }
            return radiance;
        }
        const BrdfSample bs = brdf_sample(ss, it, rng);  // direction and pdf at theta0
        if (bs.pdf <= 0.0f) break;
        const BrdfGrad bg = brdf_grad(mat, it.nrm, -it.dir, bs.dir);
        const float inv = 1.0f / (bs.pdf * (1.0f - nee));
        const V3 w = bg.brdf * inv;
        if (kGrad) {
            for (int t = 0; t < nt; ++t) {
                tl[t].d_diff = tl[t].d_diff * w;
                tl[t].d_rough = tl[t].d_rough * w;
            }
            int slot = -1;
            for (int t = 0; t < nt; ++t)
                if (tl[t].mat == mi) slot = t;
            if (slot < 0 && nt < kMaxTouched) {
                slot = nt++;
                tl[slot].mat = mi;
                tl[slot].d_diff = tl[slot].d_rough = splat(0.0f);
            }
            if (slot >= 0) {
                tl[slot].d_diff = tl[slot].d_diff + tp * bg.d_diff * inv;
                tl[slot].d_rough = tl[slot].d_rough + tp * bg.d_rough * inv;
            }
        }
        cur_pos = it.pos;
        cur_dir = bs.dir;
        tp = tp * w;
    }
    return splat(0.0f);
}

__global__ void __launch_bounds__(kPassBlock) k_frozen_forward(AdjView a, FrameParams fp, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= fp.width * fp.height) return;
    Rng rng = rng_seeded(tea64(i, fp.random));
    const V3 dir = camera_dir(fp, i % fp.width, i / fp.width, rng);
    V3 L = frozen_path<false>(a, fp, ld3(fp.cam.pos), dir, rng, splat(0.0f), nullptr);
    if (nonfinite(L)) L = splat(0.0f);
    out[3 * i] = L.x;
    out[3 * i + 1] = L.y;
    out[3 * i + 2] = L.z;
}

__global__ void __launch_bounds__(kPassBlock) k_frozen_backward(AdjView a, FrameParams fp, const float* d_img,
                                                                float* g_mat, float* g_em, int use_shared) {
    extern __shared__ float sh[];
    const uint32_t n_sh = a.num_mats * kMatGrad + a.num_emitters * kEmGrad;
    if (use_shared) {
        for (uint32_t k = threadIdx.x; k < n_sh; k += blockDim.x) sh[k] = 0.0f;
        __syncthreads();
    }
    GradSink sink{use_shared ? sh : nullptr, g_mat, g_em, a.num_mats};
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < fp.width * fp.height) {
        const V3 dl = V3{d_img[3 * i], d_img[3 * i + 1], d_img[3 * i + 2]};
        if (!nonfinite(dl) && (dl.x != 0.0f || dl.y != 0.0f || dl.z != 0.0f)) {
            Rng rng = rng_seeded(tea64(i, fp.random));
            const V3 dir = camera_dir(fp, i % fp.width, i / fp.width, rng);
            const V3 L = frozen_path<true>(a, fp, ld3(fp.cam.pos), dir, rng, dl, &sink);
            (void)L;
        }
    }
    if (use_shared) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < n_sh; k += blockDim.x) {
            const float v = sh[k];
            if (v == 0.0f) continue;
            if (k < a.num_mats * kMatGrad) atomicAdd(&g_mat[k], v);
            else atomicAdd(&g_em[k - a.num_mats * kMatGrad], v);
        }
    }
}

}  // namespace

// host side, called from api.cu
void adjoint_forward(const SceneView& eval, const crisb_material* sample_mats, uint32_t num_mats,
                     const FrameParams& fp, float* out, cudaStream_t st) {
    const AdjView a{eval, sample_mats, num_mats, eval.num_emitters};
    const uint32_t P = fp.width * fp.height;
    k_frozen_forward<<<(P + kPassBlock - 1) / kPassBlock, kPassBlock, 0, st>>>(a, fp, out);
}

void adjoint_backward(const SceneView& eval, const crisb_material* sample_mats, uint32_t num_mats,
                      const FrameParams& fp, const float* d_img, float* g_mat, float* g_em, cudaStream_t st) {
    const AdjView a{eval, sample_mats, num_mats, eval.num_emitters};
    const uint32_t P = fp.width * fp.height;
    const size_t sh_bytes = (static_cast<size_t>(num_mats) * kMatGrad + eval.num_emitters * kEmGrad) * sizeof(float);
    const int use_shared = sh_bytes <= 48u * 1024u ? 1 : 0;
    k_frozen_backward<<<(P + kPassBlock - 1) / kPassBlock, kPassBlock, use_shared ? sh_bytes : 0, st>>>(
        a, fp, d_img, g_mat, g_em, use_shared);
}

}  // namespace crisb
