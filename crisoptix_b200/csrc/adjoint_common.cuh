// adjoint_common.cuh -- pieces shared by the path-replay adjoints
// (adjoint.cu: the path tracer; restir_adjoint.cu: the resampled estimator of
// the final gather): the BRDF with its derivatives, forward-mode derivative
// entries per material, and the gradient sink behind warp-aggregated atomics.
#pragma once

#include "passes.cuh"

namespace crisb {
namespace {

constexpr int kMatGrad = 7;   // per material: d diffuse rgb, d roughness, d emission rgb
constexpr int kEmGrad = 3;    // per emitter: d colour rgb
constexpr int kMaxTouched = 16;

// d (brdf * cos) / d diffuse (per channel, channel-diagonal) and / d roughness
// for spec_usage == COLOR materials (the roughness of OCC_ROUGH_METAL materials
// lives in the specular texture and gets no gradient)
struct BrdfGrad {
    V3 brdf;
    V3 d_diff;   // d brdf_c / d diffuse_c
    V3 d_rough;  // d brdf_c / d roughness
};

RT_D BrdfGrad brdf_grad(const crisb_material& mat, V3 nrm, V3 view, V3 light) {
    BrdfGrad g;
    g.brdf = g.d_diff = g.d_rough = splat(0.0f);
    const MatVals m = mat_vals(mat);
    const float ndotv = dot(nrm, view);
    const float ndotl = dot(nrm, light);
    if (ndotv <= 0.0f || ndotl < 0.0f) return g;
    const float metal = mat.spec_usage == CRISB_SPEC_OCC_ROUGH_METAL ? mat.specular[2] : 0.0f;
    const bool rough_param = mat.spec_usage == CRISB_SPEC_COLOR;
    V3 spec = splat(0.0f), dspec_df0 = splat(0.0f), dspec_dr = splat(0.0f);
    const V3 h = normalize(light + view);
    const float ndoth = dot(h, nrm);
    const float ldoth = dot(h, light);
    if (static_cast<double>(dot(m.f0, m.f0)) > 1e-6) {
        const float r = m.rough, a2 = r * r;
        const float d = (ndoth * a2 - ndoth) * ndoth + 1.0f;
        const float D = a2 / (kPi * d * d);
        const float dD_da2 = 1.0f / (kPi * d * d) - 2.0f * a2 * ndoth * ndoth / (kPi * d * d * d);
        const float sv = sqrtf(ndotv * ndotv * (1 - a2) + a2), sl = sqrtf(ndotl * ndotl * (1 - a2) + a2);
        const float lv = ndotl * sv, ll = ndotv * sl;
        const float V = 0.5f / (lv + ll);
        const float dlv = ndotl * (1.0f - ndotv * ndotv) / (2.0f * sv);
        const float dll = ndotv * (1.0f - ndotl * ndotl) / (2.0f * sl);
        const float dV_da2 = -0.5f * (dlv + dll) / ((lv + ll) * (lv + ll));
        const float P = pow5(gmax(0.0f, 1.0f - ldoth));
        const V3 F = m.f0 + (splat(1.0f) - m.f0) * P;
        spec = D * V * F;
        dspec_df0 = splat(D * V * (1.0f - P));
        dspec_dr = ((dD_da2 * V + D * dV_da2) * 2.0f * r) * F;
    }
    g.brdf = (m.diff / kPi + spec) * ndotl;
    g.d_diff = (splat(1.0f / kPi) + dspec_df0 * (1.0f - metal)) * ndotl;
    if (rough_param) g.d_rough = dspec_dr * ndotl;
    return g;
}

struct Touched {
    uint32_t mat;
    V3 d_diff;   // d T_c / d diffuse_c of this material
    V3 d_rough;  // d T_c / d roughness of this material
};

// Warp-aggregated add: the lanes adding to the same address at this call
// combine their values (__match_any_sync on the address, shuffles to the
// group's lowest lane), which issues one atomic for the group.  Paths of
// neighbouring pixels mostly meet the same materials and emitters, so a warp
// issues a few atomics per vertex instead of up to 32 on one address.
RT_D void warp_add(float* addr, float v) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(addr));
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    float sum = v;
    unsigned rest = peers & ~(1u << leader);
    while (rest) {
        const int src = __ffs(rest) - 1;
        rest &= rest - 1u;
        const float t = __shfl_sync(peers, v, src);
        if (lane == leader) sum += t;
    }
    if (lane == leader) atomicAdd(addr, sum);
}

// gradient sink: a shared-memory block of all parameters (materials, then
// emitters) flushed once per block, or the global arrays directly when the
// block does not fit; either way behind a warp-aggregated add
struct GradSink {
    float* sh;  // null: add to global directly
    float* g_mat;
    float* g_em;
    uint32_t num_mats;
    RT_D void add_mat(uint32_t m, int k, float v) {
        if (v == 0.0f || !isfinite(v)) return;
        warp_add(sh ? &sh[m * kMatGrad + k] : &g_mat[m * kMatGrad + k], v);
    }
    RT_D void add_em(uint32_t e, int k, float v) {
        if (v == 0.0f || !isfinite(v)) return;
        warp_add(sh ? &sh[num_mats * kMatGrad + e * kEmGrad + k] : &g_em[e * kEmGrad + k], v);
    }
};

}  // namespace
}  // namespace crisb
