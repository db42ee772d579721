// records.cuh -- whole-record loads and stores of the device buffers and
// the image write shared by the pass kernels.
#pragma once

#include "passes.cuh"

namespace crisb {

RT_D uint32_t pixel_count(const FrameParams& fp) { return fp.width * fp.height; }

RT_D Res<Prefix> ld_pres(const crisb_prefix_res_rec* p, uint32_t i) {
    const crisb_prefix_res_rec r = p[i];
    return Res<Prefix>{ld_prefix(r.sample), r.w_sum, r.confidence};
}
RT_D void st_pres(crisb_prefix_res_rec* p, uint32_t i, const Res<Prefix>& r) {
    crisb_prefix_res_rec o;
    st_prefix(o.sample, r.s);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    o.pad[0] = 0;
    o.pad[1] = 0;
    p[i] = o;
}
RT_D Res<Suffix> ld_sres(const crisb_suffix_res_rec* p, uint32_t i) {
    const crisb_suffix_res_rec r = p[i];
    return Res<Suffix>{ld_suffix(r.sample), r.w_sum, r.confidence};
}
RT_D void st_sres(crisb_suffix_res_rec* p, uint32_t i, const Res<Suffix>& r) {
    crisb_suffix_res_rec o;
    st_suffix(o.sample, r.s);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    p[i] = o;
}

RT_D void store_output(const FrameParams& fp, float* out, uint32_t i, V3 radiance) {
    V3 v = radiance;
    if (fp.p.enable_accum) {
        const V3 old = V3{out[3 * i], out[3 * i + 1], out[3 * i + 2]};
        const float blend = 1.0f / static_cast<float>(fp.frame_idx + 1);
        v = blend * radiance + (1.0f - blend) * old;
    }
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
}

RT_D void invalidate(Res<Suffix>& r) {
    r.w_sum = 0.0f;
    r.conf = 0.0f;
    r.s.flags = fl_set_valid(r.s.flags, false);
}


}  // namespace crisb
