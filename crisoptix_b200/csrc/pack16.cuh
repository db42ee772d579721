// pack16.cuh -- FP16 reservoir storage: binary16 colours and barycentrics,
// octahedral directions, packed into crisb_prefix_res16_rec (80 B) and
// crisb_suffix_res16_rec (64 B).
//
// Quantisation rules (the oracle applies the same ones when it stores a
// reservoir in this mode):
//   binary16: NaN -> 0, clamp to [-65504, 65504], round to nearest even;
//   octahedral: the zero vector -> CRISB_OCT_ZERO; otherwise p = n.xy / |n|_1,
//     folded for n.z < 0, each coordinate clamped to [-1, 1] and rounded to
//     nearest even of v * 32767 as int16; decoded by the inverse fold and a
//     normalisation.  The fold's sign is the sign bit (-0 folds negative):
//     decoding a code on the fold's edge (|x| or |y| = 1) unfolds the other
//     coordinate to a signed zero, and a sign test of v >= 0 would flip it on
//     re-encoding.  With the sign bit, decoding and re-encoding every code the
//     encoder produces gives the code back, so storing a loaded record again
//     does not move it.
#pragma once

#include <cuda_fp16.h>

#include "rt_common.cuh"

namespace crisb {

RT_D uint16_t h16(float x) {
    if (isnan(x)) x = 0.0f;
    x = fminf(fmaxf(x, -65504.0f), 65504.0f);
    return __half_as_ushort(__float2half_rn(x));
}
RT_D float f16(uint16_t h) { return __half2float(__ushort_as_half(h)); }

RT_D float oct_sign(float v) { return signbit(v) ? -1.0f : 1.0f; }

RT_D uint32_t oct_encode(V3 n) {
    if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) return CRISB_OCT_ZERO;
    const float l1 = (fabsf(n.x) + fabsf(n.y)) + fabsf(n.z);
    float px = n.x / l1, py = n.y / l1;
    if (n.z < 0.0f) {
        const float tx = (1.0f - fabsf(py)) * oct_sign(px);
        const float ty = (1.0f - fabsf(px)) * oct_sign(py);
        px = tx;
        py = ty;
    }
    px = fminf(fmaxf(px, -1.0f), 1.0f);
    py = fminf(fmaxf(py, -1.0f), 1.0f);
    const int qx = static_cast<int>(rintf(px * 32767.0f));
    const int qy = static_cast<int>(rintf(py * 32767.0f));
    return (static_cast<uint32_t>(qx) & 0xFFFFu) | ((static_cast<uint32_t>(qy) & 0xFFFFu) << 16);
}

RT_D V3 oct_decode(uint32_t c) {
    if (c == CRISB_OCT_ZERO) return splat(0.0f);
    float x = static_cast<float>(static_cast<int16_t>(c & 0xFFFFu)) / 32767.0f;
    float y = static_cast<float>(static_cast<int16_t>(c >> 16)) / 32767.0f;
    const float z = (1.0f - fabsf(x)) - fabsf(y);
    if (z < 0.0f) {
        const float tx = (1.0f - fabsf(y)) * oct_sign(x);
        const float ty = (1.0f - fabsf(x)) * oct_sign(y);
        x = tx;
        y = ty;
    }
    return normalize(V3{x, y, z});
}

RT_D crisb_hit16_rec pack_hit16(const Hit& h) {
    crisb_hit16_rec o;
    o.prim = h.prim;
    o.bary[0] = h16(h.bu);
    o.bary[1] = h16(h.bv);
    o.in_dir_oct = oct_encode(h.dir);
    return o;
}
RT_D Hit unpack_hit16(const crisb_hit16_rec& h) {
    return Hit{h.prim, f16(h.bary[0]), f16(h.bary[1]), oct_decode(h.in_dir_oct)};
}

RT_D void pack_rgb16(uint16_t* o, V3 v) {
    o[0] = h16(v.x);
    o[1] = h16(v.y);
    o[2] = h16(v.z);
}
RT_D V3 unpack_rgb16(const uint16_t* o) { return V3{f16(o[0]), f16(o[1]), f16(o[2])}; }

RT_D crisb_prefix_res16_rec pack_pres16(const Res<Prefix>& r) {
    crisb_prefix_res16_rec o;
    o.rng = r.s.rng;
    o.flags = r.s.flags;
    o.p = r.s.p;
    o.path_len = r.s.path_len;
    o.primary = pack_hit16(r.s.primary);
    o.recon = pack_hit16(r.s.recon);
    o.last = pack_hit16(r.s.last);
    pack_rgb16(o.f, r.s.f);
    pack_rgb16(o.post_recon_f, r.s.prf);
    o.recon_out_dir_oct = oct_encode(r.s.rod);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    return o;
}
RT_D Res<Prefix> unpack_pres16(const crisb_prefix_res16_rec& o) {
    Res<Prefix> r;
    r.s.rng = o.rng;
    r.s.flags = o.flags;
    r.s.p = o.p;
    r.s.path_len = o.path_len;
    r.s.primary = unpack_hit16(o.primary);
    r.s.recon = unpack_hit16(o.recon);
    r.s.last = unpack_hit16(o.last);
    r.s.f = unpack_rgb16(o.f);
    r.s.prf = unpack_rgb16(o.post_recon_f);
    r.s.rod = oct_decode(o.recon_out_dir_oct);
    r.w_sum = o.w_sum;
    r.conf = o.confidence;
    return r;
}

RT_D crisb_suffix_res16_rec pack_sres16(const Res<Suffix>& r) {
    crisb_suffix_res16_rec o;
    o.rng = r.s.rng;
    o.flags = r.s.flags;
    o.p = r.s.p;
    o.recon = pack_hit16(r.s.recon);
    o.last_prefix = pack_hit16(r.s.last_prefix);
    pack_rgb16(o.f, r.s.f);
    pack_rgb16(o.post_recon_f, r.s.prf);
    o.recon_out_dir_oct = oct_encode(r.s.rod);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    return o;
}
RT_D Res<Suffix> unpack_sres16(const crisb_suffix_res16_rec& o) {
    Res<Suffix> r;
    r.s.rng = o.rng;
    r.s.flags = o.flags;
    r.s.p = o.p;
    r.s.recon = unpack_hit16(o.recon);
    r.s.last_prefix = unpack_hit16(o.last_prefix);
    r.s.f = unpack_rgb16(o.f);
    r.s.prf = unpack_rgb16(o.post_recon_f);
    r.s.rod = oct_decode(o.recon_out_dir_oct);
    r.w_sum = o.w_sum;
    r.conf = o.confidence;
    return r;
}

// whole-record vector loads / stores (records are 16-byte multiples at
// 16-byte aligned bases)
template <class T>
RT_D T ld_rec(const void* base, uint32_t i) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16");
    constexpr int kN = sizeof(T) / 16;
    const uint4* s = static_cast<const uint4*>(base) + static_cast<size_t>(i) * kN;
    uint4 v[kN];
#pragma unroll
    for (int k = 0; k < kN; ++k) v[k] = s[k];
    T r;
    memcpy(&r, v, sizeof(T));
    return r;
}
template <class T>
RT_D void st_rec(void* base, uint32_t i, const T& r) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16");
    constexpr int kN = sizeof(T) / 16;
    uint4 v[kN];
    memcpy(v, &r, sizeof(T));
    uint4* d = static_cast<uint4*>(base) + static_cast<size_t>(i) * kN;
#pragma unroll
    for (int k = 0; k < kN; ++k) d[k] = v[k];
}

}  // namespace crisb
