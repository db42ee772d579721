// rt_common.cuh -- vector math, RNG and record access shared by all kernels.
//
// Floating-point contract: this code is compiled with -fmad=false and IEEE
// division / square root, and every expression keeps the association order of
// the reference's glm expressions (vec3 dot = (x + y) + z, scalar chains
// left to right).  Together with a CPU restatement built the same way, that
// makes discrete decisions (hits, selections, neighbours) reproducible bit
// for bit.  Transcendentals the reference takes from glm are replaced by
// deterministic definitions: sin/cos via Cody-Waite reduction plus Taylor
// polynomials, pow(x, 5) via repeated squaring, the sRGB curve's x^(1/2.4)
// via double-precision series.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "crisb.h"

#define RT_HD __host__ __device__ __forceinline__
#define RT_D __device__ __forceinline__

namespace crisb {

// ---------------------------------------------------------------------------
// float3 arithmetic in glm order
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};

RT_HD V3 mk(float x, float y, float z) { return V3{x, y, z}; }
RT_HD V3 splat(float s) { return V3{s, s, s}; }
RT_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RT_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RT_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
RT_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
RT_HD V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
RT_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
RT_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
RT_HD float dot(V3 a, V3 b) {
    const float x = a.x * b.x;
    const float y = a.y * b.y;
    const float z = a.z * b.z;
    return (x + y) + z;
}
RT_HD float length(V3 v) { return sqrtf(dot(v, v)); }
RT_HD V3 normalize(V3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
RT_HD float distance(V3 p0, V3 p1) { return length(p1 - p0); }
RT_HD V3 reflect(V3 i, V3 n) { return i - n * dot(n, i) * 2.0f; }
RT_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
RT_HD float gmin(float x, float y) { return (y < x) ? y : x; }
RT_HD float gmax(float x, float y) { return (x < y) ? y : x; }
RT_HD V3 gmax(V3 a, V3 b) { return V3{gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
RT_HD float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
RT_HD bool nonfinite(float v) { return isnan(v) || isinf(v); }
RT_HD bool nonfinite(V3 v) { return nonfinite(v.x) || nonfinite(v.y) || nonfinite(v.z); }
RT_HD bool is_zero(V3 v) { return v.x == 0.0f && v.y == 0.0f && v.z == 0.0f; }
RT_HD float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
RT_HD V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }
RT_HD void st3(float* p, V3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

// Rec.709 luminance (include/graph/luminance.h:6-9)
RT_HD float luminance(V3 c) { return dot(c, V3{0.2126f, 0.7152f, 0.0722f}); }

// sin and cos of an angle in [0, 2*pi): Cody-Waite reduction by pi/2 (two-term
// split) and Taylor series of degree 9 (sin) and 10 (cos) on [-pi/4, pi/4],
// each step a correctly rounded fma.  Error below 1e-7 absolute.
RT_HD void sincos_reduced(float phi, float& s, float& c) {
    const float q = rintf(phi * 0x1.45f306p-1f);
    float r = fmaf(q, -0x1.921fb6p+0f, phi);
    r = fmaf(q, 0x1.777a5cp-25f, r);
    const float r2 = r * r;
    float ps = fmaf(r2, 0x1.71de3ap-19f, -0x1.a01a02p-13f);
    ps = fmaf(r2, ps, 0x1.111112p-7f);
    ps = fmaf(r2, ps, -0x1.555556p-3f);
    const float sn = fmaf(r * r2, ps, r);
    float pc = fmaf(r2, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = fmaf(r2, pc, -0x1.6c16c2p-10f);
    pc = fmaf(r2, pc, 0x1.555556p-5f);
    pc = fmaf(r2, pc, -0.5f);
    const float cs = fmaf(r2, pc, 1.0f);
    const int quadrant = static_cast<int>(q) & 3;
    s = quadrant == 0 ? sn : (quadrant == 1 ? cs : (quadrant == 2 ? -sn : -cs));
    c = quadrant == 0 ? cs : (quadrant == 1 ? -sn : (quadrant == 2 ? -cs : sn));
}

RT_HD uint64_t dbits(double x) {
#ifdef __CUDA_ARCH__
    return static_cast<uint64_t>(__double_as_longlong(x));
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}
RT_HD double dfrom(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(b));
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

// x^(1/2.4) of the sRGB transfer curve for a float x, evaluated in double:
// ln x = e ln 2 + 2 atanh((m - 1) / (m + 1)) with the mantissa m in
// [sqrt(1/2), sqrt(2)) (series to s^19), then exp(ln x / 2.4) = 2^k e^r with
// r in [0, ln 2) (Taylor series to r^17).  Relative error below 1e-14, so the
// float result is the correctly rounded power except within 1e-14 of a
// rounding midpoint.  NaN and negative x give NaN, +-0 gives 0, +inf gives
// +inf, as pow does.
RT_HD float srgb_root(float xf) {
    if (isnan(xf) || xf < 0.0f) return static_cast<float>(dfrom(0x7ff8000000000000ULL));
    if (xf == 0.0f) return 0.0f;
    if (isinf(xf)) return xf;
    const uint64_t b = dbits(static_cast<double>(xf));
    int e = static_cast<int>((b >> 52) & 0x7ff) - 1023;
    double m = dfrom((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e = e + 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double p = 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    const double ln2 = 0.6931471805599453;
    const double z = (static_cast<double>(e) * ln2 + 2.0 * s * p) / 2.4;
    const double k = floor(z / ln2);
    const double r = z - k * ln2;
    double t = 1.0;
    for (int i = 17; i >= 1; --i) t = 1.0 + r * t / static_cast<double>(i);
    const double scale = dfrom(static_cast<uint64_t>(static_cast<int>(k) + 1023) << 52);
    return static_cast<float>(t * scale);
}

// LinearToSrgb (src/kernel/tonemap.cu:7-21) for one channel, in the
// reference's arithmetic: both branches of the curve evaluated and blended
// by glm::lerp(if_false, if_true, cond) = if_false * (1 - cond) + if_true *
// cond, glm's clamp (NaN passes through), times 255, truncated.  So negative
// and NaN channels, +inf, and channels above FLT_MAX / 12.92 (where
// 12.92 c overflows and inf * 0 is NaN) all give 0, as in the reference.
RT_HD uint8_t srgb8(float c) {
    const float cond = c < 0.0031308f ? 1.0f : 0.0f;
    const float if_true = 12.92f * c;
    const float if_false = 1.055f * srgb_root(c) - 0.055f;
    const float g = if_false * (1.0f - cond) + if_true * cond;
    const float v = gclamp(g, 0.0f, 1.0f) * 255.0f;
    return isnan(v) ? uint8_t{0} : static_cast<uint8_t>(v);
}

// ---------------------------------------------------------------------------
// RNG: TEA-4 seeding and PCG32 on the default stream (include/util/random.h)
// ---------------------------------------------------------------------------
constexpr uint64_t kPcgMult = 0x5851f42d4c957f2dULL;
constexpr uint64_t kPcgDefaultStream = 0xda3e39cb94b95bdbULL;
constexpr uint64_t kPcgInc = (kPcgDefaultStream << 1u) | 1u;

RT_HD uint64_t tea64(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
#pragma unroll
    for (int n = 0; n < 4; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return static_cast<uint64_t>(v0) | (static_cast<uint64_t>(v1) << 32);
}

// PCG32 whose increment is fixed to the default stream: only the 64-bit state
// is carried in records.
struct Rng {
    uint64_t state;

    RT_HD uint32_t next_u32() {
        const uint64_t old = state;
        state = old * kPcgMult + kPcgInc;
        const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    RT_HD uint64_t next_u64() {
        const uint64_t lo = next_u32();
        const uint64_t hi = next_u32();
        return lo | (hi << 32);
    }
    RT_HD float next_float() {
        const uint32_t bits = (next_u32() >> 9) | 0x3f800000u;
        return __uint_as_float_hd(bits) - 1.0f;
    }
    RT_HD static float __uint_as_float_hd(uint32_t b) {
#ifdef __CUDA_ARCH__
        return __uint_as_float(b);
#else
        float f;
        __builtin_memcpy(&f, &b, 4);
        return f;
#endif
    }
};

// PCG32(seed) with the default stream: Seed(initstate, initseq)
RT_HD Rng rng_seeded(uint64_t initstate) {
    Rng r{0};
    r.next_u32();
    r.state += initstate;
    r.next_u32();
    return r;
}

// ---------------------------------------------------------------------------
// Path records in registers (FP32 layout of crisb_prefix_rec / crisb_suffix_rec)
// ---------------------------------------------------------------------------
struct Hit {  // PackedInteraction
    uint32_t prim;  // CRISB_INVALID_PRIM when invalid
    float bu, bv;
    V3 dir;
    RT_HD bool valid() const { return prim != CRISB_INVALID_PRIM; }
};

struct Isect {  // Interaction (position, normal and incoming direction)
    bool valid;
    uint32_t prim;
    float bu, bv;
    V3 pos, dir, nrm;
    RT_HD Hit pack() const { return Hit{valid ? prim : CRISB_INVALID_PRIM, bu, bv, dir}; }
};

constexpr uint32_t kFlagValid = 1u << 16;
constexpr uint32_t kFlagNee = 1u << 17;
RT_HD uint32_t fl_len(uint32_t f) { return f & 0xFFu; }
RT_HD uint32_t fl_recon(uint32_t f) { return (f >> 8) & 0xFFu; }
RT_HD uint32_t fl_set_len(uint32_t f, uint32_t l) { return (f & ~0xFFu) | (l & 0xFFu); }
RT_HD uint32_t fl_set_recon(uint32_t f, uint32_t r) { return (f & ~0xFF00u) | ((r & 0xFFu) << 8); }
RT_HD bool fl_valid(uint32_t f) { return (f & kFlagValid) != 0; }
RT_HD bool fl_nee(uint32_t f) { return (f & kFlagNee) != 0; }
RT_HD uint32_t fl_set_valid(uint32_t f, bool v) { return v ? (f | kFlagValid) : (f & ~kFlagValid); }
RT_HD uint32_t fl_set_nee(uint32_t f, bool v) { return v ? (f | kFlagNee) : (f & ~kFlagNee); }
// Suffix flags bits 24-31: the loop index of the suffix vertex at which the
// reconnection vertex was chosen (the vertex itself, or the NEE vertex whose
// light ray found it).  The reference's records have no such field (its
// reconIdx of a suffix holds the prefix length); with it the path after the
// reconnection vertex can be re-traced from the suffix's seed, since every
// suffix vertex before it took one NEE draw and three BRDF-sampling draws.
RT_HD uint32_t fl_recon_vert(uint32_t f) { return f >> 24; }
RT_HD uint32_t fl_set_recon_vert(uint32_t f, uint32_t v) { return (f & 0x00FFFFFFu) | ((v & 0xFFu) << 24); }

struct Prefix {
    uint64_t rng;
    Hit primary, recon, last;
    uint32_t flags;
    V3 f, prf;  // f, postReconF
    float p, path_len;
    V3 rod;  // reconOutDir
};

struct Suffix {
    uint64_t rng;
    Hit recon, last_prefix;
    uint32_t flags;
    V3 f, prf;
    float p;
    V3 rod;
};

template <typename T>
struct Res {
    T s;
    float w_sum;
    float conf;
};

// ---- record <-> register conversion -----------------------------------------
RT_HD Hit ld_hit(const crisb_hit_rec& h) { return Hit{h.prim, h.bary[0], h.bary[1], ld3(h.in_dir)}; }
RT_HD void st_hit(crisb_hit_rec& o, const Hit& h) {
    o.prim = h.prim;
    o.bary[0] = h.bu;
    o.bary[1] = h.bv;
    st3(o.in_dir, h.dir);
}
RT_HD Prefix ld_prefix(const crisb_prefix_rec& r) {
    Prefix p;
    p.rng = r.rng;
    p.primary = ld_hit(r.primary);
    p.recon = ld_hit(r.recon);
    p.last = ld_hit(r.last);
    p.flags = r.flags;
    p.f = ld3(r.f);
    p.prf = ld3(r.post_recon_f);
    p.p = r.p;
    p.path_len = r.path_len;
    p.rod = ld3(r.recon_out_dir);
    return p;
}
RT_HD void st_prefix(crisb_prefix_rec& r, const Prefix& p) {
    r.rng = p.rng;
    st_hit(r.primary, p.primary);
    st_hit(r.recon, p.recon);
    st_hit(r.last, p.last);
    r.flags = p.flags;
    st3(r.f, p.f);
    st3(r.post_recon_f, p.prf);
    r.p = p.p;
    r.path_len = p.path_len;
    st3(r.recon_out_dir, p.rod);
}
// The prefix record as eight 16-byte words (the same bytes as the field-wise
// forms above; records of the device arrays start 16-byte aligned): a whole
// record in 8 memory instructions instead of ~25, and the running values a
// path-machine step moves (flags, f, postReconF, p, path length, reconOutDir)
// in the last three words.
static_assert(sizeof(crisb_prefix_rec) == 128 && offsetof(crisb_prefix_rec, primary) == 8 &&
                  offsetof(crisb_prefix_rec, recon) == 32 && offsetof(crisb_prefix_rec, last) == 56 &&
                  offsetof(crisb_prefix_rec, flags) == 80 && offsetof(crisb_prefix_rec, f) == 84 &&
                  offsetof(crisb_prefix_rec, post_recon_f) == 96 && offsetof(crisb_prefix_rec, p) == 108 &&
                  offsetof(crisb_prefix_rec, path_len) == 112 && offsetof(crisb_prefix_rec, recon_out_dir) == 116,
              "prefix record layout");
static_assert(sizeof(crisb_hit_rec) == 24 && offsetof(crisb_hit_rec, bary) == 4 &&
                  offsetof(crisb_hit_rec, in_dir) == 12,
              "hit record layout");
#ifdef __CUDACC__
__device__ inline uint32_t fbits(float v) { return __float_as_uint(v); }
__device__ inline float bitsf(uint32_t v) { return __uint_as_float(v); }
// words 5-7: flags, f, postReconF, p, path length, reconOutDir
__device__ inline void ld_prefix_tail_v(const crisb_prefix_rec& r, Prefix& p) {
    const uint4* w = reinterpret_cast<const uint4*>(&r);
    const uint4 a = w[5], b = w[6], c = w[7];
    p.flags = a.x;
    p.f = V3{bitsf(a.y), bitsf(a.z), bitsf(a.w)};
    p.prf = V3{bitsf(b.x), bitsf(b.y), bitsf(b.z)};
    p.p = bitsf(b.w);
    p.path_len = bitsf(c.x);
    p.rod = V3{bitsf(c.y), bitsf(c.z), bitsf(c.w)};
}
__device__ inline void st_prefix_tail_v(crisb_prefix_rec& r, const Prefix& p) {
    uint4* w = reinterpret_cast<uint4*>(&r);
    w[5] = make_uint4(p.flags, fbits(p.f.x), fbits(p.f.y), fbits(p.f.z));
    w[6] = make_uint4(fbits(p.prf.x), fbits(p.prf.y), fbits(p.prf.z), fbits(p.p));
    w[7] = make_uint4(fbits(p.path_len), fbits(p.rod.x), fbits(p.rod.y), fbits(p.rod.z));
}
// the record's eight words from / to the fields
__device__ inline Prefix prefix_of_words(const uint4 (&w)[8]) {
    const uint4 a = w[0], b = w[1], c = w[2], d = w[3], e = w[4], f = w[5], g = w[6], h = w[7];
    Prefix p;
    p.rng = static_cast<uint64_t>(a.x) | (static_cast<uint64_t>(a.y) << 32);
    p.primary = Hit{a.z, bitsf(a.w), bitsf(b.x), V3{bitsf(b.y), bitsf(b.z), bitsf(b.w)}};
    p.recon = Hit{c.x, bitsf(c.y), bitsf(c.z), V3{bitsf(c.w), bitsf(d.x), bitsf(d.y)}};
    p.last = Hit{d.z, bitsf(d.w), bitsf(e.x), V3{bitsf(e.y), bitsf(e.z), bitsf(e.w)}};
    p.flags = f.x;
    p.f = V3{bitsf(f.y), bitsf(f.z), bitsf(f.w)};
    p.prf = V3{bitsf(g.x), bitsf(g.y), bitsf(g.z)};
    p.p = bitsf(g.w);
    p.path_len = bitsf(h.x);
    p.rod = V3{bitsf(h.y), bitsf(h.z), bitsf(h.w)};
    return p;
}
__device__ inline void words_of_prefix(const Prefix& p, uint4 (&w)[8]) {
    w[0] = make_uint4(static_cast<uint32_t>(p.rng), static_cast<uint32_t>(p.rng >> 32), p.primary.prim,
                      fbits(p.primary.bu));
    w[1] = make_uint4(fbits(p.primary.bv), fbits(p.primary.dir.x), fbits(p.primary.dir.y), fbits(p.primary.dir.z));
    w[2] = make_uint4(p.recon.prim, fbits(p.recon.bu), fbits(p.recon.bv), fbits(p.recon.dir.x));
    w[3] = make_uint4(fbits(p.recon.dir.y), fbits(p.recon.dir.z), p.last.prim, fbits(p.last.bu));
    w[4] = make_uint4(fbits(p.last.bv), fbits(p.last.dir.x), fbits(p.last.dir.y), fbits(p.last.dir.z));
    w[5] = make_uint4(p.flags, fbits(p.f.x), fbits(p.f.y), fbits(p.f.z));
    w[6] = make_uint4(fbits(p.prf.x), fbits(p.prf.y), fbits(p.prf.z), fbits(p.p));
    w[7] = make_uint4(fbits(p.path_len), fbits(p.rod.x), fbits(p.rod.y), fbits(p.rod.z));
}
__device__ inline Prefix ld_prefix_v(const crisb_prefix_rec& r) {
    const uint4* s = reinterpret_cast<const uint4*>(&r);
    uint4 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = s[k];
    return prefix_of_words(w);
}
__device__ inline void st_prefix_v(crisb_prefix_rec& r, const Prefix& p) {
    uint4 w[8];
    words_of_prefix(p, w);
    uint4* d = reinterpret_cast<uint4*>(&r);
#pragma unroll
    for (int k = 0; k < 8; ++k) d[k] = w[k];
}
#endif

RT_HD Suffix ld_suffix(const crisb_suffix_rec& r) {
    Suffix s;
    s.rng = r.rng;
    s.recon = ld_hit(r.recon);
    s.last_prefix = ld_hit(r.last_prefix);
    s.flags = r.flags;
    s.f = ld3(r.f);
    s.prf = ld3(r.post_recon_f);
    s.p = r.p;
    s.rod = ld3(r.recon_out_dir);
    return s;
}
RT_HD void st_suffix(crisb_suffix_rec& r, const Suffix& s) {
    r.rng = s.rng;
    st_hit(r.recon, s.recon);
    st_hit(r.last_prefix, s.last_prefix);
    r.flags = s.flags;
    st3(r.f, s.f);
    st3(r.post_recon_f, s.prf);
    r.p = s.p;
    st3(r.recon_out_dir, s.rod);
    r.pad = 0;
}

}  // namespace crisb
