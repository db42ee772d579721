/*
 * restir_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the oracle.
 *
 * A CPU (C++17 + OpenMP) restatement of CrisOptix's Conditional ReSTIR PT
 * frame loop, written function by function against the reference sources
 * (paths relative to the CrisOptix repository).  It checks the CUDA product;
 * the product never links it, and only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.
 *
 * Parity status: the reference application cannot be built or run here (it
 * needs the OptiX SDK and an OpenGL window) and ships no tests or golden
 * vectors.  Its unit-level device code can: oracle/Makefile `ref` compiles
 * the reference's own headers unmodified (random.h, luminance.h,
 * Reservoir.h, Camera.h, sample_emitter.h, and path_gen.h:12-72,
 * Emitter.h:6-55, brdf.cu:12-37/99-112 cut from files whose rest needs OptiX)
 * against a minimal glm (oracle/ref_shim), and tests/golden/ref_kat.npz
 * records its answers.  This restatement matches them bit for bit (TEA,
 * PCG32 seeding and draws, luminance, both pairwise MIS weights,
 * SelectSpatialNeighbor, the reconnection Jacobian, Reservoir::Update /
 * FinalizeGRIS sequences, D_GGX, V_SmithJointGGX, SpawnCameraRay, emitter
 * sampling), FresnelSchlick within 4 ulp (pow below); tests/test_ref_kat.py.
 * Above that level (traversal, the pass chain) the restatement follows the
 * cited reference lines; where the reference is non-deterministic or leans on
 * OptiX internals it fixes a deterministic definition, marked DEFINED below:
 *   - optixTrace: own BVH + watertight ray/triangle test (Woop, Benthin &
 *     Wald 2013), closest hit = smallest t, ties -> lower triangle index;
 *     a hit counts when tmin < t < tmax.  Boxes are widened by a margin
 *     (BoxMargin) so the hits are those of testing every triangle, whatever
 *     the tree.
 *   - prefix-endpoint neighbour search: the k nearest in-radius endpoints
 *     ordered by (distance, pixel index) instead of OptiX traversal order.
 *   - spatial reuse reads neighbours from the snapshot taken at pass start
 *     (the reference reads buffers other threads are writing).
 *   - glm::cos/sin -> Taylor polynomials after Cody-Waite reduction;
 *     glm::pow(x, 5) -> x^2*x^2*x.  Everything else is IEEE + - * / and sqrt with
 *     no contraction, in the reference's association order.
 *   - per-frame random: PCG32(seed, frame counter).NextUint32() instead of
 *     std::random_device (src/Renderer.cpp:9-11,215).
 *   - the NEE re-trace of the same ray in TracePrefix
 *     (include/graph/restir/path_gen.h:165-187) is deterministic and returns
 *     the interaction already in hand, so it is not re-traced.
 */
#include "oracle.h"
#include "kat.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// glm subset with glm's evaluation order (vec3 dot = (x + y) + z, etc.)
// ---------------------------------------------------------------------------
struct vec2 {
    float x = 0.0f, y = 0.0f;
};

struct vec3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    vec3() = default;
    constexpr vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit constexpr vec3(float s) : x(s), y(s), z(s) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

inline vec3 operator+(vec3 a, vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(vec3 a, vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator*(vec3 a, vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator/(vec3 a, vec3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator*(vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator/(vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline vec3 operator-(vec3 a) { return {-a.x, -a.y, -a.z}; }
inline vec3& operator*=(vec3& a, vec3 b) { a = a * b; return a; }
inline vec3& operator*=(vec3& a, float s) { a = a * s; return a; }
inline vec3& operator+=(vec3& a, vec3 b) { a = a + b; return a; }
inline vec3& operator/=(vec3& a, float s) { a = a / s; return a; }
inline bool operator==(vec3 a, vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

inline float dot(vec3 a, vec3 b) {
    const vec3 t = a * b;
    return t.x + t.y + t.z;
}
inline float length(vec3 v) { return std::sqrt(dot(v, v)); }
// glm::normalize = v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x)
inline vec3 normalize(vec3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline float distance(vec3 p0, vec3 p1) { return length(p1 - p0); }
inline vec3 reflect(vec3 I, vec3 N) { return I - N * dot(N, I) * 2.0f; }
inline vec3 cross(vec3 x, vec3 y) {
    return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
// glm::min/max: (y < x) ? y : x and (x < y) ? y : x
inline float gmin(float x, float y) { return (y < x) ? y : x; }
inline float gmax(float x, float y) { return (x < y) ? y : x; }
inline vec3 gmax(vec3 a, vec3 b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
inline float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
inline bool anyNanInf(vec3 v) {
    return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z) || std::isinf(v.x) ||
           std::isinf(v.y) || std::isinf(v.z);
}

// DEFINED: x^(1/2.4) for the sRGB curve, in double.  ln x = e ln 2 +
// 2 atanh(s), s = (m - 1) / (m + 1), mantissa m in [sqrt(1/2), sqrt(2))
// (odd series to s^19); exp(ln x / 2.4) = 2^k e^r, r = z - k ln 2 (Taylor
// series to r^17, Horner).  The reference calls glm::pow (powf); this stays
// within 1e-14 relative of the exact power.
inline float SrgbRoot(float xf) {
    if (std::isnan(xf) || xf < 0.0f) return std::numeric_limits<float>::quiet_NaN();
    if (xf == 0.0f) return 0.0f;
    if (std::isinf(xf)) return xf;
    int e = 0;
    double m = 2.0 * std::frexp(static_cast<double>(xf), &e);  // [1, 2)
    e -= 1;
    if (m > 1.4142135623730951) {
        m *= 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double p = 0.0;
    for (int k = 19; k >= 1; k -= 2) p = (k == 19) ? 1.0 / 19.0 : p * s2 + 1.0 / k;
    const double ln2 = 0.6931471805599453;
    const double z = (static_cast<double>(e) * ln2 + 2.0 * s * p) / 2.4;
    const double k = std::floor(z / ln2);
    const double r = z - k * ln2;
    double t = 1.0;
    for (int i = 17; i >= 1; --i) t = 1.0 + r * t / static_cast<double>(i);
    return static_cast<float>(t * std::ldexp(1.0, static_cast<int>(k)));
}

// LinearToSrgb / ApplySrgbGamma, src/kernel/tonemap.cu:7-21, one channel:
// both branches, glm::lerp(if_false, if_true, cond) = if_false * (1 - cond) +
// if_true * cond, glm::clamp (ternary min/max), * 255, truncation (NaN -> 0).
inline uint8_t LinearToSrgb8(float c) {
    const float cond = c < 0.0031308f ? 1.0f : 0.0f;
    const float if_true = 12.92f * c;
    const float if_false = 1.055f * SrgbRoot(c) - 0.055f;
    const float g = if_false * (1.0f - cond) + if_true * cond;
    const float lo = (g < 0.0f) ? 0.0f : g;
    const float v = ((1.0f < lo) ? 1.0f : lo) * 255.0f;
    return std::isnan(v) ? 0 : static_cast<uint8_t>(v);
}

// GetLuminance, include/graph/luminance.h:6-9
inline float GetLuminance(vec3 c) { return dot(c, vec3(0.2126f, 0.7152f, 0.0722f)); }

// DEFINED: sin/cos of phi in [0, 2pi) -- Cody-Waite reduction by pi/2 and
// Taylor polynomials (degree 9 / 10) on [-pi/4, pi/4], all steps by fmaf.
inline void SinCos(float phi, float& s, float& c) {
    const float q = std::rint(phi * 0x1.45f306p-1f);  // 2/pi
    float r = std::fma(q, -0x1.921fb6p+0f, phi);        // pi/2 high part
    r = std::fma(q, 0x1.777a5cp-25f, r);                // pi/2 low part (pi/2 - hi < 0)
    const float r2 = r * r;
    float ps = std::fma(r2, 0x1.71de3ap-19f, -0x1.a01a02p-13f);
    ps = std::fma(r2, ps, 0x1.111112p-7f);
    ps = std::fma(r2, ps, -0x1.555556p-3f);
    const float sn = std::fma(r * r2, ps, r);
    float pc = std::fma(r2, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = std::fma(r2, pc, -0x1.6c16c2p-10f);
    pc = std::fma(r2, pc, 0x1.555556p-5f);
    pc = std::fma(r2, pc, -0.5f);
    const float cs = std::fma(r2, pc, 1.0f);
    switch (static_cast<int>(q) & 3) {
        case 0: s = sn; c = cs; break;
        case 1: s = cs; c = -sn; break;
        case 2: s = -sn; c = -cs; break;
        default: s = -cs; c = sn; break;
    }
}

// ---------------------------------------------------------------------------
// RNG, include/util/random.h:7-119
// ---------------------------------------------------------------------------
constexpr uint64_t PCG32_DEFAULT_STATE = 0x853c49e6748fea9bULL;
constexpr uint64_t PCG32_DEFAULT_STREAM = 0xda3e39cb94b95bdbULL;
constexpr uint64_t PCG32_MULT = 0x5851f42d4c957f2dULL;

inline uint64_t SampleTEA64(uint32_t val0, uint32_t val1, uint32_t rounds = 4) {
    uint32_t v0 = val0, v1 = val1, s0 = 0;
    for (uint32_t n = 0; n < rounds; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return static_cast<uint64_t>(v0) | (static_cast<uint64_t>(v1) << 32);
}

struct PCG32 {
    uint64_t state = 0;
    uint64_t inc = (PCG32_DEFAULT_STREAM << 1u) | 1u;

    PCG32() = default;
    explicit PCG32(uint64_t initstate, uint64_t initseq = PCG32_DEFAULT_STREAM) {
        Seed(initstate, initseq);
    }
    void Seed(uint64_t initstate, uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        NextUint32();
        state += initstate;
        NextUint32();
    }
    uint32_t NextUint32() {
        const uint64_t oldstate = state;
        state = oldstate * PCG32_MULT + inc;
        const uint32_t xorshifted = static_cast<uint32_t>(((oldstate >> 18u) ^ oldstate) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(oldstate >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    uint64_t NextUint64() {
        const uint64_t lo = NextUint32();
        const uint64_t hi = NextUint32();
        return lo | (hi << 32);
    }
    float NextFloat() {
        const uint32_t bits = (NextUint32() >> 9) | 0x3f800000u;
        float f;
        std::memcpy(&f, &bits, 4);
        return f - 1.0f;
    }
};

// ---------------------------------------------------------------------------
// Interactions, include/graph/Interaction.h:27-184, shader/mesh_hit.cu:17-69
// ---------------------------------------------------------------------------
struct PackedInteraction {
    uint32_t prim = 0;
    vec2 bary;
    vec3 inRayDir;
    bool valid = false;
};

struct Interaction {
    uint32_t prim = 0;
    vec3 pos;
    vec3 inRayDir;
    vec3 normal;
    vec2 bary;
    bool valid = false;
    PackedInteraction Pack() const {
        PackedInteraction p;
        p.prim = prim;
        p.bary = bary;
        p.inRayDir = inRayDir;
        p.valid = valid;
        return p;
    }
};

// InterpolateBary, include/graph/Interaction.h:18-25
inline vec3 InterpolateBary(vec2 b, vec3 v0, vec3 v1, vec3 v2) {
    return ((1.0f - b.x - b.y) * v0) + (b.x * v1) + (b.y * v2);
}

struct Triangle {
    vec3 p[3];
    vec3 n[3];
    uint32_t mat;
};

// ---------------------------------------------------------------------------
// Path records, include/graph/restir/PrefixPath.h, SuffixPath.h
// ---------------------------------------------------------------------------
struct PrefixPath {
    PCG32 rng;
    PackedInteraction primaryInt, reconInt, lastInt;
    uint32_t flags = 0;
    vec3 f{0.0f, 0.0f, 0.0f};
    vec3 postReconF{0.0f, 0.0f, 0.0f};
    float p = 0.0f;
    float pathLen = 0.0f;
    vec3 reconOutDir{0.0f, 0.0f, 0.0f};

    PrefixPath() { rng.state = 0; }
    // PrefixPath(other, f, primaryInt), PrefixPath.h:60-81 (the triangle-range
    // check there cannot fail for triangles produced by this scene)
    PrefixPath(const PrefixPath& o, vec3 _f, const PackedInteraction& _primaryInt) : PrefixPath(o) {
        f = _f;
        primaryInt = _primaryInt;
    }
    PrefixPath(const PrefixPath&) = default;
    PrefixPath& operator=(const PrefixPath&) = default;

    void Reset() { flags = 0u; pathLen = 0.0f; }
    uint32_t GetLength() const { return flags & 0xFFu; }
    void SetLength(uint32_t l) { flags &= ~0xFFu; flags |= l & 0xFFu; }
    uint32_t GetReconIdx() const { return (flags >> 8u) & 0xFFu; }
    void SetReconIdx(uint32_t r) { flags &= ~0xFF00u; flags |= (r & 0xFFu) << 8u; }
    bool IsValid() const { return (flags & (1u << 16u)) != 0; }
    void SetValid(bool v) { flags &= ~(1u << 16u); if (v) flags |= 1u << 16u; }
    bool IsNee() const { return (flags & (1u << 17u)) != 0; }
    void SetNee(bool v) { flags &= ~(1u << 17u); if (v) flags |= 1u << 17u; }
};

struct SuffixPath {
    PCG32 rng;
    PackedInteraction reconInt, lastPrefixInt;
    uint32_t flags = 0;
    vec3 f{0.0f, 0.0f, 0.0f};
    vec3 postReconF{0.0f, 0.0f, 0.0f};
    float p = 0.0f;
    vec3 reconOutDir{0.0f, 0.0f, 0.0f};

    SuffixPath() { rng.state = 0; }
    // SuffixPath(other, lastPrefixInt, f), SuffixPath.h:47-62
    SuffixPath(const SuffixPath& o, const PackedInteraction& _lastPrefixInt, vec3 _f) : SuffixPath(o) {
        lastPrefixInt = _lastPrefixInt;
        f = _f;
    }
    SuffixPath(const SuffixPath&) = default;
    SuffixPath& operator=(const SuffixPath&) = default;

    void Reset() { flags = 0u; }
    uint32_t GetLength() const { return flags & 0xFFu; }
    void SetLength(uint32_t l) { flags &= ~0xFFu; flags |= l & 0xFFu; }
    uint32_t GetReconIdx() const { return (flags >> 8u) & 0xFFu; }
    void SetReconIdx(uint32_t r) { flags &= ~0xFF00u; flags |= (r & 0xFFu) << 8u; }
    bool IsValid() const { return (flags & (1u << 16u)) != 0; }
    void SetValid(bool v) { flags &= ~(1u << 16u); if (v) flags |= 1u << 16u; }
    // bits 24-31 (not in the reference's SuffixPath.h): the loop index of the
    // suffix vertex at which the reconnection vertex was chosen, so that the
    // path after it can be re-traced from `rng` by a path-replay adjoint
    uint32_t GetReconVert() const { return flags >> 24u; }
    void SetReconVert(uint32_t v) { flags &= 0x00FFFFFFu; flags |= (v & 0xFFu) << 24u; }
};

// Reservoir, include/graph/restir/Reservoir.h:8-51
template <typename T>
struct Reservoir {
    T sample;
    float wSum = 0.0f;
    float confidence = 0.0f;

    void Reset() { wSum = 0.0f; confidence = 0.0f; }
    bool Update(const T& s, float risWeight, PCG32& rng, float inputConfidence) {
        if (std::isnan(risWeight) || std::isinf(risWeight)) risWeight = 0.0f;
        wSum += risWeight;
        confidence += inputConfidence;
        confidence = gmin(confidence, CRISB_CONFIDENCE_MAX);
        if (rng.NextFloat() < risWeight / wSum) {
            sample = s;
            return true;
        }
        return false;
    }
    void FinalizeGRIS() {
        const float pHat = GetLuminance(sample.f);
        if (pHat == 0.0f) wSum = 0.0f;
        else wSum /= pHat;
    }
};

// ---- FP16 reservoir storage (crisb_params.storage == CRISB_STORAGE_FP16) ----
// The library stores reservoirs between passes with binary16 colours and
// barycentrics and octahedral directions (include/crisb.h); the oracle keeps
// FP32 reservoirs and quantises them at the same points, so that every load
// sees the value the library loads.  Rules: binary16 = NaN -> 0, clamp to
// +-65504, round to nearest even (IEEE 754 binary32 -> binary16 conversion);
// octahedral = zero vector -> a reserved code, else p = n.xy / |n|_1 folded
// for n.z < 0, clamped to [-1, 1], rounded (nearest even) to int16 units of
// 1/32767, decoded by the inverse fold and a normalisation.
uint16_t HalfBits(float f) {
    if (std::isnan(f)) f = 0.0f;
    f = std::fmin(std::fmax(f, -65504.0f), 65504.0f);
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x38800000u) {  // |f| >= 2^-14: a normal binary16
        const uint32_t m = ax & 0x7fffffu;
        uint32_t h = (((ax >> 23) - 112u) << 10) | (m >> 13);
        const uint32_t rem = m & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
        return static_cast<uint16_t>(sign | h);
    }
    if (ax < 0x33000000u) return static_cast<uint16_t>(sign);  // below 2^-25
    const uint32_t e = ax >> 23;
    const uint32_t M = (ax & 0x7fffffu) | 0x800000u;
    const uint32_t sh = 126u - e;  // 14 .. 24
    uint32_t m = M >> sh;
    const uint32_t rem = M & ((1u << sh) - 1u), half = 1u << (sh - 1u);
    if (rem > half || (rem == half && (m & 1u))) ++m;
    return static_cast<uint16_t>(sign | m);
}

float HalfValue(uint16_t h) {
    const uint32_t sign = static_cast<uint32_t>(h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t bits;
    if (e == 0) {
        const float v = std::ldexp(static_cast<float>(m), -24);  // exact
        std::memcpy(&bits, &v, 4);
    } else if (e == 31) {
        bits = m ? 0x7fc00000u : 0x7f800000u;
    } else {
        bits = ((e + 112u) << 23) | (m << 13);
    }
    bits |= sign;
    float v;
    std::memcpy(&v, &bits, 4);
    return v;
}

float Quant16(float f) { return HalfValue(HalfBits(f)); }

// the fold's sign is the sign bit (-0 folds negative), which keeps every code
// the encoder produces stable under decode + re-encode
float OctSign(float v) { return std::signbit(v) ? -1.0f : 1.0f; }

uint32_t OctEncode(vec3 n) {
    if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) return CRISB_OCT_ZERO;
    const float l1 = (std::fabs(n.x) + std::fabs(n.y)) + std::fabs(n.z);
    float px = n.x / l1, py = n.y / l1;
    if (n.z < 0.0f) {
        const float tx = (1.0f - std::fabs(py)) * OctSign(px);
        const float ty = (1.0f - std::fabs(px)) * OctSign(py);
        px = tx;
        py = ty;
    }
    px = std::fmin(std::fmax(px, -1.0f), 1.0f);
    py = std::fmin(std::fmax(py, -1.0f), 1.0f);
    const int qx = static_cast<int>(std::rint(px * 32767.0f));
    const int qy = static_cast<int>(std::rint(py * 32767.0f));
    return (static_cast<uint32_t>(qx) & 0xFFFFu) | ((static_cast<uint32_t>(qy) & 0xFFFFu) << 16);
}

vec3 OctDecode(uint32_t c) {
    if (c == CRISB_OCT_ZERO) return vec3(0.0f);
    float x = static_cast<float>(static_cast<int16_t>(c & 0xFFFFu)) / 32767.0f;
    float y = static_cast<float>(static_cast<int16_t>(c >> 16)) / 32767.0f;
    const float z = (1.0f - std::fabs(x)) - std::fabs(y);
    if (z < 0.0f) {
        const float tx = (1.0f - std::fabs(y)) * OctSign(x);
        const float ty = (1.0f - std::fabs(x)) * OctSign(y);
        x = tx;
        y = ty;
    }
    return normalize(vec3(x, y, z));
}

vec3 Quant16(vec3 v) { return vec3(Quant16(v.x), Quant16(v.y), Quant16(v.z)); }

void QuantizeHit(PackedInteraction& p) {
    p.bary.x = Quant16(p.bary.x);
    p.bary.y = Quant16(p.bary.y);
    p.inRayDir = OctDecode(OctEncode(p.inRayDir));
}
void Quantize(PrefixPath& s) {
    QuantizeHit(s.primaryInt);
    QuantizeHit(s.reconInt);
    QuantizeHit(s.lastInt);
    s.f = Quant16(s.f);
    s.postReconF = Quant16(s.postReconF);
    s.reconOutDir = OctDecode(OctEncode(s.reconOutDir));
}
void Quantize(SuffixPath& s) {
    QuantizeHit(s.reconInt);
    QuantizeHit(s.lastPrefixInt);
    s.f = Quant16(s.f);
    s.postReconF = Quant16(s.postReconF);
    s.reconOutDir = OctDecode(OctEncode(s.reconOutDir));
}

// RestirGBuffer, include/graph/restir/RestirGBuffer.h:5-28
struct GBuffer {
    PCG32 rng;
    uint32_t prevX = 0, prevY = 0;
    bool primaryIntValid = false;
    GBuffer() { rng.state = 0; }
};

struct Neighbor {
    uint32_t pixelIdx = 0;
    float distance = 0.0f;
};

// ---------------------------------------------------------------------------
// BVH + watertight triangle test (replaces optixTrace; DEFINED semantics)
// ---------------------------------------------------------------------------
struct RayPre {
    vec3 org, dir, inv;
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

inline float AbsF(float v) { return std::fabs(v); }

inline RayPre MakeRay(vec3 o, vec3 d) {
    RayPre r;
    r.org = o;
    r.dir = d;
    const float ad[3] = {AbsF(d.x), AbsF(d.y), AbsF(d.z)};
    int kz = 0;
    if (ad[1] > ad[kz]) kz = 1;
    if (ad[2] > ad[kz]) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < 0.0f) std::swap(kx, ky);
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.Sx = d[kx] / d[kz];
    r.Sy = d[ky] / d[kz];
    r.Sz = 1.0f / d[kz];
    // box-test reciprocal: zero components replaced by a signed tiny value
    auto rcp = [](float v) {
        if (std::fabs(v) < 1e-30f) v = std::copysign(1e-30f, v);
        return 1.0f / v;
    };
    r.inv = vec3(rcp(d.x), rcp(d.y), rcp(d.z));
    return r;
}

// Woop, Benthin & Wald 2013, "Watertight Ray/Triangle Intersection", JCGT 2(1).
// Returns true with t and barycentrics (u: weight of p1, v: weight of p2) when
// tmin < t < tmax.
inline bool IntersectTri(const RayPre& r, const vec3& p0, const vec3& p1, const vec3& p2,
                         float tmin, float tmax, float& tOut, float& uOut, float& vOut) {
    const vec3 A = p0 - r.org, B = p1 - r.org, C = p2 - r.org;
    const float Ax = A[r.kx] - r.Sx * A[r.kz];
    const float Ay = A[r.ky] - r.Sy * A[r.kz];
    const float Bx = B[r.kx] - r.Sx * B[r.kz];
    const float By = B[r.ky] - r.Sy * B[r.kz];
    const float Cx = C[r.kx] - r.Sx * C[r.kz];
    const float Cy = C[r.ky] - r.Sy * C[r.kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = static_cast<float>(static_cast<double>(Cx) * static_cast<double>(By) -
                               static_cast<double>(Cy) * static_cast<double>(Bx));
        V = static_cast<float>(static_cast<double>(Ax) * static_cast<double>(Cy) -
                               static_cast<double>(Ay) * static_cast<double>(Cx));
        W = static_cast<float>(static_cast<double>(Bx) * static_cast<double>(Ay) -
                               static_cast<double>(By) * static_cast<double>(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * A[r.kz];
    const float Bz = r.Sz * B[r.kz];
    const float Cz = r.Sz * C[r.kz];
    const float T = U * Az + V * Bz + W * Cz;
    const float rcpDet = 1.0f / det;
    const float t = T * rcpDet;
    if (!(t > tmin && t < tmax)) return false;
    tOut = t;
    uOut = V * rcpDet;
    vOut = W * rcpDet;
    return true;
}

struct BvhNode {
    float lo[3], hi[3];
    int32_t left = -1, right = -1;
    uint32_t first = 0, count = 0;
};

struct HitResult {
    bool hit = false;
    uint32_t prim = 0;
    float t = 0.0f, u = 0.0f, v = 0.0f;
};

// Robust slab test (Ize 2013, "Robust BVH Ray Traversal"): tfar *= 1 + 2*gamma(3).
constexpr float kSlabFarScale = 1.0000003576f;

// DEFINED: box margin.  The watertight triangle test translates vertices to
// the ray origin and shears them in float, so it accepts rays up to a few ulp
// of the origin-vertex distance outside the exact triangle, and t to a few
// ulp; a ray lying in a box face plane (a zero direction component, common
// between points of one axis-aligned face) is also cut off at t = 0 by the
// slab test.  Widening every box by 2^-17 x the scene's largest coordinate
// magnitude keeps each box test at least an order of magnitude more generous
// than those errors for rays starting within twice that magnitude, so the box
// test never rejects a ray the triangle test accepts and any tree yields the
// brute-force hits.
inline float BoxMargin(float maxAbsCoord) { return std::ldexp(std::max(maxAbsCoord, 1e-20f), -17); }

inline bool SlabHit(const RayPre& r, const BvhNode& n, float tmin, float tmax) {
    float tn = tmin, tf = tmax;
    for (int a = 0; a < 3; ++a) {
        const float o = r.org[a], inv = r.inv[a];
        float t0 = (n.lo[a] - o) * inv;
        float t1 = (n.hi[a] - o) * inv;
        if (t0 > t1) std::swap(t0, t1);
        tn = t0 > tn ? t0 : tn;
        tf = t1 < tf ? t1 : tf;
    }
    return tn <= tf * kSlabFarScale;
}

class Bvh {
  public:
    void Build(const std::vector<Triangle>& tris) {
        tris_ = &tris;
        const uint32_t n = static_cast<uint32_t>(tris.size());
        order_.resize(n);
        for (uint32_t i = 0; i < n; ++i) order_[i] = i;
        centroids_.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            const Triangle& t = tris[i];
            centroids_[i] = vec3((t.p[0].x + t.p[1].x + t.p[2].x) / 3.0f,
                                 (t.p[0].y + t.p[1].y + t.p[2].y) / 3.0f,
                                 (t.p[0].z + t.p[1].z + t.p[2].z) / 3.0f);
        }
        // DEFINED: every node box is widened by kBoxMargin x the largest
        // coordinate magnitude of the scene (BoxMargin), so that the box test
        // never rejects a ray the triangle test would accept
        float maxAbs = 0.0f;
        for (const Triangle& t : tris)
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) maxAbs = std::max(maxAbs, std::fabs(t.p[c][a]));
        margin_ = BoxMargin(maxAbs);
        nodes_.clear();
        nodes_.reserve(2 * n + 1);
        if (n > 0) BuildRec(0, n);
    }

    HitResult Closest(const RayPre& r, float tmin, float tmax) const {
        HitResult best;
        if (nodes_.empty()) return best;
        float bestT = tmax;
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const BvhNode& nd = nodes_[stack[--sp]];
            if (!SlabHit(r, nd, tmin, bestT)) continue;
            if (nd.count > 0) {
                for (uint32_t k = 0; k < nd.count; ++k) {
                    const uint32_t prim = order_[nd.first + k];
                    const Triangle& t = (*tris_)[prim];
                    float th, u, v;
                    // closest: smallest t, ties -> lower triangle index
                    if (IntersectTri(r, t.p[0], t.p[1], t.p[2], tmin, tmax, th, u, v)) {
                        if (!best.hit || th < best.t || (th == best.t && prim < best.prim)) {
                            best.hit = true;
                            best.prim = prim;
                            best.t = th;
                            best.u = u;
                            best.v = v;
                            bestT = th;
                        }
                    }
                }
            } else {
                stack[sp++] = nd.left;
                stack[sp++] = nd.right;
            }
        }
        return best;
    }

    bool Occluded(const RayPre& r, float tmin, float tmax) const {
        if (nodes_.empty()) return false;
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const BvhNode& nd = nodes_[stack[--sp]];
            if (!SlabHit(r, nd, tmin, tmax)) continue;
            if (nd.count > 0) {
                for (uint32_t k = 0; k < nd.count; ++k) {
                    const Triangle& t = (*tris_)[order_[nd.first + k]];
                    float th, u, v;
                    if (IntersectTri(r, t.p[0], t.p[1], t.p[2], tmin, tmax, th, u, v)) return true;
                }
            } else {
                stack[sp++] = nd.left;
                stack[sp++] = nd.right;
            }
        }
        return false;
    }

  private:
    int BuildRec(uint32_t first, uint32_t count) {
        const int idx = static_cast<int>(nodes_.size());
        nodes_.emplace_back();
        BvhNode nd;
        for (int a = 0; a < 3; ++a) {
            nd.lo[a] = std::numeric_limits<float>::infinity();
            nd.hi[a] = -std::numeric_limits<float>::infinity();
        }
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = first; i < first + count; ++i) {
            const Triangle& t = (*tris_)[order_[i]];
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) {
                    nd.lo[a] = std::min(nd.lo[a], t.p[c][a]);
                    nd.hi[a] = std::max(nd.hi[a], t.p[c][a]);
                }
            for (int a = 0; a < 3; ++a) {
                clo[a] = std::min(clo[a], centroids_[order_[i]][a]);
                chi[a] = std::max(chi[a], centroids_[order_[i]][a]);
            }
        }
        for (int a = 0; a < 3; ++a) {
            nd.lo[a] -= margin_;
            nd.hi[a] += margin_;
        }
        if (count <= 4) {
            nd.first = first;
            nd.count = count;
            nodes_[idx] = nd;
            return idx;
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        const uint32_t mid = first + count / 2;
        std::nth_element(order_.begin() + first, order_.begin() + mid, order_.begin() + first + count,
                         [&](uint32_t a, uint32_t b) {
                             const float ca = centroids_[a][axis], cb = centroids_[b][axis];
                             return ca < cb || (ca == cb && a < b);
                         });
        const int l = BuildRec(first, mid - first);
        const int rr = BuildRec(mid, first + count - mid);
        nd.left = l;
        nd.right = rr;
        nodes_[idx] = nd;
        return idx;
    }

    const std::vector<Triangle>* tris_ = nullptr;
    float margin_ = 0.0f;
    std::vector<uint32_t> order_;
    std::vector<vec3> centroids_;
    std::vector<BvhNode> nodes_;
};

// ---------------------------------------------------------------------------
// BRDF, shader/brdf.cu:12-338 (no textures)
// ---------------------------------------------------------------------------
constexpr float PI = 3.14159265358979323846264f;

struct BrdfEvalResult {
    vec3 brdfResult;
    float samplingPdf = 0.0f;
    vec3 emission;
    float roughness = 0.0f;
};

struct BrdfSampleResult {
    vec3 outDir;
    vec3 brdfVal;
    float samplingPdf = 0.0f;
    float roughness = 0.0f;
};

inline float P2(float x) { return x * x; }
// DEFINED: glm::pow(x, 5.0f) as x^2 * x^2 * x
inline float Pow5(float x) {
    const float x2 = x * x;
    return x2 * x2 * x;
}
// FresnelSchlick, brdf.cu:34-37
inline vec3 FresnelSchlick(vec3 F0, float VdotH) {
    return F0 + (vec3(1.0f) - F0) * Pow5(gmax(0.0f, 1.0f - VdotH));
}
// D_GGX, brdf.cu:99-104
inline float D_GGX(float NdotH, float roughness) {
    const float a2 = roughness * roughness;
    const float d = (NdotH * a2 - NdotH) * NdotH + 1.0f;
    return a2 / (PI * d * d);
}
// V_SmithJointGGX, brdf.cu:106-112
inline float V_SmithJointGGX(float NdotL, float NdotV, float roughness) {
    const float a2 = roughness * roughness;
    const float lambdaV = NdotL * std::sqrt(NdotV * NdotV * (1 - a2) + a2);
    const float lambdaL = NdotV * std::sqrt(NdotL * NdotL * (1 - a2) + a2);
    return 0.5f / (lambdaV + lambdaL);
}

struct MatVals {
    vec3 diff, specF0, emission;
    float roughness;
};

// material fetch of brdf.cu:120-138 / 219-237 over looked-up values (the
// material's constants, or texture samples where it has textures)
inline MatVals FinishMat(const crisb_material& m, vec3 diff, vec3 specF0, float roughness) {
    MatVals v;
    v.diff = diff;
    float metal = 0.0f;
    if (m.spec_usage == CRISB_SPEC_OCC_ROUGH_METAL) {
        roughness = specF0.y;
        metal = specF0.z;
        specF0 = vec3(1.0f);
    }
    // glm::mix(x, y, a) = x * (1 - a) + y * a
    v.specF0 = v.diff * (1.0f - metal) + specF0 * metal;
    v.emission = vec3(m.emission[0], m.emission[1], m.emission[2]);
    v.roughness = roughness;
    return v;
}

inline MatVals GetMat(const crisb_material& m) {
    return FinishMat(m, vec3(m.diffuse[0], m.diffuse[1], m.diffuse[2]),
                     vec3(m.specular[0], m.specular[1], m.specular[2]), m.roughness);
}

// __direct_callable__ggx_eval, brdf.cu:115-190
inline BrdfEvalResult GgxEval(const MatVals& m, const Interaction& interaction, vec3 outDir) {
    BrdfEvalResult result;
    const vec3 lightDir = outDir;
    const vec3 viewDir = -interaction.inRayDir;
    const vec3 normal = interaction.normal;
    const float nDotV = dot(normal, viewDir);
    const float nDotL = dot(normal, lightDir);
    if (nDotV <= 0.0f || nDotL < 0.0f) return result;
    const vec3 diffBrdf = m.diff / PI;
    vec3 specBrdf(0.0f);
    const float diffProb = dot(m.diff, vec3(1.0f)) / (dot(m.diff, vec3(1.0f)) + dot(m.specF0, vec3(1.0f)));
    const vec3 halfway = normalize(lightDir + viewDir);
    const float nDotH = dot(halfway, normal);
    const float lDotH = dot(halfway, lightDir);
    if (static_cast<double>(dot(m.specF0, m.specF0)) > 1e-6) {
        const float d = D_GGX(nDotH, m.roughness);
        const float v = V_SmithJointGGX(nDotL, nDotV, m.roughness);
        const vec3 f = FresnelSchlick(m.specF0, lDotH);
        specBrdf = d * v * f;
    }
    result.brdfResult = (diffBrdf + specBrdf) * nDotL;
    result.samplingPdf = diffProb * nDotL / PI +
                         (1.0f - diffProb) * D_GGX(nDotH, m.roughness) * nDotH / (4.0f * lDotH);
    result.emission = m.emission;
    result.roughness = m.roughness;
    return result;
}

// ComputeLocalFrame, brdf.cu:192-212 (columns X, Y, Z)
struct Frame3 {
    vec3 X, Y, Z;
    vec3 operator*(vec3 v) const {
        return vec3(X.x * v.x + Y.x * v.y + Z.x * v.z, X.y * v.x + Y.y * v.y + Z.y * v.z,
                    X.z * v.x + Y.z * v.y + Z.z * v.z);
    }
};
inline Frame3 ComputeLocalFrame(vec3 localZ) {
    const float x = localZ.x, y = localZ.y, z = localZ.z;
    const float sz = (z >= 0) ? 1.0f : -1.0f;
    const float a = 1 / (sz + z);
    const float ya = y * a;
    const float b = x * ya;
    const float c = x * sz;
    Frame3 f;
    f.X = vec3(c * x * a - 1, sz * b, c);
    f.Y = vec3(b, y * ya - sz, y);
    f.Z = localZ;
    return f;
}

// __direct_callable__ggx_sample, brdf.cu:214-337
inline BrdfSampleResult GgxSample(const MatVals& m, const Interaction& interaction, PCG32& rng) {
    const vec3 normal = interaction.normal;
    const vec3 viewDir = -interaction.inRayDir;
    BrdfSampleResult result;
    result.roughness = m.roughness;
    const float nDotV = dot(normal, viewDir);
    if (nDotV <= 0) {
        result.outDir = vec3(0.0f);
        result.brdfVal = vec3(0.0f);
        result.samplingPdf = 0.0f;
        return result;
    }
    const Frame3 localFrame = ComputeLocalFrame(normal);
    const float diffProb = dot(m.diff, vec3(1.0f)) / (dot(m.diff, vec3(1.0f)) + dot(m.specF0, vec3(1.0f)));
    if (rng.NextFloat() < diffProb) {
        const float phi = rng.NextFloat() * 2.0f * PI;
        const float r = std::sqrt(rng.NextFloat());
        float sphi, cphi;
        SinCos(phi, sphi, cphi);
        const float x = r * cphi;
        const float y = r * sphi;
        const float z = std::sqrt(gclamp(1.0f - P2(x) - P2(y), 0.0f, 1.0f));
        result.outDir = localFrame * vec3(x, y, z);
    } else {
        const float u = rng.NextFloat();
        const float microNormalZ = std::sqrt(gclamp((1 - u) / (1 + (P2(m.roughness) - 1) * u), 0, 1));
        const float microNormalR = std::sqrt(gclamp(1 - P2(microNormalZ), 0, 1));
        const float phi = rng.NextFloat() * 2.0f * PI;
        float sphi, cphi;
        SinCos(phi, sphi, cphi);
        const vec3 microNormal(microNormalR * cphi, microNormalR * sphi, microNormalZ);
        result.outDir = reflect(interaction.inRayDir, localFrame * microNormal);
        if (dot(result.outDir, normal) < 0.0f) {
            result.outDir = vec3(0.0f);
            result.brdfVal = vec3(0.0f);
            result.samplingPdf = 0.0f;
            return result;
        }
    }
    const vec3 diffBrdf = m.diff / PI;
    const vec3 lightDir = result.outDir;
    const float nDotL = dot(normal, lightDir);
    const vec3 halfway = normalize(lightDir + viewDir);
    const float nDotH = dot(halfway, normal);
    const float lDotH = dot(halfway, lightDir);
    vec3 specBrdf(0.0f);
    if (static_cast<double>(dot(m.specF0, m.specF0)) > 1e-6) {
        const float d = D_GGX(nDotH, m.roughness);
        const float v = V_SmithJointGGX(nDotL, nDotV, m.roughness);
        const vec3 f = FresnelSchlick(m.specF0, lDotH);
        specBrdf = d * v * f;
    }
    result.outDir = lightDir;
    result.samplingPdf = diffProb * nDotL / PI +
                         (1.0f - diffProb) * D_GGX(nDotH, m.roughness) * nDotH / (4.0f * lDotH);
    result.brdfVal = (diffBrdf + specBrdf) * nDotL;
    return result;
}

// ---------------------------------------------------------------------------
// Emitters, include/model/Emitter.h:13-55, include/graph/sample_emitter.h
// ---------------------------------------------------------------------------
struct EmitterData {
    vec3 color;
    std::vector<vec3> faces;  // 3 per face
};

struct EmitterSample {
    vec3 pos;
    vec3 color;
    float p;
};

// ---------------------------------------------------------------------------
// Camera, include/graph/Camera.h:14-22 and src/Camera.cpp:20-32
// ---------------------------------------------------------------------------
struct CameraData {
    vec3 pos, U, V, W;
};

// DEFINED: the rotation block of inverse(lookAt) is its transpose, so its
// columns are taken directly (s, u, -f) instead of glm's 4x4 cofactor inverse.
inline CameraData GetCameraData(const crisb_camera& c) {
    const vec3 pos(c.pos[0], c.pos[1], c.pos[2]);
    const vec3 viewDir(c.view_dir[0], c.view_dir[1], c.view_dir[2]);
    const vec3 up(c.up[0], c.up[1], c.up[2]);
    const vec3 center = pos + viewDir;
    const vec3 f = normalize(center - pos);       // glm::lookAtRH
    const vec3 s = normalize(cross(f, up));
    const vec3 u = cross(s, f);
    const float tanHalf = std::tan(0.5f * c.fov);
    CameraData d;
    d.pos = pos;
    d.U = normalize(s) * tanHalf * c.aspect;
    d.V = -normalize(u) * tanHalf;
    d.W = -normalize(-f);
    return d;
}

inline void SpawnCameraRay(const CameraData& cam, vec2 vp, vec3& origin, vec3& dir) {
    origin = cam.pos;
    dir = normalize(cam.U * vp.x + cam.V * vp.y + cam.W);
}

// SampleEmitter, sample_emitter.h:3-12 + EmitterData::SamplePoint, Emitter.h:21-54
inline EmitterSample SampleEmitterFrom(const std::vector<EmitterData>& emitters, PCG32& rng) {
    const size_t emitterCount = emitters.size();
    const size_t emitterIdx = rng.NextUint64() % emitterCount;
    const EmitterData& e = emitters[emitterIdx];
    const size_t faceCount = e.faces.size() / 3;
    const size_t faceIdx = rng.NextUint64() % faceCount;
    const vec3 v0 = e.faces[faceIdx * 3 + 0];
    const vec3 v1 = e.faces[faceIdx * 3 + 1];
    const vec3 v2 = e.faces[faceIdx * 3 + 2];
    float r0 = rng.NextFloat();
    float r1 = rng.NextFloat();
    float r2 = rng.NextFloat();
    const float rSum = r0 + r1 + r2;
    r0 /= rSum;
    r1 /= rSum;
    r2 /= rSum;
    const vec3 point = r0 * v0 + r1 * v1 + r2 * v2;
    return {point, e.color, 1.0f};
}

// SelectSpatialNeighbor, path_gen.h:50-57, with the window radius R as a
// parameter (the reference's WINDOW_RADIUS = 10, path_gen.h:12)
inline void SelectSpatialNeighborR(uint32_t px, uint32_t py, uint32_t R, PCG32& rng, uint32_t& nx, uint32_t& ny) {
    const uint32_t WS = 2 * R + 1;
    const uint32_t x = (px + R) - (rng.NextUint32() % WS);
    const uint32_t y = (py + R) - (rng.NextUint32() % WS);
    if (x == px && y == py) {
        nx = px + 1;
        ny = py + 1;
        return;
    }
    nx = x;
    ny = y;
}

// ---------------------------------------------------------------------------
// The renderer state and passes
// ---------------------------------------------------------------------------
struct Scene {
    std::vector<Triangle> tris;
    std::vector<crisb_material> mats;
    std::vector<EmitterData> emitters;
    Bvh bvh;
    float sceneSize = 0.0f;
};

uint32_t FrameRandom(uint64_t seed, uint64_t frameCounter) {
    PCG32 r(seed, frameCounter);
    return r.NextUint32();
}

}  // namespace

struct oracle_ctx {
    Scene scene;
    crisb_params params{};
    uint32_t width = 0, height = 0;
    uint64_t frameIdx = 0;
    uint64_t frameCounter = 0;
    uint32_t random = 0;
    int front = 0, back = 0;
    CameraData cam;
    CameraData prevCam;       // this frame's previous camera (REPROJECT)
    bool hasPrevCam = false;
    CameraData lastCam;       // the last RenderFrame's camera
    bool hasLastCam = false;
    std::vector<float> motion;  // 2 per pixel (VECTORS)

    std::vector<Reservoir<PrefixPath>> prefixRes[2];
    std::vector<PrefixPath> canonPrefix;
    std::vector<Reservoir<SuffixPath>> suffixRes[2];
    std::vector<SuffixPath> canonSuffix;
    std::vector<GBuffer> gbuf;
    // prefix entries: point + radius (the AABB of prefix_store_entries.cu)
    std::vector<vec3> entryPos;
    std::vector<float> entryRad;
    std::vector<uint8_t> entryValid;
    std::vector<Neighbor> neighbors;
    std::vector<uint32_t> neighCount;
    // uniform grid over valid entries (host acceleration for the kNN)
    float gridCell = 1.0f;
    vec3 gridOrigin, gridMax;
    std::vector<std::pair<uint64_t, uint32_t>> gridEntries;

    uint32_t K() const { return static_cast<uint32_t>(std::max(params.gather_m - 1, 0)); }

    // ---- tracing wrappers --------------------------------------------------
    // TraceWithDataPointer + __closesthit__mesh / __miss__main
    void TraceClosest(vec3 origin, vec3 dir, float tmin, float tmax, Interaction& it) const {
        const RayPre r = MakeRay(origin, dir);
        const HitResult h = scene.bvh.Closest(r, tmin, tmax);
        it.inRayDir = dir;
        if (!h.hit) {
            it.valid = false;
            return;
        }
        it.valid = true;
        it.prim = h.prim;
        it.bary.x = h.u;
        it.bary.y = h.v;
        const Triangle& t = scene.tris[h.prim];
        it.pos = InterpolateBary(it.bary, t.p[0], t.p[1], t.p[2]);
        it.normal = normalize(InterpolateBary(it.bary, t.n[0], t.n[1], t.n[2]));
    }
    // TraceOcclusion, include/graph/trace.h:64-88
    bool TraceOcclusion(vec3 origin, vec3 dir, float tmin, float tmax) const {
        return scene.bvh.Occluded(MakeRay(origin, dir), tmin, tmax);
    }
    // Interaction(PackedInteraction, transforms), Interaction.h:115-172:
    // interpolated position and (unnormalised) normal, identity transform
    Interaction Unpack(const PackedInteraction& p) const {
        Interaction it;
        it.valid = p.valid;
        it.inRayDir = p.inRayDir;
        it.prim = p.prim;
        it.bary = p.bary;
        if (!it.valid) return it;
        if (p.prim >= scene.tris.size()) {
            it.valid = false;
            return it;
        }
        const Triangle& t = scene.tris[p.prim];
        it.pos = InterpolateBary(it.bary, t.p[0], t.p[1], t.p[2]);
        it.normal = InterpolateBary(it.bary, t.n[0], t.n[1], t.n[2]);
        return it;
    }
    const crisb_material& MatOf(const Interaction& it) const { return scene.mats[scene.tris[it.prim].mat]; }
    BrdfEvalResult Eval(const Interaction& it, vec3 dir) const { return GgxEval(MatValsAt(it), it, dir); }
    BrdfSampleResult Sample(const Interaction& it, PCG32& rng) const { return GgxSample(MatValsAt(it), it, rng); }

    // ---- textures: tex2D of src/Texture.cpp:44-72 and GetFromTexIfPossible,
    // shader/brdf.cu:64-97 ----------------------------------------------------
    struct Texture {
        uint32_t width = 0, height = 0;
        std::vector<uint32_t> texels;  // RGBA8 words, first row first
    };
    std::vector<float> triUv;                   // 6 per triangle (corner uvs)
    std::vector<Texture> textures;
    std::vector<std::array<int32_t, 3>> matTex;  // diffuse, specular, roughness

    struct Rgba {
        float r, g, b, a;
    };
    static Rgba Texel(uint32_t w) {
        return Rgba{static_cast<float>(w & 0xffu) / 255.0f, static_cast<float>((w >> 8) & 0xffu) / 255.0f,
                    static_cast<float>((w >> 16) & 0xffu) / 255.0f, static_cast<float>(w >> 24) / 255.0f};
    }
    // DEFINED after the CUDA programming guide's linear filtering of
    // normalised, wrapped coordinates: x_B = frac(u) * width - 0.5, i =
    // floor(x_B), alpha = frac(x_B) with 8 fractional bits (rounded), texels
    // i and i + 1 wrapped; (1-a)(1-b) T00 + a(1-b) T10 + (1-a) b T01 + a b T11.
    Rgba TexSample(int t, float u, float v) const {
        const Texture& tx = textures[static_cast<size_t>(t)];
        const int W = static_cast<int>(tx.width), H = static_cast<int>(tx.height);
        if (!std::isfinite(u)) u = 0.0f;
        if (!std::isfinite(v)) v = 0.0f;
        const float x = (u - std::floor(u)) * static_cast<float>(W) - 0.5f;
        const float y = (v - std::floor(v)) * static_cast<float>(H) - 0.5f;
        const float xf = std::floor(x), yf = std::floor(y);
        const float a = std::floor((x - xf) * 256.0f + 0.5f) * (1.0f / 256.0f);
        const float b = std::floor((y - yf) * 256.0f + 0.5f) * (1.0f / 256.0f);
        const int i0 = ((static_cast<int>(xf) % W) + W) % W, j0 = ((static_cast<int>(yf) % H) + H) % H;
        const int i1 = (i0 + 1) % W, j1 = (j0 + 1) % H;
        const Rgba t00 = Texel(tx.texels[static_cast<size_t>(j0) * W + i0]);
        const Rgba t10 = Texel(tx.texels[static_cast<size_t>(j0) * W + i1]);
        const Rgba t01 = Texel(tx.texels[static_cast<size_t>(j1) * W + i0]);
        const Rgba t11 = Texel(tx.texels[static_cast<size_t>(j1) * W + i1]);
        const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
        auto mix = [&](float c00, float c10, float c01, float c11) {
            return ((w00 * c00 + w10 * c10) + w01 * c01) + w11 * c11;
        };
        return Rgba{mix(t00.r, t10.r, t01.r, t11.r), mix(t00.g, t10.g, t01.g, t11.g),
                    mix(t00.b, t10.b, t01.b, t11.b), mix(t00.a, t10.a, t01.a, t11.a)};
    }
    MatVals MatValsAt(const Interaction& it) const {
        const crisb_material& m = MatOf(it);
        vec3 diff(m.diffuse[0], m.diffuse[1], m.diffuse[2]);
        vec3 f0(m.specular[0], m.specular[1], m.specular[2]);
        float rough = m.roughness;
        if (!matTex.empty()) {
            const std::array<int32_t, 3>& t = matTex[scene.tris[it.prim].mat];
            if (t[0] >= 0 || t[1] >= 0 || t[2] >= 0) {
                // Interaction::uv = InterpolateBary of the corner uvs (Interaction.h:171)
                const float* c = &triUv[6 * static_cast<size_t>(it.prim)];
                const float w = 1.0f - it.bary.x - it.bary.y;
                const float u = (w * c[0] + it.bary.x * c[2]) + it.bary.y * c[4];
                const float v = (w * c[1] + it.bary.x * c[3]) + it.bary.y * c[5];
                if (t[0] >= 0) {
                    const Rgba s = TexSample(t[0], u, v);
                    diff = vec3(s.r, s.g, s.b);
                }
                if (t[1] >= 0) {
                    const Rgba s = TexSample(t[1], u, v);
                    f0 = vec3(s.r, s.g, s.b);
                }
                if (t[2] >= 0) rough = TexSample(t[2], u, v).r;
            }
        }
        return FinishMat(m, diff, f0, rough);
    }

    EmitterSample SampleEmitter(PCG32& rng) const { return SampleEmitterFrom(scene.emitters, rng); }

    bool IsPixelValid(uint32_t x, uint32_t y) const { return x < width && y < height; }

    // ---- prevPixelCoord, prefix_gen_temp_reuse.cu:130-136 -----------------
    // DEFINED (CRISB_MOTION_*): NONE keeps pixelCoord; VECTORS is the
    // commented-out uvec2(vec2(pixelCoord) + vec2(0.5) + motionVector) with
    // the GPU's saturating float -> uint conversion; REPROJECT takes the
    // pixel of the previous frame's camera whose footprint [x, x + 1) holds
    // the primary hit.  No previous pixel is stored as (0xffff, 0xffff).
    static constexpr uint32_t kNoPrev = 0xffffu;
    static uint32_t ToUintSat(float v) {
        if (!(v > 0.0f)) return 0u;
        if (v >= 4294967296.0f) return 0xffffffffu;
        return static_cast<uint32_t>(v);
    }
    void SetPrev(uint32_t px, uint32_t py, uint32_t& prevX, uint32_t& prevY) const {
        const bool ok = IsPixelValid(px, py);
        prevX = ok ? px : kNoPrev;
        prevY = ok ? py : kNoPrev;
    }
    void PrevFromMotion(uint32_t x, uint32_t y, uint32_t& prevX, uint32_t& prevY) const {
        const size_t i = static_cast<size_t>(y) * width + x;
        const float fx = (static_cast<float>(x) + 0.5f) + motion[2 * i];
        const float fy = (static_cast<float>(y) + 0.5f) + motion[2 * i + 1];
        SetPrev(ToUintSat(fx), ToUintSat(fy), prevX, prevY);
    }
    void PrevFromReprojection(vec3 p, uint32_t& prevX, uint32_t& prevY) const {
        prevX = prevY = kNoPrev;
        const vec3 d = p - prevCam.pos;
        const float t = dot(d, prevCam.W) / dot(prevCam.W, prevCam.W);
        if (!(t > 0.0f)) return;
        const float ux = dot(d, prevCam.U) / (t * dot(prevCam.U, prevCam.U));
        const float uy = dot(d, prevCam.V) / (t * dot(prevCam.V, prevCam.V));
        const float xc = (ux + 1.0f) * 0.5f * static_cast<float>(width);
        const float yc = (uy + 1.0f) * 0.5f * static_cast<float>(height);
        if (!(xc >= 0.0f && xc < static_cast<float>(width) && yc >= 0.0f && yc < static_cast<float>(height))) return;
        SetPrev(static_cast<uint32_t>(xc), static_cast<uint32_t>(yc), prevX, prevY);
    }

    // ---- path generation, include/graph/restir/path_gen.h -----------------
    // ComputeCanonicalPairwiseMISWeight, path_gen.h:15-31
    static float CanonMis(vec3 bAtB, vec3 bAtN, float jac, float K, float cM, float nM) {
        float w = 1.f;
        if (GetLuminance(bAtB) > 0.f) {
            const float atBasisTerm = GetLuminance(bAtB) * cM;
            w = atBasisTerm / (atBasisTerm + GetLuminance(bAtN) * jac * nM * K);
        }
        return w;
    }
    // ComputeNeighborPairwiseMISWeight, path_gen.h:33-48
    static float NeighMis(vec3 nAtB, vec3 nAtN, float jac, float K, float cM, float nM) {
        float w = 0.f;
        if (GetLuminance(nAtN) > 0.f) {
            w = GetLuminance(nAtN) * nM / (GetLuminance(nAtN) * nM + GetLuminance(nAtB) * jac * cM / K);
        }
        return w;
    }
    void SelectSpatialNeighbor(uint32_t px, uint32_t py, PCG32& rng, uint32_t& nx, uint32_t& ny) const {
        SelectSpatialNeighborR(px, py, static_cast<uint32_t>(params.window_radius), rng, nx, ny);
    }
    // CalcReconnectionJacobian, path_gen.h:59-72
    static float ReconJacobian(vec3 oldXi, vec3 newXi, vec3 targetPos, vec3 targetNormal) {
        const float term1 = std::fabs(dot(normalize(newXi - targetPos), targetNormal) /
                                      dot(normalize(oldXi - targetPos), targetNormal));
        const float term2 = dot(targetPos - oldXi, targetPos - oldXi);
        const float term3 = dot(targetPos - newXi, targetPos - newXi);
        const float result = term1 * term2 / term3;
        if (std::isinf(result) || std::isnan(result)) return 0.0f;
        return gmax(0.0f, result);
    }

    // TracePrefix, path_gen.h:74-250 (prefix is modified in place)
    void TracePrefix(PrefixPath& prefix, vec3 origin, vec3 dir, PCG32& rng) const {
        vec3 currentPos = origin;
        vec3 currentDir = dir;
        prefix.Reset();
        prefix.rng = rng;
        prefix.p = 1.0f;
        prefix.f = vec3(1.0f);
        prefix.postReconF = vec3(1.0f);
        prefix.SetValid(true);
        Interaction interaction;
        const int type = params.renderer_type;
        const uint32_t maxLen = type == CRISB_RENDERER_RESTIR_PT ? static_cast<uint32_t>(params.max_path_len)
                                                                 : static_cast<uint32_t>(params.prefix_len);
        bool postRecon = false;
        for (uint32_t traceIdx = 0; traceIdx < maxLen; ++traceIdx) {
            TraceClosest(currentPos, currentDir, 1e-3f, 1e16f, interaction);
            if (!interaction.valid) {
                prefix.SetValid(false);
                return;
            }
            prefix.pathLen += distance(currentPos, interaction.pos);
            prefix.SetLength(prefix.GetLength() + 1);
            if (prefix.GetLength() == 1) prefix.primaryInt = interaction.Pack();
            if (type == CRISB_RENDERER_CONDITIONAL_RESTIR && traceIdx == maxLen - 1) {
                if (!postRecon) {
                    prefix.reconInt = interaction.Pack();
                    prefix.SetReconIdx(prefix.GetLength());
                    prefix.reconOutDir = vec3(0.0f);
                }
                prefix.SetValid(true);
                prefix.lastInt = interaction.Pack();
                return;
            }
            const bool forceNee = type == CRISB_RENDERER_RESTIR_PT && traceIdx == maxLen - 1;
            if (rng.NextFloat() < params.nee_prob || forceNee) {
                prefix.p *= params.nee_prob;
                const EmitterSample emitterSample = SampleEmitter(rng);
                const vec3 lightDir = normalize(emitterSample.pos - interaction.pos);
                const float dist = length(emitterSample.pos - interaction.pos);
                if (TraceOcclusion(interaction.pos, lightDir, 1e-3f, dist)) {
                    prefix.SetValid(false);
                    return;
                }
                if (!postRecon) {
                    // re-trace of the same ray (path_gen.h:167-174) yields `interaction`
                    prefix.reconInt = interaction.Pack();
                    prefix.SetReconIdx(prefix.GetLength());
                    prefix.reconOutDir = currentDir;
                    postRecon = true;
                }
                const BrdfEvalResult brdfEvalResult = Eval(interaction, lightDir);
                if (brdfEvalResult.samplingPdf <= 0.0f) {
                    prefix.SetValid(false);
                    return;
                }
                const float distFactor = 1.0f / (dist * dist);
                prefix.f *= brdfEvalResult.brdfResult * emitterSample.color * distFactor;
                if (postRecon) prefix.postReconF *= brdfEvalResult.brdfResult * emitterSample.color * distFactor;
                if (prefix.GetLength() == 1) prefix.f += brdfEvalResult.emission * distFactor;
                prefix.SetNee(true);
                prefix.SetValid(true);
                prefix.lastInt = interaction.Pack();
                return;
            }
            const BrdfSampleResult brdfSampleResult = Sample(interaction, rng);
            if (brdfSampleResult.samplingPdf <= 0.0f) {
                prefix.SetValid(false);
                return;
            }
            const float reconDistance = distance(currentPos, interaction.pos);
            const float reconRoughness = brdfSampleResult.roughness;
            const bool intCanRecon = reconDistance > params.recon_min_distance &&
                                     reconRoughness > params.recon_min_roughness && prefix.GetLength() >= 2;
            if (!postRecon && intCanRecon) {
                prefix.reconInt = interaction.Pack();
                prefix.SetReconIdx(prefix.GetLength());
                prefix.reconOutDir = brdfSampleResult.outDir;
                postRecon = true;
            }
            currentPos = interaction.pos;
            currentDir = brdfSampleResult.outDir;
            prefix.f *= brdfSampleResult.brdfVal;
            prefix.p *= brdfSampleResult.samplingPdf * (1.0f - params.nee_prob);
            if (postRecon) prefix.postReconF *= brdfSampleResult.brdfVal;
        }
        prefix.lastInt = interaction.Pack();
    }

    // TraceSuffix, path_gen.h:252-387 (suffix is modified in place)
    void TraceSuffix(SuffixPath& suffix, const PrefixPath& prefix, PCG32& rng) const {
        suffix.f = vec3(1.0f);
        suffix.p = 1.0f;
        suffix.postReconF = vec3(1.0f);
        suffix.rng = rng;
        suffix.lastPrefixInt = prefix.lastInt;
        suffix.Reset();
        if (!prefix.IsValid() || prefix.IsNee()) return;
        const uint32_t maxLen = static_cast<uint32_t>(params.max_path_len) - prefix.GetLength();
        Interaction interaction = Unpack(prefix.lastInt);
        if (!interaction.valid) return;
        bool postRecon = false;
        vec3 lastDir(0.0f);
        for (uint32_t vertIdx = 0; vertIdx < maxLen; ++vertIdx) {
            const vec3 lastPos = interaction.pos;
            if (suffix.GetLength() > 0) {
                TraceClosest(lastPos, lastDir, 1e-3f, 1e16f, interaction);
                if (!interaction.valid) return;
            }
            const bool forceNee = vertIdx == maxLen - 1;
            if (rng.NextFloat() < params.nee_prob || forceNee) {
                if (!forceNee) suffix.p *= params.nee_prob;
                const EmitterSample emitter = SampleEmitter(rng);
                const vec3 lightVec = emitter.pos - interaction.pos;
                const float lightLen = length(lightVec);
                const vec3 lightDir = normalize(lightVec);
                if (anyNanInf(lightDir)) return;
                if (TraceOcclusion(interaction.pos, lightDir, 1e-3f, lightLen)) return;
                const BrdfEvalResult brdfEvalResult = Eval(interaction, lightDir);
                if (brdfEvalResult.samplingPdf <= 0.0f) return;
                suffix.SetLength(suffix.GetLength() + 1);
                if (!postRecon) {
                    Interaction reconInt;
                    TraceClosest(interaction.pos, lightDir, 1e-3f, 1e16f, reconInt);
                    if (!reconInt.valid) return;
                    suffix.reconInt = reconInt.Pack();
                    suffix.SetReconIdx(suffix.GetLength());
                    suffix.SetReconVert(vertIdx);
                    suffix.reconOutDir = vec3(0.0f);
                    postRecon = true;
                }
                const float distFactor = 1.0f / (lightLen * lightLen);
                suffix.f *= brdfEvalResult.brdfResult * emitter.color * distFactor;
                suffix.postReconF *= emitter.color * distFactor;
                if (suffix.GetReconIdx() < suffix.GetLength()) suffix.postReconF *= brdfEvalResult.brdfResult;
                suffix.SetValid(true);
                return;
            }
            const BrdfSampleResult brdfSampleResult = Sample(interaction, rng);
            if (brdfSampleResult.samplingPdf <= 0.0f) return;
            suffix.p *= brdfSampleResult.samplingPdf * (1.0f - params.nee_prob);
            suffix.f *= brdfSampleResult.brdfVal;
            if (postRecon) suffix.postReconF *= brdfSampleResult.brdfVal;
            const float reconDistance = distance(lastPos, interaction.pos);
            const float reconRoughness = brdfSampleResult.roughness;
            const bool intCanRecon = reconDistance > params.recon_min_distance &&
                                     reconRoughness > params.recon_min_roughness && prefix.GetLength() >= 1;
            if (!postRecon && intCanRecon) {
                suffix.reconInt = interaction.Pack();
                suffix.SetReconIdx(prefix.GetLength());
                suffix.SetReconVert(vertIdx);
                suffix.reconOutDir = brdfSampleResult.outDir;
                postRecon = true;
            }
            lastDir = brdfSampleResult.outDir;
            suffix.SetLength(suffix.GetLength() + 1);
        }
    }

    // TraceCompletePath, path_gen.h:389-472
    vec3 TraceCompletePath(vec3 origin, vec3 dir, PCG32& rng) const {
        vec3 currentPos = origin;
        vec3 currentDir = dir;
        size_t currentDepth = 0;
        vec3 radiance(0.0f);
        vec3 throughput(1.0f);
        for (uint32_t traceIdx = 0; traceIdx < static_cast<uint32_t>(params.max_path_len); ++traceIdx) {
            Interaction interaction;
            TraceClosest(currentPos, currentDir, 1e-3f, 1e16f, interaction);
            if (!interaction.valid) break;
            ++currentDepth;
            if (rng.NextFloat() < params.nee_prob) {
                throughput /= params.nee_prob;
                const EmitterSample emitterSample = SampleEmitter(rng);
                const vec3 lightDir = normalize(emitterSample.pos - interaction.pos);
                const float dist = length(emitterSample.pos - interaction.pos);
                if (TraceOcclusion(interaction.pos, lightDir, 1e-3f, dist)) return vec3(0.0f);
                const BrdfEvalResult brdfEvalResult = Eval(interaction, lightDir);
                const float distFactor = 1.0f / (dist * dist);
                radiance = throughput * brdfEvalResult.brdfResult * emitterSample.color * distFactor;
                if (currentDepth == 1) radiance += brdfEvalResult.emission;
                break;
            }
            const BrdfSampleResult brdfSampleResult = Sample(interaction, rng);
            if (brdfSampleResult.samplingPdf <= 0.0f) break;
            currentPos = interaction.pos;
            currentDir = brdfSampleResult.outDir;
            throughput *= brdfSampleResult.brdfVal / brdfSampleResult.samplingPdf;
            throughput /= (1.0f - params.nee_prob);
        }
        return radiance;
    }

    // TracePrefixForFinalGather, path_gen.h:474-531
    bool TracePrefixForFinalGather(vec3& throughput, float& p, Interaction& lastInt, vec3 origin, vec3 dir,
                                   size_t maxLen, PCG32& rng) const {
        vec3 currentPos = origin;
        vec3 currentDir = dir;
        throughput = vec3(1.0f);
        p = 1.0f;
        lastInt.valid = false;
        for (uint32_t traceIdx = 0; traceIdx < maxLen; ++traceIdx) {
            TraceClosest(currentPos, currentDir, 1e-3f, 1e16f, lastInt);
            if (!lastInt.valid) return false;
            const BrdfSampleResult brdfSampleResult = Sample(lastInt, rng);
            if (brdfSampleResult.samplingPdf <= 0.0f) return false;
            currentPos = lastInt.pos;
            currentDir = brdfSampleResult.outDir;
            throughput *= brdfSampleResult.brdfVal;
            p *= brdfSampleResult.samplingPdf;
        }
        return true;
    }

    // ---- shift mappings ------------------------------------------------------
    // prefix CalcCurrContribInOtherDomain, include/graph/restir/prefix_reuse.h:10-99
    vec3 ShiftPrefix(const PrefixPath& srcPrefix, const PrefixPath& dstPrefix, float& jacobian) const {
        jacobian = 0.0f;
        if (!srcPrefix.IsValid() || !srcPrefix.IsValid() || srcPrefix.GetReconIdx() < 2) return vec3(0.0f);
        const Interaction srcPrimaryInt = Unpack(srcPrefix.primaryInt);
        if (!srcPrimaryInt.valid) return vec3(0.0f);
        Interaction dstPrimaryInt = Unpack(dstPrefix.primaryInt);
        if (!dstPrimaryInt.valid) return vec3(0.0f);
        Interaction srcReconInt = Unpack(srcPrefix.reconInt);
        if (!srcReconInt.valid) return vec3(0.0f);
        const uint32_t reconVertCount =
            static_cast<uint32_t>(std::max<int>(static_cast<int>(srcPrefix.GetReconIdx() - 2), 0));
        Interaction& currInt = dstPrimaryInt;
        PCG32 srcRng = srcPrefix.rng;
        vec3 throughput(1.0f);
        for (uint32_t idx = 0; idx < reconVertCount; ++idx) {
            srcRng.NextFloat();
            const BrdfSampleResult brdf = Sample(currInt, srcRng);
            if (brdf.samplingPdf <= 0.0f) return vec3(0.0f);
            throughput *= brdf.brdfVal;
            const vec3 pos = currInt.pos;
            TraceClosest(pos, brdf.outDir, 1e-3f, 1e16f, currInt);
            if (!currInt.valid) return vec3(0.0f);
        }
        const vec3 reconVec = srcReconInt.pos - currInt.pos;
        const float reconLen = length(reconVec);
        const vec3 reconDir = normalize(reconVec);
        if (std::isinf(reconLen) || anyNanInf(reconDir)) return vec3(0.0f);
        if (TraceOcclusion(currInt.pos, reconDir, 1e-3f, reconLen)) return vec3(0.0f);
        const BrdfEvalResult brdf1 = Eval(currInt, reconDir);
        if (brdf1.samplingPdf <= 0.0f) return vec3(0.0f);
        throughput *= brdf1.brdfResult;
        srcReconInt.inRayDir = reconDir;
        const BrdfEvalResult brdf2 = Eval(srcReconInt, srcPrefix.reconOutDir);
        if (brdf2.samplingPdf <= 0.0f) return vec3(0.0f);
        throughput *= brdf2.brdfResult;
        jacobian = ReconJacobian(srcPrimaryInt.pos, currInt.pos, srcReconInt.pos, srcReconInt.normal);
        return gmax(vec3(0.0f), throughput * srcPrefix.postReconF);
    }

    // suffix CalcCurrContribInOtherDomain, include/graph/restir/suffix_reuse.h:10-108
    vec3 ShiftSuffix(const SuffixPath& srcSuffix, const Interaction& dstLastPrefixInt, float& jacobian) const {
        jacobian = 0.0f;
        if (!srcSuffix.IsValid()) return vec3(0.0f);
        if (!dstLastPrefixInt.valid) return vec3(0.0f);
        const Interaction srcLastPrefixInt = Unpack(srcSuffix.lastPrefixInt);
        if (!srcLastPrefixInt.valid) return vec3(0.0f);
        Interaction srcReconInt = Unpack(srcSuffix.reconInt);
        if (!srcReconInt.valid) return vec3(0.0f);
        const uint32_t reconVertCount =
            static_cast<uint32_t>(std::max<int>(static_cast<int>(srcSuffix.GetReconIdx() - 1), 0));
        Interaction currInt = dstLastPrefixInt;
        PCG32 srcRng = srcSuffix.rng;
        vec3 throughput(1.0f);
        for (uint32_t idx = 0; idx < reconVertCount; ++idx) {
            srcRng.NextFloat();
            const BrdfSampleResult brdf = Sample(currInt, srcRng);
            if (brdf.samplingPdf <= 0.0f) return vec3(0.0f);
            throughput *= brdf.brdfVal;
            const vec3 oldPos = currInt.pos;
            TraceClosest(oldPos, brdf.outDir, 1e-3f, 1e16f, currInt);
            if (!currInt.valid) return vec3(0.0f);
        }
        const vec3 reconVec = srcReconInt.pos - currInt.pos;
        const float reconLen = length(reconVec);
        const vec3 reconDir = normalize(reconVec);
        if (anyNanInf(reconDir)) return vec3(0.0f);
        if (TraceOcclusion(currInt.pos, reconDir, 1e-3f, reconLen)) return vec3(0.0f);
        const BrdfEvalResult brdf1 = Eval(currInt, reconDir);
        if (brdf1.samplingPdf <= 0.0f) return vec3(0.0f);
        throughput *= brdf1.brdfResult;
        if (srcSuffix.GetReconIdx() < srcSuffix.GetLength()) {
            srcReconInt.inRayDir = reconDir;
            if (srcSuffix.reconOutDir == vec3(0.0f)) return vec3(0.0f);
            const BrdfEvalResult brdf2 = Eval(srcReconInt, srcSuffix.reconOutDir);
            if (brdf2.samplingPdf <= 0.0f) return vec3(0.0f);
            throughput *= brdf2.brdfResult;
        }
        jacobian = ReconJacobian(srcLastPrefixInt.pos, currInt.pos, srcReconInt.pos, srcReconInt.normal);
        return throughput * srcSuffix.postReconF;
    }

    // suffix_reuse.h:111-123
    vec3 ShiftSuffix(const SuffixPath& srcSuffix, const SuffixPath& dstSuffix, float& jacobian) const {
        const Interaction dstLastPrefixInt = Unpack(dstSuffix.lastPrefixInt);
        if (!dstLastPrefixInt.valid) return vec3(0.0f);
        return ShiftSuffix(srcSuffix, dstLastPrefixInt, jacobian);
    }

    // Test infrastructure (not in the reference): the postReconF of a valid
    // suffix sample re-traced from its seed past its reconnection vertex, as
    // the resampled-path adjoint re-traces it -- the random state advanced
    // four draws per suffix vertex up to and including the one whose loop
    // index the flags carry (GetReconVert), then TraceSuffix's loop from the
    // next vertex along reconOutDir.  `checkable` is false for samples that
    // reconnected at their NEE vertex (postReconF = colour * 1/d^2 of a light
    // sample whose vertex is not stored).
    vec3 ReplayPostRecon(const SuffixPath& s, bool& checkable) const {
        const uint32_t len = s.GetLength(), r = s.GetReconVert();
        checkable = r + 1 < len;
        if (!checkable) return vec3(0.0f);
        const uint32_t maxLen = static_cast<uint32_t>(params.max_path_len - params.prefix_len);
        PCG32 rng = s.rng;
        for (uint32_t k = 0; k < 4 * (r + 1); ++k) rng.NextFloat();
        vec3 pos = Unpack(s.reconInt).pos, dir = s.reconOutDir;
        vec3 prf(1.0f);
        for (uint32_t vertIdx = r + 1; vertIdx < maxLen; ++vertIdx) {
            Interaction it;
            TraceClosest(pos, dir, 1e-3f, 1e16f, it);
            if (!it.valid) return vec3(NAN);
            const bool forceNee = vertIdx == maxLen - 1;
            if (rng.NextFloat() < params.nee_prob || forceNee) {
                const EmitterSample emitter = SampleEmitter(rng);
                const vec3 lightVec = emitter.pos - it.pos;
                const float lightLen = length(lightVec);
                const BrdfEvalResult e = Eval(it, normalize(lightVec));
                const float distFactor = 1.0f / (lightLen * lightLen);
                prf *= emitter.color * distFactor;
                if (s.GetReconIdx() < len) prf *= e.brdfResult;
                return prf;
            }
            const BrdfSampleResult b = Sample(it, rng);
            prf *= b.brdfVal;
            pos = it.pos;
            dir = b.outDir;
        }
        return vec3(NAN);
    }

    // ---- passes ----------------------------------------------------------------
    vec3 PixelJitterDir(uint32_t x, uint32_t y, PCG32& rng) const {
        // Next2d: x drawn first (DEFINED: left-to-right argument evaluation)
        const float jx = rng.NextFloat();
        const float jy = rng.NextFloat();
        vec2 uv;
        uv.x = (static_cast<float>(x) + jx) / static_cast<float>(width);
        uv.y = (static_cast<float>(y) + jy) / static_cast<float>(height);
        uv.x = 2.0f * uv.x - 1.0f;
        uv.y = 2.0f * uv.y - 1.0f;
        vec3 o, d;
        SpawnCameraRay(cam, uv, o, d);
        return d;
    }

    void StoreOutput(float* out, size_t pixelIdx, vec3 radiance) const {
        vec3 v = radiance;
        if (params.enable_accum) {
            const vec3 oldVal(out[3 * pixelIdx], out[3 * pixelIdx + 1], out[3 * pixelIdx + 2]);
            const float blendFactor = 1.0f / static_cast<float>(frameIdx + 1);
            v = blendFactor * radiance + (1.0f - blendFactor) * oldVal;
        }
        out[3 * pixelIdx] = v.x;
        out[3 * pixelIdx + 1] = v.y;
        out[3 * pixelIdx + 2] = v.z;
    }

    // PrefixGenTempReuse, shader/prefix_gen_temp_reuse.cu:11-98
    bool PrefixGenTempReuse(size_t pixelIdx, uint32_t& prevX, uint32_t& prevY, vec3 origin, vec3 dir, PCG32& rng) {
        TracePrefix(canonPrefix[pixelIdx], origin, dir, rng);
        const PrefixPath& canon = canonPrefix[pixelIdx];
        if (params.motion_mode == CRISB_MOTION_REPROJECT) {
            prevX = prevY = kNoPrev;
            if (canon.IsValid() && hasPrevCam) {
                const Interaction it = Unpack(canon.primaryInt);
                if (it.valid) PrevFromReprojection(it.pos, prevX, prevY);
            }
        }
        if (!canon.IsValid()) return false;
        const float canonPHat = GetLuminance(canon.f);
        Reservoir<PrefixPath>& currRes = prefixRes[front][pixelIdx];
        currRes.Reset();
        if (!params.prefix_enable_temporal || !IsPixelValid(prevX, prevY)) {
            currRes.Update(canon, canonPHat / canon.p, rng, 1.0f);
            currRes.FinalizeGRIS();
            return true;
        }
        // the reference reads back[pixelIdx] (prefix_gen_temp_reuse.cu:42), the
        // same pixel as prevPixelIdx under CRISB_MOTION_NONE
        const size_t prevPixelIdx = static_cast<size_t>(prevY) * width + prevX;
        const Reservoir<PrefixPath>& prevRes = prefixRes[back][prevPixelIdx];
        const PrefixPath& prevPrefix = prevRes.sample;
        const bool skipBecauseOfNee = params.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR && prevPrefix.IsNee();
        if (prevRes.wSum <= 0.0f || !prevPrefix.IsValid() || skipBecauseOfNee) {
            currRes.Update(canon, canonPHat / canon.p, rng, 1.0f);
            currRes.FinalizeGRIS();
            return true;
        }
        float jacobianCanonToPrev = 0.0f, jacobianPrevToCanon = 0.0f;
        const vec3 fFromCanonOfPrev = ShiftPrefix(prevPrefix, canon, jacobianPrevToCanon);
        const vec3 fFromPrevOfCanon = ShiftPrefix(canon, prevPrefix, jacobianCanonToPrev);
        const float pFromCanonOfPrev = GetLuminance(fFromCanonOfPrev) * jacobianPrevToCanon;
        constexpr float pairwiseK = 1.0f;
        const float prevMisWeight =
            NeighMis(fFromCanonOfPrev, prevPrefix.f, jacobianPrevToCanon, pairwiseK, 1.0f, prevRes.confidence);
        const float canonMisWeight =
            1.0f + CanonMis(canon.f, fFromPrevOfCanon, jacobianCanonToPrev, pairwiseK, 1.0f, prevRes.confidence);
        const float canonRisWeight = canonMisWeight * canonPHat / canon.p;
        currRes.Update(canon, canonRisWeight, rng, 1.0f);
        const float prevRisWeight = prevMisWeight * pFromCanonOfPrev * prevRes.wSum;
        const PrefixPath shiftedPrevPrefix(prevPrefix, fFromCanonOfPrev, canon.primaryInt);
        currRes.Update(shiftedPrevPrefix, prevRisWeight, rng, prevRes.confidence);
        if (currRes.wSum > 0.0f) {
            currRes.wSum /= pairwiseK + 1.0f;
            currRes.FinalizeGRIS();
        }
        return true;
    }

    // __raygen__prefix_gen_temp_reuse, shader/prefix_gen_temp_reuse.cu:100-193
    void PassPrefixGenTempReuse(float* out) {
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) {
            const uint32_t x = static_cast<uint32_t>(pi % width), y = static_cast<uint32_t>(pi / width);
            const size_t pixelIdx = static_cast<size_t>(pi);
            PCG32 rng(SampleTEA64(static_cast<uint32_t>(pixelIdx), random));
            vec3 outputRadiance(0.0f);
            const vec3 dir = PixelJitterDir(x, y, rng);
            const vec3 origin = cam.pos;
            const int type = params.renderer_type;
            if (type == CRISB_RENDERER_CONDITIONAL_RESTIR || type == CRISB_RENDERER_RESTIR_PT) {
                uint32_t prevX = x, prevY = y;
                if (params.motion_mode == CRISB_MOTION_VECTORS) PrevFromMotion(x, y, prevX, prevY);
                const bool validPrimaryInt = PrefixGenTempReuse(pixelIdx, prevX, prevY, origin, dir, rng);
                if (type == CRISB_RENDERER_RESTIR_PT && !params.prefix_enable_spatial) {
                    if (validPrimaryInt) {
                        const Reservoir<PrefixPath>& r = prefixRes[front][pixelIdx];
                        outputRadiance = r.wSum * r.sample.f;
                    }
                    StoreOutput(out, pixelIdx, outputRadiance);
                }
                GBuffer& g = gbuf[pixelIdx];
                g.rng = rng;
                g.prevX = prevX;
                g.prevY = prevY;
                g.primaryIntValid = validPrimaryInt;
            } else {
                outputRadiance = TraceCompletePath(origin, dir, rng);
                if (anyNanInf(outputRadiance)) outputRadiance = vec3(0.0f);
                StoreOutput(out, pixelIdx, outputRadiance);
            }
        }
        // Copy front to back reservoir for spatial reuse
        // (prefix_gen_temp_reuse.cu:159-164), after every pixel's temporal
        // reuse: other pixels read back[prevPixelIdx] during the pass
        const int type = params.renderer_type;
        if ((type == CRISB_RENDERER_RESTIR_PT && params.prefix_enable_spatial) ||
            (type == CRISB_RENDERER_CONDITIONAL_RESTIR && params.suffix_enable_spatial)) {
#pragma omp parallel for schedule(static)
            for (int64_t pi = 0; pi < P; ++pi) prefixRes[back][pi] = prefixRes[front][pi];
        }
    }

    // PrefixSpatialReuse, shader/prefix_spatial_reuse.cu:11-134 (neighbours read
    // from the pass-start snapshot `snap`)
    bool PrefixSpatialReuse(uint32_t x, uint32_t y, const std::vector<Reservoir<PrefixPath>>& snap) {
        const size_t currPixelIdx = static_cast<size_t>(y) * width + x;
        Reservoir<PrefixPath>& currRes = prefixRes[front][currPixelIdx];
        const PrefixPath currPrefix = currRes.sample;
        if (!currPrefix.IsValid()) return false;
        const PrefixPath& canon = canonPrefix[currPixelIdx];
        if (!canon.IsValid() || !canon.primaryInt.valid) return false;
        PCG32& rng = gbuf[currPixelIdx].rng;
        const float currResWSum = currRes.wSum;
        const float currResConfidence = currRes.confidence;
        currRes.Reset();
        const int neighCount = params.prefix_spatial_count;
        float canonMisWeight = 1.0f;
        uint32_t validNeighCount = 0, validNeighFlags = 0;
        uint32_t nxs[CRISB_MAX_SPATIAL_NEIGH], nys[CRISB_MAX_SPATIAL_NEIGH];
        for (int n = 0; n < neighCount; ++n) {
            SelectSpatialNeighbor(x, y, rng, nxs[n], nys[n]);
            if (!IsPixelValid(nxs[n], nys[n])) continue;
            const size_t ni = static_cast<size_t>(nys[n]) * width + nxs[n];
            if (!gbuf[ni].primaryIntValid) continue;
            const PrefixPath& np = snap[ni].sample;
            const bool skipBecauseOfNee = params.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR && np.IsNee();
            if (!np.IsValid() || skipBecauseOfNee) continue;
            ++validNeighCount;
            validNeighFlags |= 1u << n;
        }
        const float pairwiseK = static_cast<float>(validNeighCount);
        for (int n = 0; n < neighCount; ++n) {
            if (!((validNeighFlags >> n) & 1u)) continue;
            const size_t ni = static_cast<size_t>(nys[n]) * width + nxs[n];
            const Reservoir<PrefixPath>& neighRes = snap[ni];
            const PrefixPath& neighPrefix = neighRes.sample;
            float jacobianNeighToCanon = 0.0f;
            const vec3 fFromCanonOfNeigh = ShiftPrefix(neighPrefix, currPrefix, jacobianNeighToCanon);
            const float pFromCanonOfNeigh = GetLuminance(fFromCanonOfNeigh) * jacobianNeighToCanon;
            float jacobianCanonToNeigh = 0.0f;
            const vec3 fFromNeighOfCanon = ShiftPrefix(currPrefix, neighPrefix, jacobianCanonToNeigh);
            float neighMisWeight = NeighMis(fFromCanonOfNeigh, neighPrefix.f, jacobianNeighToCanon, pairwiseK,
                                            currResConfidence, neighRes.confidence);
            if (std::isnan(neighMisWeight) || std::isinf(neighMisWeight)) neighMisWeight = 0.0f;
            const float neighRisWeight = neighMisWeight * pFromCanonOfNeigh * neighRes.wSum;
            currRes.Update(PrefixPath(neighPrefix, fFromCanonOfNeigh, currPrefix.primaryInt), neighRisWeight, rng,
                           neighRes.confidence);
            canonMisWeight += CanonMis(currPrefix.f, fFromNeighOfCanon, jacobianCanonToNeigh, pairwiseK,
                                       currResConfidence, neighRes.confidence);
        }
        if (std::isinf(canonMisWeight) || std::isnan(canonMisWeight)) canonMisWeight = 0.0f;
        const float canonRisWeight = canonMisWeight * currResWSum * GetLuminance(currPrefix.f);
        currRes.Update(currPrefix, canonRisWeight, rng, currResConfidence);
        if (currRes.wSum > 0.0f) {
            currRes.wSum /= pairwiseK + 1.0f;
            currRes.FinalizeGRIS();
        }
        return true;
    }

    // __raygen__prefix_spatial_reuse, shader/prefix_spatial_reuse.cu:136-177
    void PassPrefixSpatialReuse(float* out, int roundIdx) {
        const std::vector<Reservoir<PrefixPath>> snap = prefixRes[back];
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) {
            const uint32_t x = static_cast<uint32_t>(pi % width), y = static_cast<uint32_t>(pi / width);
            vec3 outputRadiance(0.0f);
            if (PrefixSpatialReuse(x, y, snap) && params.renderer_type == CRISB_RENDERER_RESTIR_PT) {
                const Reservoir<PrefixPath>& r = prefixRes[front][pi];
                outputRadiance = r.wSum * r.sample.f;
            }
            if (params.renderer_type == CRISB_RENDERER_RESTIR_PT && roundIdx == params.prefix_spatial_rounds - 1)
                StoreOutput(out, static_cast<size_t>(pi), outputRadiance);
        }
        prefixRes[back] = prefixRes[front];
    }

    void InvalidateSuffixReservoir(size_t pixelIdx) {
        Reservoir<SuffixPath>& r = suffixRes[front][pixelIdx];
        r.Reset();
        r.sample.SetValid(false);
    }

    // SuffixGenTempReuse, shader/suffix_gen_temp_reuse.cu:19-112
    void SuffixGenTempReuse(size_t pixelIdx) {
        const PrefixPath& prefix = prefixRes[front][pixelIdx].sample;
        if (!prefix.IsValid() || prefix.IsNee()) {
            InvalidateSuffixReservoir(pixelIdx);
            return;
        }
        PCG32& rng = gbuf[pixelIdx].rng;
        TraceSuffix(canonSuffix[pixelIdx], prefix, rng);
        const SuffixPath& canon = canonSuffix[pixelIdx];
        if (!canon.IsValid()) {
            InvalidateSuffixReservoir(pixelIdx);
            return;
        }
        const float canonPHat = GetLuminance(canon.f);
        Reservoir<SuffixPath>& currRes = suffixRes[front][pixelIdx];
        currRes.Reset();
        const uint32_t prevX = gbuf[pixelIdx].prevX, prevY = gbuf[pixelIdx].prevY;
        if (!params.suffix_enable_temporal || !IsPixelValid(prevX, prevY)) {
            currRes.Update(canon, canonPHat / canon.p, rng, 1.0f);
            currRes.FinalizeGRIS();
            return;
        }
        const size_t prevPixelIdx = static_cast<size_t>(prevY) * width + prevX;
        const Reservoir<SuffixPath>& prevRes = suffixRes[back][prevPixelIdx];
        const SuffixPath& prevSuffix = prevRes.sample;
        if (prevRes.wSum <= 0.0f || !prevSuffix.IsValid()) {
            currRes.Update(canon, canonPHat / canon.p, rng, 1.0f);
            currRes.FinalizeGRIS();
            return;
        }
        float jacobianCanonToPrev = 0.0f, jacobianPrevToCanon = 0.0f;
        const vec3 fFromCanonOfPrev = ShiftSuffix(prevSuffix, canon, jacobianPrevToCanon);
        const vec3 fFromPrevOfCanon = ShiftSuffix(canon, prevSuffix, jacobianCanonToPrev);
        const float pFromCanonOfPrev = GetLuminance(fFromCanonOfPrev) * jacobianPrevToCanon;
        constexpr float pairwiseK = 1.0f;
        const float prevConfidence = prevRes.confidence;
        const float prevMisWeight =
            NeighMis(fFromCanonOfPrev, prevSuffix.f, jacobianPrevToCanon, pairwiseK, 1.0f, prevConfidence);
        const float canonMisWeight =
            1.0f + CanonMis(canon.f, fFromPrevOfCanon, jacobianCanonToPrev, pairwiseK, 1.0f, prevConfidence);
        const float canonRisWeight = canonMisWeight * canonPHat / canon.p;
        currRes.Update(canon, canonRisWeight, rng, 1.0f);
        const float prevRisWeight = prevMisWeight * pFromCanonOfPrev * prevRes.wSum;
        const SuffixPath shiftedPrevSuffix(prevSuffix, canon.lastPrefixInt, fFromCanonOfPrev);
        currRes.Update(shiftedPrevSuffix, prevRisWeight, rng, prevConfidence);
        if (currRes.wSum > 0.0f) {
            currRes.wSum /= pairwiseK + 1.0f;
            currRes.FinalizeGRIS();
        }
    }

    // __raygen__suffix_gen_temp_reuse, shader/suffix_gen_temp_reuse.cu:114-134
    void PassSuffixGenTempReuse() {
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) SuffixGenTempReuse(static_cast<size_t>(pi));
        // "Swap buffers" (suffix_gen_temp_reuse.cu:129-133) after every pixel:
        // other pixels read back[prevPixelIdx] during the pass
#pragma omp parallel for schedule(static)
        for (int64_t pi = 0; pi < P; ++pi) suffixRes[back][pi] = suffixRes[front][pi];
    }

    // SuffixSpatialReuse, shader/suffix_spatial_reuse.cu:16-145 (neighbours
    // read from the pass-start snapshot `snap`)
    void SuffixSpatialReuse(uint32_t x, uint32_t y, const std::vector<Reservoir<SuffixPath>>& snap) {
        const size_t currPixelIdx = static_cast<size_t>(y) * width + x;
        const PrefixPath& prefix = prefixRes[front][currPixelIdx].sample;
        if (!prefix.IsValid() || prefix.IsNee()) {
            InvalidateSuffixReservoir(currPixelIdx);
            return;
        }
        Reservoir<SuffixPath>& currRes = suffixRes[front][currPixelIdx];
        const SuffixPath currSuffix = currRes.sample;
        if (!currSuffix.IsValid()) {
            InvalidateSuffixReservoir(currPixelIdx);
            return;
        }
        const SuffixPath& canon = canonSuffix[currPixelIdx];
        if (!canon.IsValid()) {
            InvalidateSuffixReservoir(currPixelIdx);
            return;
        }
        PCG32& rng = gbuf[currPixelIdx].rng;
        const float currResWSum = currRes.wSum;
        const float currResConfidence = currRes.confidence;
        currRes.Reset();
        const int neighCount = params.suffix_spatial_count;
        float canonMisWeight = 1.0f;
        uint32_t validNeighCount = 0, validNeighFlags = 0;
        uint32_t nxs[CRISB_MAX_SPATIAL_NEIGH], nys[CRISB_MAX_SPATIAL_NEIGH];
        for (int n = 0; n < neighCount; ++n) {
            SelectSpatialNeighbor(x, y, rng, nxs[n], nys[n]);
            if (!IsPixelValid(nxs[n], nys[n])) continue;
            const size_t ni = static_cast<size_t>(nys[n]) * width + nxs[n];
            if (!gbuf[ni].primaryIntValid) continue;
            if (!snap[ni].sample.IsValid()) continue;
            ++validNeighCount;
            validNeighFlags |= 1u << n;
        }
        const float pairwiseK = static_cast<float>(validNeighCount);
        for (int n = 0; n < neighCount; ++n) {
            if (!((validNeighFlags >> n) & 1u)) continue;
            const size_t ni = static_cast<size_t>(nys[n]) * width + nxs[n];
            const Reservoir<SuffixPath>& neighRes = snap[ni];
            const SuffixPath& neighSuffix = neighRes.sample;
            float jacobianNeighToCanon = 0.0f;
            const vec3 fFromCanonOfNeigh = ShiftSuffix(neighSuffix, currSuffix, jacobianNeighToCanon);
            const float pFromCanonOfNeigh = GetLuminance(fFromCanonOfNeigh) * jacobianNeighToCanon;
            float jacobianCanonToNeigh = 0.0f;
            const vec3 fFromNeighOfCanon = ShiftSuffix(currSuffix, neighSuffix, jacobianCanonToNeigh);
            float neighMisWeight = NeighMis(fFromCanonOfNeigh, neighSuffix.f, jacobianNeighToCanon, pairwiseK,
                                            currResConfidence, neighRes.confidence);
            if (std::isnan(neighMisWeight) || std::isinf(neighMisWeight)) neighMisWeight = 0.0f;
            const float neighRisWeight = neighMisWeight * pFromCanonOfNeigh * neighRes.wSum;
            currRes.Update(SuffixPath(neighSuffix, currSuffix.lastPrefixInt, fFromCanonOfNeigh), neighRisWeight, rng,
                           neighRes.confidence);
            canonMisWeight += CanonMis(currSuffix.f, fFromNeighOfCanon, jacobianCanonToNeigh, pairwiseK,
                                       currResConfidence, neighRes.confidence);
        }
        if (std::isinf(canonMisWeight) || std::isnan(canonMisWeight)) canonMisWeight = 0.0f;
        const float canonRisWeight = canonMisWeight * currResWSum * GetLuminance(currSuffix.f);
        currRes.Update(currSuffix, canonRisWeight, rng, currResConfidence);
        if (currRes.wSum > 0.0f) {
            currRes.wSum /= pairwiseK + 1.0f;
            currRes.FinalizeGRIS();
        }
    }

    // __raygen__suffix_spatial_reuse, shader/suffix_spatial_reuse.cu:147-167
    void PassSuffixSpatialReuse() {
        const std::vector<Reservoir<SuffixPath>> snap = suffixRes[back];
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) {
            SuffixSpatialReuse(static_cast<uint32_t>(pi % width), static_cast<uint32_t>(pi / width), snap);
        }
        suffixRes[back] = suffixRes[front];
    }

    // __raygen__prefix_store_entries, shader/prefix_store_entries.cu:9-53, and
    // the acceleration structure rebuild (src/PrefixAccelStruct.cpp:14-26)
    // replaced by a uniform grid over the valid entries.
    void PassPrefixStoreEntries() {
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(static)
        for (int64_t pi = 0; pi < P; ++pi) {
            const PrefixPath& prefix = prefixRes[front][pi].sample;
            const SuffixPath& suffix = suffixRes[front][pi].sample;
            const Interaction lastPrefixInt = Unpack(prefix.lastInt);
            if (prefix.IsValid() && suffix.IsValid() && lastPrefixInt.valid) {
                float radius = params.gather_radius;
                if (params.gather_radius_type == CRISB_RADIUS_PATH_LENGTH) radius *= prefix.pathLen / 4.5f;
                const vec3 pos = lastPrefixInt.pos;
                const float minX = pos.x - radius, maxX = pos.x + radius;
                entryPos[pi] = pos;
                // prefix_search_hit.cu:42: radius = (aabb.maxX - aabb.minX) / 2
                entryRad[pi] = (maxX - minX) / 2.0f;
                entryValid[pi] = 1;
            } else {
                entryPos[pi] = vec3(0.0f);
                entryRad[pi] = 0.0f;
                entryValid[pi] = 0;
            }
        }
        float maxR = 0.0f;
        vec3 lo(INFINITY), hi(-INFINITY);
        for (int64_t pi = 0; pi < P; ++pi) {
            if (!entryValid[pi]) continue;
            maxR = std::max(maxR, entryRad[pi]);
            lo = vec3(std::min(lo.x, entryPos[pi].x), std::min(lo.y, entryPos[pi].y), std::min(lo.z, entryPos[pi].z));
            hi = vec3(std::max(hi.x, entryPos[pi].x), std::max(hi.y, entryPos[pi].y), std::max(hi.z, entryPos[pi].z));
        }
        gridCell = std::max(maxR * 1.001f, 1e-6f);
        gridOrigin = lo;
        gridMax = hi;
        gridEntries.clear();
        for (int64_t pi = 0; pi < P; ++pi) {
            if (!entryValid[pi]) continue;
            gridEntries.emplace_back(CellKey(entryPos[pi]), static_cast<uint32_t>(pi));
        }
        std::sort(gridEntries.begin(), gridEntries.end());
    }

    static int64_t CellCoord(float v, float o, float h) { return static_cast<int64_t>(std::floor((v - o) / h)); }
    static uint64_t PackCell(int64_t cx, int64_t cy, int64_t cz) {
        return (static_cast<uint64_t>(cx + (1 << 20)) << 42) | (static_cast<uint64_t>(cy + (1 << 20)) << 21) |
               static_cast<uint64_t>(cz + (1 << 20));
    }
    uint64_t CellKey(vec3 p) const {
        return PackCell(CellCoord(p.x, gridOrigin.x, gridCell), CellCoord(p.y, gridOrigin.y, gridCell),
                        CellCoord(p.z, gridOrigin.z, gridCell));
    }

    // __intersection__prefix_entry, shader/prefix_search_hit.cu:9-73 over all
    // entries (DEFINED order: k nearest by (distance, pixel index)).
    uint32_t QueryNeighbors(size_t pixelIdx, vec3 queryPos) {
        const uint32_t k = K();
        Neighbor* list = neighbors.data() + pixelIdx * k;
        uint32_t count = 0;
        if (gridEntries.empty() || k == 0) {
            neighCount[pixelIdx] = 0;
            return 0;
        }
        // a non-finite query finds nothing; a query more than one cell outside
        // the entries' bounds cannot be within any entry's radius
        if (anyNanInf(queryPos)) {
            neighCount[pixelIdx] = 0;
            return 0;
        }
        for (int a = 0; a < 3; ++a) {
            const float q = queryPos[a], o = gridOrigin[a];
            if (q < o - 2.0f * gridCell || q > gridMax[a] + 2.0f * gridCell) {
                neighCount[pixelIdx] = 0;
                return 0;
            }
        }
        const int64_t cx = CellCoord(queryPos.x, gridOrigin.x, gridCell);
        const int64_t cy = CellCoord(queryPos.y, gridOrigin.y, gridCell);
        const int64_t cz = CellCoord(queryPos.z, gridOrigin.z, gridCell);
        for (int64_t dx = -1; dx <= 1; ++dx)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dz = -1; dz <= 1; ++dz) {
                    const uint64_t key = PackCell(cx + dx, cy + dy, cz + dz);
                    auto it = std::lower_bound(gridEntries.begin(), gridEntries.end(),
                                               std::make_pair(key, uint32_t(0)));
                    for (; it != gridEntries.end() && it->first == key; ++it) {
                        const uint32_t j = it->second;
                        const float d = distance(queryPos, entryPos[j]);
                        if (d > entryRad[j]) continue;
                        // insert (d, j) into the sorted list of at most k entries
                        if (count == k) {
                            const Neighbor& w = list[k - 1];
                            if (!(d < w.distance || (d == w.distance && j < w.pixelIdx))) continue;
                            --count;
                        }
                        uint32_t pos = count;
                        while (pos > 0 && (d < list[pos - 1].distance ||
                                           (d == list[pos - 1].distance && j < list[pos - 1].pixelIdx))) {
                            list[pos] = list[pos - 1];
                            --pos;
                        }
                        list[pos].pixelIdx = j;
                        list[pos].distance = d;
                        ++count;
                    }
                }
        neighCount[pixelIdx] = count;
        return count;
    }

    // FinalGatherCanon, shader/final_gather.cu:69-188
    vec3 FinalGatherCanon(size_t pixelIdx, vec3 origin, vec3 dir, uint32_t k, PCG32& rng) {
        PrefixPath canonPrefix2;
        TracePrefix(canonPrefix2, origin, dir, rng);
        if (!canonPrefix2.IsValid()) return vec3(0.0f);
        if (canonPrefix2.IsNee()) return canonPrefix2.f / canonPrefix2.p;
        SuffixPath canonSuffix2;
        TraceSuffix(canonSuffix2, canonPrefix2, rng);
        if (!canonSuffix2.IsValid()) return vec3(0.0f);
        const vec3 canonContrib = canonPrefix2.f * canonSuffix2.f / (canonPrefix2.p * canonSuffix2.p);
        if (k == 0) return canonContrib;
        const Interaction lastPrefixInt = Unpack(canonSuffix2.lastPrefixInt);
        const uint32_t neighCountQ = QueryNeighbors(pixelIdx, lastPrefixInt.pos);
        const Neighbor* list = neighbors.data() + pixelIdx * K();
        uint32_t validNeighCount = 0, validNeighFlags = 0;
        for (uint32_t n = 0; n < neighCountQ; ++n) {
            const SuffixPath& ns = suffixRes[front][list[n].pixelIdx].sample;
            if (!ns.IsValid()) continue;
            ++validNeighCount;
            validNeighFlags |= 1u << n;
        }
        vec3 suffixContrib(0.0f);
        const float pairwiseK = static_cast<float>(validNeighCount);
        float canonMisWeight = 1.0f;
        for (uint32_t n = 0; n < neighCountQ; ++n) {
            if (!(validNeighFlags & (1u << n))) continue;
            const Reservoir<SuffixPath>& neighRes = suffixRes[front][list[n].pixelIdx];
            const SuffixPath& neighSuffix = neighRes.sample;
            float jacobianNeighToCanon = 0.0f;
            const vec3 fFromCanonOfNeigh = ShiftSuffix(neighSuffix, canonSuffix2, jacobianNeighToCanon);
            float jacobianCanonToNeigh = 0.0f;
            const vec3 fFromNeighOfCanon = ShiftSuffix(canonSuffix2, neighSuffix, jacobianCanonToNeigh);
            float neighMisWeight =
                NeighMis(fFromCanonOfNeigh, neighSuffix.f, jacobianNeighToCanon, pairwiseK, 1.0f, neighRes.confidence);
            if (std::isnan(neighMisWeight) || std::isinf(neighMisWeight)) neighMisWeight = 0.0f;
            const vec3 neighContrib = neighMisWeight * fFromCanonOfNeigh * neighRes.wSum * jacobianNeighToCanon;
            if (!anyNanInf(neighContrib)) suffixContrib += neighContrib;
            canonMisWeight +=
                CanonMis(canonSuffix2.f, fFromNeighOfCanon, jacobianCanonToNeigh, pairwiseK, 1.0f, neighRes.confidence);
        }
        vec3 gatherContrib = suffixContrib * canonPrefix2.f / canonPrefix2.p;
        gatherContrib /= static_cast<float>(validNeighCount + 1);
        vec3 result = gatherContrib + (canonContrib * canonMisWeight);
        result /= pairwiseK + 1.0f;
        if (anyNanInf(result)) return vec3(0.0f);
        return result;
    }

    // FinalGatherNotCanon, shader/final_gather.cu:190-288
    vec3 FinalGatherNotCanon(size_t pixelIdx, vec3 origin, vec3 dir, uint32_t k, PCG32& rng) {
        if (k == 0) return vec3(0.0f);
        Interaction lastPrefixInt;
        vec3 prefixThroughput(0.0f);
        float prefixP = 0.0f;
        if (!TracePrefixForFinalGather(prefixThroughput, prefixP, lastPrefixInt, origin, dir,
                                       static_cast<size_t>(params.prefix_len), rng))
            return vec3(0.0f);
        const uint32_t neighCountQ = QueryNeighbors(pixelIdx, lastPrefixInt.pos);
        const Neighbor* list = neighbors.data() + pixelIdx * K();
        uint32_t validNeighCount = 0, validNeighFlags = 0;
        for (uint32_t n = 0; n < neighCountQ; ++n) {
            if (!suffixRes[front][list[n].pixelIdx].sample.IsValid()) continue;
            ++validNeighCount;
            validNeighFlags |= 1u << n;
        }
        vec3 suffixContrib(0.0f);
        const float pairwiseK = static_cast<float>(validNeighCount);
        for (uint32_t n = 0; n < neighCountQ; ++n) {
            if (!(validNeighFlags & (1u << n))) continue;
            const Reservoir<SuffixPath>& neighRes = suffixRes[front][list[n].pixelIdx];
            const SuffixPath& neighSuffix = neighRes.sample;
            float jacobianNeighToCanon = 0.0f;
            const vec3 fFromCanonOfNeigh = ShiftSuffix(neighSuffix, lastPrefixInt, jacobianNeighToCanon);
            float neighMisWeight =
                NeighMis(fFromCanonOfNeigh, neighSuffix.f, jacobianNeighToCanon, pairwiseK, 1.0f, neighRes.confidence);
            if (std::isnan(neighMisWeight) || std::isinf(neighMisWeight)) neighMisWeight = 0.0f;
            const vec3 neighContrib = neighMisWeight * fFromCanonOfNeigh * neighRes.wSum * jacobianNeighToCanon;
            if (!anyNanInf(neighContrib)) suffixContrib += neighContrib;
        }
        vec3 result = suffixContrib * prefixThroughput / prefixP;
        result /= static_cast<float>(params.gather_n);
        result /= pairwiseK + 1.0f;
        if (anyNanInf(result)) return vec3(0.0f);
        return result;
    }

    // GetRadiance + __raygen__final_gather, shader/final_gather.cu:290-356
    void PassFinalGather(float* out) {
        const int64_t P = static_cast<int64_t>(width) * height;
        const uint32_t k = K();
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) {
            const size_t pixelIdx = static_cast<size_t>(pi);
            const uint32_t x = static_cast<uint32_t>(pi % width), y = static_cast<uint32_t>(pi / width);
            neighCount[pixelIdx] = 0;
            vec3 outputRadiance(0.0f);
            if (canonPrefix[pixelIdx].primaryInt.valid) {
                PCG32& rng = gbuf[pixelIdx].rng;
                const vec3 dir = PixelJitterDir(x, y, rng);
                const vec3 origin = cam.pos;
                outputRadiance += FinalGatherCanon(pixelIdx, origin, dir, k, rng);
                for (int prefixIdx = 1; prefixIdx < params.gather_n; ++prefixIdx)
                    outputRadiance += FinalGatherNotCanon(pixelIdx, origin, dir, k, rng);
                if (anyNanInf(outputRadiance)) outputRadiance = vec3(0.0f);
            }
            StoreOutput(out, pixelIdx, outputRadiance);
        }
    }

    // Renderer::LaunchFrame, src/Renderer.cpp:209-406
    // the library stores every reservoir it writes at the end of a pass; in
    // FP16 storage the stored values are the quantised ones
    void QuantizeReservoirs() {
        if (params.storage != CRISB_STORAGE_FP16) return;
        const int64_t P = static_cast<int64_t>(width) * height;
#pragma omp parallel for schedule(static)
        for (int64_t pi = 0; pi < P; ++pi) {
            for (int b = 0; b < 2; ++b) {
                Quantize(prefixRes[b][pi].sample);
                Quantize(suffixRes[b][pi].sample);
            }
        }
    }

    void RenderFrame(const crisb_camera& c, float* out, double* passMs) {
        using clk = std::chrono::steady_clock;
        auto t0 = clk::now();
        auto lap = [&](int slot) {
            if (!passMs) return;
            const auto t1 = clk::now();
            passMs[slot] += std::chrono::duration<double, std::milli>(t1 - t0).count();
            t0 = t1;
        };
        if (passMs)
            for (int i = 0; i < 6; ++i) passMs[i] = 0.0;
        ++frameIdx;
        if (c.changed || !params.enable_accum) frameIdx = 0;
        random = FrameRandom(params.seed, frameCounter);
        ++frameCounter;
        cam = GetCameraData(c);
        prevCam = lastCam;
        hasPrevCam = hasLastCam;
        lastCam = cam;
        hasLastCam = true;
        if (front == 0) {
            front = 1;
            back = 0;
        } else {
            front = 0;
            back = 1;
        }
        PassPrefixGenTempReuse(out);
        QuantizeReservoirs();
        lap(0);
        const int type = params.renderer_type;
        if (type == CRISB_RENDERER_CONDITIONAL_RESTIR || type == CRISB_RENDERER_RESTIR_PT) {
            if (params.prefix_enable_spatial)
                for (int r = 0; r < params.prefix_spatial_rounds; ++r) {
                    PassPrefixSpatialReuse(out, r);
                    QuantizeReservoirs();
                }
            lap(1);
            if (type == CRISB_RENDERER_CONDITIONAL_RESTIR) {
                PassSuffixGenTempReuse();
                QuantizeReservoirs();
                lap(2);
                if (params.suffix_enable_spatial && params.suffix_spatial_count > 0)
                    for (int r = 0; r < params.suffix_spatial_rounds; ++r) {
                        PassSuffixSpatialReuse();
                        QuantizeReservoirs();
                    }
                lap(3);
                PassPrefixStoreEntries();
                lap(4);
                PassFinalGather(out);
                lap(5);
            }
        }
    }
};

namespace {

void PackHit(const PackedInteraction& p, crisb_hit_rec& h) {
    h.prim = p.valid ? p.prim : CRISB_INVALID_PRIM;
    h.bary[0] = p.bary.x;
    h.bary[1] = p.bary.y;
    h.in_dir[0] = p.inRayDir.x;
    h.in_dir[1] = p.inRayDir.y;
    h.in_dir[2] = p.inRayDir.z;
}
void Put3(float* d, vec3 v) {
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}
void PackPrefix(const PrefixPath& s, crisb_prefix_rec& r) {
    std::memset(&r, 0, sizeof(r));
    r.rng = s.rng.state;
    PackHit(s.primaryInt, r.primary);
    PackHit(s.reconInt, r.recon);
    PackHit(s.lastInt, r.last);
    r.flags = s.flags;
    Put3(r.f, s.f);
    Put3(r.post_recon_f, s.postReconF);
    r.p = s.p;
    r.path_len = s.pathLen;
    Put3(r.recon_out_dir, s.reconOutDir);
}
crisb_hit16_rec PackHit16(const PackedInteraction& p) {
    crisb_hit16_rec h;
    h.prim = p.valid ? p.prim : CRISB_INVALID_PRIM;
    h.bary[0] = HalfBits(p.bary.x);
    h.bary[1] = HalfBits(p.bary.y);
    h.in_dir_oct = OctEncode(p.inRayDir);
    return h;
}
void Put16(uint16_t* d, vec3 v) {
    d[0] = HalfBits(v.x);
    d[1] = HalfBits(v.y);
    d[2] = HalfBits(v.z);
}
void PackPrefixRes16(const Reservoir<PrefixPath>& r, crisb_prefix_res16_rec& o) {
    std::memset(&o, 0, sizeof(o));
    const PrefixPath& s = r.sample;
    o.rng = s.rng.state;
    o.flags = s.flags;
    o.p = s.p;
    o.path_len = s.pathLen;
    o.primary = PackHit16(s.primaryInt);
    o.recon = PackHit16(s.reconInt);
    o.last = PackHit16(s.lastInt);
    Put16(o.f, s.f);
    Put16(o.post_recon_f, s.postReconF);
    o.recon_out_dir_oct = OctEncode(s.reconOutDir);
    o.w_sum = r.wSum;
    o.confidence = r.confidence;
}
void PackSuffixRes16(const Reservoir<SuffixPath>& r, crisb_suffix_res16_rec& o) {
    std::memset(&o, 0, sizeof(o));
    const SuffixPath& s = r.sample;
    o.rng = s.rng.state;
    o.flags = s.flags;
    o.p = s.p;
    o.recon = PackHit16(s.reconInt);
    o.last_prefix = PackHit16(s.lastPrefixInt);
    Put16(o.f, s.f);
    Put16(o.post_recon_f, s.postReconF);
    o.recon_out_dir_oct = OctEncode(s.reconOutDir);
    o.w_sum = r.wSum;
    o.confidence = r.confidence;
}
void PackSuffix(const SuffixPath& s, crisb_suffix_rec& r) {
    std::memset(&r, 0, sizeof(r));
    r.rng = s.rng.state;
    PackHit(s.reconInt, r.recon);
    PackHit(s.lastPrefixInt, r.last_prefix);
    r.flags = s.flags;
    Put3(r.f, s.f);
    Put3(r.post_recon_f, s.postReconF);
    r.p = s.p;
    Put3(r.recon_out_dir, s.reconOutDir);
}

}  // namespace

extern "C" {

oracle_ctx* oracle_create(const float* tri_pos, const float* tri_nrm, const uint32_t* tri_mat, uint32_t num_tris,
                          const crisb_material* mats, uint32_t num_mats, const crisb_emitter* emitters,
                          uint32_t num_emitters, const float* emitter_faces, uint32_t num_faces, uint32_t width,
                          uint32_t height, const crisb_params* params) {
    if (!tri_pos || !tri_nrm || !tri_mat || !mats || !params || width == 0 || height == 0) return nullptr;
    auto ctx = std::make_unique<oracle_ctx>();
    Scene& s = ctx->scene;
    s.tris.resize(num_tris);
    vec3 lo(0.0f), hi(0.0f);  // Scene::GetSceneSize starts min/max at the origin
    for (uint32_t i = 0; i < num_tris; ++i) {
        Triangle& t = s.tris[i];
        for (int c = 0; c < 3; ++c) {
            t.p[c] = vec3(tri_pos[9 * i + 3 * c], tri_pos[9 * i + 3 * c + 1], tri_pos[9 * i + 3 * c + 2]);
            t.n[c] = vec3(tri_nrm[9 * i + 3 * c], tri_nrm[9 * i + 3 * c + 1], tri_nrm[9 * i + 3 * c + 2]);
            lo = vec3(gmin(lo.x, t.p[c].x), gmin(lo.y, t.p[c].y), gmin(lo.z, t.p[c].z));
            hi = vec3(gmax(hi.x, t.p[c].x), gmax(hi.y, t.p[c].y), gmax(hi.z, t.p[c].z));
        }
        t.mat = tri_mat[i];
        if (t.mat >= num_mats) return nullptr;
    }
    s.sceneSize = distance(lo, hi);
    s.mats.assign(mats, mats + num_mats);
    for (uint32_t e = 0; e < num_emitters; ++e) {
        EmitterData d;
        d.color = vec3(emitters[e].color[0], emitters[e].color[1], emitters[e].color[2]);
        if (emitters[e].num_faces == 0 || emitters[e].first_face + emitters[e].num_faces > num_faces) return nullptr;
        for (uint32_t f = 0; f < emitters[e].num_faces; ++f)
            for (int c = 0; c < 3; ++c) {
                const float* v = emitter_faces + 9 * (emitters[e].first_face + f) + 3 * c;
                d.faces.push_back(vec3(v[0], v[1], v[2]));
            }
        s.emitters.push_back(std::move(d));
    }
    if (s.emitters.empty()) return nullptr;
    s.bvh.Build(s.tris);
    ctx->width = width;
    ctx->height = height;
    if (oracle_set_params(ctx.get(), params) != 0) return nullptr;
    const size_t P = static_cast<size_t>(width) * height;
    for (int b = 0; b < 2; ++b) {
        ctx->prefixRes[b].resize(P);
        ctx->suffixRes[b].resize(P);
    }
    ctx->canonPrefix.resize(P);
    ctx->canonSuffix.resize(P);
    ctx->gbuf.resize(P);
    ctx->entryPos.resize(P);
    ctx->entryRad.resize(P);
    ctx->entryValid.resize(P);
    ctx->neighCount.assign(P, 0);
    ctx->neighbors.assign(P * ctx->K(), Neighbor{});
    return ctx.release();
}

void oracle_destroy(oracle_ctx* ctx) { delete ctx; }

int oracle_set_params(oracle_ctx* ctx, const crisb_params* p) {
    if (!ctx || !p) return CRISB_ERR_INVALID_ARGUMENT;
    if (p->prefix_spatial_count < 0 || p->prefix_spatial_count > CRISB_MAX_SPATIAL_NEIGH ||
        p->suffix_spatial_count < 0 || p->suffix_spatial_count > CRISB_MAX_SPATIAL_NEIGH || p->gather_m < 1 ||
        p->gather_m > CRISB_MAX_GATHER_M || p->gather_n < 1 || p->max_path_len < 1 || p->prefix_len < 1 ||
        p->window_radius < 0 || p->motion_mode < CRISB_MOTION_NONE || p->motion_mode > CRISB_MOTION_REPROJECT)
        return CRISB_ERR_INVALID_ARGUMENT;
    const uint32_t oldK = ctx->K();
    ctx->params = *p;
    if (ctx->K() != oldK) {
        ctx->neighbors.assign(static_cast<size_t>(ctx->width) * ctx->height * ctx->K(), Neighbor{});
    }
    return CRISB_OK;
}

int oracle_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

float oracle_scene_size(const oracle_ctx* ctx) { return ctx ? ctx->scene.sceneSize : 0.0f; }

namespace {
bool MotionReady(const oracle_ctx* ctx) {
    return ctx->params.motion_mode != CRISB_MOTION_VECTORS ||
           ctx->motion.size() == 2 * static_cast<size_t>(ctx->width) * ctx->height;
}
}  // namespace

int oracle_render_frame(oracle_ctx* ctx, const crisb_camera* cam, float* out_rgb) {
    if (!ctx || !cam || !out_rgb || !MotionReady(ctx)) return CRISB_ERR_INVALID_ARGUMENT;
    ctx->RenderFrame(*cam, out_rgb, nullptr);
    return CRISB_OK;
}

int oracle_render_frame_timed(oracle_ctx* ctx, const crisb_camera* cam, float* out_rgb, double* pass_ms) {
    if (!ctx || !cam || !out_rgb || !MotionReady(ctx)) return CRISB_ERR_INVALID_ARGUMENT;
    ctx->RenderFrame(*cam, out_rgb, pass_ms);
    return CRISB_OK;
}

int oracle_set_textures(oracle_ctx* ctx, const float* tri_uvs, uint32_t num_tris, const crisb_texture* textures,
                        uint32_t num_textures, const int32_t* material_textures) {
    if (!ctx || num_tris != ctx->scene.tris.size()) return CRISB_ERR_INVALID_ARGUMENT;
    if (!material_textures) {
        ctx->matTex.clear();
        return CRISB_OK;
    }
    const size_t M = ctx->scene.mats.size();
    std::vector<std::array<int32_t, 3>> mt(M);
    for (size_t m = 0; m < M; ++m)
        for (int k = 0; k < 3; ++k) {
            const int32_t t = material_textures[3 * m + k];
            if (t < -1 || t >= static_cast<int64_t>(num_textures)) return CRISB_ERR_INVALID_ARGUMENT;
            mt[m][k] = t;
        }
    if (!tri_uvs || (num_textures && !textures)) return CRISB_ERR_INVALID_ARGUMENT;
    std::vector<oracle_ctx::Texture> tx(num_textures);
    for (uint32_t t = 0; t < num_textures; ++t) {
        if (!textures[t].rgba || textures[t].width == 0 || textures[t].height == 0) return CRISB_ERR_INVALID_ARGUMENT;
        tx[t].width = textures[t].width;
        tx[t].height = textures[t].height;
        tx[t].texels.resize(static_cast<size_t>(tx[t].width) * tx[t].height);
        std::memcpy(tx[t].texels.data(), textures[t].rgba, 4 * tx[t].texels.size());
    }
    ctx->triUv.assign(tri_uvs, tri_uvs + 6 * static_cast<size_t>(num_tris));
    ctx->textures = std::move(tx);
    ctx->matTex = std::move(mt);
    return CRISB_OK;
}

void oracle_tex_sample(const uint8_t* rgba, uint32_t width, uint32_t height, const float* uv, uint32_t n,
                       float* out) {
    oracle_ctx::Texture t;
    t.width = width;
    t.height = height;
    t.texels.resize(static_cast<size_t>(width) * height);
    std::memcpy(t.texels.data(), rgba, 4 * t.texels.size());
    oracle_ctx probe;
    probe.textures.push_back(std::move(t));
    for (uint32_t i = 0; i < n; ++i) {
        const oracle_ctx::Rgba c = probe.TexSample(0, uv[2 * i], uv[2 * i + 1]);
        out[4 * i] = c.r;
        out[4 * i + 1] = c.g;
        out[4 * i + 2] = c.b;
        out[4 * i + 3] = c.a;
    }
}

int oracle_set_motion_vectors(oracle_ctx* ctx, const float* motion, uint32_t num_pixels) {
    if (!ctx) return CRISB_ERR_INVALID_ARGUMENT;
    if (!motion) {
        ctx->motion.clear();
        return CRISB_OK;
    }
    if (num_pixels != ctx->width * ctx->height) return CRISB_ERR_INVALID_ARGUMENT;
    ctx->motion.assign(motion, motion + 2 * static_cast<size_t>(num_pixels));
    return CRISB_OK;
}

uint64_t oracle_frame_index(const oracle_ctx* ctx) { return ctx ? ctx->frameIdx : 0; }
uint32_t oracle_frame_random(const oracle_ctx* ctx) { return ctx ? ctx->random : 0; }

size_t oracle_dump_size(const oracle_ctx* ctx, int id) {
    if (!ctx) return 0;
    const size_t P = static_cast<size_t>(ctx->width) * ctx->height;
    switch (id) {
        case CRISB_BUF_PREFIX_RES_FRONT:
        case CRISB_BUF_PREFIX_RES_BACK:
            return P * (ctx->params.storage == CRISB_STORAGE_FP16 ? sizeof(crisb_prefix_res16_rec)
                                                                   : sizeof(crisb_prefix_res_rec));
        case CRISB_BUF_CANON_PREFIX: return P * sizeof(crisb_prefix_rec);
        case CRISB_BUF_SUFFIX_RES_FRONT:
        case CRISB_BUF_SUFFIX_RES_BACK:
            return P * (ctx->params.storage == CRISB_STORAGE_FP16 ? sizeof(crisb_suffix_res16_rec)
                                                                   : sizeof(crisb_suffix_res_rec));
        case CRISB_BUF_CANON_SUFFIX: return P * sizeof(crisb_suffix_rec);
        case CRISB_BUF_GBUFFER: return P * sizeof(crisb_gbuffer_rec);
        case CRISB_BUF_NEIGHBORS: return P * ctx->K() * sizeof(crisb_neighbor_rec);
        case CRISB_BUF_NEIGHBOR_COUNT: return P * sizeof(uint32_t);
        default: return 0;
    }
}

int oracle_check_post_recon(const oracle_ctx* ctx, uint32_t* checked, uint32_t* mismatched, uint32_t* nee_recon) {
    if (!ctx || !checked || !mismatched || !nee_recon) return CRISB_ERR_INVALID_ARGUMENT;
    if (ctx->params.renderer_type != CRISB_RENDERER_CONDITIONAL_RESTIR) return CRISB_ERR_INVALID_ARGUMENT;
    *checked = *mismatched = *nee_recon = 0;
    for (const auto& res : ctx->suffixRes[ctx->front]) {
        if (!res.sample.IsValid()) continue;
        bool checkable = false;
        const vec3 v = ctx->ReplayPostRecon(res.sample, checkable);
        if (!checkable) {
            ++*nee_recon;
            continue;
        }
        ++*checked;
        if (std::memcmp(&v, &res.sample.postReconF, sizeof(v)) != 0) ++*mismatched;
    }
    return CRISB_OK;
}

int oracle_dump(const oracle_ctx* ctx, int id, void* dst, size_t bytes) {
    if (!ctx || !dst || bytes != oracle_dump_size(ctx, id) || bytes == 0) return CRISB_ERR_INVALID_ARGUMENT;
    const size_t P = static_cast<size_t>(ctx->width) * ctx->height;
    switch (id) {
        case CRISB_BUF_PREFIX_RES_FRONT:
        case CRISB_BUF_PREFIX_RES_BACK: {
            const auto& v = ctx->prefixRes[id == CRISB_BUF_PREFIX_RES_FRONT ? ctx->front : ctx->back];
            if (ctx->params.storage == CRISB_STORAGE_FP16) {
                auto* o16 = static_cast<crisb_prefix_res16_rec*>(dst);
                for (size_t i = 0; i < P; ++i) PackPrefixRes16(v[i], o16[i]);
                return CRISB_OK;
            }
            auto* o = static_cast<crisb_prefix_res_rec*>(dst);
            for (size_t i = 0; i < P; ++i) {
                std::memset(&o[i], 0, sizeof(o[i]));
                PackPrefix(v[i].sample, o[i].sample);
                o[i].w_sum = v[i].wSum;
                o[i].confidence = v[i].confidence;
            }
            return CRISB_OK;
        }
        case CRISB_BUF_CANON_PREFIX: {
            auto* o = static_cast<crisb_prefix_rec*>(dst);
            for (size_t i = 0; i < P; ++i) PackPrefix(ctx->canonPrefix[i], o[i]);
            return CRISB_OK;
        }
        case CRISB_BUF_SUFFIX_RES_FRONT:
        case CRISB_BUF_SUFFIX_RES_BACK: {
            const auto& v = ctx->suffixRes[id == CRISB_BUF_SUFFIX_RES_FRONT ? ctx->front : ctx->back];
            if (ctx->params.storage == CRISB_STORAGE_FP16) {
                auto* o16 = static_cast<crisb_suffix_res16_rec*>(dst);
                for (size_t i = 0; i < P; ++i) PackSuffixRes16(v[i], o16[i]);
                return CRISB_OK;
            }
            auto* o = static_cast<crisb_suffix_res_rec*>(dst);
            for (size_t i = 0; i < P; ++i) {
                std::memset(&o[i], 0, sizeof(o[i]));
                PackSuffix(v[i].sample, o[i].sample);
                o[i].w_sum = v[i].wSum;
                o[i].confidence = v[i].confidence;
            }
            return CRISB_OK;
        }
        case CRISB_BUF_CANON_SUFFIX: {
            auto* o = static_cast<crisb_suffix_rec*>(dst);
            for (size_t i = 0; i < P; ++i) PackSuffix(ctx->canonSuffix[i], o[i]);
            return CRISB_OK;
        }
        case CRISB_BUF_GBUFFER: {
            auto* o = static_cast<crisb_gbuffer_rec*>(dst);
            for (size_t i = 0; i < P; ++i) {
                o[i].rng = ctx->gbuf[i].rng.state;
                o[i].prev_xy = ctx->gbuf[i].prevX | (ctx->gbuf[i].prevY << 16);
                o[i].flags = ctx->gbuf[i].primaryIntValid ? 1u : 0u;
            }
            return CRISB_OK;
        }
        case CRISB_BUF_NEIGHBORS: {
            auto* o = static_cast<crisb_neighbor_rec*>(dst);
            const uint32_t k = ctx->K();
            for (size_t i = 0; i < P; ++i)
                for (uint32_t n = 0; n < k; ++n) {
                    const bool used = n < ctx->neighCount[i];
                    o[i * k + n].pixel = used ? ctx->neighbors[i * k + n].pixelIdx : 0u;
                    o[i * k + n].dist = used ? ctx->neighbors[i * k + n].distance : 0.0f;
                }
            return CRISB_OK;
        }
        case CRISB_BUF_NEIGHBOR_COUNT: {
            std::memcpy(dst, ctx->neighCount.data(), bytes);
            return CRISB_OK;
        }
        default: return CRISB_ERR_INVALID_ARGUMENT;
    }
}

static int TraceImpl(const oracle_ctx* ctx, const float* rays, crisb_trace_hit* hits, uint32_t n, int any_hit,
                     bool brute) {
    if (!ctx || !rays || !hits) return CRISB_ERR_INVALID_ARGUMENT;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
        const float* r = rays + 8 * i;
        const vec3 o(r[0], r[1], r[2]), d(r[4], r[5], r[6]);
        const float tmin = r[3], tmax = r[7];
        const RayPre rp = MakeRay(o, d);
        crisb_trace_hit h{CRISB_INVALID_PRIM, 0.0f, 0.0f, 0.0f};
        if (!brute) {
            if (any_hit) {
                h.prim = ctx->scene.bvh.Occluded(rp, tmin, tmax) ? 1u : 0u;
            } else {
                const HitResult hr = ctx->scene.bvh.Closest(rp, tmin, tmax);
                if (hr.hit) h = {hr.prim, hr.t, hr.u, hr.v};
            }
        } else {
            bool found = false;
            for (uint32_t t = 0; t < ctx->scene.tris.size(); ++t) {
                const Triangle& tr = ctx->scene.tris[t];
                float th, u, v;
                if (!IntersectTri(rp, tr.p[0], tr.p[1], tr.p[2], tmin, tmax, th, u, v)) continue;
                if (any_hit) {
                    found = true;
                    break;
                }
                if (!found || th < h.t || (th == h.t && t < h.prim)) {
                    h = {t, th, u, v};
                    found = true;
                }
            }
            if (any_hit) h.prim = found ? 1u : 0u;
        }
        hits[i] = h;
    }
    return CRISB_OK;
}

int oracle_trace(const oracle_ctx* ctx, const float* rays, crisb_trace_hit* hits, uint32_t n, int any_hit) {
    return TraceImpl(ctx, rays, hits, n, any_hit, false);
}

int oracle_trace_bruteforce(const oracle_ctx* ctx, const float* rays, crisb_trace_hit* hits, uint32_t n,
                            int any_hit) {
    return TraceImpl(ctx, rays, hits, n, any_hit, true);
}

int oracle_pt_accumulate(oracle_ctx* ctx, const crisb_camera* cam, uint32_t spp, uint64_t seed, double* accum) {
    if (!ctx || !cam || !accum) return CRISB_ERR_INVALID_ARGUMENT;
    ctx->cam = GetCameraData(*cam);
    const int64_t P = static_cast<int64_t>(ctx->width) * ctx->height;
    for (uint32_t s = 0; s < spp; ++s) {
        const uint32_t rnd = FrameRandom(seed, s);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t pi = 0; pi < P; ++pi) {
            const uint32_t x = static_cast<uint32_t>(pi % ctx->width), y = static_cast<uint32_t>(pi / ctx->width);
            PCG32 rng(SampleTEA64(static_cast<uint32_t>(pi), rnd));
            const vec3 dir = ctx->PixelJitterDir(x, y, rng);
            vec3 L = ctx->TraceCompletePath(ctx->cam.pos, dir, rng);
            if (anyNanInf(L)) L = vec3(0.0f);
            accum[3 * pi] += L.x;
            accum[3 * pi + 1] += L.y;
            accum[3 * pi + 2] += L.z;
        }
    }
    return CRISB_OK;
}

void oracle_pcg32(uint64_t initstate, uint64_t initseq, uint32_t n, uint32_t* out) {
    PCG32 r(initstate, initseq);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.NextUint32();
}

uint64_t oracle_tea64(uint32_t v0, uint32_t v1) { return SampleTEA64(v0, v1); }

void oracle_srgb_root(const float* in, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = SrgbRoot(in[i]);
}

uint32_t oracle_srgb8_first_decrease(uint32_t lo_bits, uint32_t hi_bits) {
    uint32_t first = 0;
#pragma omp parallel for schedule(static) reduction(min : first)
    for (int64_t chunk = 0; chunk < (static_cast<int64_t>(hi_bits) - lo_bits + 65535) / 65536; ++chunk) {
        const uint32_t b0 = lo_bits + static_cast<uint32_t>(chunk) * 65536u;
        const uint32_t b1 = std::min<uint64_t>(static_cast<uint64_t>(b0) + 65536u, hi_bits);
        float f;
        memcpy(&f, &b0, sizeof f);
        uint8_t prev = LinearToSrgb8(f);
        for (uint32_t b = b0 + 1; b <= b1; ++b) {
            memcpy(&f, &b, sizeof f);
            const uint8_t cur = LinearToSrgb8(f);
            if (cur < prev && (first == 0 || b < first)) first = b;
            prev = cur;
        }
    }
    return first;
}

int oracle_tonemap_srgb8(const float* rgb, uint8_t* out, uint32_t num_pixels) {
    if ((!rgb || !out) && num_pixels) return CRISB_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < 3 * num_pixels; ++i) out[i] = LinearToSrgb8(rgb[i]);
    return CRISB_OK;
}

void oracle_half(const float* in, uint32_t n, uint16_t* bits, float* back) {
    for (uint32_t i = 0; i < n; ++i) {
        bits[i] = HalfBits(in[i]);
        back[i] = HalfValue(bits[i]);
    }
}

void oracle_oct(const float* dirs, uint32_t n, uint32_t* codes, float* decoded) {
    for (uint32_t i = 0; i < n; ++i) {
        codes[i] = OctEncode(vec3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        const vec3 d = OctDecode(codes[i]);
        decoded[3 * i] = d.x;
        decoded[3 * i + 1] = d.y;
        decoded[3 * i + 2] = d.z;
    }
}

uint64_t oracle_oct_unstable(const uint32_t* codes, uint32_t n) {
    uint64_t bad = 0;
#pragma omp parallel for reduction(+ : bad)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
        const uint32_t c1 = OctEncode(OctDecode(codes[i]));
        if (OctEncode(OctDecode(c1)) != c1) ++bad;
    }
    return bad;
}

void oracle_sincos(const float* phi, uint32_t n, float* s, float* c) {
    for (uint32_t i = 0; i < n; ++i) SinCos(phi[i], s[i], c[i]);
}

int oracle_camera_data(const crisb_camera* cam, crisb_camera_data* out) {
    if (!cam || !out) return CRISB_ERR_INVALID_ARGUMENT;
    const CameraData d = GetCameraData(*cam);
    Put3(out->pos, d.pos);
    Put3(out->u, d.U);
    Put3(out->v, d.V);
    Put3(out->w, d.W);
    return CRISB_OK;
}

uint32_t oracle_frame_random_for(uint64_t seed, uint64_t frame_counter) { return FrameRandom(seed, frame_counter); }

/* known-answer-test hooks (kat.h): the oracle's own unit-level functions */
namespace {
uint64_t KatGet64(const uint32_t* w) { return static_cast<uint64_t>(w[0]) | (static_cast<uint64_t>(w[1]) << 32); }
void KatPut64(uint32_t* w, uint64_t v) {
    w[0] = static_cast<uint32_t>(v);
    w[1] = static_cast<uint32_t>(v >> 32);
}
float KatGetF(const uint32_t* w) {
    float f;
    std::memcpy(&f, w, 4);
    return f;
}
void KatPutF(uint32_t* w, float f) { std::memcpy(w, &f, 4); }
vec3 KatGet3(const uint32_t* w) { return vec3(KatGetF(w), KatGetF(w + 1), KatGetF(w + 2)); }
void KatPut3(uint32_t* w, vec3 v) {
    KatPutF(w, v.x);
    KatPutF(w + 1, v.y);
    KatPutF(w + 2, v.z);
}
PCG32 KatRng(const uint32_t* w) {
    PCG32 r;
    r.state = KatGet64(w);
    r.inc = KatGet64(w + 2);
    return r;
}
struct KatSample {
    vec3 f;
    uint32_t id = 0;
};

void KatEval(int fn, const uint32_t* in, uint32_t* out) {
    switch (fn) {
        case KAT_TEA64:
            KatPut64(out, SampleTEA64(in[0], in[1]));
            break;
        case KAT_PCG_SEED: {
            const PCG32 r(KatGet64(in), KatGet64(in + 2));
            KatPut64(out, r.state);
            KatPut64(out + 2, r.inc);
            break;
        }
        case KAT_PCG_DRAWS: {
            PCG32 r = KatRng(in);
            out[0] = r.NextUint32();
            KatPutF(out + 1, r.NextFloat());
            KatPut64(out + 2, r.NextUint64());
            KatPut64(out + 4, r.state);
            break;
        }
        case KAT_LUMINANCE:
            KatPutF(out, GetLuminance(KatGet3(in)));
            break;
        case KAT_MIS_CANON:
            KatPutF(out, oracle_ctx::CanonMis(KatGet3(in), KatGet3(in + 3), KatGetF(in + 6), KatGetF(in + 7),
                                              KatGetF(in + 8), KatGetF(in + 9)));
            break;
        case KAT_MIS_NEIGH:
            KatPutF(out, oracle_ctx::NeighMis(KatGet3(in), KatGet3(in + 3), KatGetF(in + 6), KatGetF(in + 7),
                                              KatGetF(in + 8), KatGetF(in + 9)));
            break;
        case KAT_SELECT_NEIGHBOR: {
            PCG32 r = KatRng(in + 2);
            SelectSpatialNeighborR(in[0], in[1], 10u, r, out[0], out[1]);
            KatPut64(out + 2, r.state);
            break;
        }
        case KAT_JACOBIAN:
            KatPutF(out, oracle_ctx::ReconJacobian(KatGet3(in), KatGet3(in + 3), KatGet3(in + 6), KatGet3(in + 9)));
            break;
        case KAT_RESERVOIR: {
            PCG32 r = KatRng(in);
            Reservoir<KatSample> res;
            res.wSum = KatGetF(in + 4);
            res.confidence = KatGetF(in + 5);
            res.sample.f = KatGet3(in + 6);
            res.sample.id = KAT_RES_STEPS;
            const uint32_t* c = in + 9;
            for (uint32_t st = 0; st < KAT_RES_STEPS; ++st, c += 5) {
                KatSample k;
                k.f = KatGet3(c + 2);
                k.id = st;
                out[3 * st] = res.Update(k, KatGetF(c), r, KatGetF(c + 1)) ? 1u : 0u;
                KatPutF(out + 3 * st + 1, res.wSum);
                KatPutF(out + 3 * st + 2, res.confidence);
            }
            res.FinalizeGRIS();
            uint32_t* o = out + 3 * KAT_RES_STEPS;
            o[0] = res.sample.id;
            KatPutF(o + 1, res.wSum);
            KatPut64(o + 2, r.state);
            break;
        }
        case KAT_GGX:
            KatPutF(out, D_GGX(KatGetF(in), KatGetF(in + 3)));
            KatPutF(out + 1, V_SmithJointGGX(KatGetF(in + 1), KatGetF(in + 2), KatGetF(in + 3)));
            KatPut3(out + 2, FresnelSchlick(KatGet3(in + 5), KatGetF(in + 4)));
            break;
        case KAT_CAMERA_RAY: {
            CameraData cd;
            cd.pos = KatGet3(in);
            cd.U = KatGet3(in + 3);
            cd.V = KatGet3(in + 6);
            cd.W = KatGet3(in + 9);
            vec3 o, d;
            vec2 vp;
            vp.x = KatGetF(in + 12);
            vp.y = KatGetF(in + 13);
            SpawnCameraRay(cd, vp, o, d);
            KatPut3(out, d);
            break;
        }
        default:
            break;
    }
}
}  // namespace

int oracle_kat(int fn, const void* in, uint32_t n, void* out) {
    static const int kIn[] = KAT_IN_WORDS;
    static const int kOut[] = KAT_OUT_WORDS;
    if (fn < 1 || fn > KAT_NUM_FN) return CRISB_ERR_INVALID_ARGUMENT;
    const uint32_t* i = static_cast<const uint32_t*>(in);
    uint32_t* o = static_cast<uint32_t*>(out);
    for (uint32_t k = 0; k < n; ++k)
        KatEval(fn, i + static_cast<size_t>(k) * kIn[fn], o + static_cast<size_t>(k) * kOut[fn]);
    return CRISB_OK;
}

int oracle_kat_emitter(const crisb_emitter* ems, uint32_t num_emitters, const float* faces, const uint64_t* states,
                       uint32_t n, float* out, uint64_t* state_out) {
    if (!ems || num_emitters == 0) return CRISB_ERR_INVALID_ARGUMENT;
    std::vector<EmitterData> table(num_emitters);
    for (uint32_t e = 0; e < num_emitters; ++e) {
        table[e].color = vec3(ems[e].color[0], ems[e].color[1], ems[e].color[2]);
        for (uint32_t f = 0; f < ems[e].num_faces; ++f)
            for (int c = 0; c < 3; ++c) {
                const float* v = faces + 9 * (static_cast<size_t>(ems[e].first_face) + f) + 3 * c;
                table[e].faces.push_back(vec3(v[0], v[1], v[2]));
            }
    }
    for (uint32_t k = 0; k < n; ++k) {
        PCG32 r;
        r.state = states[2 * k];
        r.inc = states[2 * k + 1];
        const EmitterSample s = SampleEmitterFrom(table, r);
        const float v[6] = {s.pos.x, s.pos.y, s.pos.z, s.color.x, s.color.y, s.color.z};
        std::memcpy(out + 6 * static_cast<size_t>(k), v, sizeof v);
        state_out[k] = r.state;
    }
    return CRISB_OK;
}

}  // extern "C"
