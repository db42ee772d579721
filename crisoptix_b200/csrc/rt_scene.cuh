// rt_scene.cuh -- device view of the scene: BVH traversal, surface
// interactions, the reference BRDF and emitter sampling.
//
// Replaces OptiX's optixTrace + __closesthit__mesh / __miss__* programs
// (include/graph/trace.h:25-88, shader/mesh_hit.cu:17-69, shader/miss.cu) and
// the ggx direct callables (shader/brdf.cu:99-337).  Hit semantics: a
// triangle is hit when tmin < t < tmax; the closest hit is the smallest t with
// ties going to the lower triangle index, so the result does not depend on the
// traversal order.
#pragma once

#include "bvh_build.h"
#include "rt_common.cuh"

namespace crisb {

// device error word bits
constexpr int kDevErrStack = 1;
constexpr int kDevErrIterations = 2;
constexpr int kDevErrKnn = 4;

constexpr int kTraversalStack = 64;
// visit caps: a closest-hit query visits well under a thousand nodes; the
// caps only bound the work of a malformed tree (the error word records it)
constexpr uint32_t kMaxNodeVisits = 1u << 16;
constexpr uint32_t kKnnMaxVisits = 1u << 21;
// robust slab test: tfar *= 1 + 2*gamma(3) (Ize 2013, "Robust BVH Ray Traversal")
constexpr float kSlabFarScale = 1.0000003576f;

// BVH2 node of the prefix-endpoint search structure: boxes of both children
// + child links.  A child link >= 0 is an inner node; a negative link
// -1-first marks a leaf of `count` entries starting at `first` in leaf order.
struct BvhNode {
    float4 a;  // l.lo.xyz, l.hi.x
    float4 b;  // l.hi.yz, r.lo.xy
    float4 c;  // r.lo.z, r.hi.xyz
    int4 d;    // left link, right link, left count, right count
};

struct SceneView {
    const Bvh4Node* nodes;  // 4-wide scene BVH, root at 0 (when qnodes is null)
    const Bvh8QNode* qnodes = nullptr;  // compressed 8-wide scene BVH, root at 0, or null
    const float4* tris;   // 3 per triangle in leaf order; tris[3i+2].w = triangle index bits
    const float4* shade;  // 5 per triangle in scene order: p0 p1 p2 n0 n1 n2 material
    const crisb_material* mats;
    const crisb_emitter* emitters;
    const float* emitter_faces;
    uint32_t num_emitters;
    uint32_t num_tris;
    int* err;
    // [closest, shadow] or null; shift kernels get a view offset by 2 so
    // their rays land in [2, 3] and their job count in [4]
    unsigned long long* ray_count;
    unsigned long long* trav_count;  // [node visits, triangle tests] or null
    // textures (null without): per-triangle corner uvs in scene order, per
    // material (diffuse, specular, roughness, -) texture or -1, texel words
    // (RGBA8, first row first) and per texture (first word, width, height, -)
    const float2* uvs = nullptr;
    const int4* mat_tex = nullptr;
    const uint32_t* texels = nullptr;
    const uint4* tex_info = nullptr;
};

struct RayPre {
    V3 org, dir, inv;
    int kx, ky, kz;
    float sx, sy, sz;
};

RT_HD float rcp_box(float v) {
    if (fabsf(v) < 1e-30f) v = copysignf(1e-30f, v);
    return 1.0f / v;
}

RT_HD RayPre make_ray(V3 o, V3 d) {
    RayPre r;
    r.org = o;
    r.dir = d;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) {
        kz = 1;
        m = ay;
    }
    if (az > m) kz = 2;
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (comp(d, kz) < 0.0f) {
        const int t = kx;
        kx = ky;
        ky = t;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    const float dz = comp(d, kz);
    r.sx = comp(d, kx) / dz;
    r.sy = comp(d, ky) / dz;
    r.sz = 1.0f / dz;
    r.inv = V3{rcp_box(d.x), rcp_box(d.y), rcp_box(d.z)};
    return r;
}

// Watertight ray/triangle test (Woop, Benthin & Wald, JCGT 2013).  u and v
// are the barycentric weights of p1 and p2 (OptiX's convention).
RT_HD bool intersect_tri(const RayPre& r, V3 p0, V3 p1, V3 p2, float tmin, float tmax, float& t_out,
                         float& u_out, float& v_out) {
    const V3 A = p0 - r.org, B = p1 - r.org, C = p2 - r.org;
    const float akz = comp(A, r.kz), bkz = comp(B, r.kz), ckz = comp(C, r.kz);
    const float Ax = comp(A, r.kx) - r.sx * akz;
    const float Ay = comp(A, r.ky) - r.sy * akz;
    const float Bx = comp(B, r.kx) - r.sx * bkz;
    const float By = comp(B, r.ky) - r.sy * bkz;
    const float Cx = comp(C, r.kx) - r.sx * ckz;
    const float Cy = comp(C, r.ky) - r.sy * ckz;
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
    const float Az = r.sz * akz;
    const float Bz = r.sz * bkz;
    const float Cz = r.sz * ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float rcp_det = 1.0f / det;
    const float t = T * rcp_det;
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = V * rcp_det;
    v_out = W * rcp_det;
    return true;
}

RT_D bool slab(const RayPre& r, float lox, float loy, float loz, float hix, float hiy, float hiz, float tmin,
               float tmax, float& tnear) {
    float t0 = (lox - r.org.x) * r.inv.x, t1 = (hix - r.org.x) * r.inv.x;
    float tn = fminf(t0, t1), tf = fmaxf(t0, t1);
    t0 = (loy - r.org.y) * r.inv.y;
    t1 = (hiy - r.org.y) * r.inv.y;
    tn = fmaxf(tn, fminf(t0, t1));
    tf = fminf(tf, fmaxf(t0, t1));
    t0 = (loz - r.org.z) * r.inv.z;
    t1 = (hiz - r.org.z) * r.inv.z;
    tn = fmaxf(tn, fminf(t0, t1));
    tf = fminf(tf, fmaxf(t0, t1));
    tn = fmaxf(tn, tmin);
    tf = fminf(tf, tmax);
    tnear = tn;
    return tn <= tf * kSlabFarScale;
}

struct TraceResult {
    uint32_t prim;  // CRISB_INVALID_PRIM: miss
    float t, u, v;
};

RT_D void dev_error(const SceneView& s, int code) {
    if (s.err) atomicOr(s.err, code);
}

// statistics: one warp-aggregated atomic per call site
RT_D void count_ray(const SceneView& s, int which) {
    if (!s.ray_count) return;
    const unsigned m = __activemask();
    if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&s.ray_count[which], static_cast<unsigned long long>(__popc(m)));
}

// Traversal of one ray as a resumable state: step() visits one node (both
// child boxes, leaf triangles) and reports whether the ray is finished.  The
// stack is kept apart from the scalar state so the latter stays in registers.
struct TravStack {
    int node[kTraversalStack];
    float t[kTraversalStack];
};

template <bool kAnyHit>
struct Trav {
    RayPre r;
    float tmin, tmax;
    TraceResult best;
    int sp, cur;
    uint32_t visits, tris;

    RT_D void init(const RayPre& ray, float t0, float t1) {
        r = ray;
        tmin = t0;
        tmax = t1;
        best = TraceResult{CRISB_INVALID_PRIM, t1, 0.0f, 0.0f};
        sp = 0;
        cur = 0;
        visits = 0;
        tris = 0;
    }

    RT_D float bound() const { return best.prim == CRISB_INVALID_PRIM ? tmax : best.t; }

    // slab() with the near / far plane of each axis chosen by the sign of the
    // inverse direction: the same values as the min / max form, since
    // (lo - o) * inv <= (hi - o) * inv exactly when inv > 0 (rounding is
    // monotonic) and the inverse direction is never zero or NaN.  (One FMA per
    // plane against a per-ray org * inv measured no faster: 13.67 against
    // 13.59 ms of traversal per 1080p frame; the traversal is latency-bound.)
    RT_D bool slab_nf(float nx, float fx, float ny, float fy, float nz, float fz, float tmax_, float& tnear) const {
        float tn = (nx - r.org.x) * r.inv.x, tf = (fx - r.org.x) * r.inv.x;
        tn = fmaxf(tn, (ny - r.org.y) * r.inv.y);
        tf = fminf(tf, (fy - r.org.y) * r.inv.y);
        tn = fmaxf(tn, (nz - r.org.z) * r.inv.z);
        tf = fminf(tf, (fz - r.org.z) * r.inv.z);
        tn = fmaxf(tn, tmin);
        tf = fminf(tf, tmax_);
        tnear = tn;
        return tn <= tf * kSlabFarScale;
    }

    // triangles [first, first + count) of the leaf order; true when an
    // any-hit query is answered
    RT_D bool leaf(const SceneView& s, int first, int count) {
        tris += static_cast<uint32_t>(count);
        for (int k = 0; k < count; ++k) {
            const float4 q0 = __ldg(&s.tris[3 * (first + k) + 0]);
            const float4 q1 = __ldg(&s.tris[3 * (first + k) + 1]);
            const float4 q2 = __ldg(&s.tris[3 * (first + k) + 2]);
            const uint32_t prim = __float_as_uint(q2.w);
            float t, u, v;
            if (!intersect_tri(r, V3{q0.x, q0.y, q0.z}, V3{q1.x, q1.y, q1.z}, V3{q2.x, q2.y, q2.z}, tmin, tmax, t,
                               u, v))
                continue;
            if (kAnyHit) {
                best.prim = prim;
                best.t = t;
                return true;
            }
            if (best.prim == CRISB_INVALID_PRIM || t < best.t || (t == best.t && prim < best.prim)) {
                best.prim = prim;
                best.t = t;
                best.u = u;
                best.v = v;
            }
        }
        return false;
    }

    // one wide node: the four child boxes, the triangles of every leaf child
    // that is hit, then the nearest inner child next and the others pushed
    // far to near
    RT_D bool step(const SceneView& s, TravStack& st) {
        if (s.num_tris == 0) return true;
        if (++visits > kMaxNodeVisits) {
            dev_error(s, kDevErrIterations);
            return true;
        }
        // rows of the node: lo_x hi_x lo_y hi_y lo_z hi_z (kBvhWidth / 4
        // float4 per plane over the children), links, counts.  Per axis the
        // near plane is lo for a positive inverse direction and hi otherwise,
        // so min(t_lo, t_hi) of the slab test is the near plane's t.
        constexpr int kQ = kBvhWidth / 4;
        const float4* np = reinterpret_cast<const float4*>(s.nodes + cur);
        const int sx = signbit(r.inv.x) ? 1 : 0, sy = signbit(r.inv.y) ? 1 : 0, sz = signbit(r.inv.z) ? 1 : 0;
        const float bnd = bound();
        int link[kBvhWidth];
        int cnt[kBvhWidth];
        float tn[kBvhWidth];
        bool hit[kBvhWidth];
#pragma unroll
        for (int j = 0; j < kQ; ++j) {
            const float4 nx = __ldg(np + sx * kQ + j), fx = __ldg(np + (1 - sx) * kQ + j);
            const float4 ny = __ldg(np + (2 + sy) * kQ + j), fy = __ldg(np + (3 - sy) * kQ + j);
            const float4 nz = __ldg(np + (4 + sz) * kQ + j), fz = __ldg(np + (5 - sz) * kQ + j);
            const int4 lk = __ldg(reinterpret_cast<const int4*>(np + 6 * kQ + j));
            const int4 ct = __ldg(reinterpret_cast<const int4*>(np + 7 * kQ + j));
            link[4 * j + 0] = lk.x;
            link[4 * j + 1] = lk.y;
            link[4 * j + 2] = lk.z;
            link[4 * j + 3] = lk.w;
            cnt[4 * j + 0] = ct.x;
            cnt[4 * j + 1] = ct.y;
            cnt[4 * j + 2] = ct.z;
            cnt[4 * j + 3] = ct.w;
            hit[4 * j + 0] = lk.x != kNoChild && slab_nf(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, bnd, tn[4 * j + 0]);
            hit[4 * j + 1] = lk.y != kNoChild && slab_nf(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, bnd, tn[4 * j + 1]);
            hit[4 * j + 2] = lk.z != kNoChild && slab_nf(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, bnd, tn[4 * j + 2]);
            hit[4 * j + 3] = lk.w != kNoChild && slab_nf(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, bnd, tn[4 * j + 3]);
        }
#pragma unroll
        for (int c = 0; c < kBvhWidth; ++c) {
            if (!hit[c] || link[c] >= 0) continue;
            hit[c] = false;
            if (leaf(s, -1 - link[c], cnt[c])) return true;
        }
        // inner children still in front of the closest hit, nearest first
        const float cut = bound() * kSlabFarScale;
#pragma unroll
        for (int c = 0; c < kBvhWidth; ++c)
            if (!hit[c] || tn[c] > cut) tn[c] = INFINITY;
        auto cswap = [&](int i, int j) {
            if (tn[j] < tn[i]) {
                const float t = tn[i];
                tn[i] = tn[j];
                tn[j] = t;
                const int l = link[i];
                link[i] = link[j];
                link[j] = l;
            }
        };
        if (kAnyHit) {
            // any hit ends the ray: the visiting order only moves work
            // around, so the first child hit goes next and the rest are pushed
            // as they come
            int nh = 0;
#pragma unroll
            for (int c = 0; c < kBvhWidth; ++c) nh += tn[c] < INFINITY ? 1 : 0;
            if (nh > 0) {
                if (sp + nh - 1 > kTraversalStack) {
                    dev_error(s, kDevErrStack);
                    return true;
                }
                bool first = true;
#pragma unroll
                for (int c = 0; c < kBvhWidth; ++c) {
                    if (!(tn[c] < INFINITY)) continue;
                    if (first) {
                        cur = link[c];
                        first = false;
                    } else {
                        st.node[sp] = link[c];
                        st.t[sp++] = tn[c];
                    }
                }
                return false;
            }
        } else if (kBvhWidth == 4) {
            cswap(0, 1);
            cswap(2, 3);
            cswap(0, 2);
            cswap(1, 3);
            cswap(1, 2);
        } else {
            // Batcher's odd-even merge network for 8 keys (19 comparators)
            cswap(0, 1);
            cswap(2, 3);
            cswap(4, 5);
            cswap(6, 7);
            cswap(0, 2);
            cswap(1, 3);
            cswap(4, 6);
            cswap(5, 7);
            cswap(1, 2);
            cswap(5, 6);
            cswap(0, 4);
            cswap(1, 5);
            cswap(2, 6);
            cswap(3, 7);
            cswap(2, 4);
            cswap(3, 5);
            cswap(1, 2);
            cswap(3, 4);
            cswap(5, 6);
        }
        int nh = 0;
#pragma unroll
        for (int c = 0; c < kBvhWidth; ++c) nh += tn[c] < INFINITY ? 1 : 0;
        if (nh > 0) {
            if (sp + nh - 1 > kTraversalStack) {
                dev_error(s, kDevErrStack);
                return true;
            }
#pragma unroll
            for (int j = kBvhWidth - 1; j >= 1; --j) {
                if (j < nh) {
                    st.node[sp] = link[j];
                    st.t[sp++] = tn[j];
                }
            }
            cur = link[0];
            return false;
        }
        // pop, skipping entries now beyond the closest hit
        while (sp > 0) {
            --sp;
            if (st.t[sp] <= bound() * kSlabFarScale) {
                cur = st.node[sp];
                return false;
            }
        }
        return true;
    }
};

// statistics: node visits and triangle tests of a finished ray (one
// warp-aggregated atomic each)
RT_D void count_trav(const SceneView& s, uint32_t visits, uint32_t tris) {
    if (!s.trav_count) return;
    const unsigned m = __activemask();
    const uint32_t v = __reduce_add_sync(m, visits), t = __reduce_add_sync(m, tris);
    if ((threadIdx.x & 31) == __ffs(m) - 1) {
        atomicAdd(&s.trav_count[0], static_cast<unsigned long long>(v));
        atomicAdd(&s.trav_count[1], static_cast<unsigned long long>(t));
    }
}

// ---- compressed 8-wide tree ------------------------------------------------------
constexpr int kQStack = 32;

// 2^e for a grid exponent e in [-126, 127]
RT_D float exp2_int(int e) { return __int_as_float((e + 127) << 23); }

// packed pairs of floats (sm_100 f32x2 arithmetic: two IEEE round-to-nearest
// operations per instruction) and three-input min / max
RT_D uint64_t pk2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
RT_D void upk2(uint64_t v, float& lo, float& hi) { asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v)); }
RT_D uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
RT_D uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
RT_D float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
RT_D float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Closest or first hit over the compressed tree (Bvh8QNode).  A child plane
// at grid step q is met at t = q * (2^e * inv) + (p - o) * inv, one FMA per
// plane on two per-node terms per axis; against the subtract-and-multiply
// form on the decoded plane this adds roundings of |p - o| and |X - o| size,
// far inside the box margin, so the test stays conservative and the hits are
// those of testing every triangle (the tree only changes the speed).  Hit
// children go into one mask: inner children at bit 24 + (slot ^ octant), leaf
// triangles at their bits 0-23.  Inner children are taken lowest bit first
// (near to far in the octant order); the rest of a node's hit inner children
// wait on the stack as one group (child base, bits, inner mask, the least
// entry t of the group, which culls the group once a closer hit is known).
// Traversal state of one ray over the compressed tree; step() visits one
// node (its eight child boxes, then the triangles of its hit leaf children)
// and picks the next, reporting when the ray is finished.  `any`: first hit
// (occlusion) instead of the closest.  The group stack is kept apart so the
// scalar state stays in registers.
struct QTrav {
    RayPre r;
    float tmin, tmax0;
    TraceResult best;
    uint32_t node, visits, ntris;
    int sp;
    uint32_t oct;
    bool any;

    RT_D void init(const RayPre& ray, float t0, float t1, bool any_hit) {
        r = ray;
        tmin = t0;
        tmax0 = t1;
        best = TraceResult{CRISB_INVALID_PRIM, t1, 0.0f, 0.0f};
        node = 0;
        visits = 0;
        ntris = 0;
        sp = 0;
        oct = (signbit(r.inv.x) ? 1u : 0u) | (signbit(r.inv.y) ? 2u : 0u) | (signbit(r.inv.z) ? 4u : 0u);
        any = any_hit;
    }

    RT_D bool step(const SceneView& s, uint4* stk) {
        if (s.num_tris == 0) return true;
        if (++visits > kMaxNodeVisits) {
            dev_error(s, kDevErrIterations);
            return true;
        }
        const uint32_t ox = oct & 1u, oy = (oct >> 1) & 1u, oz = oct >> 2;
        const float4* np = reinterpret_cast<const float4*>(s.qnodes + node);
        const float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
        const uint32_t ew = __float_as_uint(n0.w);
        const float sx = exp2_int(static_cast<int>(static_cast<int8_t>(ew & 0xffu))) * r.inv.x;
        const float sy = exp2_int(static_cast<int>(static_cast<int8_t>((ew >> 8) & 0xffu))) * r.inv.y;
        const float sz = exp2_int(static_cast<int>(static_cast<int8_t>((ew >> 16) & 0xffu))) * r.inv.z;
        const float bx = (n0.x - r.org.x) * r.inv.x;
        const float by = (n0.y - r.org.y) * r.inv.y;
        const float bz = (n0.z - r.org.z) * r.inv.z;
        // per axis (near, far) pairs share the scale and the offset
        const uint64_t sx2 = pk2(sx, sx), sy2 = pk2(sy, sy), sz2 = pk2(sz, sz);
        const uint64_t bx2 = pk2(bx, bx), by2 = pk2(by, by), bz2 = pk2(bz, bz);
        const uint64_t m23 = pk2(-8388608.0f, -8388608.0f);
        const float bnd = best.t;
        uint32_t hits = 0;
        float gmin = INFINITY;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t meta = __float_as_uint(h ? n1.w : n1.z);
            const uint32_t lx = __float_as_uint(h ? n2.y : n2.x), hx = __float_as_uint(h ? n3.w : n3.z);
            const uint32_t ly = __float_as_uint(h ? n2.w : n2.z), hy = __float_as_uint(h ? n4.y : n4.x);
            const uint32_t lz = __float_as_uint(h ? n3.y : n3.x), hz = __float_as_uint(h ? n4.w : n4.z);
            const uint32_t nx = ox ? hx : lx, fx = ox ? lx : hx;
            const uint32_t ny = oy ? hy : ly, fy = oy ? ly : hy;
            const uint32_t nz = oz ? hz : lz, fz = oz ? lz : hz;
            // per byte: inner children have meta bits 4 and 3 set
            const uint32_t inner4 = (meta & (meta << 1)) & 0x10101010u;
            const uint32_t bit4 = (meta ^ ((inner4 >> 4) * oct)) & 0x1f1f1f1fu;
            const uint32_t cnt4 = (meta >> 5) & 0x07070707u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                // byte j of the near and far words as the floats 2^23 + q,
                // minus 2^23 (exact), then t = q * s + b per plane
                const uint32_t sel = 0x7440u + static_cast<uint32_t>(j);
                const uint64_t qx = add2(pk2(__uint_as_float(__byte_perm(nx, 0x4B000000u, sel)),
                                             __uint_as_float(__byte_perm(fx, 0x4B000000u, sel))), m23);
                const uint64_t qy = add2(pk2(__uint_as_float(__byte_perm(ny, 0x4B000000u, sel)),
                                             __uint_as_float(__byte_perm(fy, 0x4B000000u, sel))), m23);
                const uint64_t qz = add2(pk2(__uint_as_float(__byte_perm(nz, 0x4B000000u, sel)),
                                             __uint_as_float(__byte_perm(fz, 0x4B000000u, sel))), m23);
                float tnx, tfx, tny, tfy, tnz, tfz;
                upk2(fma2(qx, sx2, bx2), tnx, tfx);
                upk2(fma2(qy, sy2, by2), tny, tfy);
                upk2(fma2(qz, sz2, bz2), tnz, tfz);
                const float tn = max3f(tnx, tny, fmaxf(tnz, tmin));
                const float tf = min3f(tfx, tfy, fminf(tfz, bnd));
                if (tn <= tf * kSlabFarScale) {
                    const uint32_t sh = 8u * static_cast<uint32_t>(j);
                    hits |= ((cnt4 >> sh) & 7u) << ((bit4 >> sh) & 31u);
                    if ((inner4 >> (sh + 4u)) & 1u) gmin = fminf(gmin, tn);
                }
            }
        }
        // the node's leaf triangles
        const uint32_t tbase = __float_as_uint(n1.y);
        uint32_t tmask = hits & 0x00ffffffu;
        while (tmask) {
            const uint32_t k = static_cast<uint32_t>(__ffs(tmask) - 1);
            tmask &= tmask - 1u;
            ++ntris;
            if (triangle(s, tbase + k)) return true;
        }
        // next node: this node's nearest inner child, else a group from the stack
        uint32_t gbase = __float_as_uint(n1.x), gbits = hits >> 24, gim = ew >> 24;
        float gt = gmin;
        if (!any && gt > best.t * kSlabFarScale) gbits = 0;
        if (gbits == 0) {
            while (sp > 0) {
                const uint4 e = stk[--sp];
                if (any || __uint_as_float(e.z) <= best.t * kSlabFarScale) {
                    gbase = e.x;
                    gbits = e.y & 0xffu;
                    gim = e.y >> 8;
                    gt = __uint_as_float(e.z);
                    break;
                }
            }
            if (gbits == 0) return true;
        }
        const uint32_t b = static_cast<uint32_t>(__ffs(gbits) - 1);
        gbits &= gbits - 1u;
        const uint32_t slot = b ^ oct;
        node = gbase + static_cast<uint32_t>(__popc(gim & ((1u << slot) - 1u)));
        if (gbits) {
            if (sp >= kQStack) {
                dev_error(s, kDevErrStack);
                return true;
            }
            stk[sp++] = make_uint4(gbase, gbits | (gim << 8), __float_as_uint(gt), 0u);
        }
        return false;
    }

    // one leaf triangle; true when a first-hit query is answered
    RT_D bool triangle(const SceneView& s, uint32_t slot) {
        const float4 q0 = __ldg(&s.tris[3 * slot + 0]);
        const float4 q1 = __ldg(&s.tris[3 * slot + 1]);
        const float4 q2 = __ldg(&s.tris[3 * slot + 2]);
        const uint32_t prim = __float_as_uint(q2.w);
        float t, u, v;
        if (!intersect_tri(r, V3{q0.x, q0.y, q0.z}, V3{q1.x, q1.y, q1.z}, V3{q2.x, q2.y, q2.z}, tmin, tmax0, t,
                           u, v))
            return false;
        if (any) {
            best.prim = prim;
            best.t = t;
            return true;
        }
        if (best.prim == CRISB_INVALID_PRIM || t < best.t || (t == best.t && prim < best.prim)) {
            best.prim = prim;
            best.t = t;
            best.u = u;
            best.v = v;
        }
        return false;
    }
};

template <bool kAnyHit>
RT_D TraceResult traverse_q(const SceneView& s, const RayPre& r, float tmin, float tmax) {
    QTrav t;
    uint4 stk[kQStack];
    t.init(r, tmin, tmax, kAnyHit);
    while (!t.step(s, stk)) {
    }
    count_trav(s, t.visits, t.ntris);
    return t.best;
}

// closest or first hit over the 4-wide tree
template <bool kAnyHit>
RT_D TraceResult traverse_wide4(const SceneView& s, const RayPre& r, float tmin, float tmax) {
    Trav<kAnyHit> t;
    TravStack st;
    t.init(r, tmin, tmax);
    while (!t.step(s, st)) {
    }
    count_trav(s, t.visits, t.tris);
    return t.best;
}

// node formats of the scene tree
constexpr int kFmtWide4 = 0;
constexpr int kFmtCompressed8 = 1;

// traversal for a format fixed at compile time (the queue traversal kernel
// is instantiated per format, so it carries only one traversal)
template <int kFmt, bool kAnyHit>
RT_D TraceResult traverse_fmt(const SceneView& s, const RayPre& r, float tmin, float tmax) {
    if (kFmt == kFmtCompressed8) return traverse_q<kAnyHit>(s, r, tmin, tmax);
    return traverse_wide4<kAnyHit>(s, r, tmin, tmax);
}

// Closest hit (any_hit == false) or first hit (any_hit == true) over the
// scene tree, whichever format it has.
template <bool kAnyHit>
RT_D TraceResult traverse(const SceneView& s, const RayPre& r, float tmin, float tmax) {
    if (s.qnodes) return traverse_q<kAnyHit>(s, r, tmin, tmax);
    return traverse_wide4<kAnyHit>(s, r, tmin, tmax);
}

// ---- interactions -------------------------------------------------------------
struct ShadeTri {
    V3 p0, p1, p2, n0, n1, n2;
    uint32_t mat;
};

RT_D ShadeTri load_shade(const SceneView& s, uint32_t prim) {
    const float4* q = s.shade + 5 * static_cast<size_t>(prim);
    const float4 a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
    ShadeTri t;
    t.p0 = V3{a.x, a.y, a.z};
    t.p1 = V3{a.w, b.x, b.y};
    t.p2 = V3{b.z, b.w, c.x};
    t.n0 = V3{c.y, c.z, c.w};
    t.n1 = V3{d.x, d.y, d.z};
    t.n2 = V3{d.w, e.x, e.y};
    t.mat = __float_as_uint(e.z);
    return t;
}

// InterpolateBary (include/graph/Interaction.h:18-25)
RT_HD V3 interp(float bu, float bv, V3 v0, V3 v1, V3 v2) {
    return ((1.0f - bu - bv) * v0) + (bu * v1) + (bv * v2);
}

// optixTrace + __closesthit__mesh / __miss__main: interaction with the
// normalised interpolated normal.  On a miss only valid and dir change.
RT_D void trace_closest(const SceneView& s, V3 o, V3 d, float tmin, float tmax, Isect& it) {
    count_ray(s, 0);
    const RayPre r = make_ray(o, d);
    const TraceResult h = traverse<false>(s, r, tmin, tmax);
    it.dir = d;
    if (h.prim == CRISB_INVALID_PRIM) {
        it.valid = false;
        return;
    }
    it.valid = true;
    it.prim = h.prim;
    it.bu = h.u;
    it.bv = h.v;
    const ShadeTri t = load_shade(s, h.prim);
    it.pos = interp(it.bu, it.bv, t.p0, t.p1, t.p2);
    it.nrm = normalize(interp(it.bu, it.bv, t.n0, t.n1, t.n2));
}

// TraceOcclusion (include/graph/trace.h:64-88)
RT_D bool occluded(const SceneView& s, V3 o, V3 d, float tmin, float tmax) {
    count_ray(s, 1);
    const RayPre r = make_ray(o, d);
    return traverse<true>(s, r, tmin, tmax).prim != CRISB_INVALID_PRIM;
}

// Interaction(PackedInteraction, transforms) (include/graph/Interaction.h:115-172):
// interpolated position and unnormalised normal.
RT_D Isect unpack(const SceneView& s, const Hit& h) {
    Isect it;
    it.valid = h.valid() && h.prim < s.num_tris;
    it.prim = h.prim;
    it.bu = h.bu;
    it.bv = h.bv;
    it.dir = h.dir;
    it.pos = splat(0.0f);
    it.nrm = splat(0.0f);
    if (!it.valid) return it;
    const ShadeTri t = load_shade(s, h.prim);
    it.pos = interp(it.bu, it.bv, t.p0, t.p1, t.p2);
    it.nrm = interp(it.bu, it.bv, t.n0, t.n1, t.n2);
    return it;
}

RT_D uint32_t material_of(const SceneView& s, uint32_t prim) {
    return __float_as_uint(__ldg(&s.shade[5 * static_cast<size_t>(prim) + 4].z));
}

// ---- BRDF (shader/brdf.cu) ---------------------------------------------------------
constexpr float kPi = 3.14159265358979323846264f;

struct BrdfEval {
    V3 brdf;
    float pdf;
    V3 emission;
    float roughness;
};
struct BrdfSample {
    V3 dir;
    V3 brdf;
    float pdf;
    float roughness;
};
struct MatVals {
    V3 diff, f0, emission;
    float rough;
};

// tex2D<float4> of the reference's texture objects (src/Texture.cpp:44-72:
// normalised coordinates, cudaAddressModeWrap, cudaFilterModeLinear,
// cudaReadModeNormalizedFloat on uchar4 texels), DEFINED in software after the
// CUDA programming guide's linear-filtering formula: the coordinate's
// fraction scaled to texels, x_B = x - 0.5, i = floor(x_B), alpha = frac(x_B)
// held with 8 fractional bits (rounded here), neighbours i and i + 1 wrapped,
// result = (1-a)(1-b) T[i,j] + a(1-b) T[i+1,j] + (1-a) b T[i,j+1] + a b
// T[i+1,j+1] in that order, texel channels c / 255.  Non-finite
// coordinates read as 0.
RT_HD float tex_frac_weight(float a) { return floorf(a * 256.0f + 0.5f) * (1.0f / 256.0f); }

RT_D float4 texel_rgba(uint32_t w) {
    return make_float4(static_cast<float>(w & 0xffu) / 255.0f, static_cast<float>((w >> 8) & 0xffu) / 255.0f,
                       static_cast<float>((w >> 16) & 0xffu) / 255.0f, static_cast<float>(w >> 24) / 255.0f);
}

RT_D float4 tex_sample(const uint32_t* texels, const uint4* tex_info, int tex, float u, float v) {
    const uint4 info = tex_info[tex];
    const int W = static_cast<int>(info.y), H = static_cast<int>(info.z);
    if (!(u - u == 0.0f)) u = 0.0f;  // NaN or infinite
    if (!(v - v == 0.0f)) v = 0.0f;
    const float x = (u - floorf(u)) * static_cast<float>(W) - 0.5f;
    const float y = (v - floorf(v)) * static_cast<float>(H) - 0.5f;
    const float xf = floorf(x), yf = floorf(y);
    const float a = tex_frac_weight(x - xf), b = tex_frac_weight(y - yf);
    int i0 = static_cast<int>(xf) % W, j0 = static_cast<int>(yf) % H;
    if (i0 < 0) i0 += W;
    if (j0 < 0) j0 += H;
    const int i1 = i0 + 1 == W ? 0 : i0 + 1, j1 = j0 + 1 == H ? 0 : j0 + 1;
    const uint32_t* t = texels + info.x;
    // ((w00 T00 + w10 T10) + w01 T01) + w11 T11, one texel live at a time
    float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // set by the first add
    auto add = [&](uint32_t word, float w, bool first) {
        const float4 c = texel_rgba(word);
        acc = first ? make_float4(w * c.x, w * c.y, w * c.z, w * c.w)
                    : make_float4(acc.x + w * c.x, acc.y + w * c.y, acc.z + w * c.z, acc.w + w * c.w);
    };
    add(__ldg(t + static_cast<size_t>(j0) * W + i0), (1.0f - a) * (1.0f - b), true);
    add(__ldg(t + static_cast<size_t>(j0) * W + i1), a * (1.0f - b), false);
    add(__ldg(t + static_cast<size_t>(j1) * W + i0), (1.0f - a) * b, false);
    add(__ldg(t + static_cast<size_t>(j1) * W + i1), a * b, false);
    return acc;
}

struct TexVals {
    V3 diff, f0;
    float rough;
};

// GetFromTexIfPossible for a textured material (mt: diffuse, specular,
// roughness texture or -1) at uv = InterpolateBary of the corner uvs
// (include/graph/Interaction.h:171).  Inlined: a non-inlined form raised
// the shading kernel from 128 to 156 registers (the call's saved registers).
RT_D TexVals textured_vals(const float2* uvs, const uint32_t* texels, const uint4* tex_info,
                                              int4 mt, uint32_t prim, float bu, float bv, TexVals v) {
    const float2 a = uvs[3 * static_cast<size_t>(prim)], b = uvs[3 * static_cast<size_t>(prim) + 1],
                 c = uvs[3 * static_cast<size_t>(prim) + 2];
    const float w = 1.0f - bu - bv;
    const float u = (w * a.x + bu * b.x) + bv * c.x, t = (w * a.y + bu * b.y) + bv * c.y;
    if (mt.x >= 0) {
        const float4 q = tex_sample(texels, tex_info, mt.x, u, t);
        v.diff = V3{q.x, q.y, q.z};
    }
    if (mt.y >= 0) {
        const float4 q = tex_sample(texels, tex_info, mt.y, u, t);
        v.f0 = V3{q.x, q.y, q.z};
    }
    if (mt.z >= 0) v.rough = tex_sample(texels, tex_info, mt.z, u, t).x;
    return v;
}

// the metal workflow and mix of shader/brdf.cu:129-138 over looked-up values
RT_D MatVals finish_mat(const crisb_material& m, V3 diff, V3 f0, float rough) {
    MatVals v;
    v.diff = diff;
    float metal = 0.0f;
    if (m.spec_usage == CRISB_SPEC_OCC_ROUGH_METAL) {
        rough = f0.y;
        metal = f0.z;
        f0 = splat(1.0f);
    }
    v.f0 = v.diff * (1.0f - metal) + f0 * metal;  // glm::mix
    v.emission = V3{m.emission[0], m.emission[1], m.emission[2]};
    v.rough = rough;
    return v;
}

// material values at an interaction: GetFromTexIfPossible for the diffuse
// colour, specF0 and roughness (shader/brdf.cu:64-97,120-138)
// kTex = false compiles the texture lookup out (kernels instantiated for
// untextured scenes keep their register budget).
template <bool kTex = true>
RT_D MatVals mat_vals(const SceneView& s, const Isect& it) {
    const uint32_t mi = material_of(s, it.prim);
    const crisb_material& m = s.mats[mi];
    TexVals v{V3{m.diffuse[0], m.diffuse[1], m.diffuse[2]}, V3{m.specular[0], m.specular[1], m.specular[2]},
              m.roughness};
    if (kTex && s.mat_tex) {
        const int4 mt = s.mat_tex[mi];
        if (mt.x >= 0 || mt.y >= 0 || mt.z >= 0)
            v = textured_vals(s.uvs, s.texels, s.tex_info, mt, it.prim, it.bu, it.bv, v);
    }
    return finish_mat(m, v.diff, v.f0, v.rough);
}

// the material without its textures (constant values)
RT_D MatVals mat_vals(const crisb_material& m) {
    return finish_mat(m, V3{m.diffuse[0], m.diffuse[1], m.diffuse[2]}, V3{m.specular[0], m.specular[1], m.specular[2]},
                      m.roughness);
}

RT_D float pow5(float x) {
    const float x2 = x * x;
    return x2 * x2 * x;
}
RT_D float d_ggx(float ndoth, float rough) {
    const float a2 = rough * rough;
    const float d = (ndoth * a2 - ndoth) * ndoth + 1.0f;
    return a2 / (kPi * d * d);
}
RT_D float v_smith(float ndotl, float ndotv, float rough) {
    const float a2 = rough * rough;
    const float lv = ndotl * sqrtf(ndotv * ndotv * (1 - a2) + a2);
    const float ll = ndotv * sqrtf(ndotl * ndotl * (1 - a2) + a2);
    return 0.5f / (lv + ll);
}
RT_D V3 fresnel(V3 f0, float vdoth) { return f0 + (splat(1.0f) - f0) * pow5(gmax(0.0f, 1.0f - vdoth)); }
RT_D float diff_prob(const MatVals& m) {
    const float sd = dot(m.diff, splat(1.0f));
    return sd / (dot(m.diff, splat(1.0f)) + dot(m.f0, splat(1.0f)));
}

// brdf * cos and the mixture pdf shared by eval and sample
RT_D void brdf_value(const MatVals& m, V3 nrm, V3 view, V3 light, float ndotl, float ndotv, float dprob, V3& brdf,
                     float& pdf) {
    const V3 diff_brdf = m.diff / kPi;
    V3 spec = splat(0.0f);
    const V3 h = normalize(light + view);
    const float ndoth = dot(h, nrm);
    const float ldoth = dot(h, light);
    if (static_cast<double>(dot(m.f0, m.f0)) > 1e-6) {
        const float d = d_ggx(ndoth, m.rough);
        const float v = v_smith(ndotl, ndotv, m.rough);
        const V3 f = fresnel(m.f0, ldoth);
        spec = d * v * f;
    }
    brdf = (diff_brdf + spec) * ndotl;
    pdf = dprob * ndotl / kPi + (1.0f - dprob) * d_ggx(ndoth, m.rough) * ndoth / (4.0f * ldoth);
}

// __direct_callable__ggx_eval, shader/brdf.cu:115-190
template <bool kTex = true>
RT_D BrdfEval brdf_eval(const SceneView& s, const Isect& it, V3 out_dir) {
    BrdfEval r;
    r.brdf = splat(0.0f);
    r.pdf = 0.0f;
    r.emission = splat(0.0f);
    r.roughness = 0.0f;
    const MatVals m = mat_vals<kTex>(s, it);
    const V3 view = -it.dir;
    const float ndotv = dot(it.nrm, view);
    const float ndotl = dot(it.nrm, out_dir);
    if (ndotv <= 0.0f || ndotl < 0.0f) return r;
    brdf_value(m, it.nrm, view, out_dir, ndotl, ndotv, diff_prob(m), r.brdf, r.pdf);
    r.emission = m.emission;
    r.roughness = m.rough;
    return r;
}

// ComputeLocalFrame (shader/brdf.cu:192-212) applied to a local vector
RT_D V3 local_to_world(V3 z, V3 v) {
    const float sz = (z.z >= 0) ? 1.0f : -1.0f;
    const float a = 1 / (sz + z.z);
    const float ya = z.y * a;
    const float b = z.x * ya;
    const float c = z.x * sz;
    const V3 X = V3{c * z.x * a - 1, sz * b, c};
    const V3 Y = V3{b, z.y * ya - sz, z.y};
    return V3{X.x * v.x + Y.x * v.y + z.x * v.z, X.y * v.x + Y.y * v.y + z.y * v.z,
              X.z * v.x + Y.z * v.y + z.z * v.z};
}

// __direct_callable__ggx_sample, shader/brdf.cu:214-337
template <bool kTex = true>
RT_D BrdfSample brdf_sample(const SceneView& s, const Isect& it, Rng& rng) {
    const MatVals m = mat_vals<kTex>(s, it);
    BrdfSample r;
    r.roughness = m.rough;
    r.dir = splat(0.0f);
    r.brdf = splat(0.0f);
    r.pdf = 0.0f;
    const V3 nrm = it.nrm;
    const V3 view = -it.dir;
    const float ndotv = dot(nrm, view);
    if (ndotv <= 0) return r;
    const float dprob = diff_prob(m);
    V3 dir;
    if (rng.next_float() < dprob) {
        const float phi = rng.next_float() * 2.0f * kPi;
        const float rr = sqrtf(rng.next_float());
        float sp, cp;
        sincos_reduced(phi, sp, cp);
        const float x = rr * cp;
        const float y = rr * sp;
        const float z = sqrtf(gclamp(1.0f - x * x - y * y, 0.0f, 1.0f));
        dir = local_to_world(nrm, V3{x, y, z});
    } else {
        const float u = rng.next_float();
        const float mz = sqrtf(gclamp((1 - u) / (1 + (m.rough * m.rough - 1) * u), 0, 1));
        const float mr = sqrtf(gclamp(1 - mz * mz, 0, 1));
        const float phi = rng.next_float() * 2.0f * kPi;
        float sp, cp;
        sincos_reduced(phi, sp, cp);
        dir = reflect(it.dir, local_to_world(nrm, V3{mr * cp, mr * sp, mz}));
        if (dot(dir, nrm) < 0.0f) return r;
    }
    const float ndotl = dot(nrm, dir);
    r.dir = dir;
    brdf_value(m, nrm, view, dir, ndotl, ndotv, dprob, r.brdf, r.pdf);
    return r;
}

// ---- emitters (include/graph/sample_emitter.h, include/model/Emitter.h:21-54) ----
struct EmitterSample {
    V3 pos;
    V3 color;
    uint32_t index;  // the emitter chosen
};

RT_D EmitterSample sample_emitter(const SceneView& s, Rng& rng) {
    const uint64_t ei = rng.next_u64() % static_cast<uint64_t>(s.num_emitters);
    const crisb_emitter e = s.emitters[ei];
    const uint64_t fi = rng.next_u64() % static_cast<uint64_t>(e.num_faces);
    const float* f = s.emitter_faces + 9 * (static_cast<size_t>(e.first_face) + fi);
    const V3 v0 = V3{f[0], f[1], f[2]}, v1 = V3{f[3], f[4], f[5]}, v2 = V3{f[6], f[7], f[8]};
    float r0 = rng.next_float();
    float r1 = rng.next_float();
    float r2 = rng.next_float();
    const float rsum = r0 + r1 + r2;
    r0 /= rsum;
    r1 /= rsum;
    r2 /= rsum;
    EmitterSample es;
    es.pos = r0 * v0 + r1 * v1 + r2 * v2;
    es.color = V3{e.color[0], e.color[1], e.color[2]};
    es.index = static_cast<uint32_t>(ei);
    return es;
}

}  // namespace crisb
