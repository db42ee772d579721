// knn.cuh -- the prefix-endpoint neighbour search (device side).
//
// Replaces the OptiX custom-primitive acceleration structure over per-pixel
// AABBs and its intersection program (src/PrefixAccelStruct.cpp:14-221,
// shader/prefix_search_hit.cu:9-73).  An entry is an endpoint position with a
// radius; a query point q collects every entry j with |p_j - q| <= r_j and
// keeps the k nearest, ordered by (distance, entry index) -- a deterministic
// definition of the reference's "first k hits in traversal order".  The
// entries sit in an LBVH (lbvh.cuh) whose boxes are conservative: an entry
// that passes the distance test always has q inside its box.
#pragma once

#include "lbvh.cuh"

namespace crisb {

struct KnnView {
    const BvhNode* nodes;
    const float4* leaf;       // leaf order: x, y, z, radius
    const uint32_t* index;    // leaf order -> entry index
    const uint32_t* n;        // number of entries in the structure
};

struct NeighborList {
    float dist[CRISB_MAX_GATHER_M];
    uint32_t pix[CRISB_MAX_GATHER_M];
    uint32_t count;
};

// float <-> order-preserving unsigned, for atomic min / max of floats
RT_D unsigned int float_to_ordered(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
RT_D float ordered_to_float(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// conservative box of an entry: a candidate passes dist <= radius only if the
// query lies inside this box
RT_D lbvh::Box entry_box(float4 e) {
    const float h = e.w * 1.0001f + 4e-7f * (fabsf(e.x) + fabsf(e.y) + fabsf(e.z) + 1.0f);
    lbvh::Box bx;
    bx.lo[0] = e.x - h;
    bx.lo[1] = e.y - h;
    bx.lo[2] = e.z - h;
    bx.hi[0] = e.x + h;
    bx.hi[1] = e.y + h;
    bx.hi[2] = e.z + h;
    return bx;
}

RT_D bool knn_before(float d, uint32_t p, float d2, uint32_t p2) { return d < d2 || (d == d2 && p < p2); }

RT_D void knn_error(int* err, int code) {
    if (err) atomicOr(err, code);
}

// The k (<= CRISB_MAX_GATHER_M) nearest entries whose radius covers q.  A
// query that visits more than max_visits nodes stops with the neighbours found
// so far and sets kDevErrKnn in *err.
RT_D void knn_query(const KnnView& v, int* err, V3 q, uint32_t k, NeighborList& nl,
                    uint32_t max_visits = kKnnMaxVisits) {
    nl.count = 0;
    const uint32_t n = *v.n;
    if (n == 0 || k == 0 || nonfinite(q)) return;
    int stack[kTraversalStack];
    int sp = 0;
    int cur = 0;
    uint32_t visits = 0;
    while (true) {
        if (++visits > max_visits) {
            knn_error(err, kDevErrKnn);
            return;
        }
        const BvhNode nd = v.nodes[cur];
        const bool in_l = q.x >= nd.a.x && q.y >= nd.a.y && q.z >= nd.a.z && q.x <= nd.a.w && q.y <= nd.b.x &&
                          q.z <= nd.b.y;
        const bool in_r = q.x >= nd.b.z && q.y >= nd.b.w && q.z >= nd.c.x && q.x <= nd.c.y && q.y <= nd.c.z &&
                          q.z <= nd.c.w;
        const int links[2] = {nd.d.x, nd.d.y};
        const int counts[2] = {nd.d.z, nd.d.w};
        bool go[2] = {in_l, in_r};
        for (int c = 0; c < 2; ++c) {
            if (!go[c] || links[c] >= 0) continue;
            go[c] = false;
            const int first = -1 - links[c];
            for (int t = 0; t < counts[c]; ++t) {
                const float4 e = v.leaf[first + t];
                const uint32_t j = v.index[first + t];
                const float d = distance(q, V3{e.x, e.y, e.z});
                if (d > e.w) continue;
                if (nl.count == k) {
                    if (!knn_before(d, j, nl.dist[k - 1], nl.pix[k - 1])) continue;
                    --nl.count;
                }
                uint32_t pos = nl.count;
                while (pos > 0 && knn_before(d, j, nl.dist[pos - 1], nl.pix[pos - 1])) {
                    nl.dist[pos] = nl.dist[pos - 1];
                    nl.pix[pos] = nl.pix[pos - 1];
                    --pos;
                }
                nl.dist[pos] = d;
                nl.pix[pos] = j;
                ++nl.count;
            }
        }
        if (go[0] && go[1]) {
            if (sp >= kTraversalStack) {
                knn_error(err, kDevErrStack);
                return;
            }
            stack[sp++] = links[1];
            cur = links[0];
        } else if (go[0]) {
            cur = links[0];
        } else if (go[1]) {
            cur = links[1];
        } else {
            if (sp == 0) return;
            cur = stack[--sp];
        }
    }
}

}  // namespace crisb
