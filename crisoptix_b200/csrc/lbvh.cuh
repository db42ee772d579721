// lbvh.cuh -- linear BVH construction on the device.
//
// 30-bit Morton codes of primitive centroids, made unique by the primitive
// index in the low 32 bits, sorted with a device radix sort; the binary radix
// tree of Karras (HPG 2012, "Maximizing Parallelism in the Construction of
// BVHs, Octrees, and k-d Trees"); bounding boxes by an atomic bottom-up pass;
// and emission into two-child nodes (rt_scene.cuh BvhNode) where any subtree
// of at most `leaf_max` primitives becomes one leaf.  The primitive count is
// read from device memory so that a per-frame build needs no host round trip.
#pragma once

#include <cstdint>

#include "rt_scene.cuh"

namespace crisb {
namespace lbvh {

struct Box {
    float lo[3];
    float hi[3];
};

RT_D uint32_t expand_bits10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

RT_D uint32_t morton30(float x, float y, float z) {
    const uint32_t xi = static_cast<uint32_t>(fminf(fmaxf(x * 1024.0f, 0.0f), 1023.0f));
    const uint32_t yi = static_cast<uint32_t>(fminf(fmaxf(y * 1024.0f, 0.0f), 1023.0f));
    const uint32_t zi = static_cast<uint32_t>(fminf(fmaxf(z * 1024.0f, 0.0f), 1023.0f));
    return (expand_bits10(xi) << 2) | (expand_bits10(yi) << 1) | expand_bits10(zi);
}

// key for centroid c inside bounds [lo, hi]
RT_D uint64_t morton_key(const float* lo, const float* hi, float cx, float cy, float cz, uint32_t idx) {
    const float ex = fmaxf(hi[0] - lo[0], 1e-30f), ey = fmaxf(hi[1] - lo[1], 1e-30f),
                ez = fmaxf(hi[2] - lo[2], 1e-30f);
    const uint32_t m = morton30((cx - lo[0]) / ex, (cy - lo[1]) / ey, (cz - lo[2]) / ez);
    return (static_cast<uint64_t>(m) << 32) | idx;
}

// Work arrays of one build, capacity = max primitive count.
struct Work {
    uint64_t* keys_in;
    uint64_t* keys;        // sorted
    int* inner_parent;     // capacity
    int* leaf_parent;      // capacity
    int* inner_left;       // encoded: >= 0 inner, < 0 leaf (-1 - leaf)
    int* inner_right;
    int* range_lo;
    int* range_hi;
    Box* inner_box;
    Box* leaf_box;
    int* flags;
    uint32_t* n;           // device primitive count
    BvhNode* nodes;        // capacity (>= 1)
    uint32_t* order;       // leaf order -> primitive index
    int* err;
};

RT_D int delta(const uint64_t* keys, int n, int i, int j) {
    if (j < 0 || j > n - 1) return -1;
    return __clzll(static_cast<long long>(keys[i] ^ keys[j]));
}

#ifdef CRISB_LBVH_KERNELS
// Karras radix tree: one thread per inner node i in [0, n-2]
__global__ void k_karras(Work w) {
    const int n = static_cast<int>(*w.n);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const uint64_t* k = w.keys;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) {
        lmax *= 2;
        if (lmax > (1 << 30)) break;
    }
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    int left, right;
    if (lo == gamma) {
        left = -1 - gamma;
        w.leaf_parent[gamma] = i;
    } else {
        left = gamma;
        w.inner_parent[gamma] = i;
    }
    if (hi == gamma + 1) {
        right = -1 - (gamma + 1);
        w.leaf_parent[gamma + 1] = i;
    } else {
        right = gamma + 1;
        w.inner_parent[gamma + 1] = i;
    }
    w.inner_left[i] = left;
    w.inner_right[i] = right;
    w.range_lo[i] = lo;
    w.range_hi[i] = hi;
    w.flags[i] = 0;
    if (i == 0) w.inner_parent[0] = -1;
}

RT_D Box ld_box_cg(const Box* b) {
    Box r;
    const float* p = reinterpret_cast<const float*>(b);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        r.lo[a] = __ldcg(p + a);
        r.hi[a] = __ldcg(p + 3 + a);
    }
    return r;
}

RT_D Box box_union(const Box& a, const Box& b) {
    Box r;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r.lo[c] = fminf(a.lo[c], b.lo[c]);
        r.hi[c] = fmaxf(a.hi[c], b.hi[c]);
    }
    return r;
}

// Bottom-up boxes: leaf boxes must already be in w.leaf_box (leaf order).
// One thread per leaf; the second child to arrive at an inner node computes
// its box and continues upward.
__global__ void k_refit(Work w) {
    const int n = static_cast<int>(*w.n);
    const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n || n < 2) return;
    int node = w.leaf_parent[leaf];
    for (int guard = 0; node >= 0 && guard < 128; ++guard) {
        __threadfence();
        if (atomicAdd(&w.flags[node], 1) == 0) return;
        __threadfence();
        const int l = w.inner_left[node], r = w.inner_right[node];
        const Box bl = l >= 0 ? ld_box_cg(&w.inner_box[l]) : ld_box_cg(&w.leaf_box[-1 - l]);
        const Box br = r >= 0 ? ld_box_cg(&w.inner_box[r]) : ld_box_cg(&w.leaf_box[-1 - r]);
        const Box u = box_union(bl, br);
        float* dst = reinterpret_cast<float*>(&w.inner_box[node]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            __stcg(dst + a, u.lo[a]);
            __stcg(dst + 3 + a, u.hi[a]);
        }
        node = w.inner_parent[node];
    }
}

RT_D void put_child(BvhNode& nd, int side, const Box& b, int link, int count) {
    if (side == 0) {
        nd.a = make_float4(b.lo[0], b.lo[1], b.lo[2], b.hi[0]);
        nd.b.x = b.hi[1];
        nd.b.y = b.hi[2];
        nd.d.x = link;
        nd.d.z = count;
    } else {
        nd.b.z = b.lo[0];
        nd.b.w = b.lo[1];
        nd.c = make_float4(b.lo[2], b.hi[0], b.hi[1], b.hi[2]);
        nd.d.y = link;
        nd.d.w = count;
    }
}

// Emit BVH2 nodes.  One thread per inner node; node 0 is the root.  With n < 2
// the root holds the single leaf (or nothing).
__global__ void k_emit(Work w, int leaf_max) {
    const int n = static_cast<int>(*w.n);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < 2) {
        if (i != 0) return;
        BvhNode nd;
        nd.d = make_int4(-1, -1, 0, 0);
        Box empty;
        for (int a = 0; a < 3; ++a) {
            empty.lo[a] = 1.0f;
            empty.hi[a] = -1.0f;
        }
        put_child(nd, 0, n == 1 ? w.leaf_box[0] : empty, -1, n == 1 ? 1 : 0);
        put_child(nd, 1, empty, -1, 0);
        w.nodes[0] = nd;
        return;
    }
    if (i >= n - 1) return;
    BvhNode nd;
    const int links[2] = {w.inner_left[i], w.inner_right[i]};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int l = links[c];
        if (l < 0) {
            put_child(nd, c, w.leaf_box[-1 - l], l, 1);
        } else {
            const int cnt = w.range_hi[l] - w.range_lo[l] + 1;
            if (cnt <= leaf_max) put_child(nd, c, w.inner_box[l], -1 - w.range_lo[l], cnt);
            else put_child(nd, c, w.inner_box[l], l, 0);
        }
    }
    w.nodes[i] = nd;
}

// leaf order -> primitive index from the sorted keys
__global__ void k_order(Work w) {
    const uint32_t n = *w.n;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    w.order[i] = static_cast<uint32_t>(w.keys[i] & 0xFFFFFFFFull);
}

#endif  // CRISB_LBVH_KERNELS

}  // namespace lbvh
}  // namespace crisb
