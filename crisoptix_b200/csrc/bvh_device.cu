// bvh_device.cu -- build_wide_bvh_device (bvh_device.h).
#include "bvh_device.h"

#include <algorithm>
#include <cfloat>
#include <cstring>

#include "radix_sort.h"

namespace crisb {
namespace {

// PLOC's search window: with the compressed nodes' SAH distribution, radius
// 8 / 16 / 24 / 32 / 48 / 64 rendered the 1080p workload in 17.05 / 17.29 /
// 16.98 / 17.02 / 17.06 / 17.41 ms per frame
constexpr int kPlocRadius = 32;
constexpr int kBlock = 256;
constexpr float kTriCost = 2.0f;
constexpr float kNodeCost = 1.0f;
constexpr uint32_t kLeafyBit = 0x80000000u;  // in BNode.meta: the SAH makes this subtree one leaf

// binary node: box, children (< 0: none; ids < n are triangles in sorted
// order), meta = triangle count | kLeafyBit
struct BNode {
    float lo[3], hi[3];
    int left, right;
    uint32_t meta;
    float cost;
};

inline unsigned blocks(uint32_t n, int b = kBlock) { return (std::max<uint32_t>(n, 1) + b - 1) / b; }

__device__ float area_of(const float* lo, const float* hi) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

__device__ unsigned int ordered(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ float unordered(unsigned int u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }

__device__ uint32_t spread10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// ---- 1. centroid bounds, Morton keys ----------------------------------------------------
__global__ void k_bounds_init(unsigned int* cb) {
    if (threadIdx.x < 3) cb[threadIdx.x] = ordered(FLT_MAX);
    else if (threadIdx.x < 6) cb[threadIdx.x] = ordered(-FLT_MAX);
}

__global__ void k_centroid_bounds(const float* __restrict__ pos, uint32_t n, unsigned int* cb) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, d[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (t < n) {
        const float* p = pos + 9 * static_cast<size_t>(t);
        for (int a = 0; a < 3; ++a) c[a] = d[a] = (p[a] + p[3 + a] + p[6 + a]) * (1.0f / 3.0f);
    }
    for (int a = 0; a < 3; ++a) {
        float lo = c[a], hi = d[a];
        for (int off = 16; off > 0; off >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, off));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&cb[a], ordered(lo));
            atomicMax(&cb[3 + a], ordered(hi));
        }
    }
}

__global__ void k_keys(const float* __restrict__ pos, uint32_t n, const unsigned int* cb, uint64_t* keys) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* p = pos + 9 * static_cast<size_t>(t);
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float lo = unordered(cb[a]), hi = unordered(cb[3 + a]);
        const float c = (p[a] + p[3 + a] + p[6 + a]) * (1.0f / 3.0f);
        const float ext = fmaxf(hi - lo, 1e-30f);
        q[a] = static_cast<uint32_t>(fminf(fmaxf((c - lo) / ext * 1024.0f, 0.0f), 1023.0f));
    }
    const uint32_t m = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    keys[t] = (static_cast<uint64_t>(m) << 32) | t;
}

// leaves in sorted order: node i is triangle order[i]
__global__ void k_leaves(const float* __restrict__ pos, uint32_t n, const uint64_t* __restrict__ sorted,
                         uint32_t* order, BNode* nodes, int* cluster) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = static_cast<uint32_t>(sorted[i] & 0xFFFFFFFFull);
    order[i] = t;
    const float* p = pos + 9 * static_cast<size_t>(t);
    BNode b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = fminf(fminf(p[a], p[3 + a]), p[6 + a]);
        b.hi[a] = fmaxf(fmaxf(p[a], p[3 + a]), p[6 + a]);
    }
    b.left = b.right = -1;
    b.meta = 1u | kLeafyBit;
    b.cost = kTriCost * area_of(b.lo, b.hi);
    nodes[i] = b;
    cluster[i] = static_cast<int>(i);
}

// ---- 2. PLOC ---------------------------------------------------------------------------
// nearest neighbour within kPlocRadius positions by union surface area
// (ties: the lower position)
__global__ void __launch_bounds__(kBlock) k_nearest(const int* __restrict__ cluster, uint32_t count,
                                                    const BNode* __restrict__ nodes, int* __restrict__ nn) {
    constexpr int kWin = kBlock + 2 * kPlocRadius;
    __shared__ float slo[3][kWin], shi[3][kWin];
    const int b0 = static_cast<int>(blockIdx.x) * kBlock;
    for (int t = threadIdx.x; t < kWin; t += kBlock) {
        const int j = b0 - kPlocRadius + t;
        if (j >= 0 && j < static_cast<int>(count)) {
            const BNode& nd = nodes[cluster[j]];
            for (int a = 0; a < 3; ++a) {
                slo[a][t] = nd.lo[a];
                shi[a][t] = nd.hi[a];
            }
        }
    }
    __syncthreads();
    const int i = b0 + static_cast<int>(threadIdx.x);
    if (i >= static_cast<int>(count)) return;
    const int li = i - b0 + kPlocRadius;
    float best = FLT_MAX;
    int bj = -1;
    const int j0 = max(0, i - kPlocRadius), j1 = min(static_cast<int>(count) - 1, i + kPlocRadius);
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int lj = j - b0 + kPlocRadius;
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(slo[a][li], slo[a][lj]);
            hi[a] = fmaxf(shi[a][li], shi[a][lj]);
        }
        const float ar = area_of(lo, hi);
        if (ar < best) {
            best = ar;
            bj = j;
        }
    }
    nn[i] = bj;
}

__global__ void k_merge_flags(const int* __restrict__ nn, uint32_t count, uint32_t* mflag, uint32_t* kflag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == static_cast<int>(i);
    mflag[i] = mutual && static_cast<int>(i) < j ? 1u : 0u;
    kflag[i] = mutual && static_cast<int>(i) > j ? 0u : 1u;
}

// no mutual pair in the window (only possible with exactly equal areas):
// merge the first two clusters
__global__ void k_force_pair(int* nn) {
    nn[0] = 1;
    nn[1] = 0;
}

__global__ void k_apply(const int* __restrict__ cluster, uint32_t count, const int* __restrict__ nn,
                        const uint32_t* __restrict__ mflag, const uint32_t* __restrict__ kflag,
                        const uint32_t* __restrict__ mpos, const uint32_t* __restrict__ kpos, uint32_t next_id,
                        int leaf_max, BNode* nodes, int* out_cluster) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || !kflag[i]) return;
    if (!mflag[i]) {
        out_cluster[kpos[i]] = cluster[i];
        return;
    }
    const int l = cluster[i], r = cluster[nn[i]];
    const BNode a = nodes[l], b = nodes[r];
    BNode m;
    for (int k = 0; k < 3; ++k) {
        m.lo[k] = fminf(a.lo[k], b.lo[k]);
        m.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    m.left = l;
    m.right = r;
    const uint32_t cnt = (a.meta & ~kLeafyBit) + (b.meta & ~kLeafyBit);
    const float ar = area_of(m.lo, m.hi);
    const float split = kNodeCost * ar + a.cost + b.cost;
    const float leaf = kTriCost * static_cast<float>(cnt) * ar;
    const bool leafy = cnt <= static_cast<uint32_t>(leaf_max) && leaf <= split;
    m.meta = cnt | (leafy ? kLeafyBit : 0u);
    m.cost = leafy ? leaf : split;
    const uint32_t id = next_id + mpos[i];
    nodes[id] = m;
    out_cluster[kpos[i]] = static_cast<int>(id);
}

// ---- 4. collapse into wide nodes -------------------------------------------------------
__device__ bool is_leaf_child(const BNode& b, uint32_t n_tris, int id) {
    return static_cast<uint32_t>(id) < n_tris || (b.meta & kLeafyBit);
}

// children of the wide node standing for binary node b: open the inner child
// with the largest surface area until there are kW
template <int kW>
__device__ int gather_children(const BNode* nodes, uint32_t n_tris, int b, int ch[kW]) {
    const BNode& root = nodes[b];
    if (static_cast<uint32_t>(b) < n_tris || (root.meta & kLeafyBit)) {
        ch[0] = b;  // a single leaf (only the root can be one)
        return 1;
    }
    int k = 2;
    ch[0] = root.left;
    ch[1] = root.right;
    while (k < kW) {
        int best = -1;
        float best_area = -1.0f;
        for (int c = 0; c < k; ++c) {
            const BNode& nd = nodes[ch[c]];
            if (is_leaf_child(nd, n_tris, ch[c])) continue;
            const float ar = area_of(nd.lo, nd.hi);
            if (ar > best_area) {
                best_area = ar;
                best = c;
            }
        }
        if (best < 0) break;
        const BNode& nd = nodes[ch[best]];
        for (int c = k; c > best + 1; --c) ch[c] = ch[c - 1];
        ch[best] = nd.left;
        ch[best + 1] = nd.right;
        ++k;
    }
    return k;
}

template <int kW>
__global__ void k_collapse_count(const int* __restrict__ level, uint32_t nl, const BNode* __restrict__ nodes,
                                 uint32_t n_tris, uint32_t* inner_cnt, uint32_t* tri_cnt) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nl) return;
    int ch[kW];
    const int k = gather_children<kW>(nodes, n_tris, level[e], ch);
    uint32_t ni = 0, nt = 0;
    for (int c = 0; c < k; ++c) {
        const BNode& nd = nodes[ch[c]];
        if (is_leaf_child(nd, n_tris, ch[c])) nt += nd.meta & ~kLeafyBit;
        else ++ni;
    }
    inner_cnt[e] = ni;
    tri_cnt[e] = nt;
}

// the triangles of leafy subtree `root`, left to right, from position `tri`
// of the leaf order; returns the position after them
__device__ uint32_t write_leaf_tris(const BNode* __restrict__ nodes, uint32_t n_tris, const uint32_t* __restrict__ order,
                                    const float* __restrict__ pos, int root, uint32_t tri, float4* tris) {
    int stack[2 * 8];
    int sp = 0;
    stack[sp++] = root;
    while (sp > 0) {
        const int id = stack[--sp];
        if (static_cast<uint32_t>(id) < n_tris) {
            const uint32_t t = order[id];
            const float* p = pos + 9 * static_cast<size_t>(t);
            tris[3 * tri + 0] = make_float4(p[0], p[1], p[2], 0.0f);
            tris[3 * tri + 1] = make_float4(p[3], p[4], p[5], 0.0f);
            tris[3 * tri + 2] = make_float4(p[6], p[7], p[8], __uint_as_float(t));
            ++tri;
        } else if (sp + 2 <= 2 * 8) {
            stack[sp++] = nodes[id].right;
            stack[sp++] = nodes[id].left;
        }
    }
    return tri;
}

__global__ void k_collapse_write(const int* __restrict__ level, uint32_t nl, const BNode* __restrict__ nodes,
                                 uint32_t n_tris, const uint32_t* __restrict__ order, const float* __restrict__ pos,
                                 const uint32_t* __restrict__ inner_off, const uint32_t* __restrict__ tri_off,
                                 uint32_t node_base, uint32_t child_base, uint32_t tri_base, float margin,
                                 Bvh4Node* out, float4* tris, int* next_level) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nl) return;
    int ch[4];
    const int k = gather_children<4>(nodes, n_tris, level[e], ch);
    Bvh4Node w;
    for (int c = 0; c < kBvhWidth; ++c) {
        w.link[c] = kNoChild;
        w.count[c] = 0;
        w.lo_x[c] = w.lo_y[c] = w.lo_z[c] = 0.0f;
        w.hi_x[c] = w.hi_y[c] = w.hi_z[c] = 0.0f;
    }
    uint32_t inner = inner_off[e], tri = tri_base + tri_off[e];
    for (int c = 0; c < k; ++c) {
        const BNode& nd = nodes[ch[c]];
        w.lo_x[c] = nd.lo[0] - margin;
        w.lo_y[c] = nd.lo[1] - margin;
        w.lo_z[c] = nd.lo[2] - margin;
        w.hi_x[c] = nd.hi[0] + margin;
        w.hi_y[c] = nd.hi[1] + margin;
        w.hi_z[c] = nd.hi[2] + margin;
        if (is_leaf_child(nd, n_tris, ch[c])) {
            const uint32_t first = tri;
            tri = write_leaf_tris(nodes, n_tris, order, pos, ch[c], tri, tris);
            w.link[c] = -1 - static_cast<int>(first);
            w.count[c] = static_cast<int>(tri - first);
        } else {
            w.link[c] = static_cast<int>(child_base + inner);
            next_level[inner] = ch[c];
            ++inner;
        }
    }
    out[node_base + e] = w;
}

// ---- 3b. SAH-optimal distribution into compressed nodes (after Ylitie, Karras
// & Laine 2017, section 4.1, restated): per binary node n and slot budget j,
// C(n, j) = the least cost of representing n's subtree in at most j child
// slots of a wide node, a slot being a leaf of at most kQLeafMax triangles
// (cost kQTri x triangles x area) or a wide node (cost kQNode x area + the
// best distribution of n's subtree over its eight slots).  Areas are the
// probabilities of hitting the slot's box, so costs are expected work per ray
// up to one factor.  Bottom-up in PLOC merge order (children are always made
// before their parent).  Triangle cost 1 per node visit: on the 1080p
// workload 0.15 / 0.3 / 0.6 / 1.0 / 1.5 / 2.5 gave 12.14 / 11.93 / 11.52 /
// 11.42 / 11.47 / 11.44 ms of traversal per frame (the greedy collapse, whose
// nodes hold 4.1 of 8 children: 12.17 ms).
constexpr float kQNode = 1.0f;
constexpr float kQTri = 1.0f;

struct DpCell {
    float c[8];      // C(n, j + 1)
    uint8_t dec[8];  // [0]: 1 = one slot is a leaf; [j]: bits 0-2 = the left budget k of the
                     // best split of j + 1 slots, bit 7 = C(n, j + 1) takes one slot
};

__global__ void k_dp_leaves(const BNode* __restrict__ nodes, uint32_t n, DpCell* dp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DpCell d;
    const float c = kQTri * area_of(nodes[i].lo, nodes[i].hi);
    for (int j = 0; j < 8; ++j) {
        d.c[j] = c;
        d.dec[j] = 0x80;
    }
    d.dec[0] = 1;
    dp[i] = d;
}

__global__ void k_dp_inner(const BNode* __restrict__ nodes, uint32_t first, uint32_t count, DpCell* dp) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const uint32_t id = first + e;
    const BNode& nd = nodes[id];
    const DpCell& L = dp[nd.left];
    const DpCell& R = dp[nd.right];
    float cl[8], cr[8];
    for (int j = 0; j < 8; ++j) {
        cl[j] = L.c[j];
        cr[j] = R.c[j];
    }
    DpCell d;
    float dist[8];  // dist[j]: the best split of j + 1 slots between the children
    uint8_t dk[8];
    dist[0] = INFINITY;
    dk[0] = 0;
    for (int j = 1; j < 8; ++j) {
        float best = INFINITY;
        uint8_t bk = 1;
        for (int k = 1; k <= j; ++k) {  // k slots left, j + 1 - k right
            const float v = cl[k - 1] + cr[j - k];
            if (v < best) {
                best = v;
                bk = static_cast<uint8_t>(k);
            }
        }
        dist[j] = best;
        dk[j] = bk;
    }
    const float ar = area_of(nd.lo, nd.hi);
    const uint32_t tris = nd.meta & ~kLeafyBit;
    const float leaf = tris <= static_cast<uint32_t>(kQLeafMax) ? kQTri * static_cast<float>(tris) * ar : INFINITY;
    const float node = kQNode * ar + dist[7];
    const float single = fminf(leaf, node);
    d.dec[0] = leaf <= node ? 1 : 0;
    d.c[0] = single;
    for (int j = 1; j < 8; ++j) {
        const bool one = single <= dist[j];
        d.c[j] = one ? single : dist[j];
        d.dec[j] = static_cast<uint8_t>(dk[j] | (one ? 0x80 : 0));
    }
    dp[id] = d;
}

// the slots of the compressed node standing for binary node b: its best
// distribution over eight slots (ch: binary node ids, leaf: a leaf slot);
// a whole-scene leaf root is one leaf slot
__device__ int gather_slots_dp(const BNode* nodes, const DpCell* dp, uint32_t n_tris, int b, int ch[8],
                               bool leaf[8]) {
    if (static_cast<uint32_t>(b) < n_tris || dp[b].dec[0] == 1) {
        ch[0] = b;
        leaf[0] = true;
        return 1;
    }
    // explicit stack of (node, budget, split only); left parts come out first
    int sn[16], sj[16];
    bool sd[16];
    int sp = 0, k = 0;
    sn[sp] = b;
    sj[sp] = 8;
    sd[sp++] = true;
    while (sp > 0 && k < 8) {
        --sp;
        const int id = sn[sp], j = sj[sp];
        const bool split_only = sd[sp];
        const DpCell& d = dp[id];
        const bool inner = static_cast<uint32_t>(id) >= n_tris;
        if (!inner || j == 1 || (!split_only && (d.dec[j - 1] & 0x80))) {
            ch[k] = id;
            leaf[k] = !inner || d.dec[0] == 1;
            ++k;
            continue;
        }
        const int kl = d.dec[j - 1] & 7;
        if (sp + 2 > 16) break;
        const BNode& nd = nodes[id];
        sn[sp] = nd.right;
        sj[sp] = j - kl;
        sd[sp++] = false;
        sn[sp] = nd.left;
        sj[sp] = kl;
        sd[sp++] = false;
    }
    return k;
}

__global__ void k_dp_count(const int* __restrict__ level, uint32_t nl, const BNode* __restrict__ nodes,
                           const DpCell* __restrict__ dp, uint32_t n_tris, uint32_t* inner_cnt, uint32_t* tri_cnt) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nl) return;
    int ch[8];
    bool lf[8];
    const int k = gather_slots_dp(nodes, dp, n_tris, level[e], ch, lf);
    uint32_t ni = 0, nt = 0;
    for (int c = 0; c < k; ++c) {
        if (lf[c]) nt += static_cast<uint32_t>(ch[c]) < n_tris ? 1u : (nodes[ch[c]].meta & ~kLeafyBit);
        else ++ni;
    }
    inner_cnt[e] = ni;
    tri_cnt[e] = nt;
}

// one compressed node per binary node of the level: the slots of its best
// distribution placed in octant slots (greedy: the cheapest remaining (child, slot) pair
// first, cost = centroid offset from the node's centre along the slot's
// diagonal, ties to the lower child then slot), boxes widened by `margin`
// then quantised outward in double precision
__global__ void k_qcollapse_write(const int* __restrict__ level, uint32_t nl, const BNode* __restrict__ nodes,
                                  uint32_t n_tris, const uint32_t* __restrict__ order, const float* __restrict__ pos,
                                  const uint32_t* __restrict__ inner_off, const uint32_t* __restrict__ tri_off,
                                  uint32_t node_base, uint32_t child_base, uint32_t tri_base, float margin,
                                  const DpCell* __restrict__ dp, Bvh8QNode* out, float4* tris, int* next_level) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nl) return;
    int ch[8];
    bool lf[8];
    const int k = gather_slots_dp(nodes, dp, n_tris, level[e], ch, lf);
    float lo[8][3], hi[8][3], plo[3], phi[3];
    for (int a = 0; a < 3; ++a) {
        plo[a] = FLT_MAX;
        phi[a] = -FLT_MAX;
    }
    for (int c = 0; c < k; ++c) {
        const BNode& nd = nodes[ch[c]];
        for (int a = 0; a < 3; ++a) {
            lo[c][a] = nd.lo[a] - margin;
            hi[c][a] = nd.hi[a] + margin;
            plo[a] = fminf(plo[a], lo[c][a]);
            phi[a] = fmaxf(phi[a], hi[c][a]);
        }
    }
    int slot_child[8];
    for (int t = 0; t < 8; ++t) slot_child[t] = -1;
    uint32_t used_c = 0, used_s = 0;
    for (int r = 0; r < k; ++r) {
        float best = FLT_MAX;
        int bc = -1, bs = -1;
        for (int c = 0; c < k; ++c) {
            if ((used_c >> c) & 1u) continue;
            float off[3];
            for (int a = 0; a < 3; ++a) off[a] = (lo[c][a] + hi[c][a]) - (plo[a] + phi[a]);
            for (int t = 0; t < 8; ++t) {
                if ((used_s >> t) & 1u) continue;
                const float cost = ((t & 1) ? -off[0] : off[0]) + ((t & 2) ? -off[1] : off[1]) +
                                   ((t & 4) ? -off[2] : off[2]);
                if (bc < 0 || cost < best) {
                    best = cost;
                    bc = c;
                    bs = t;
                }
            }
        }
        used_c |= 1u << bc;
        used_s |= 1u << bs;
        slot_child[bs] = bc;
    }
    Bvh8QNode w;
    memset(&w, 0, sizeof(w));
    int ex[3];
    double scale[3];
    float porg[3];
    for (int a = 0; a < 3; ++a) {
        const double ext = k > 0 ? static_cast<double>(phi[a]) - static_cast<double>(plo[a]) : 0.0;
        int x = -126;
        if (ext > 0.0) {
            frexp(ext / 255.0, &x);  // ext / 255 < 2^x
            x = max(x, -126);
        }
        porg[a] = k > 0 ? plo[a] : 0.0f;
        ex[a] = x;
        scale[a] = ldexp(1.0, x);
    }
    w.px = porg[0];
    w.py = porg[1];
    w.pz = porg[2];
    w.ex = static_cast<int8_t>(ex[0]);
    w.ey = static_cast<int8_t>(ex[1]);
    w.ez = static_cast<int8_t>(ex[2]);
    w.child_base = child_base + inner_off[e];
    w.tri_base = tri_base + tri_off[e];
    uint8_t* qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z};
    uint8_t* qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
    uint32_t cursor = 0, rank = 0;
    for (int t = 0; t < 8; ++t) {
        const int c = slot_child[t];
        if (c < 0) continue;
        for (int a = 0; a < 3; ++a) {
            const double p = static_cast<double>(porg[a]);
            const double l = floor((static_cast<double>(lo[c][a]) - p) / scale[a]);
            const double h = ceil((static_cast<double>(hi[c][a]) - p) / scale[a]);
            qlo[a][t] = static_cast<uint8_t>(fmin(fmax(l, 0.0), 255.0));
            qhi[a][t] = static_cast<uint8_t>(fmin(fmax(h, 0.0), 255.0));
        }
        if (lf[c]) {
            const uint32_t first = w.tri_base + cursor;
            const uint32_t cnt = write_leaf_tris(nodes, n_tris, order, pos, ch[c], first, tris) - first;
            w.meta[t] = static_cast<uint8_t>((((1u << cnt) - 1u) << 5) | cursor);
            cursor += cnt;
        } else {
            w.meta[t] = static_cast<uint8_t>(0x38u | static_cast<uint32_t>(t));
            w.imask |= static_cast<uint8_t>(1u << t);
            next_level[inner_off[e] + rank] = ch[c];
            ++rank;
        }
    }
    out[node_base + e] = w;
}

template <class T>
cudaError_t dev_alloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

cudaError_t build_wide_bvh_device(const float* pos, uint32_t n, int leaf_max, float margin, bool compressed,
                                  cudaStream_t st, DeviceWideBvh* out) {
    if (compressed) leaf_max = std::min(leaf_max, kQLeafMax);
    *out = DeviceWideBvh{};
    cudaError_t e = cudaSuccess;
    // scratch
    uint64_t *keys = nullptr, *sorted = nullptr;
    uint32_t* order = nullptr;
    BNode* nodes = nullptr;
    int *cl[2] = {nullptr, nullptr}, *nn = nullptr;
    uint32_t *mflag = nullptr, *kflag = nullptr, *mpos = nullptr, *kpos = nullptr, *totals = nullptr;
    unsigned int* cb = nullptr;
    void* sort_temp = nullptr;
    void* scan_temp = nullptr;
    int* level[2] = {nullptr, nullptr};
    DpCell* dp = nullptr;
    std::vector<uint32_t> made;  // per PLOC iteration: first node id and count
    const uint32_t m = std::max<uint32_t>(n, 1);
    auto fail = [&](cudaError_t err) {
        cudaFree(keys);
        cudaFree(sorted);
        cudaFree(order);
        cudaFree(nodes);
        cudaFree(cl[0]);
        cudaFree(cl[1]);
        cudaFree(nn);
        cudaFree(mflag);
        cudaFree(kflag);
        cudaFree(mpos);
        cudaFree(kpos);
        cudaFree(totals);
        cudaFree(cb);
        cudaFree(sort_temp);
        cudaFree(scan_temp);
        cudaFree(level[0]);
        cudaFree(level[1]);
        cudaFree(dp);
        if (err != cudaSuccess) {
            cudaFree(out->nodes);
            cudaFree(out->qnodes);
            cudaFree(out->tris);
            *out = DeviceWideBvh{};
        }
        return err;
    };
#define TRY(x)                           \
    do {                                 \
        e = (x);                         \
        if (e != cudaSuccess) return fail(e); \
    } while (0)
    const size_t sort_bytes = rsort::temp_bytes(m);
    TRY(dev_alloc(&keys, m));
    TRY(dev_alloc(&sorted, m));
    TRY(dev_alloc(&order, m));
    TRY(dev_alloc(&nodes, 2 * static_cast<size_t>(m)));
    TRY(dev_alloc(&cl[0], m));
    TRY(dev_alloc(&cl[1], m));
    TRY(dev_alloc(&nn, m));
    TRY(dev_alloc(&mflag, m));
    TRY(dev_alloc(&kflag, m));
    TRY(dev_alloc(&mpos, m));
    TRY(dev_alloc(&kpos, m));
    TRY(dev_alloc(&totals, 4));
    TRY(dev_alloc(&cb, 8));
    TRY(cudaMalloc(&sort_temp, sort_bytes));
    TRY(cudaMalloc(&scan_temp, rsort::scan_temp_bytes(m)));
    auto scan = [&](const uint32_t* in, uint32_t* o, uint32_t cnt, uint32_t* total) {
        return rsort::exclusive_scan(in, o, cnt, total, scan_temp, st);
    };
    TRY(dev_alloc(&level[0], m));
    TRY(dev_alloc(&level[1], m));
    if (compressed) TRY(dev_alloc(&out->qnodes, m));
    else TRY(dev_alloc(&out->nodes, m));
    TRY(dev_alloc(&out->tris, 3 * static_cast<size_t>(m)));
    TRY(cudaMemsetAsync(out->tris, 0, 3 * static_cast<size_t>(m) * sizeof(float4), st));

    // 1. keys, sort, leaves
    k_bounds_init<<<1, 32, 0, st>>>(cb);
    if (n > 0) {
        k_centroid_bounds<<<blocks(n), kBlock, 0, st>>>(pos, n, cb);
        k_keys<<<blocks(n), kBlock, 0, st>>>(pos, n, cb, keys);
        TRY(rsort::sort_high32(keys, sorted, sort_temp, sort_bytes, n, st));
        k_leaves<<<blocks(n), kBlock, 0, st>>>(pos, n, sorted, order, nodes, cl[0]);
    }
    TRY(cudaGetLastError());

    // 2. PLOC until one cluster is left
    uint32_t count = n, next_id = n;
    int cur = 0;
    for (uint32_t iter = 0; count > 1; ++iter) {
        if (iter > 2 * n + 8) return fail(cudaErrorUnknown);
        k_nearest<<<blocks(count), kBlock, 0, st>>>(cl[cur], count, nodes, nn);
        k_merge_flags<<<blocks(count), kBlock, 0, st>>>(nn, count, mflag, kflag);
        TRY(scan(mflag, mpos, count, totals));
        uint32_t merges = 0;
        TRY(cudaMemcpyAsync(&merges, totals, sizeof(merges), cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        if (merges == 0) {
            k_force_pair<<<1, 1, 0, st>>>(nn);
            k_merge_flags<<<blocks(count), kBlock, 0, st>>>(nn, count, mflag, kflag);
            TRY(scan(mflag, mpos, count, totals));
            merges = 1;
        }
        TRY(scan(kflag, kpos, count, totals + 1));
        k_apply<<<blocks(count), kBlock, 0, st>>>(cl[cur], count, nn, mflag, kflag, mpos, kpos, next_id, leaf_max,
                                                  nodes, cl[cur ^ 1]);
        TRY(cudaGetLastError());
        made.push_back(next_id);
        made.push_back(merges);
        next_id += merges;
        count -= merges;
        cur ^= 1;
    }
    int root = 0;
    if (n > 0) TRY(cudaMemcpyAsync(&root, cl[cur], sizeof(int), cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));

    // 4. collapse level by level; the root wide node at 0
    if (n == 0) {
        if (compressed) {
            Bvh8QNode q;
            std::memset(&q, 0, sizeof(q));
            q.ex = q.ey = q.ez = -126;
            TRY(cudaMemcpyAsync(out->qnodes, &q, sizeof(q), cudaMemcpyHostToDevice, st));
        } else {
            Bvh4Node w;
            std::memset(&w, 0, sizeof(w));
            for (int c = 0; c < kBvhWidth; ++c) w.link[c] = kNoChild;
            TRY(cudaMemcpyAsync(out->nodes, &w, sizeof(w), cudaMemcpyHostToDevice, st));
        }
        out->num_nodes = 1;
        TRY(cudaStreamSynchronize(st));
        return fail(cudaSuccess);
    }
    TRY(cudaMemcpyAsync(level[0], &root, sizeof(int), cudaMemcpyHostToDevice, st));
    if (compressed) {
        // 3b. slot costs bottom-up, one launch per PLOC iteration
        TRY(dev_alloc(&dp, 2 * static_cast<size_t>(m)));
        k_dp_leaves<<<blocks(n), kBlock, 0, st>>>(nodes, n, dp);
        for (size_t it = 0; it + 1 < made.size(); it += 2)
            k_dp_inner<<<blocks(made[it + 1]), kBlock, 0, st>>>(nodes, made[it], made[it + 1], dp);
        TRY(cudaGetLastError());
    }
    uint32_t nl = 1, node_base = 0, tri_base = 0;
    int lv = 0, depth = 0;
    while (nl > 0) {
        const uint32_t child_base = node_base + nl;
        if (compressed) k_dp_count<<<blocks(nl), kBlock, 0, st>>>(level[lv], nl, nodes, dp, n, mflag, kflag);
        else k_collapse_count<4><<<blocks(nl), kBlock, 0, st>>>(level[lv], nl, nodes, n, mflag, kflag);
        TRY(scan(mflag, mpos, nl, totals));
        TRY(scan(kflag, kpos, nl, totals + 1));
        uint32_t tot[2] = {0, 0};
        TRY(cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        if (child_base + tot[0] > m || tri_base + tot[1] > n) return fail(cudaErrorUnknown);
        if (compressed)
            k_qcollapse_write<<<blocks(nl), kBlock, 0, st>>>(level[lv], nl, nodes, n, order, pos, mpos, kpos,
                                                             node_base, child_base, tri_base, margin, dp,
                                                             out->qnodes, out->tris, level[lv ^ 1]);
        else
            k_collapse_write<<<blocks(nl), kBlock, 0, st>>>(level[lv], nl, nodes, n, order, pos, mpos, kpos,
                                                            node_base, child_base, tri_base, margin, out->nodes,
                                                            out->tris, level[lv ^ 1]);
        TRY(cudaGetLastError());
        node_base = child_base;
        tri_base += tot[1];
        nl = tot[0];
        lv ^= 1;
        ++depth;
    }
    TRY(cudaStreamSynchronize(st));
    if (tri_base != n) return fail(cudaErrorUnknown);
    out->num_nodes = node_base;
    out->binary_depth = depth;
    return fail(cudaSuccess);
#undef TRY
}

}  // namespace crisb
