// bvh_build.cpp -- binned-SAH binary BVH over triangles, collapsed into a
// 4-wide BVH (Wald 2007 "On fast Construction of SAH-based Bounding Volume
// Hierarchies" for the binning; greedy collapse by surface area as in Wald,
// Benthin & Boulos 2008 "Getting rid of packets").  Subtrees above a size
// threshold are built on separate host threads; the result does not depend on
// the thread schedule (every split works on its own index range and the wide
// tree is laid out by a depth-first walk from the root).
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>

namespace crisb {
namespace {

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    bool empty() const { return lo[0] > hi[0]; }
    float area() const {
        if (empty()) return 0.0f;
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

struct BinNode {
    Box box;
    int left = -1, right = -1;  // both -1: leaf over [first, first + count)
    uint32_t first = 0, count = 0;
};

constexpr int kBins = 32;
constexpr float kCostNode = 1.0f;
constexpr float kCostTri = 2.0f;
constexpr uint32_t kParallelMin = 1u << 15;

struct Builder {
    const std::vector<Box>& prim_box;
    const std::vector<float>& cent;  // 3 per triangle
    std::vector<uint32_t>& idx;
    std::vector<BinNode>& nodes;
    std::atomic<uint32_t> next{0};
    std::atomic<int> max_depth{0};
    std::atomic<int> threads{0};
    int leaf_max, median_depth, max_threads;

    Builder(const std::vector<Box>& pb, const std::vector<float>& c, std::vector<uint32_t>& i,
            std::vector<BinNode>& n, int lm, int md)
        : prim_box(pb), cent(c), idx(i), nodes(n), leaf_max(lm), median_depth(md) {
        max_threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    }

    uint32_t alloc() {
        const uint32_t i = next.fetch_add(1);
        if (i >= nodes.size()) throw std::runtime_error("bvh build: node pool exhausted");
        return i;
    }

    void make_leaf(BinNode& nd, uint32_t b, uint32_t e) {
        nd.left = nd.right = -1;
        nd.first = b;
        nd.count = e - b;
    }

    // split [b, e) in place; returns the first index of the right side, or b
    // when no split is possible
    uint32_t split(uint32_t b, uint32_t e, const Box& box, int depth, bool& force_leaf) {
        const uint32_t n = e - b;
        force_leaf = false;
        Box cb;
        for (uint32_t i = b; i < e; ++i) cb.grow(&cent[3 * idx[i]]);
        int axis = 0;
        float ext[3];
        for (int a = 0; a < 3; ++a) ext[a] = cb.hi[a] - cb.lo[a];
        if (ext[1] > ext[axis]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        auto median = [&](int ax) {
            const uint32_t mid = b + n / 2;
            std::nth_element(idx.begin() + b, idx.begin() + mid, idx.begin() + e, [&](uint32_t x, uint32_t y) {
                const float cx = cent[3 * x + ax], cy = cent[3 * y + ax];
                return cx < cy || (cx == cy && x < y);
            });
            return mid;
        };
        if (!(ext[axis] > 0.0f)) {  // coincident centroids
            if (n <= static_cast<uint32_t>(leaf_max)) {
                force_leaf = true;
                return b;
            }
            return median(axis);
        }
        if (depth >= median_depth) return median(axis);
        // binned SAH over all three axes
        float best_cost = INFINITY;
        int best_axis = -1, best_bin = -1;
        for (int a = 0; a < 3; ++a) {
            if (!(ext[a] > 0.0f)) continue;
            Box bins[kBins];
            uint32_t cnt[kBins] = {};
            const float scale = kBins / ext[a];
            for (uint32_t i = b; i < e; ++i) {
                const uint32_t t = idx[i];
                int k = static_cast<int>((cent[3 * t + a] - cb.lo[a]) * scale);
                k = std::min(std::max(k, 0), kBins - 1);
                ++cnt[k];
                bins[k].grow(prim_box[t]);
            }
            float right_area[kBins];
            uint32_t right_cnt[kBins];
            Box acc;
            uint32_t c = 0;
            for (int k = kBins - 1; k > 0; --k) {
                acc.grow(bins[k]);
                c += cnt[k];
                right_area[k] = acc.area();
                right_cnt[k] = c;
            }
            acc = Box();
            c = 0;
            for (int k = 0; k < kBins - 1; ++k) {
                acc.grow(bins[k]);
                c += cnt[k];
                if (c == 0 || right_cnt[k + 1] == 0) continue;
                const float cost = acc.area() * c + right_area[k + 1] * right_cnt[k + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_bin = k;
                }
            }
        }
        if (best_axis < 0) return median(axis);
        const float parent = box.area();
        const float split_cost = kCostNode + (parent > 0.0f ? kCostTri * best_cost / parent : INFINITY);
        if (n <= static_cast<uint32_t>(leaf_max) && kCostTri * n <= split_cost) {
            force_leaf = true;
            return b;
        }
        const float lo = cb.lo[best_axis], scale = kBins / ext[best_axis];
        const auto mid = std::partition(idx.begin() + b, idx.begin() + e, [&](uint32_t t) {
            int k = static_cast<int>((cent[3 * t + best_axis] - lo) * scale);
            k = std::min(std::max(k, 0), kBins - 1);
            return k <= best_bin;
        });
        const uint32_t m = static_cast<uint32_t>(mid - idx.begin());
        if (m == b || m == e) return median(axis);
        return m;
    }

    void build(uint32_t node, uint32_t b, uint32_t e, int depth) {
        while (true) {
            BinNode& nd = nodes[node];
            nd.box = Box();
            for (uint32_t i = b; i < e; ++i) nd.box.grow(prim_box[idx[i]]);
            int d = max_depth.load();
            while (depth > d && !max_depth.compare_exchange_weak(d, depth)) {
            }
            if (e - b <= 1) {
                make_leaf(nd, b, e);
                return;
            }
            bool force_leaf = false;
            const uint32_t m = split(b, e, nd.box, depth, force_leaf);
            if (force_leaf) {
                make_leaf(nd, b, e);
                return;
            }
            const uint32_t l = alloc(), r = alloc();
            nd.left = static_cast<int>(l);
            nd.right = static_cast<int>(r);
            nd.first = b;
            nd.count = e - b;
            // the larger side on another thread while threads are free
            const bool big = std::min(m - b, e - m) >= kParallelMin;
            if (big && threads.fetch_add(1) < max_threads - 1) {
                auto f = std::async(std::launch::async, [this, l, b, m, depth] { build(l, b, m, depth + 1); });
                build(r, m, e, depth + 1);
                f.get();
                threads.fetch_sub(1);
                return;
            }
            if (big) threads.fetch_sub(1);
            build(l, b, m, depth + 1);
            node = r;
            b = m;
            ++depth;
        }
    }
};

struct Collapser {
    const std::vector<BinNode>& bin;
    std::vector<Bvh4Node>& out;
    float margin;  // widening of every emitted child box (box_margin)
    int max_stack = 0;

    bool is_leaf(int i) const { return bin[i].left < 0; }

    // children of the wide node standing for binary inner node `i`
    void gather(int i, int ch[kBvhWidth], int& k) const {
        ch[0] = bin[i].left;
        ch[1] = bin[i].right;
        k = 2;
        while (k < kBvhWidth) {
            int pick = -1;
            float best = -1.0f;
            for (int c = 0; c < k; ++c) {
                if (is_leaf(ch[c])) continue;
                const float a = bin[ch[c]].box.area();
                if (a > best) {
                    best = a;
                    pick = c;
                }
            }
            if (pick < 0) break;
            const int p = ch[pick];
            ch[pick] = bin[p].left;
            ch[k++] = bin[p].right;
        }
    }

    // lays out the subtree of binary inner node `i` at wide index `w`;
    // returns the worst-case stack entries below it
    int emit(int i, uint32_t w) {
        int ch[kBvhWidth], k;
        gather(i, ch, k);
        const float m = margin;
        Bvh4Node nd;
        int inner = 0;
        for (int c = 0; c < kBvhWidth; ++c) {
            nd.link[c] = kNoChild;
            nd.count[c] = 0;
            nd.lo_x[c] = nd.lo_y[c] = nd.lo_z[c] = 0.0f;
            nd.hi_x[c] = nd.hi_y[c] = nd.hi_z[c] = 0.0f;
        }
        for (int c = 0; c < k; ++c) {
            const Box& bx = bin[ch[c]].box;
            nd.lo_x[c] = bx.lo[0] - m;
            nd.lo_y[c] = bx.lo[1] - m;
            nd.lo_z[c] = bx.lo[2] - m;
            nd.hi_x[c] = bx.hi[0] + m;
            nd.hi_y[c] = bx.hi[1] + m;
            nd.hi_z[c] = bx.hi[2] + m;
            if (is_leaf(ch[c])) {
                nd.link[c] = -1 - static_cast<int>(bin[ch[c]].first);
                nd.count[c] = static_cast<int>(bin[ch[c]].count);
            } else {
                ++inner;
            }
        }
        // depth-first pre-order: each inner child right after its elder
        // siblings' subtrees
        int below = 0;
        for (int c = 0; c < k; ++c) {
            if (is_leaf(ch[c])) continue;
            const uint32_t cw = static_cast<uint32_t>(out.size());
            nd.link[c] = static_cast<int>(cw);
            out.emplace_back();
            below = std::max(below, emit(ch[c], cw));
        }
        out[w] = nd;
        return std::max(inner - 1, 0) + below;
    }
};

}  // namespace

WideBvh build_wide_bvh(const float* pos, uint32_t n, int leaf_max, int median_depth) {
    WideBvh r;
    r.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) r.order[i] = i;
    if (n == 0) {
        Bvh4Node nd;
        std::memset(&nd, 0, sizeof(nd));
        for (int c = 0; c < kBvhWidth; ++c) nd.link[c] = kNoChild;
        r.nodes.push_back(nd);
        return r;
    }
    std::vector<Box> prim_box(n);
    std::vector<float> cent(3 * static_cast<size_t>(n));
    for (uint32_t t = 0; t < n; ++t) {
        const float* p = pos + 9 * static_cast<size_t>(t);
        Box b;
        b.grow(p);
        b.grow(p + 3);
        b.grow(p + 6);
        prim_box[t] = b;
        for (int a = 0; a < 3; ++a) cent[3 * t + a] = (p[a] + p[3 + a] + p[6 + a]) * (1.0f / 3.0f);
    }
    std::vector<BinNode> bin(2 * static_cast<size_t>(n));
    Builder bld(prim_box, cent, r.order, bin, leaf_max, median_depth);
    const uint32_t root = bld.alloc();
    bld.build(root, 0, n, 0);
    r.max_depth = bld.max_depth.load();
    float max_abs = 0.0f;
    for (size_t i = 0; i < 9 * static_cast<size_t>(n); ++i) max_abs = std::max(max_abs, std::fabs(pos[i]));
    const float margin = box_margin(max_abs);
    Collapser col{bin, r.nodes, margin};
    r.nodes.reserve(bld.next.load() / 2 + 1);
    r.nodes.emplace_back();
    if (bin[root].left < 0) {
        // a single leaf: one wide node with one leaf child
        Bvh4Node nd;
        std::memset(&nd, 0, sizeof(nd));
        for (int c = 0; c < kBvhWidth; ++c) nd.link[c] = kNoChild;
        const Box& bx = bin[root].box;
        nd.lo_x[0] = bx.lo[0] - margin;
        nd.lo_y[0] = bx.lo[1] - margin;
        nd.lo_z[0] = bx.lo[2] - margin;
        nd.hi_x[0] = bx.hi[0] + margin;
        nd.hi_y[0] = bx.hi[1] + margin;
        nd.hi_z[0] = bx.hi[2] + margin;
        nd.link[0] = -1;
        nd.count[0] = static_cast<int>(n);
        r.nodes[0] = nd;
    } else {
        r.max_stack = col.emit(static_cast<int>(root), 0);
    }
    return r;
}

int validate_wide_bvh(const WideBvh& bvh, const float* pos, uint32_t n, int leaf_max) {
    auto fail = [](const char* what) { throw std::runtime_error(std::string("bvh check: ") + what); };
    const size_t nn = bvh.nodes.size();
    if (nn == 0) fail("no root");
    if (bvh.order.size() != n) fail("leaf order size");
    std::vector<uint8_t> seen_tri(n, 0), seen_node(nn, 0);
    struct Item {
        uint32_t node;
        int stack;  // entries pushed above this node
    };
    std::vector<Item> todo{{0, 0}};
    seen_node[0] = 1;
    int max_stack = 0;
    auto inside = [](float v, float lo, float hi) { return v >= lo && v <= hi; };
    // box of every inner node's subtree is checked against its triangles by
    // walking leaves; inner child boxes are checked to contain their
    // children's boxes
    while (!todo.empty()) {
        const Item it = todo.back();
        todo.pop_back();
        max_stack = std::max(max_stack, it.stack);
        const Bvh4Node& nd = bvh.nodes[it.node];
        int inner = 0;
        for (int c = 0; c < kBvhWidth; ++c) {
            const int l = nd.link[c];
            if (l == kNoChild) continue;
            if (l >= 0) {
                ++inner;
                continue;
            }
            const int64_t first = -1 - static_cast<int64_t>(l);
            const int cnt = nd.count[c];
            if (cnt < 1 || cnt > leaf_max || first + cnt > static_cast<int64_t>(n)) fail("leaf range");
            for (int k = 0; k < cnt; ++k) {
                const uint32_t slot = static_cast<uint32_t>(first + k);
                if (seen_tri[slot]) fail("triangle in two leaves");
                seen_tri[slot] = 1;
                const uint32_t prim = bvh.order[slot];
                if (prim >= n) fail("leaf order entry");
                const float* p = pos + 9 * static_cast<size_t>(prim);
                for (int v = 0; v < 3; ++v)
                    if (!inside(p[3 * v], nd.lo_x[c], nd.hi_x[c]) || !inside(p[3 * v + 1], nd.lo_y[c], nd.hi_y[c]) ||
                        !inside(p[3 * v + 2], nd.lo_z[c], nd.hi_z[c]))
                        fail("leaf box does not contain its triangle");
            }
        }
        const int pushed = std::max(inner - 1, 0);
        for (int c = 0; c < kBvhWidth; ++c) {
            const int l = nd.link[c];
            if (l == kNoChild || l < 0) continue;
            if (static_cast<size_t>(l) >= nn || l == 0) fail("inner link out of range");
            if (seen_node[l]) fail("inner node reached twice");
            seen_node[l] = 1;
            const Bvh4Node& ch = bvh.nodes[l];
            for (int g = 0; g < kBvhWidth; ++g) {
                if (ch.link[g] == kNoChild) continue;
                if (ch.lo_x[g] < nd.lo_x[c] || ch.hi_x[g] > nd.hi_x[c] || ch.lo_y[g] < nd.lo_y[c] ||
                    ch.hi_y[g] > nd.hi_y[c] || ch.lo_z[g] < nd.lo_z[c] || ch.hi_z[g] > nd.hi_z[c])
                    fail("child box outside its parent's box");
            }
            todo.push_back({static_cast<uint32_t>(l), it.stack + pushed});
        }
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!seen_tri[i]) fail("triangle in no leaf");
    for (size_t i = 0; i < nn; ++i)
        if (!seen_node[i]) fail("unreachable node");
    if (max_stack > bvh.max_stack) fail("stack bound");
    return max_stack;
}

int validate_qbvh(const std::vector<Bvh8QNode>& nodes, const std::vector<uint32_t>& order, const float* pos,
                  uint32_t n, float margin) {
    auto fail = [](const char* what) { throw std::runtime_error(std::string("compressed bvh check: ") + what); };
    const size_t nn = nodes.size();
    if (nn == 0) fail("no root");
    if (order.size() != n) fail("leaf order size");
    std::vector<uint8_t> seen_tri(n, 0), seen_node(nn, 0);
    std::vector<int> depth(nn, 0);
    // top-down: links, leaves, depth; children always lie after their parent
    std::vector<uint32_t> todo{0};
    seen_node[0] = 1;
    depth[0] = 1;
    int max_depth = 1;
    while (!todo.empty()) {
        const uint32_t v = todo.back();
        todo.pop_back();
        const Bvh8QNode& nd = nodes[v];
        max_depth = std::max(max_depth, depth[v]);
        for (int a = 0; a < 3; ++a) {
            const int e = a == 0 ? nd.ex : a == 1 ? nd.ey : nd.ez;
            if (e < -126 || e > 100) fail("grid exponent out of range");
        }
        int rank = 0;
        for (int c = 0; c < 8; ++c) {
            const uint32_t m = nd.meta[c];
            const bool inner_bit = (nd.imask >> c) & 1u;
            if (m == 0) {
                if (inner_bit) fail("empty slot marked inner");
                continue;
            }
            if (nd.qlo_x[c] > nd.qhi_x[c] || nd.qlo_y[c] > nd.qhi_y[c] || nd.qlo_z[c] > nd.qhi_z[c])
                fail("inverted child box");
            if ((m & 0x18u) == 0x18u) {
                if (m != (0x38u | static_cast<uint32_t>(c)) || !inner_bit) fail("inner slot meta");
                const uint64_t ch = static_cast<uint64_t>(nd.child_base) + static_cast<uint64_t>(rank++);
                if (ch >= nn || ch <= v) fail("inner link out of range");
                if (seen_node[ch]) fail("inner node reached twice");
                seen_node[ch] = 1;
                depth[ch] = depth[v] + 1;
                todo.push_back(static_cast<uint32_t>(ch));
                continue;
            }
            if (inner_bit) fail("leaf slot marked inner");
            const uint32_t cb = m >> 5, off = m & 31u;
            const uint32_t cnt = cb == 1u ? 1u : cb == 3u ? 2u : cb == 7u ? 3u : 0u;
            if (cnt == 0 || off + cnt > static_cast<uint32_t>(kQTrisPerNode)) fail("leaf meta");
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint64_t slot = static_cast<uint64_t>(nd.tri_base) + off + k;
                if (slot >= n) fail("leaf range");
                if (seen_tri[slot]) fail("triangle in two leaves");
                seen_tri[slot] = 1;
                if (order[slot] >= n) fail("leaf order entry");
            }
        }
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!seen_tri[i]) fail("triangle in no leaf");
    for (size_t i = 0; i < nn; ++i)
        if (!seen_node[i]) fail("unreachable node");
    // bottom-up: subtree bounds against the decoded child boxes
    std::vector<double> sub(6 * nn);
    const double half = 0.5 * static_cast<double>(margin);
    for (size_t v = nn; v-- > 0;) {
        const Bvh8QNode& nd = nodes[v];
        double box[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        const double p[3] = {nd.px, nd.py, nd.pz};
        const int e[3] = {nd.ex, nd.ey, nd.ez};
        const uint8_t* qlo[3] = {nd.qlo_x, nd.qlo_y, nd.qlo_z};
        const uint8_t* qhi[3] = {nd.qhi_x, nd.qhi_y, nd.qhi_z};
        int rank = 0;
        for (int c = 0; c < 8; ++c) {
            const uint32_t m = nd.meta[c];
            if (m == 0) continue;
            double cb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
            if ((m & 0x18u) == 0x18u) {
                const size_t ch = nd.child_base + static_cast<size_t>(rank++);
                for (int a = 0; a < 6; ++a) cb[a] = sub[6 * ch + a];
            } else {
                const uint32_t cbits = m >> 5, off = m & 31u;
                const uint32_t cnt = cbits == 1u ? 1u : cbits == 3u ? 2u : 3u;
                for (uint32_t k = 0; k < cnt; ++k) {
                    const float* t = pos + 9 * static_cast<size_t>(order[nd.tri_base + off + k]);
                    for (int vtx = 0; vtx < 3; ++vtx)
                        for (int a = 0; a < 3; ++a) {
                            cb[a] = std::min(cb[a], static_cast<double>(t[3 * vtx + a]));
                            cb[3 + a] = std::max(cb[3 + a], static_cast<double>(t[3 * vtx + a]));
                        }
                }
            }
            for (int a = 0; a < 3; ++a) {
                const double lo = p[a] + std::ldexp(static_cast<double>(qlo[a][c]), e[a]);
                const double hi = p[a] + std::ldexp(static_cast<double>(qhi[a][c]), e[a]);
                if (lo > cb[a] - half || hi < cb[3 + a] + half) fail("child box does not contain its subtree");
                box[a] = std::min(box[a], cb[a]);
                box[3 + a] = std::max(box[3 + a], cb[3 + a]);
            }
        }
        for (int a = 0; a < 6; ++a) sub[6 * v + a] = box[a];
    }
    return max_depth;
}

}  // namespace crisb
