// bvh_build.h -- node formats of the scene BVH and its host builder and validators.
//
// Stands in for the OptiX GAS/IAS build of the reference
// (src/Scene.cpp:73-160, src/Mesh.cpp:54-120): a binned-SAH binary
// tree over the flattened triangles, collapsed greedily (largest surface area
// first) into 4-wide nodes.  Every child box is widened by box_margin(): the
// watertight triangle test accepts rays a few ulp of the origin-vertex
// distance outside the exact triangle (and t to a few ulp), and the slab test
// cuts a ray lying in a box face plane off at t = 0, so exact boxes can reject
// a ray the triangle test accepts.  With the margin, the box test is at least
// an order of magnitude more generous than those errors, every tree gives the
// hits of testing all triangles, and the tree shape only changes speed.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace crisb {

#ifndef CRISB_BVH_WIDTH
#define CRISB_BVH_WIDTH 4
#endif
// children per node (4: one 128-byte line per node; 8: two).  8-wide nodes
// cut node visits from 16.3 to 10.1 per ray on the 1080p workload but doubled
// the traversal time (27.3 against 13.6 ms per frame): the eight box tests
// and the sort of eight children per step cost more than the saved steps.
constexpr int kBvhWidth = CRISB_BVH_WIDTH;
static_assert(kBvhWidth == 4 || kBvhWidth == 8, "BVH width 4 or 8");

// wide node: child boxes as structure of arrays, child links (>= 0 inner
// node, -1-first a leaf of `count` triangles starting at `first` in leaf
// order, kNoChild an empty slot)
struct alignas(128) Bvh4Node {
    float lo_x[kBvhWidth], hi_x[kBvhWidth], lo_y[kBvhWidth], hi_y[kBvhWidth], lo_z[kBvhWidth], hi_z[kBvhWidth];
    int link[kBvhWidth];
    int count[kBvhWidth];
};
static_assert(sizeof(Bvh4Node) == 32 * kBvhWidth, "node size");

constexpr int kNoChild = 0x7fffffff;

// box widening for a scene whose largest coordinate magnitude is max_abs:
// 2^-17 x max_abs (rays are taken to start within twice that magnitude)
inline float box_margin(float max_abs) { return std::ldexp(max_abs > 1e-20f ? max_abs : 1e-20f, -17); }

struct WideBvh {
    std::vector<Bvh4Node> nodes;  // root at 0
    std::vector<uint32_t> order;  // leaf order -> triangle index
    int max_stack = 0;            // worst-case traversal stack entries
    int max_depth = 0;            // depth of the binary tree
};

// Compressed 8-wide node (80 bytes, five 16-byte loads), after Ylitie, Karras
// & Laine 2017 ("Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs").  Per axis the child boxes lie on the grid
// p + 2^e * q, q in [0, 255], rounded outward from boxes already widened by
// box_margin().  Inner children are stored contiguously from child_base in
// slot order, leaf triangles contiguously (leaf order) from tri_base.  Per
// slot, meta is
//   0                   an empty slot,
//   0b001'11sss         an inner child (sss = the slot),
//   0b ccc'ooooo        a leaf: ccc = 1, 3 or 7 for 1-3 triangles at
//                       tri_base + ooooo (ooooo < 24).
// Children are placed in slots by the octant of their centroid relative to
// the node's (slot bit a set: toward +a), so a ray whose direction signs give
// octant o (bit a set: negative along a) meets the child in slot o ^ k
// roughly k-th.
struct alignas(16) Bvh8QNode {
    float px, py, pz;
    int8_t ex, ey, ez;
    uint8_t imask;  // bit s: slot s holds an inner child
    uint32_t child_base, tri_base;
    uint8_t meta[8];
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8], qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(Bvh8QNode) == 80, "compressed node size");
constexpr int kQLeafMax = 3;      // triangles per leaf child of a compressed node
constexpr int kQTrisPerNode = 24;  // triangles per compressed node
// the compressed format needs |coordinates| below this (the slab test's
// per-node terms stay finite for every ray direction; larger scenes use
// 4-wide nodes)
constexpr float kQMaxCoord = 1.6e7f;

// Structural check of a compressed tree: node links in range and each node
// reached once, leaves of 1-3 triangles inside the node's 24, every triangle
// in exactly one leaf, every decoded child box containing its subtree's
// triangles widened by half the margin (compared in double precision), grid
// exponents in range.  `order`: leaf order -> triangle.  Returns the depth of
// the tree (the traversal's group-stack bound).  Throws std::runtime_error.
int validate_qbvh(const std::vector<Bvh8QNode>& nodes, const std::vector<uint32_t>& order, const float* pos,
                  uint32_t num_tris, float margin);

// `pos`: 9 floats per triangle (three vertices).  Leaves hold at most
// `leaf_max` triangles; below `median_depth` binary levels the SAH split is
// replaced by object-median splits so the depth stays logarithmic.
WideBvh build_wide_bvh(const float* pos, uint32_t num_tris, int leaf_max, int median_depth);

// Structural check before the tree goes to the device: links in range, every
// triangle in exactly one leaf, leaves of at most `leaf_max` triangles, child
// boxes containing their subtrees, each inner node reached once, and the
// traversal stack bound recomputed (it must not exceed bvh.max_stack, and is
// returned).  Throws std::runtime_error on a failure.
int validate_wide_bvh(const WideBvh& bvh, const float* pos, uint32_t num_tris, int leaf_max);

}  // namespace crisb
