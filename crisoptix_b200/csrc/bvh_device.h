// bvh_device.h -- the scene BVH built on the device (compressed 8-wide or 4-wide nodes).
//
// Stands in for the OptiX GAS/IAS build of the reference (src/Scene.cpp:73-160,
// src/Mesh.cpp:54-120) on the GPU:
//   1. 30-bit Morton codes of the triangle centroids, sorted with the
//      library's radix sort (radix_sort.h);
//   2. a binary tree by PLOC -- parallel locally-ordered clustering (Meister &
//      Bittner, IEEE TVCG 2018): in sorted order every cluster finds the
//      cluster within kPlocRadius positions whose union box has the smallest
//      surface area, mutual nearest neighbours merge, the survivors are
//      compacted, until one cluster is left; node ids come from scans, so the
//      tree does not depend on thread scheduling;
//   3. per node, the surface-area-heuristic choice between a leaf and a split
//      (triangle cost 2, node cost 1, leaves of at most leaf_max triangles),
//      made bottom-up as the nodes are created;
//   4. a top-down collapse into the 4-wide nodes of bvh_build.h, level by
//      level: a wide node opens its children largest surface area first until
//      it has four; leaf children store their triangles contiguously in leaf
//      order; child boxes are widened by box_margin().  Or, for compressed
//      nodes (Bvh8QNode), the SAH-optimal distribution of every subtree over
//      eight child slots (leaves of up to kQLeafMax triangles; after Ylitie,
//      Karras & Laine 2017), found bottom-up in PLOC merge order and taken
//      top-down level by level; children placed in octant slots, boxes
//      quantised outward on the node's grid.
// The 4-wide tree lands in the same node and triangle layouts the host
// builder (bvh_build.h) produces, so its traversal is shared; the compressed
// tree keeps the same leaf-ordered triangle layout.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "bvh_build.h"

namespace crisb {

struct DeviceWideBvh {
    Bvh4Node* nodes = nullptr;    // device, root at 0 (4-wide build)
    Bvh8QNode* qnodes = nullptr;  // device, root at 0 (compressed 8-wide build)
    uint32_t num_nodes = 0;
    float4* tris = nullptr;     // device, 3 per triangle in leaf order, triangle id bits in tris[3i+2].w
    int binary_depth = 0;       // levels of the collapse
};

// Builds from world-space positions on the device (pos_dev: 9 floats per
// triangle).  `compressed`: the collapse makes compressed 8-wide nodes
// (Bvh8QNode, leaves of at most kQLeafMax triangles) instead of 4-wide ones.
// Allocates nodes (or qnodes) and tris with cudaMalloc (free them with
// cudaFree); synchronises `st` between clustering and collapse steps.
// Returns cudaSuccess or the first CUDA error.
cudaError_t build_wide_bvh_device(const float* pos_dev, uint32_t n, int leaf_max, float margin, bool compressed,
                                  cudaStream_t st, DeviceWideBvh* out);

}  // namespace crisb
