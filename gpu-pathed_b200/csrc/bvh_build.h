// Host BVH construction: binned-SAH binary tree collapsed to a W-wide tree (W = 2, 4, 8).
//
// The reference has no acceleration structure on its CUDA path: World::hit scans every
// triangle and then every sphere (src/world.cu:5-41). The wide BVH replaces that scan. Its
// child boxes are padded outward by a few ulps of their coordinates so that traversal never
// culls a primitive the reference's scan would accept; the closest-hit rule (total order on
// t, ties to the highest triangle index, triangles before spheres) is applied in the leaf
// test, so the order in which leaves are visited does not change the result.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "host_scene.h"

namespace pt {

struct BvhBuild {
    int width = 4;
    int root = 0;
    int num_nodes = 0;
    int depth = 0;              // wide-tree depth, root level = 1
    int max_leaf = 0;           // largest leaf
    std::vector<uint8_t> nodes; // num_nodes * sizeof(BvhNode<width>)
    std::vector<float> prims;   // 12 floats (3 float4) per leaf entry
    std::vector<int> prim_order;// leaf entry -> primitive id (>= 0 triangle, ~id sphere)
    double build_ms = 0.0;
    double sah_cost = 0.0;
};

// max_leaf in [1, 16]. Returns false with a message on invalid input.
bool build_bvh(const HostScene& s, int width, int max_leaf, BvhBuild& out, std::string& err);

// Structural self-check used by the tests: every primitive referenced exactly once, every
// primitive contained in the padded boxes of all its ancestors, child codes in range.
bool check_bvh(const HostScene& s, const BvhBuild& b, std::string& err);

// Quantized nodes (qnode_bytes(b.width) each) against the float nodes they replace: the same
// child codes, and every decoded child box, fmaf(q, scale, origin) per plane, containing the
// float child box.
bool check_qnodes(const BvhBuild& b, const std::vector<uint8_t>& q, std::string& err);

// Append a scene's BVH to the shared BVH of a batch (node, leaf-entry and primitive-id
// offsets applied; the scene's primitives start at tri_base / sph_base). Returns its root.
int append_bvh(const BvhBuild& b, int tri_base, int sph_base, BvhBuild& into);

}  // namespace pt
