// The host's BVH builder: a binned surface-area-heuristic tree over the scene's primitive boxes, in double, with
// leaves of one primitive kind and boxes rounded outward to float (a float box must contain what the float tests
// accept, src/gpu/bvh.cuh:129-187). The reference splits at the object median on the longest axis (bvh.ixx:53-73,
// bvh.cuh:382-435); the SAH tree visits fewer nodes per ray for the same hits, and the first-hit parity test compares
// hits in source index space, so the two trees need not agree node for node.
#pragma once

#include <cstdint>
#include <vector>

#include "device_types.h"

namespace rtb
{
struct build_prim
{
    double lo[3];
    double hi[3];
    int32_t kind;   // kind_sphere, kind_quad, kind_triangle
    int32_t source; // index in that kind's source table
};

struct bvh_options
{
    int max_leaf_size = 1;   // 1..7
    int bins = 32;
    double node_cost = 1.0;  // the SAH's cost of a node fetch, in primitive tests
    int threads = 0;         // host threads for the subtrees (0: every hardware thread); the tree is the same for any
};

struct bvh_result
{
    std::vector<bvh_node> nodes;
    std::vector<int32_t> order[3]; // per kind, the source indices in leaf order: the kind's device array order
    int32_t depth = 0;
    int64_t leaves = 0;
};

// Throws std::runtime_error when the tree would be deeper than the traversal stack (max_bvh_depth)
bvh_result build_bvh(std::vector<build_prim> prims, const bvh_options& options);

// The binary tree collapsed four wide (each node takes its children's children, the largest first, while it has
// fewer than four); returns the wide tree's depth. The children's boxes are the binary nodes' own, so both walks
// test the same boxes.
int32_t collapse_bvh4(const std::vector<bvh_node>& nodes, std::vector<bvh4_node>& out);

// A double bound rounded to float toward -inf / +inf
float round_down(double x);
float round_up(double x);
} // namespace rtb
