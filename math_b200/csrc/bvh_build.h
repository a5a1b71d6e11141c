// Binned-SAH BVH builder for mesh facets.
//
// Reproduces the reference's build (src/geometry/accelerators/bvh_build.h:79-221,
// bvh_split.h:47-315, bvh.cpp:35-86) with the same fixed intersection costs the
// CPU oracle uses, so both produce the same tree: 32 buckets on the axis of
// largest centroid extent, SAH cost with a traversal cost of twice a box
// test, a leaf when no split is cheaper, objects partitioned in place with
// std::partition's element order, and nodes flattened depth first with the
// first child next to its parent.
#pragma once

#include <cstdint>
#include <vector>

namespace nbpt::host
{
// Intersections per second of one primitive per unit of space dimension; a
// cost is dimension / rate seconds.  The CPU oracle pins the reference's
// run-time measured costs to the same values (oracle/pinned_costs.cpp).
inline constexpr double BOX_R_RATE = 2.4e9;
inline constexpr double SIMPLEX_RATE = 0.8e9;

// Entries of the traversal stack (the reference's BvhStack holds 64,
// src/geometry/accelerators/bvh_stack.h:26).  Depth-first traversal keeps at
// most one entry per interior node above the current node, so a tree whose
// leaves are at most this deep (root at depth 0) never overflows it; both
// builders refuse deeper trees, which only degenerate meshes produce.
inline constexpr int BVH_MAX_DEPTH = 64;

template <int N, typename T>
struct BuiltBvh final
{
        std::vector<T> lo;                 // [node][N]
        std::vector<T> hi;                 // [node][N]
        std::vector<std::uint32_t> offset; // leaf: first index slot, interior: second child
        std::vector<std::uint32_t> count;  // 0 for interior nodes
        std::vector<std::uint32_t> axis;
        std::vector<std::uint32_t> indices; // facet per leaf slot
        int depth = 0;                      // of the deepest leaf, the root at 0
};

// vertices: [V][N] in T; facets: [F][N] vertex indices.  Throws
// std::runtime_error if a leaf lies deeper than BVH_MAX_DEPTH.
template <int N, typename T>
BuiltBvh<N, T> build_facet_bvh(const std::vector<T>& vertices, const std::vector<int>& facets);
} // namespace nbpt::host
