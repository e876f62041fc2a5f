// Host BVH builder: binned-SAH binary tree collapsed into a 4-wide tree whose
// nodes are exactly one 128-byte L2 line.  Replaces Bvh::Build/BuildImpl
// (accelerator/bvh.cpp:16-496); the tree differs from the reference's (leaves
// of up to max_leaf triangles, full-depth SAH, wide nodes), which changes only
// the visit order, never the set of accepted triangles.
#pragma once

#include <cstdint>
#include <vector>

namespace bg {

// Child slot encoding of a wide node.
//   internal child : index of the child node (0 <= c < 2^31 - 1)
//   leaf child     : bit 31 set, bits 27..30 = count-1, bits 0..26 = first triangle
//   empty slot     : kEmptyChild (its box is inverted, so it is never entered)
constexpr int32_t kEmptyChild = 0x7fffffff;
constexpr int kLeafStartBits = 27;
constexpr int32_t kMaxLeafStart = (1 << kLeafStartBits) - 1;

inline int32_t encode_leaf(int32_t start, int32_t count) {
    return int32_t(0x80000000u | (uint32_t(count - 1) << kLeafStartBits) | uint32_t(start));
}

struct alignas(16) WideNode4 {      // 128 bytes: one L2 line
    float lox[4], hix[4];
    float loy[4], hiy[4];
    float loz[4], hiz[4];
    int32_t child[4];
    int32_t pad[4];
};
static_assert(sizeof(WideNode4) == 128, "wide node must be one 128-byte line");

struct BuildParams {
    int max_leaf = 4;       // triangles per leaf
    int bins = 32;          // SAH bins per axis
    float cost_node = 1.0f; // SAH traversal cost relative to a triangle test
    int threads = 0;        // 0 = hardware concurrency
};

struct BuildResult {
    std::vector<WideNode4> nodes;   // root at index 0 (always an internal node)
    std::vector<int32_t> order;     // leaf order: order[k] = original triangle index
    int max_depth = 0;
    int max_stack = 0;              // worst-case traversal stack entries
    int64_t nleaves = 0;
};

// lo/hi/centroid: world-space triangle boxes, 3 floats each, n entries.
// Non-finite boxes are treated as a point at the origin.
BuildResult build_wide_bvh(const float* lo, const float* hi, int64_t n, const BuildParams& p);

}  // namespace bg
