// Host BVH builder: binned-SAH binary tree collapsed into a 4-wide tree whose
// nodes are exactly one 128-byte L2 line, and into an 8-wide tree of
// compressed (quantised) 96-byte nodes.  Replaces Bvh::Build/BuildImpl
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

// 8-wide compressed node: three 32-byte sectors.
//   header: per axis a = x, y, z the plane grid step s_a = 2^(e_a - 127) and
//           o2_a = (k_a - 2^23) * s_a, where k_a * s_a is the grid origin
//           (|k_a| < 2^23 - 256).  A quantised plane q in [0, 255] lies at
//           P = (k_a + q) * s_a, which fmaf(2^23 + q, s_a, o2_a) gives exactly
//           (all three values and the result are representable floats).
//   q boxes: qx = {lo bytes of slots 0-3, lo 4-7, hi 0-3, hi 4-7}, same for y, z;
//           lo planes are rounded down and hi planes up, so every child box
//           contains the exact box of its triangles.
//   slots:  children are assigned to slots so that slot (i ^ octant) is
//           roughly the i-th child met by a ray whose direction has sign bits
//           `octant` (bit k set: component k negative); `valid` marks used slots.
struct alignas(32) QNode8 {
    float o2x, o2y, o2z;
    uint32_t meta;          // e_x | e_y << 8 | e_z << 16 | valid << 24
    int32_t child[8];       // same encoding as WideNode4::child
    uint32_t qx[4], qy[4], qz[4];
};
static_assert(sizeof(QNode8) == 96, "compressed node must be three 32-byte sectors");

struct BuildParams {
    int max_leaf = 4;       // triangles per leaf
    int bins = 32;          // SAH bins per axis
    float cost_node = 1.0f; // SAH traversal cost relative to a triangle test
    int threads = 0;        // 0 = hardware concurrency
    bool wide4 = true;      // emit the 4-wide tree
    bool wide8 = true;      // emit the 8-wide compressed tree
};

struct BuildResult {
    std::vector<WideNode4> nodes;   // root at index 0 (always an internal node)
    std::vector<int32_t> order;     // leaf order: order[k] = original triangle index
    int max_depth = 0;
    int max_stack = 0;              // worst-case traversal stack entries
    int64_t nleaves = 0;
    std::vector<QNode8> nodes8;     // 8-wide tree over the same leaves (root at 0)
    int max_depth8 = 0;
    int max_stack8 = 0;
};

// Quantisation of one axis of an 8-wide node whose children span [L, H]:
// returns the exponent e (grid step 2^e) and the origin index k.  Exposed for tests.
constexpr int kQMaxExp = 104;
int qnode_axis(float L, float H, double* k);

// lo/hi/centroid: world-space triangle boxes, 3 floats each, n entries.
// Non-finite boxes are treated as a point at the origin.
BuildResult build_wide_bvh(const float* lo, const float* hi, int64_t n, const BuildParams& p);

}  // namespace bg
