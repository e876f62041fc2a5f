// Device BVH build, from world-space triangle boxes in HBM to the 4-wide and
// 8-wide node arrays and the leaf order, with nothing but counters crossing
// to the host.  Replaces the host binned-SAH build (Bvh::Build,
// accelerator/bvh.cpp:16-496) when build time matters more than tree quality;
// hits are identical whichever tree is traversed.
//
//  1. Morton order: 63-bit codes of the box centroids (21 bits per axis over
//     the centroid bounds), CUB radix sort.  Leaf p is the p-th triangle in
//     that order; internal nodes are numbered n, n + 1, ...
//  2. Binary tree, one of
//     - builder 1, LBVH (Karras, "Maximizing Parallelism in the Construction
//       of BVHs, Octrees, and k-d Trees", HPG 2012): one thread per internal
//       node finds its key range and split by binary search;
//     - builder 2, PLOC (Meister and Bittner, "Parallel Locally-Ordered
//       Clustering for Bounding Volume Hierarchy Construction", TVCG 2018):
//       the sorted triangles are clusters; every round each cluster finds the
//       neighbour within 16 positions whose union box has the least surface
//       area, mutual pairs merge, and the survivors are compacted in order.
//  3. Bottom-up pass (the second child to finish computes its parent):
//     boxes, triangle counts, and the SAH choice between a subtree as one leaf
//     (count x area) and as a split (area + the children's costs; one node
//     visit costs one triangle test); subtrees of at most max_leaf triangles
//     that are cheaper as a leaf become leaves.
//  4. Top-down collapse, one launch per level of the wide tree: each wide node
//     opens the largest-area internal child until it has 4 (or 8) children,
//     the same rule as the host collapse; its internal children get node
//     slots and join the next level.  Leaf triangles are numbered in
//     left-to-right order of the binary tree, so every leaf is one range of
//     the leaf order.  8-wide nodes are quantised on the device (qnode.h).
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <vector>

#include "bvh_build.h"
#include "internal.h"
#include "qnode.h"

namespace bg {
namespace {

constexpr int kBT = 256;            // threads per block of the build kernels
constexpr int kBGrid = 148 * 8;     // blocks of the grid-stride launches
constexpr int kPlocRadius = 16;
constexpr int kMaxWideLevels = 128; // deeper trees exceed every traversal stack anyway

__device__ __forceinline__ unsigned int f2ord(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// centroid bounds, as order-preserving integers (min over x,y,z then max)
__global__ void k_centroid_bounds(const float* __restrict__ lo, const float* __restrict__ hi, int64_t n,
                                  unsigned int* __restrict__ cb) {
    unsigned int mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned int c = f2ord(0.5f * (lo[3 * i + k] + hi[3 * i + k]));
            mn[k] = min(mn[k], c);
            mx[k] = max(mx[k], c);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[k] = min(mn[k], __shfl_down_sync(0xffffffffu, mn[k], off));
            mx[k] = max(mx[k], __shfl_down_sync(0xffffffffu, mx[k], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(cb + k, mn[k]);
            atomicMax(cb + 3 + k, mx[k]);
        }
    }
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {   // 21 bits -> every third of 63
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const float* __restrict__ lo, const float* __restrict__ hi, int64_t n,
                         const unsigned int* __restrict__ cb, uint64_t* __restrict__ keys, int32_t* __restrict__ idx) {
    float cmin[3], scale[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        cmin[k] = ord2f(cb[k]);
        const float ext = ord2f(cb[3 + k]) - cmin[k];
        scale[k] = ext > 0.f ? 2097151.f / ext : 0.f;
    }
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint64_t key = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (lo[3 * i + k] + hi[3 * i + k]);
            float q = (c - cmin[k]) * scale[k];
            q = fminf(fmaxf(q, 0.f), 2097151.f);
            key |= spread21(uint64_t(q)) << (2 - k);
        }
        keys[i] = key;
        idx[i] = int32_t(i);
    }
}

// node boxes of the leaves (node p = Morton position p); a non-finite box is a
// point at the origin, as in the host builder.  cl (optional): cl[p] = p.
__global__ void k_leaf_boxes(const float* __restrict__ lo, const float* __restrict__ hi,
                             const int32_t* __restrict__ sorted, int64_t n, float* __restrict__ box,
                             int32_t* __restrict__ cl) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        const int64_t t = sorted[p];
        bool finite = true;
        for (int k = 0; k < 3; ++k) finite = finite && isfinite(lo[3 * t + k]) && isfinite(hi[3 * t + k]);
        float* b = box + 6 * p;
        for (int k = 0; k < 3; ++k) {
            b[k] = finite ? lo[3 * t + k] : 0.f;
            b[3 + k] = finite ? hi[3 * t + k] : 0.f;
        }
        if (cl) cl[p] = int32_t(p);
    }
}

// ---------------------------------------------------------------- LBVH
// common-prefix length of sorted keys i and j (ties broken by index); -1 outside [0, n)
__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a != b) return __clzll(a ^ b);
    return 64 + __clzll(uint64_t(i) ^ uint64_t(j));
}

// Internal node n + i (i < n - 1; the root is n): children and parents in
// the unified numbering (leaves 0..n-1, internal nodes n..2n-2).
__global__ void k_radix_tree(const uint64_t* __restrict__ keys, int64_t n, int32_t* __restrict__ left,
                             int32_t* __restrict__ right, int32_t* __restrict__ parent) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n - 1; i += int64_t(gridDim.x) * blockDim.x) {
        const int d = delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1) >= 0 ? 1 : -1;
        const int dmin = delta(keys, n, i, i - d);
        int64_t lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int64_t l = 0;
        for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int64_t j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int64_t s = 0;
        for (int64_t t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int64_t g = i + s * d + (d < 0 ? -1 : 0);
        const int64_t lo_ = d > 0 ? i : j, hi_ = d > 0 ? j : i;
        const int32_t me = int32_t(n + i);
        const int32_t a = lo_ == g ? int32_t(g) : int32_t(n + g);
        const int32_t b = hi_ == g + 1 ? int32_t(g + 1) : int32_t(n + g + 1);
        left[me] = a;
        right[me] = b;
        parent[a] = me;
        parent[b] = me;
        if (i == 0) parent[me] = -1;
    }
}

// ---------------------------------------------------------------- PLOC
__device__ __forceinline__ float merged_area(const float* a, const float* b) {
    const float ex = fmaxf(a[3], b[3]) - fminf(a[0], b[0]);
    const float ey = fmaxf(a[4], b[4]) - fminf(a[1], b[1]);
    const float ez = fmaxf(a[5], b[5]) - fminf(a[2], b[2]);
    return ex * ey + ey * ez + ez * ex;
}

// Equal areas (duplicate triangles) are ordered by a key symmetric in the
// pair: nearer positions first, then pairs whose lower end is even, so a run
// of identical clusters pairs up as (0,1), (2,3), ... instead of all pointing
// at one end.  With a symmetric total order on pairs the smallest pair is
// always mutual, so every round merges.
__device__ __forceinline__ bool tie_before(int i, int j, int k) {   // is pair (i,j) before pair (i,k)?
    if (k < 0) return true;
    const int dj = abs(i - j), dk = abs(i - k);
    if (dj != dk) return dj < dk;
    const int lj = min(i, j), lk = min(i, k);
    if ((lj & 1) != (lk & 1)) return (lj & 1) == 0;
    return lj < lk;
}

// The cluster count m lives on the device (written by the compaction), so the
// rounds run back to back; m_bound >= m sizes the launches and CUB passes.
__global__ void k_ploc_nn(const int32_t* __restrict__ cl, const int* __restrict__ m_dev,
                          const float* __restrict__ box, int32_t* __restrict__ nn) {
    const int m = *m_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const float* bi = box + 6 * size_t(cl[i]);
        float best = FLT_MAX;
        int bj = -1;
        const int j0 = max(0, i - kPlocRadius), j1 = min(m - 1, i + kPlocRadius);
        for (int j = j0; j <= j1; ++j) {
            if (j == i) continue;
            const float a = merged_area(bi, box + 6 * size_t(cl[j]));
            if (a < best || (a == best && tie_before(i, j, bj))) { best = a; bj = j; }
        }
        nn[i] = bj;
    }
}

// leader of a mutual pair (the lower index) creates the merged node
__global__ void k_ploc_flags(const int32_t* __restrict__ nn, const int* __restrict__ m_dev, int m_bound,
                             int32_t* __restrict__ lead, int32_t* __restrict__ keep) {
    const int m = *m_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m_bound; i += gridDim.x * blockDim.x) {
        if (i >= m) { lead[i] = 0; keep[i] = 0; continue; }
        const int j = nn[i];
        const bool mutual = j >= 0 && nn[j] == i;
        lead[i] = (mutual && i < j) ? 1 : 0;
        keep[i] = (mutual && i > j) ? 0 : 1;       // the higher partner disappears
    }
}

__global__ void k_ploc_merge(int32_t* __restrict__ cl, const int32_t* __restrict__ nn, const int* __restrict__ m_dev,
                             const int32_t* __restrict__ lead, const int32_t* __restrict__ lead_scan,
                             const int32_t* __restrict__ base_dev, float* __restrict__ box, int32_t* __restrict__ left,
                             int32_t* __restrict__ right, int32_t* __restrict__ parent) {
    const int m = *m_dev;
    const int32_t base = *base_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (!lead[i]) continue;
        const int j = nn[i];
        const int32_t node = base + lead_scan[i];
        const int32_t a = cl[i], b = cl[j];
        const float* ba = box + 6 * size_t(a);
        const float* bb = box + 6 * size_t(b);
        float* o = box + 6 * size_t(node);
        for (int k = 0; k < 3; ++k) { o[k] = fminf(ba[k], bb[k]); o[3 + k] = fmaxf(ba[3 + k], bb[3 + k]); }
        left[node] = a;
        right[node] = b;
        parent[a] = node;
        parent[b] = node;
        cl[i] = node;
    }
}

// next free node index += this round's merges
__global__ void k_ploc_advance(int32_t* __restrict__ base_dev, const int32_t* __restrict__ lead_scan,
                               const int32_t* __restrict__ lead, int m_bound) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *base_dev += lead_scan[m_bound - 1] + lead[m_bound - 1];
}

// ---------------------------------------------------------------- bottom-up SAH
__device__ __forceinline__ float half_area(const float* b) {
    const float ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
    return ex * ey + ey * ez + ez * ex;
}

// One thread per leaf climbs while it is the second child to arrive; boxes,
// counts and costs of other threads' nodes are read through L2 (ld.cg) after
// the arrival counter shows them complete.
__global__ void k_bottom_up(int64_t n, const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                            const int32_t* __restrict__ parent, float* box, int32_t* cnt, float* cost,
                            uint8_t* __restrict__ mk, int* __restrict__ visits, int max_leaf, float cost_node,
                            int* __restrict__ nopen) {          // nopen[0]: non-leaf internal nodes, [1]: error
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        __stcg(cnt + p, 1);
        __stcg(cost + p, half_area(box + 6 * p));
        mk[p] = 1;
        __threadfence();
        int32_t v = parent[p];
        for (int64_t steps = 0; v >= 0; ++steps) {
            if (steps >= n) { atomicOr(nopen + 1, 1); break; }   // a parent cycle: report, never spin
            if (atomicAdd(visits + v, 1) == 0) break;      // the sibling finishes this node
            __threadfence();
            const int32_t a = left[v], c = right[v];
            float ub[6];
            for (int k = 0; k < 3; ++k) {
                ub[k] = fminf(__ldcg(box + 6 * size_t(a) + k), __ldcg(box + 6 * size_t(c) + k));
                ub[3 + k] = fmaxf(__ldcg(box + 6 * size_t(a) + 3 + k), __ldcg(box + 6 * size_t(c) + 3 + k));
            }
            const int32_t tot = __ldcg(cnt + a) + __ldcg(cnt + c);
            const float av = half_area(ub);
            const float split = cost_node * av + __ldcg(cost + a) + __ldcg(cost + c);
            const float as_leaf = float(tot) * av;
            const bool leaf = tot <= max_leaf && as_leaf <= split;
            for (int k = 0; k < 6; ++k) __stcg(box + 6 * size_t(v) + k, ub[k]);
            __stcg(cnt + v, tot);
            __stcg(cost + v, leaf ? as_leaf : split);
            mk[v] = leaf ? 1 : 0;
            if (!leaf) atomicAdd(nopen, 1);
            __threadfence();
            v = parent[v];
        }
    }
}

// ---------------------------------------------------------------- top-down collapse
struct CItem {                // one wide node to fill
    int32_t v;                // its binary node
    int32_t slot;             // its index in the wide node array
    int32_t off;              // first leaf-order position of its triangles
    int16_t depth, stack;     // depth (root 1) and traversal stack entries above it
};
static_assert(sizeof(CItem) == 16, "collapse item is 16 bytes");

struct CollapseArgs {
    const int32_t* left;
    const int32_t* right;
    const float* box;
    const int32_t* cnt;
    const uint8_t* mk;
    const int32_t* sorted;    // Morton position -> triangle
    int32_t* order;           // leaf order written by this pass (nullptr: not written)
    int64_t n;
    int* counts;              // [3] frontier sizes, a ring over the levels
    int* nodecount;           // wide node slots handed out
    int* stats;               // [0] max depth, [1] max stack, [2] flags: 1 overflow, 2 quantisation failed
    int capacity;             // wide node slots and frontier entries available
};

__device__ __forceinline__ float box_area2(const float* b) {   // full surface area, as the host collapse
    const float e0 = b[3] - b[0], e1 = b[4] - b[1], e2 = b[5] - b[2];
    if (e0 < 0.f || e1 < 0.f || e2 < 0.f) return 0.f;
    return 2.f * (e0 * e1 + e0 * e2 + e1 * e2);
}

__device__ __forceinline__ int32_t leaf_code(int32_t start, int32_t count) {
    return int32_t(0x80000000u | (uint32_t(count - 1) << kLeafStartBits) | uint32_t(start));
}

// triangles of leaf subtree v, left to right, at order[off ...]
__device__ void write_leaf_order(const CollapseArgs& A, int32_t v, int32_t off) {
    int32_t st[34];
    int sp = 0;
    st[sp++] = v;
    while (sp > 0) {
        const int32_t u = st[--sp];
        if (u < A.n) {
            if (off < A.n) A.order[off] = A.sorted[u];
            ++off;
            continue;
        }
        if (sp > 31) { atomicOr(A.stats + 2, 1); return; }
        st[sp++] = A.right[u];
        st[sp++] = A.left[u];
    }
}

template <int W>
__global__ void __launch_bounds__(kBT) k_collapse(const CItem* __restrict__ cur, CItem* __restrict__ next, int level,
                                                  CollapseArgs A, void* __restrict__ out) {
    const int m = min(A.counts[level % 3], A.capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0) A.counts[(level + 2) % 3] = 0;   // the level after next appends there
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const CItem it = cur[i];
        int32_t kv[W], ko[W];
        kv[0] = A.left[it.v];
        kv[1] = A.right[it.v];
        ko[0] = it.off;
        ko[1] = it.off + A.cnt[kv[0]];
        int nk = 2;
        while (nk < W) {          // open the largest-area internal child
            int best = -1;
            float ba = -1.f;
            for (int j = 0; j < nk; ++j) {
                const int32_t c = kv[j];
                if (c >= A.n && !A.mk[c]) {
                    const float a = box_area2(A.box + 6 * size_t(c));
                    if (a > ba) { ba = a; best = j; }
                }
            }
            if (best < 0) break;
            const int32_t c = kv[best], o = ko[best];
            const int32_t l = A.left[c];
            kv[best] = l;
            ko[best] = o;
            kv[nk] = A.right[c];
            ko[nk] = o + A.cnt[l];
            ++nk;
        }
        const int stack_here = it.stack + nk - 1;
        atomicMax(A.stats + 0, int(it.depth));
        atomicMax(A.stats + 1, stack_here);
        int32_t codes[W];
        for (int j = 0; j < nk; ++j) {
            const int32_t c = kv[j];
            if (c < A.n || A.mk[c]) {
                codes[j] = leaf_code(ko[j], A.cnt[c]);
                if (A.order) write_leaf_order(A, c, ko[j]);
                continue;
            }
            const int slot = atomicAdd(A.nodecount, 1);
            const int q = atomicAdd(A.counts + (level + 1) % 3, 1);
            if (slot >= A.capacity || q >= A.capacity) {
                atomicOr(A.stats + 2, 1);
                codes[j] = kEmptyChild;
                continue;
            }
            next[q] = CItem{c, slot, ko[j], int16_t(it.depth + 1), int16_t(stack_here)};
            codes[j] = slot;
        }
        if constexpr (W == 4) {
            WideNode4 w;
            for (int j = 0; j < 4; ++j) {
                if (j < nk) {
                    const float* b = A.box + 6 * size_t(kv[j]);
                    w.lox[j] = b[0]; w.loy[j] = b[1]; w.loz[j] = b[2];
                    w.hix[j] = b[3]; w.hiy[j] = b[4]; w.hiz[j] = b[5];
                    w.child[j] = codes[j];
                } else {
                    w.lox[j] = w.loy[j] = w.loz[j] = FLT_MAX;
                    w.hix[j] = w.hiy[j] = w.hiz[j] = -FLT_MAX;
                    w.child[j] = kEmptyChild;
                }
                w.pad[j] = 0;
            }
            static_cast<WideNode4*>(out)[it.slot] = w;
        } else {
            float kb[8][6];
            for (int j = 0; j < nk; ++j)
                for (int k = 0; k < 6; ++k) kb[j][k] = A.box[6 * size_t(kv[j]) + k];
            QNode8 q;
            if (!fill_qnode8(q, kb, codes, nk)) atomicOr(A.stats + 2, 2);
            static_cast<QNode8*>(out)[it.slot] = q;
        }
    }
}

struct WideOut {
    int64_t nodes = 0;
    int max_depth = 0, max_stack = 0;
    bool quant_ok = true;
};

// Runs the collapse of width W from the root; the nodes land in `nodes`
// (grown to the exact size).  order != nullptr: this pass writes the leaf order.
template <int W>
int run_collapse(CollapseArgs A, int32_t root, int capacity, int32_t* order, DevBuf& nodes, WideOut& r) {
    const size_t node_bytes = W == 4 ? sizeof(WideNode4) : sizeof(QNode8);
    struct Scratch {
        ScratchBuf items0, items1, ctr, out;
    } S;
    int rc;
    if ((rc = S.items0.ensure(size_t(capacity) * sizeof(CItem))) ||
        (rc = S.items1.ensure(size_t(capacity) * sizeof(CItem))) || (rc = S.ctr.ensure(8 * sizeof(int))) ||
        (rc = S.out.ensure(size_t(capacity) * node_bytes)))
        return rc;
    const int init[8] = {1, 0, 0, 1, 0, 0, 0, 0};   // counts ring, nodecount (root = slot 0), stats
    BG_CUDA(cudaMemcpy(S.ctr.ptr, init, sizeof(init), cudaMemcpyHostToDevice));
    const CItem root_item{root, 0, 0, 1, 0};
    BG_CUDA(cudaMemcpy(S.items0.ptr, &root_item, sizeof(CItem), cudaMemcpyHostToDevice));
    int* ctr = S.ctr.as<int>();
    A.counts = ctr;
    A.nodecount = ctr + 3;
    A.stats = ctr + 4;
    A.capacity = capacity;
    A.order = order;
    const int grid = int(std::min<int64_t>(kBGrid, (int64_t(capacity) + kBT - 1) / kBT));
    for (int level = 0;; ++level) {
        if (level >= kMaxWideLevels)
            return set_error(BG_ERR_UNSUPPORTED, "device BVH deeper than %d %d-wide levels", kMaxWideLevels, W);
        CItem* cur = (level & 1) ? S.items1.as<CItem>() : S.items0.as<CItem>();
        CItem* nxt = (level & 1) ? S.items0.as<CItem>() : S.items1.as<CItem>();
        k_collapse<W><<<grid, kBT>>>(cur, nxt, level, A, S.out.ptr);
        if ((level & 7) == 7) {
            BG_CUDA(cudaGetLastError());
            int pending = 0;
            BG_CUDA(cudaMemcpy(&pending, ctr + (level + 1) % 3, sizeof(int), cudaMemcpyDeviceToHost));
            if (pending == 0) break;
        }
    }
    int h[8];
    BG_CUDA(cudaMemcpy(h, ctr, sizeof(h), cudaMemcpyDeviceToHost));
    if ((h[6] & 1) || h[3] > capacity)
        return set_error(BG_ERR_OVERFLOW, "device BVH collapse exceeded its %d node slots", capacity);
    r.nodes = h[3];
    r.max_depth = h[4];
    r.max_stack = h[5];
    r.quant_ok = !(h[6] & 2);
    if ((rc = nodes.ensure(size_t(r.nodes) * node_bytes))) return rc;
    BG_CUDA(cudaMemcpy(nodes.ptr, S.out.ptr, size_t(r.nodes) * node_bytes, cudaMemcpyDeviceToDevice));
    return BG_OK;
}

}  // namespace

int gpu_build_bvh(const float* lo, const float* hi, int64_t n, int builder, const BuildParams& bp, int32_t* order,
                  DevBuf& nodes4, DevBuf& nodes8, DeviceBvh& out) {
    if (n < 2) return set_error(BG_ERR_INVALID_ARG, "device build needs at least 2 triangles");
    if (n > (int64_t(1) << 29)) return set_error(BG_ERR_UNSUPPORTED, "device build: too many triangles");
    if (builder < 1 || builder > 3) return set_error(BG_ERR_INVALID_ARG, "device builder %d", builder);
    struct Scratch {
        ScratchBuf cb, keys, keys2, idx, sorted, left, right, parent, box, cnt, cost, mk, visits, nopen, tmp;
        ScratchBuf cl, cl2, nn, lead, scan, keep, nsel;
    } S;
    const size_t N = size_t(n), NN = 2 * N - 1;
    int rc;
    if ((rc = S.cb.ensure(32)) || (rc = S.keys.ensure(N * 8)) || (rc = S.keys2.ensure(N * 8)) ||
        (rc = S.idx.ensure(N * 4)) || (rc = S.sorted.ensure(N * 4)) || (rc = S.left.ensure(NN * 4)) ||
        (rc = S.right.ensure(NN * 4)) || (rc = S.parent.ensure(NN * 4)) || (rc = S.box.ensure(NN * 24)) ||
        (rc = S.cnt.ensure(NN * 4)) || (rc = S.cost.ensure(NN * 4)) || (rc = S.mk.ensure(NN)) ||
        (rc = S.visits.ensure(NN * 4)) || (rc = S.nopen.ensure(2 * sizeof(int))))
        return rc;
    if (builder == 2 &&
        ((rc = S.cl.ensure(N * 4)) || (rc = S.cl2.ensure(N * 4)) || (rc = S.nn.ensure(N * 4)) ||
         (rc = S.lead.ensure(N * 4)) || (rc = S.scan.ensure(N * 4)) || (rc = S.keep.ensure(N * 4)) ||
         (rc = S.nsel.ensure(8))))
        return rc;
    const int blocks = int(std::min<int64_t>(kBGrid, (n + kBT - 1) / kBT));
    int32_t root = int32_t(n);
    if (builder == 3) {
        // top-down binned SAH on the device (sah_build.cu): tree and final order
        if ((rc = sah_binary_tree(lo, hi, n, S.sorted.as<int32_t>(), S.left.as<int32_t>(), S.right.as<int32_t>(),
                                  S.parent.as<int32_t>())))
            return rc;
        k_leaf_boxes<<<blocks, kBT>>>(lo, hi, S.sorted.as<int32_t>(), n, S.box.as<float>(), nullptr);
        BG_CUDA(cudaGetLastError());
    } else {
        const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        BG_CUDA(cudaMemcpy(S.cb.ptr, init, sizeof(init), cudaMemcpyHostToDevice));
        k_centroid_bounds<<<blocks, kBT>>>(lo, hi, n, S.cb.as<unsigned int>());
        k_morton<<<blocks, kBT>>>(lo, hi, n, S.cb.as<unsigned int>(), S.keys.as<uint64_t>(), S.idx.as<int32_t>());
        BG_CUDA(cudaGetLastError());
        size_t b1 = 0, b2 = 0, b3 = 0;
        BG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, S.keys.as<uint64_t>(), S.keys2.as<uint64_t>(),
                                                S.idx.as<int32_t>(), S.sorted.as<int32_t>(), int(n), 0, 63));
        if (builder == 2) {
            BG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b2, S.lead.as<int32_t>(), S.scan.as<int32_t>(), int(n)));
            BG_CUDA(cub::DeviceSelect::Flagged(nullptr, b3, S.cl.as<int32_t>(), S.keep.as<int32_t>(),
                                               S.cl2.as<int32_t>(), S.nsel.as<int32_t>(), int(n)));
        }
        const size_t tb = std::max(b1, std::max(b2, b3));
        if ((rc = S.tmp.ensure(tb))) return rc;
        size_t tbytes = tb;
        BG_CUDA(cub::DeviceRadixSort::SortPairs(S.tmp.ptr, tbytes, S.keys.as<uint64_t>(), S.keys2.as<uint64_t>(),
                                                S.idx.as<int32_t>(), S.sorted.as<int32_t>(), int(n), 0, 63));
        BG_CUDA(cudaMemset(S.parent.ptr, 0xff, NN * 4));
        k_leaf_boxes<<<blocks, kBT>>>(lo, hi, S.sorted.as<int32_t>(), n, S.box.as<float>(),
                                      builder == 2 ? S.cl.as<int32_t>() : nullptr);
        BG_CUDA(cudaGetLastError());
        if (builder == 1) {
            k_radix_tree<<<blocks, kBT>>>(S.keys2.as<uint64_t>(), n, S.left.as<int32_t>(), S.right.as<int32_t>(),
                                          S.parent.as<int32_t>());
            BG_CUDA(cudaGetLastError());
        } else {
            int* m_dev = S.nsel.as<int>();              // [0] clusters (written by the compaction), [1] next node
            int32_t* base_dev = S.nsel.as<int32_t>() + 1;
            const int32_t init_mb[2] = {int32_t(n), int32_t(n)};
            BG_CUDA(cudaMemcpy(S.nsel.ptr, init_mb, sizeof(init_mb), cudaMemcpyHostToDevice));
            int32_t* cl = S.cl.as<int32_t>();
            int32_t* cl2 = S.cl2.as<int32_t>();
            // every round merges at least one pair (the smallest pair is mutual), so
            // m falls by at least one per round while above 1; the host reads m
            // every kPlocCheck rounds to shrink the launch bound and to stop
            constexpr int kPlocCheck = 4;
            int m_bound = int(n);
            while (m_bound > 1) {
                for (int r = 0; r < kPlocCheck; ++r) {
                    const int g = std::min(kBGrid, (m_bound + kBT - 1) / kBT);
                    k_ploc_nn<<<g, kBT>>>(cl, m_dev, S.box.as<float>(), S.nn.as<int32_t>());
                    k_ploc_flags<<<g, kBT>>>(S.nn.as<int32_t>(), m_dev, m_bound, S.lead.as<int32_t>(), S.keep.as<int32_t>());
                    tbytes = tb;
                    BG_CUDA(cub::DeviceScan::ExclusiveSum(S.tmp.ptr, tbytes, S.lead.as<int32_t>(), S.scan.as<int32_t>(),
                                                          m_bound));
                    k_ploc_merge<<<g, kBT>>>(cl, S.nn.as<int32_t>(), m_dev, S.lead.as<int32_t>(), S.scan.as<int32_t>(),
                                             base_dev, S.box.as<float>(), S.left.as<int32_t>(), S.right.as<int32_t>(),
                                             S.parent.as<int32_t>());
                    k_ploc_advance<<<1, 32>>>(base_dev, S.scan.as<int32_t>(), S.lead.as<int32_t>(), m_bound);
                    tbytes = tb;
                    BG_CUDA(cub::DeviceSelect::Flagged(S.tmp.ptr, tbytes, cl, S.keep.as<int32_t>(), cl2, m_dev, m_bound));
                    std::swap(cl, cl2);
                }
                BG_CUDA(cudaGetLastError());
                int m = 0;
                BG_CUDA(cudaMemcpy(&m, m_dev, sizeof(int), cudaMemcpyDeviceToHost));
                if (m >= m_bound) return set_error(BG_ERR_STATE, "device PLOC build made no progress");
                m_bound = m;
            }
            int32_t next_node = 0;
            BG_CUDA(cudaMemcpy(&next_node, base_dev, sizeof(int32_t), cudaMemcpyDeviceToHost));
            if (next_node != int32_t(NN)) return set_error(BG_ERR_STATE, "device PLOC build: %d nodes", next_node);
            BG_CUDA(cudaMemcpy(&root, cl, 4, cudaMemcpyDeviceToHost));
        }
    }
    BG_CUDA(cudaMemset(S.visits.ptr, 0, NN * 4));
    BG_CUDA(cudaMemset(S.nopen.ptr, 0, 2 * sizeof(int)));
    k_bottom_up<<<blocks, kBT>>>(n, S.left.as<int32_t>(), S.right.as<int32_t>(), S.parent.as<int32_t>(),
                                 S.box.as<float>(), S.cnt.as<int32_t>(), S.cost.as<float>(), S.mk.as<uint8_t>(),
                                 S.visits.as<int>(), bp.max_leaf, bp.cost_node, S.nopen.as<int>());
    BG_CUDA(cudaGetLastError());
    int nopen[2] = {0, 0};
    BG_CUDA(cudaMemcpy(nopen, S.nopen.ptr, sizeof(nopen), cudaMemcpyDeviceToHost));
    if (nopen[1]) return set_error(BG_ERR_STATE, "device BVH build: the binary tree has a parent cycle");
    const int capacity = nopen[0] + 1;     // every wide node opens a distinct non-leaf binary node (or the root)
    CollapseArgs A{};
    A.left = S.left.as<int32_t>();
    A.right = S.right.as<int32_t>();
    A.box = S.box.as<float>();
    A.cnt = S.cnt.as<int32_t>();
    A.mk = S.mk.as<uint8_t>();
    A.sorted = S.sorted.as<int32_t>();
    A.n = n;
    out = DeviceBvh{};
    if (bp.wide4) {
        WideOut w;
        if ((rc = run_collapse<4>(A, root, capacity, order, nodes4, w))) return rc;
        out.nnodes4 = w.nodes;
        out.max_depth4 = w.max_depth;
        out.max_stack4 = w.max_stack;
    }
    if (bp.wide8) {
        WideOut w;
        if ((rc = run_collapse<8>(A, root, capacity, bp.wide4 ? nullptr : order, nodes8, w))) return rc;
        out.quant_ok = w.quant_ok;
        out.nnodes8 = w.quant_ok ? w.nodes : 0;
        out.max_depth8 = w.quant_ok ? w.max_depth : 0;
        out.max_stack8 = w.quant_ok ? w.max_stack : 0;
    }
    return BG_OK;
}

}  // namespace bg
