// Device BVH builder: a linear BVH over 63-bit Morton codes of the triangle
// centroids (Karras, "Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees", HPG 2012), built in four kernels and a CUB radix
// sort; subtrees of at most max_leaf triangles become leaves, and the binary
// tree is handed to the host collapse that emits the 4-wide and 8-wide node
// layouts.  Replaces the host binned-SAH build (Bvh::Build,
// accelerator/bvh.cpp:16-496) when build time matters more than tree quality
// (bg_build_opts.builder = 1); hits are identical either way.
#include <cub/cub.cuh>

#include <cfloat>
#include <vector>

#include "bvh_build.h"
#include "internal.h"

namespace bg {
namespace {

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

// common-prefix length of sorted keys i and j (ties broken by index); -1 outside [0, n)
__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a != b) return __clzll(a ^ b);
    return 64 + __clzll(uint64_t(i) ^ uint64_t(j));
}

// Internal node i of n - 1: children (>= 0 internal, < 0 leaf ~p), key range, parents.
__global__ void k_radix_tree(const uint64_t* __restrict__ keys, int64_t n, int32_t* __restrict__ left,
                             int32_t* __restrict__ right, int32_t* __restrict__ first, int32_t* __restrict__ last,
                             int32_t* __restrict__ parent_int, int32_t* __restrict__ parent_leaf) {
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
        first[i] = int32_t(lo_);
        last[i] = int32_t(hi_);
        if (lo_ == g) { left[i] = ~int32_t(g); parent_leaf[g] = int32_t(i); }
        else { left[i] = int32_t(g); parent_int[g] = int32_t(i); }
        if (hi_ == g + 1) { right[i] = ~int32_t(g + 1); parent_leaf[g + 1] = int32_t(i); }
        else { right[i] = int32_t(g + 1); parent_int[g + 1] = int32_t(i); }
    }
}

// Bottom-up boxes: the second child to finish computes its parent's box.
__global__ void k_boxes(const float* __restrict__ lo, const float* __restrict__ hi, const int32_t* __restrict__ order,
                        int64_t n, const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                        const int32_t* __restrict__ parent_int, const int32_t* __restrict__ parent_leaf,
                        int* __restrict__ visits, float* __restrict__ box) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        int32_t node = parent_leaf[p];
        while (node >= 0) {
            __threadfence();
            if (atomicAdd(visits + node, 1) == 0) break;     // the sibling will finish this node
            __threadfence();
            float b[6];
            for (int k = 0; k < 3; ++k) { b[k] = FLT_MAX; b[3 + k] = -FLT_MAX; }
            const int32_t ch[2] = {left[node], right[node]};
            for (int c = 0; c < 2; ++c) {
                if (ch[c] < 0) {
                    const int32_t t = order[~ch[c]];
                    for (int k = 0; k < 3; ++k) { b[k] = fminf(b[k], lo[3 * t + k]); b[3 + k] = fmaxf(b[3 + k], hi[3 * t + k]); }
                } else {
                    const volatile float* cbx = box + 6 * size_t(ch[c]);
                    for (int k = 0; k < 3; ++k) { b[k] = fminf(b[k], cbx[k]); b[3 + k] = fmaxf(b[3 + k], cbx[3 + k]); }
                }
            }
            volatile float* out = box + 6 * size_t(node);
            for (int k = 0; k < 6; ++k) out[k] = b[k];
            node = node == 0 ? -1 : parent_int[node];
        }
    }
}

}  // namespace

// Builds the binary LBVH of n triangle boxes (host arrays) on the device and
// converts it to the host BinaryTree the wide collapses read.
int gpu_build_tree(const float* lo_h, const float* hi_h, int64_t n, int max_leaf, BinaryTree& t) {
    if (n < 2) return set_error(BG_ERR_INVALID_ARG, "device build needs at least 2 triangles");
    if (n > (int64_t(1) << 30)) return set_error(BG_ERR_UNSUPPORTED, "device build: too many triangles");
    struct Scratch {
        DevBuf lo, hi, cb, keys, keys2, idx, idx2, left, right, first, last, pint, pleaf, vis, box, tmp;
        ~Scratch() {
            for (DevBuf* b : {&lo, &hi, &cb, &keys, &keys2, &idx, &idx2, &left, &right, &first, &last, &pint, &pleaf,
                              &vis, &box, &tmp})
                b->release();
        }
    } S;
    DevBuf &dlo = S.lo, &dhi = S.hi, &dcb = S.cb, &dkeys = S.keys, &dkeys2 = S.keys2, &didx = S.idx, &didx2 = S.idx2,
           &dleft = S.left, &dright = S.right, &dfirst = S.first, &dlast = S.last, &dpint = S.pint,
           &dpleaf = S.pleaf, &dvis = S.vis, &dbox = S.box, &dtmp = S.tmp;
    const size_t N = size_t(n);
    int rc;
    if ((rc = dlo.ensure(N * 12)) || (rc = dhi.ensure(N * 12)) || (rc = dcb.ensure(32)) ||
        (rc = dkeys.ensure(N * 8)) || (rc = dkeys2.ensure(N * 8)) || (rc = didx.ensure(N * 4)) ||
        (rc = didx2.ensure(N * 4)) || (rc = dleft.ensure(N * 4)) || (rc = dright.ensure(N * 4)) ||
        (rc = dfirst.ensure(N * 4)) || (rc = dlast.ensure(N * 4)) || (rc = dpint.ensure(N * 4)) ||
        (rc = dpleaf.ensure(N * 4)) || (rc = dvis.ensure(N * 4)) || (rc = dbox.ensure(N * 24)))
        return rc;
    BG_CUDA(cudaMemcpy(dlo.ptr, lo_h, N * 12, cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemcpy(dhi.ptr, hi_h, N * 12, cudaMemcpyHostToDevice));
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BG_CUDA(cudaMemcpy(dcb.ptr, init, sizeof(init), cudaMemcpyHostToDevice));
    const int blocks = 1024, threads = 256;
    k_centroid_bounds<<<blocks, threads>>>(dlo.as<float>(), dhi.as<float>(), n, dcb.as<unsigned int>());
    k_morton<<<blocks, threads>>>(dlo.as<float>(), dhi.as<float>(), n, dcb.as<unsigned int>(), dkeys.as<uint64_t>(),
                                  didx.as<int32_t>());
    BG_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    BG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dkeys.as<uint64_t>(), dkeys2.as<uint64_t>(),
                                            didx.as<int32_t>(), didx2.as<int32_t>(), int(n), 0, 63));
    if ((rc = dtmp.ensure(tmp_bytes))) return rc;
    BG_CUDA(cub::DeviceRadixSort::SortPairs(dtmp.ptr, tmp_bytes, dkeys.as<uint64_t>(), dkeys2.as<uint64_t>(),
                                            didx.as<int32_t>(), didx2.as<int32_t>(), int(n), 0, 63));
    BG_CUDA(cudaMemset(dpint.ptr, 0xff, N * 4));
    BG_CUDA(cudaMemset(dvis.ptr, 0, N * 4));
    k_radix_tree<<<blocks, threads>>>(dkeys2.as<uint64_t>(), n, dleft.as<int32_t>(), dright.as<int32_t>(),
                                      dfirst.as<int32_t>(), dlast.as<int32_t>(), dpint.as<int32_t>(),
                                      dpleaf.as<int32_t>());
    k_boxes<<<blocks, threads>>>(dlo.as<float>(), dhi.as<float>(), didx2.as<int32_t>(), n, dleft.as<int32_t>(),
                                 dright.as<int32_t>(), dpint.as<int32_t>(), dpleaf.as<int32_t>(), dvis.as<int>(),
                                 dbox.as<float>());
    BG_CUDA(cudaGetLastError());
    const size_t ni = N - 1;
    std::vector<int32_t> L(ni), R(ni), F(ni), La(ni);
    std::vector<float> B(ni * 6);
    t.order.resize(N);
    BG_CUDA(cudaMemcpy(L.data(), dleft.ptr, ni * 4, cudaMemcpyDeviceToHost));
    BG_CUDA(cudaMemcpy(R.data(), dright.ptr, ni * 4, cudaMemcpyDeviceToHost));
    BG_CUDA(cudaMemcpy(F.data(), dfirst.ptr, ni * 4, cudaMemcpyDeviceToHost));
    BG_CUDA(cudaMemcpy(La.data(), dlast.ptr, ni * 4, cudaMemcpyDeviceToHost));
    BG_CUDA(cudaMemcpy(B.data(), dbox.ptr, ni * 24, cudaMemcpyDeviceToHost));
    BG_CUDA(cudaMemcpy(t.order.data(), didx2.ptr, N * 4, cudaMemcpyDeviceToHost));
    // host tree: internal nodes keep their index; a child that is a single
    // triangle, or an internal node over <= max_leaf triangles, becomes a leaf node
    t.box.clear(); t.left.clear(); t.right.clear(); t.start.clear(); t.count.clear();
    t.box.reserve(ni * 6 * 2);
    auto add_node = [&](const float* b, int32_t l, int32_t r, int32_t s, int32_t c) {
        t.box.insert(t.box.end(), b, b + 6);
        t.left.push_back(l); t.right.push_back(r); t.start.push_back(s); t.count.push_back(c);
        return int32_t(t.left.size() - 1);
    };
    for (size_t i = 0; i < ni; ++i) add_node(&B[6 * i], -1, -1, 0, 0);
    const float* hlo = lo_h;
    const float* hhi = hi_h;
    auto leaf_of = [&](int32_t p) {
        const int32_t tri = t.order[size_t(p)];
        float b[6] = {hlo[3 * tri], hlo[3 * tri + 1], hlo[3 * tri + 2], hhi[3 * tri], hhi[3 * tri + 1], hhi[3 * tri + 2]};
        return add_node(b, -1, -1, p, 1);
    };
    for (size_t i = 0; i < ni; ++i) {
        const int32_t size = La[i] - F[i] + 1;
        if (size <= max_leaf) {               // a small subtree: one leaf over its range
            t.start[i] = F[i];
            t.count[i] = size;
            continue;
        }
        t.left[i] = L[i] < 0 ? leaf_of(~L[i]) : L[i];
        t.right[i] = R[i] < 0 ? leaf_of(~R[i]) : R[i];
    }
    return BG_OK;
}

}  // namespace bg
