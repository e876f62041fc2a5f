// Device binned-SAH builder (bg_build_opts.builder = 3): the same top-down
// binned SAH as the host builder (Bvh::Build with its FindSahSplit,
// accelerator/bvh.cpp:16-496; cost = node + (NL AL + NR AR) / A), run on the
// GPU level by level.  It produces the binary tree in the numbering the other
// device builders use (leaf p = the triangle at final position p, internal
// nodes n, n + 1, ...), so the bottom-up SAH leaf choice and the wide
// collapses of gpu_build.cu follow unchanged.
//
//  * Tasks of more than kSmallTask triangles are split together, one pass over
//    all triangles per level: centroid bounds per task, then 32 bins per axis
//    (count and box) per task, both with warp-aggregated atomics (lanes of a
//    warp mostly share a task, so one lane per (task, bin) group issues the
//    atomics); one warp per task sweeps the bins for the cheapest split; the
//    triangles are partitioned stably through one exclusive scan of their
//    left flags over the whole array.
//  * Tasks of at most kSmallTask triangles are finished by one warp each, in
//    registers (two triangles per lane): 8 bins per axis from warp reductions,
//    partition by ballots, depth first with a small stack.
//  * Splits fall back to the median position when every bin split leaves a
//    side empty (coincident centroids) and from depth kMedianDepth on, which
//    bounds the depth of the tree.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>

#include "internal.h"

namespace bg {
namespace {

constexpr int kST = 256;             // threads per block
constexpr int kSGrid = 148 * 8;      // blocks of the grid-stride launches
constexpr int kBins = 32;            // bins per axis of the large tasks (one per lane of the split warp)
constexpr int kSmallTask = 64;       // tasks of at most this many triangles are finished by one warp
constexpr int kSmallBins = 8;        // bins per axis inside the warp builder
constexpr int kTinyTask = 4;         // at most this many: split at the median position
constexpr int kMedianDepth = 48;     // from this depth on: median splits
constexpr int kMaxLevels = 256;      // large-task levels (median splits from kMedianDepth bound them)
constexpr int kStatWords = 6 + 3 * kBins * 7;   // per large task: centroid bounds + bins (count, lo3, hi3)

struct Task {
    int32_t begin, end, node, depth;
};

__device__ __forceinline__ unsigned f2o(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}
__device__ __forceinline__ float half_area6(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float ex = hx - lx, ey = hy - ly, ez = hz - lz;
    return ex * ey + ey * ez + ez * ex;
}
// bin of centroid coordinate c; scale = nb / extent (0 for a flat extent)
__device__ __forceinline__ int bin_of(float c, float cmin, float scale, int nb) {
    const int b = int((c - cmin) * scale);
    return min(nb - 1, max(0, b));
}
__device__ __forceinline__ float bin_scale(float cmin, float cmax, int nb) {
    const float ext = cmax - cmin;
    return ext > 0.f ? float(nb) / ext : 0.f;
}

// sanitised boxes (a non-finite box is a point at the origin, as in the host
// builder), centroids, identity order, every position in task 0 (or in the
// small phase when the whole scene is one small task)
__global__ void k_sah_prep(const float* __restrict__ lo, const float* __restrict__ hi, int64_t n,
                           float* __restrict__ box6, float4* __restrict__ cen, int32_t* __restrict__ idx,
                           int32_t* __restrict__ task_of, int32_t first_task) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        bool finite = true;
        for (int k = 0; k < 3; ++k) finite = finite && isfinite(lo[3 * i + k]) && isfinite(hi[3 * i + k]);
        float b[6];
        for (int k = 0; k < 3; ++k) {
            b[k] = finite ? lo[3 * i + k] : 0.f;
            b[3 + k] = finite ? hi[3 * i + k] : 0.f;
        }
        for (int k = 0; k < 6; ++k) box6[6 * i + k] = b[k];
        cen[i] = make_float4(0.5f * (b[0] + b[3]), 0.5f * (b[1] + b[4]), 0.5f * (b[2] + b[5]), 0.f);
        idx[i] = int32_t(i);
        task_of[i] = first_task;
    }
}

__global__ void k_sah_stats_init(unsigned* __restrict__ stats, int64_t ntasks) {
    const int64_t total = ntasks * kStatWords;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const int w = int(i % kStatWords);
        unsigned v;
        if (w < 6) v = w < 3 ? 0xffffffffu : 0u;              // centroid min / max
        else {
            const int c = (w - 6) % 7;                         // count, lo xyz, hi xyz
            v = c == 0 ? 0u : (c <= 3 ? 0xffffffffu : 0u);
        }
        stats[i] = v;
    }
}

// centroid bounds per large task
__global__ void k_sah_cbounds(int64_t n, const int32_t* __restrict__ task_of, const int32_t* __restrict__ idx,
                              const float4* __restrict__ cen, unsigned* __restrict__ stats) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t p0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) & ~int64_t(31); p0 < n; p0 += stride) {
        const int64_t p = p0 + lane;
        const int t = p < n ? task_of[p] : -1;
        const unsigned am = __ballot_sync(0xffffffffu, t >= 0);
        if (t < 0) continue;
        const float4 c = cen[idx[p]];
        const unsigned g = __match_any_sync(am, t);
        const unsigned v[6] = {__reduce_min_sync(g, f2o(c.x)), __reduce_min_sync(g, f2o(c.y)),
                               __reduce_min_sync(g, f2o(c.z)), __reduce_max_sync(g, f2o(c.x)),
                               __reduce_max_sync(g, f2o(c.y)), __reduce_max_sync(g, f2o(c.z))};
        if (lane == __ffs(g) - 1) {
            unsigned* s = stats + size_t(t) * kStatWords;
            for (int k = 0; k < 3; ++k) { atomicMin(s + k, v[k]); atomicMax(s + 3 + k, v[3 + k]); }
        }
    }
}

// count and box per (task, axis, bin)
__global__ void k_sah_bins(int64_t n, const int32_t* __restrict__ task_of, const int32_t* __restrict__ idx,
                           const float4* __restrict__ cen, const float* __restrict__ box6, unsigned* __restrict__ stats) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t p0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) & ~int64_t(31); p0 < n; p0 += stride) {
        const int64_t p = p0 + lane;
        const int t = p < n ? task_of[p] : -1;
        const unsigned am = __ballot_sync(0xffffffffu, t >= 0);
        if (t < 0) continue;
        const int tri = idx[p];
        const float4 c = cen[tri];
        const float cc[3] = {c.x, c.y, c.z};
        unsigned bx[6];
        for (int k = 0; k < 6; ++k) bx[k] = f2o(box6[6 * size_t(tri) + k]);
        unsigned* s = stats + size_t(t) * kStatWords;
        for (int a = 0; a < 3; ++a) {
            const float cmin = o2f(s[a]), cmax = o2f(s[3 + a]);
            const int b = bin_of(cc[a], cmin, bin_scale(cmin, cmax, kBins), kBins);
            const unsigned g = __match_any_sync(am, t * kBins + b);
            const unsigned r[6] = {__reduce_min_sync(g, bx[0]), __reduce_min_sync(g, bx[1]),
                                   __reduce_min_sync(g, bx[2]), __reduce_max_sync(g, bx[3]),
                                   __reduce_max_sync(g, bx[4]), __reduce_max_sync(g, bx[5])};
            if (lane == __ffs(g) - 1) {
                unsigned* w = s + 6 + (a * kBins + b) * 7;
                atomicAdd(w, unsigned(__popc(g)));
                for (int k = 0; k < 3; ++k) { atomicMin(w + 1 + k, r[k]); atomicMax(w + 4 + k, r[3 + k]); }
            }
        }
    }
}

// One warp per large task: sweep the 32 bins of each axis for the cheapest
// split; split_axis = -1 asks for the median position.
__global__ void k_sah_split(int ntasks, const Task* __restrict__ tasks, const unsigned* __restrict__ stats,
                            int32_t* __restrict__ split_axis, int32_t* __restrict__ split_bin) {
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntasks; t += nwarps) {
        const unsigned* s = stats + size_t(t) * kStatWords;
        float best = FLT_MAX;
        int best_key = 0x7fffffff;   // axis * 32 + split (lowest wins ties)
        for (int a = 0; a < 3; ++a) {
            const unsigned* w = s + 6 + (a * kBins + lane) * 7;
            const unsigned cnt = w[0];
            // inclusive prefix (bins 0..lane) and suffix (bins lane..31) of counts and boxes
            unsigned pc = cnt, sc = cnt;
            unsigned pl[3] = {w[1], w[2], w[3]}, ph[3] = {w[4], w[5], w[6]};
            unsigned sl[3] = {w[1], w[2], w[3]}, sh[3] = {w[4], w[5], w[6]};
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned qc = __shfl_up_sync(0xffffffffu, pc, o);
                const unsigned rc = __shfl_down_sync(0xffffffffu, sc, o);
                unsigned ql[3], qh[3], rl[3], rh[3];
                for (int k = 0; k < 3; ++k) {
                    ql[k] = __shfl_up_sync(0xffffffffu, pl[k], o);
                    qh[k] = __shfl_up_sync(0xffffffffu, ph[k], o);
                    rl[k] = __shfl_down_sync(0xffffffffu, sl[k], o);
                    rh[k] = __shfl_down_sync(0xffffffffu, sh[k], o);
                }
                if (lane >= o) {
                    pc += qc;
                    for (int k = 0; k < 3; ++k) { pl[k] = min(pl[k], ql[k]); ph[k] = max(ph[k], qh[k]); }
                }
                if (lane + o < 32) {
                    sc += rc;
                    for (int k = 0; k < 3; ++k) { sl[k] = min(sl[k], rl[k]); sh[k] = max(sh[k], rh[k]); }
                }
            }
            // split after bin `lane`: left = prefix(lane), right = suffix(lane + 1)
            const unsigned nr = __shfl_down_sync(0xffffffffu, sc, 1);
            unsigned rl2[3], rh2[3];
            for (int k = 0; k < 3; ++k) {
                rl2[k] = __shfl_down_sync(0xffffffffu, sl[k], 1);
                rh2[k] = __shfl_down_sync(0xffffffffu, sh[k], 1);
            }
            if (lane < 31 && pc > 0 && nr > 0) {
                const float al = half_area6(o2f(pl[0]), o2f(pl[1]), o2f(pl[2]), o2f(ph[0]), o2f(ph[1]), o2f(ph[2]));
                const float ar = half_area6(o2f(rl2[0]), o2f(rl2[1]), o2f(rl2[2]), o2f(rh2[0]), o2f(rh2[1]),
                                            o2f(rh2[2]));
                const float cost = float(pc) * al + float(nr) * ar;
                const int key = a * 32 + lane;
                if (cost < best || (cost == best && key < best_key)) { best = cost; best_key = key; }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {       // warp argmin
            const float ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int ok = __shfl_xor_sync(0xffffffffu, best_key, o);
            if (ob < best || (ob == best && ok < best_key)) { best = ob; best_key = ok; }
        }
        if (lane == 0) {
            const bool median = best_key == 0x7fffffff || tasks[t].depth >= kMedianDepth;
            split_axis[t] = median ? -1 : best_key / 32;
            split_bin[t] = median ? 0 : best_key % 32;
        }
    }
}

__global__ void k_sah_flags(int64_t n, const int32_t* __restrict__ task_of, const int32_t* __restrict__ idx,
                            const float4* __restrict__ cen, const Task* __restrict__ tasks,
                            const unsigned* __restrict__ stats, const int32_t* __restrict__ split_axis,
                            const int32_t* __restrict__ split_bin, int32_t* __restrict__ flags) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        const int t = task_of[p];
        int f = 0;
        if (t >= 0) {
            const int ax = split_axis[t];
            if (ax < 0) {
                const Task T = tasks[t];
                f = (p - T.begin) < (T.end - T.begin) / 2 ? 1 : 0;
            } else {
                const unsigned* s = stats + size_t(t) * kStatWords;
                const float4 c = cen[idx[p]];
                const float cc = ax == 0 ? c.x : (ax == 1 ? c.y : c.z);
                const float cmin = o2f(s[ax]), cmax = o2f(s[3 + ax]);
                f = bin_of(cc, cmin, bin_scale(cmin, cmax, kBins), kBins) <= split_bin[t] ? 1 : 0;
            }
        }
        flags[p] = f;
    }
}

struct SahCounters {
    int nodes;       // internal nodes handed out (the root is node n + 0)
    int nlarge;      // next level's large tasks
    int nsmall;      // small tasks
    int err;         // 1: a capacity or consistency check failed
};

// Per large task: child ranges, node ids, tree links, next-level tasks.
__global__ void k_sah_children(int ntasks, const Task* __restrict__ tasks, const int32_t* __restrict__ scan,
                               const int32_t* __restrict__ flags, int64_t n, int32_t* __restrict__ left,
                               int32_t* __restrict__ right, int32_t* __restrict__ parent, Task* __restrict__ next,
                               int cap_large, Task* __restrict__ small, int cap_small, SahCounters* __restrict__ ctr,
                               int32_t* __restrict__ child_code, int32_t* __restrict__ nleft_of) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x) {
        const Task T = tasks[t];
        const int nl = scan[T.end - 1] + flags[T.end - 1] - scan[T.begin];
        const int size = T.end - T.begin;
        nleft_of[t] = nl;
        if (nl <= 0 || nl >= size) { atomicOr(&ctr->err, 1); child_code[2 * t] = child_code[2 * t + 1] = -1; continue; }
        int32_t ids[2];
        for (int side = 0; side < 2; ++side) {
            const int b = side ? T.begin + nl : T.begin, e = side ? T.end : T.begin + nl;
            int code = -1;                                   // -1: a finished leaf
            if (e - b == 1) {
                ids[side] = b;                               // leaf id = its final position
            } else {
                const int k = atomicAdd(&ctr->nodes, 1);
                ids[side] = int32_t(n) + k;
                if (int64_t(k) >= n - 1) { atomicOr(&ctr->err, 1); ids[side] = b; continue; }
                const Task C{b, e, ids[side], T.depth + 1};
                if (e - b > kSmallTask) {
                    const int q = atomicAdd(&ctr->nlarge, 1);
                    if (q >= cap_large) atomicOr(&ctr->err, 1); else { next[q] = C; code = q; }
                } else {
                    const int q = atomicAdd(&ctr->nsmall, 1);
                    if (q >= cap_small) atomicOr(&ctr->err, 1); else small[q] = C;
                    code = -2;                               // finished by a warp in the small phase
                }
            }
            child_code[2 * t + side] = code;
        }
        left[T.node] = ids[0];
        right[T.node] = ids[1];
        parent[ids[0]] = T.node;
        parent[ids[1]] = T.node;
    }
}

// stable partition of every large task by its flags; positions of other tasks are copied
__global__ void k_sah_scatter(int64_t n, const int32_t* __restrict__ task_of, const int32_t* __restrict__ idx,
                              const int32_t* __restrict__ scan, const int32_t* __restrict__ flags,
                              const Task* __restrict__ tasks, const int32_t* __restrict__ nleft_of,
                              const int32_t* __restrict__ child_code, int32_t* __restrict__ idx2,
                              int32_t* __restrict__ task_of2) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        const int t = task_of[p];
        if (t < 0) { idx2[p] = idx[p]; task_of2[p] = t; continue; }
        const int b = tasks[t].begin;
        const int lr = scan[p] - scan[b];
        int64_t np;
        int code;
        if (flags[p]) { np = b + lr; code = child_code[2 * t]; }
        else { np = b + nleft_of[t] + (p - b - lr); code = child_code[2 * t + 1]; }
        idx2[np] = idx[p];
        task_of2[np] = code;
    }
}

// One warp per small task: the whole subtree, depth first, in registers.
__global__ void k_sah_small(int nsmall_cap, const Task* __restrict__ small, SahCounters* __restrict__ ctr,
                            const float4* __restrict__ cen, const float* __restrict__ box6, int32_t* __restrict__ idx,
                            int64_t n, int32_t* __restrict__ left, int32_t* __restrict__ right,
                            int32_t* __restrict__ parent) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int ns = min(ctr->nsmall, nsmall_cap);
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < ns; w += nwarps) {
        int4 st[kSmallTask + 2];                       // (begin, end, node, depth)
        int sp = 0;
        st[sp++] = make_int4(small[w].begin, small[w].end, small[w].node, small[w].depth);
        while (sp > 0) {
            const int4 cur = st[--sp];
            const int b = cur.x, e = cur.y, size = e - b;
            // the node's triangles, two per lane
            const bool v0 = lane < size, v1 = lane + 32 < size;
            const int id0 = v0 ? idx[b + lane] : 0, id1 = v1 ? idx[b + 32 + lane] : 0;
            __syncwarp();                            // every lane has read before any lane writes below
            int nl;
            unsigned left0 = 0, left1 = 0;           // ballots of "goes left"
            bool f0 = false, f1 = false;
            bool median = size <= kTinyTask || cur.w >= kMedianDepth;
            int best_axis = -1, best_split = 0;
            float c0[3] = {0.f, 0.f, 0.f}, c1[3] = {0.f, 0.f, 0.f};
            if (!median) {
                const float4 a0 = v0 ? cen[id0] : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 a1 = v1 ? cen[id1] : make_float4(0.f, 0.f, 0.f, 0.f);
                c0[0] = a0.x; c0[1] = a0.y; c0[2] = a0.z;
                c1[0] = a1.x; c1[1] = a1.y; c1[2] = a1.z;
                unsigned bl0[3], bh0[3], bl1[3], bh1[3];
                for (int k = 0; k < 3; ++k) {
                    bl0[k] = v0 ? f2o(box6[6 * size_t(id0) + k]) : 0xffffffffu;
                    bh0[k] = v0 ? f2o(box6[6 * size_t(id0) + 3 + k]) : 0u;
                    bl1[k] = v1 ? f2o(box6[6 * size_t(id1) + k]) : 0xffffffffu;
                    bh1[k] = v1 ? f2o(box6[6 * size_t(id1) + 3 + k]) : 0u;
                }
                float best = FLT_MAX;
                for (int a = 0; a < 3; ++a) {
                    const float cmin = o2f(__reduce_min_sync(full, min(v0 ? f2o(c0[a]) : 0xffffffffu,
                                                                        v1 ? f2o(c1[a]) : 0xffffffffu)));
                    const float cmax = o2f(__reduce_max_sync(full, max(v0 ? f2o(c0[a]) : 0u, v1 ? f2o(c1[a]) : 0u)));
                    const float sc = bin_scale(cmin, cmax, kSmallBins);
                    const int bn0 = bin_of(c0[a], cmin, sc, kSmallBins), bn1 = bin_of(c1[a], cmin, sc, kSmallBins);
                    unsigned cnt[kSmallBins];
                    float lo[kSmallBins][3], hi[kSmallBins][3];
                    for (int j = 0; j < kSmallBins; ++j) {
                        const bool i0 = v0 && bn0 == j, i1 = v1 && bn1 == j;
                        cnt[j] = __popc(__ballot_sync(full, i0)) + __popc(__ballot_sync(full, i1));
                        for (int k = 0; k < 3; ++k) {
                            lo[j][k] = o2f(__reduce_min_sync(full, min(i0 ? bl0[k] : 0xffffffffu, i1 ? bl1[k] : 0xffffffffu)));
                            hi[j][k] = o2f(__reduce_max_sync(full, max(i0 ? bh0[k] : 0u, i1 ? bh1[k] : 0u)));
                        }
                    }
                    // every lane sweeps the same 7 splits
                    unsigned nlc = 0;
                    float ll[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                    for (int s = 0; s < kSmallBins - 1; ++s) {
                        nlc += cnt[s];
                        for (int k = 0; k < 3; ++k) { ll[k] = fminf(ll[k], lo[s][k]); lh[k] = fmaxf(lh[k], hi[s][k]); }
                        unsigned nrc = 0;
                        float rl[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                        for (int j = s + 1; j < kSmallBins; ++j) {
                            nrc += cnt[j];
                            for (int k = 0; k < 3; ++k) { rl[k] = fminf(rl[k], lo[j][k]); rh[k] = fmaxf(rh[k], hi[j][k]); }
                        }
                        if (nlc == 0 || nrc == 0) continue;
                        const float cost = float(nlc) * half_area6(ll[0], ll[1], ll[2], lh[0], lh[1], lh[2]) +
                                           float(nrc) * half_area6(rl[0], rl[1], rl[2], rh[0], rh[1], rh[2]);
                        if (cost < best) { best = cost; best_axis = a; best_split = s; }
                    }
                }
                if (best_axis < 0) median = true;
                else {
                    const float cmin = o2f(__reduce_min_sync(full, min(v0 ? f2o(c0[best_axis]) : 0xffffffffu,
                                                                        v1 ? f2o(c1[best_axis]) : 0xffffffffu)));
                    const float cmax = o2f(__reduce_max_sync(full, max(v0 ? f2o(c0[best_axis]) : 0u,
                                                                        v1 ? f2o(c1[best_axis]) : 0u)));
                    const float sc = bin_scale(cmin, cmax, kSmallBins);
                    f0 = v0 && bin_of(c0[best_axis], cmin, sc, kSmallBins) <= best_split;
                    f1 = v1 && bin_of(c1[best_axis], cmin, sc, kSmallBins) <= best_split;
                }
            }
            if (median) {
                f0 = v0 && lane < size / 2;
                f1 = v1 && lane + 32 < size / 2;
            }
            left0 = __ballot_sync(full, f0);
            left1 = __ballot_sync(full, f1);
            nl = __popc(left0) + __popc(left1);
            const unsigned below = (1u << lane) - 1u;
            const unsigned any0 = __ballot_sync(full, v0), any1 = __ballot_sync(full, v1);
            // stable partition: left triangles first, in position order
            if (v0) {
                const int r = f0 ? __popc(left0 & below) : nl + __popc(any0 & ~left0 & below);
                idx[b + r] = id0;
            }
            if (v1) {
                const int r = f1 ? __popc(left0) + __popc(left1 & below)
                                 : nl + __popc(any0 & ~left0) + __popc(any1 & ~left1 & below);
                idx[b + r] = id1;
            }
            __syncwarp();
            if (nl <= 0 || nl >= size) { if (lane == 0) atomicOr(&ctr->err, 1); continue; }
            int32_t ids[2];
            for (int side = 0; side < 2; ++side) {
                const int cb = side ? b + nl : b, ce = side ? e : b + nl;
                int id = cb;                                     // a single triangle: leaf at its position
                if (ce - cb > 1) {
                    int k = 0;
                    if (lane == 0) k = atomicAdd(&ctr->nodes, 1);
                    k = __shfl_sync(full, k, 0);
                    if (int64_t(k) >= n - 1 || sp >= kSmallTask + 2) { if (lane == 0) atomicOr(&ctr->err, 1); }
                    else {
                        id = int32_t(n) + k;
                        st[sp++] = make_int4(cb, ce, id, cur.w + 1);
                    }
                }
                ids[side] = id;
            }
            if (lane == 0) {
                left[cur.z] = ids[0];
                right[cur.z] = ids[1];
                parent[ids[0]] = cur.z;
                parent[ids[1]] = cur.z;
            }
        }
    }
}

int grid_of(int64_t n, int per = kST) {
    return int(std::max<int64_t>(1, std::min<int64_t>(kSGrid, (n + per - 1) / per)));
}

}  // namespace

int sah_binary_tree(const float* lo, const float* hi, int64_t n, int32_t* sorted, int32_t* left, int32_t* right,
                    int32_t* parent) {
    if (n < 2) return set_error(BG_ERR_INVALID_ARG, "device SAH build needs at least 2 triangles");
    const size_t N = size_t(n);
    const int64_t cap_large = n / (kSmallTask + 1) + 2;     // large tasks hold > kSmallTask triangles each
    const int64_t cap_small = n / 2 + 2;
    struct Scratch {
        ScratchBuf box6, cen, idx2, task_of, task_of2, flags, scan, tasks, next, small, stats, split_axis,
            split_bin, child_code, nleft, ctr, tmp;
    } S;
    int rc;
    if ((rc = S.box6.ensure(N * 24)) || (rc = S.cen.ensure(N * 16)) || (rc = S.idx2.ensure(N * 4)) ||
        (rc = S.task_of.ensure(N * 4)) || (rc = S.task_of2.ensure(N * 4)) || (rc = S.flags.ensure(N * 4)) ||
        (rc = S.scan.ensure(N * 4)) || (rc = S.tasks.ensure(size_t(cap_large) * sizeof(Task))) ||
        (rc = S.next.ensure(size_t(cap_large) * sizeof(Task))) ||
        (rc = S.small.ensure(size_t(cap_small) * sizeof(Task))) ||
        (rc = S.stats.ensure(size_t(cap_large) * kStatWords * 4)) ||
        (rc = S.split_axis.ensure(size_t(cap_large) * 4)) || (rc = S.split_bin.ensure(size_t(cap_large) * 4)) ||
        (rc = S.child_code.ensure(size_t(cap_large) * 8)) || (rc = S.nleft.ensure(size_t(cap_large) * 4)) ||
        (rc = S.ctr.ensure(sizeof(SahCounters))))
        return rc;
    size_t tb = 0;
    BG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, S.flags.as<int32_t>(), S.scan.as<int32_t>(), int(n)));
    if ((rc = S.tmp.ensure(tb))) return rc;
    int32_t* idx = sorted;                      // the order is built in place in `sorted` (and idx2)
    int32_t* idx2 = S.idx2.as<int32_t>();
    int32_t* tof = S.task_of.as<int32_t>();
    int32_t* tof2 = S.task_of2.as<int32_t>();
    Task* cur = S.tasks.as<Task>();
    Task* nxt = S.next.as<Task>();
    const bool large_root = n > kSmallTask;
    SahCounters c0{1, 0, large_root ? 0 : 1, 0};
    BG_CUDA(cudaMemcpy(S.ctr.ptr, &c0, sizeof(c0), cudaMemcpyHostToDevice));
    const Task root{0, int32_t(n), int32_t(n), 0};
    BG_CUDA(cudaMemcpy(large_root ? static_cast<void*>(cur) : S.small.ptr, &root, sizeof(root), cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemset(parent, 0xff, (2 * N - 1) * 4));
    const int gb = grid_of(n);
    k_sah_prep<<<gb, kST>>>(lo, hi, n, S.box6.as<float>(), S.cen.as<float4>(), idx, tof, large_root ? 0 : -2);
    BG_CUDA(cudaGetLastError());
    SahCounters* ctr = S.ctr.as<SahCounters>();
    int ntasks = large_root ? 1 : 0;
    for (int level = 0; ntasks > 0; ++level) {
        if (level >= kMaxLevels) return set_error(BG_ERR_UNSUPPORTED, "device SAH build deeper than %d levels", kMaxLevels);
        unsigned* stats = S.stats.as<unsigned>();
        k_sah_stats_init<<<grid_of(int64_t(ntasks) * kStatWords), kST>>>(stats, ntasks);
        k_sah_cbounds<<<gb, kST>>>(n, tof, idx, S.cen.as<float4>(), stats);
        k_sah_bins<<<gb, kST>>>(n, tof, idx, S.cen.as<float4>(), S.box6.as<float>(), stats);
        k_sah_split<<<grid_of(int64_t(ntasks) * 32), kST>>>(ntasks, cur, stats, S.split_axis.as<int32_t>(),
                                                            S.split_bin.as<int32_t>());
        k_sah_flags<<<gb, kST>>>(n, tof, idx, S.cen.as<float4>(), cur, stats, S.split_axis.as<int32_t>(),
                                 S.split_bin.as<int32_t>(), S.flags.as<int32_t>());
        size_t tbytes = tb;
        BG_CUDA(cub::DeviceScan::ExclusiveSum(S.tmp.ptr, tbytes, S.flags.as<int32_t>(), S.scan.as<int32_t>(), int(n)));
        BG_CUDA(cudaMemset(&ctr->nlarge, 0, sizeof(int)));
        k_sah_children<<<grid_of(ntasks), kST>>>(ntasks, cur, S.scan.as<int32_t>(), S.flags.as<int32_t>(), n, left,
                                                 right, parent, nxt, int(cap_large), S.small.as<Task>(),
                                                 int(cap_small), ctr, S.child_code.as<int32_t>(),
                                                 S.nleft.as<int32_t>());
        k_sah_scatter<<<gb, kST>>>(n, tof, idx, S.scan.as<int32_t>(), S.flags.as<int32_t>(), cur,
                                   S.nleft.as<int32_t>(), S.child_code.as<int32_t>(), idx2, tof2);
        BG_CUDA(cudaGetLastError());
        SahCounters h;
        BG_CUDA(cudaMemcpy(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost));
        if (h.err) return set_error(BG_ERR_STATE, "device SAH build: a split or capacity check failed");
        ntasks = std::min<int>(h.nlarge, int(cap_large));
        std::swap(cur, nxt);
        std::swap(tof, tof2);
        // the scattered order lives in idx2 now: keep the caller's buffer current
        BG_CUDA(cudaMemcpyAsync(idx, idx2, N * 4, cudaMemcpyDeviceToDevice, 0));
    }
    k_sah_small<<<grid_of(int64_t(cap_small) * 32), kST>>>(int(cap_small), S.small.as<Task>(), ctr,
                                                           S.cen.as<float4>(), S.box6.as<float>(), idx, n, left,
                                                           right, parent);
    BG_CUDA(cudaGetLastError());
    SahCounters h;
    BG_CUDA(cudaMemcpy(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.err) return set_error(BG_ERR_STATE, "device SAH build: a split or capacity check failed");
    if (int64_t(h.nodes) != n - 1) return set_error(BG_ERR_STATE, "device SAH build: %d internal nodes for %lld triangles",
                                                  h.nodes, (long long)n);
    return BG_OK;
}

}  // namespace bg
