// Closest-hit / any-hit traversal of the 4-wide BVH and of the 8-wide
// compressed BVH.
//
// Replaces Bvh::Intersect(ray, Hit&) and Bvh::Intersect(ray)
// (accelerator/bvh.cpp:499-647) together with Mesh::IntersectShape /
// IntersectFace (primitive/mesh.cpp:7-45, 216-261):
//   * a triangle is accepted when its Moller-Trumbore t is in (tmin, best],
//     computed with the reference's exact operation order in the bundle's
//     object space (ray transformed by minv as transform_ray does,
//     math/mathutils.h:154-157; skipped for identity bundles, where it is exact);
//   * the box test is this project's own: a slab test with a relative slack of
//     4e-7 on the exit distance (more than the 2*gamma(3) rounding bound of
//     (lo - o) * (1/d)), so no box that holds an accepted triangle is culled.
// Children are visited nearest-first; stack entries keep their entry distance
// and are culled against the current closest hit, widened by the same slack,
// when popped.
#pragma once

#include <type_traits>

#include "device_common.cuh"
#include "scene_types.h"
#include "../../include/banshee_gpu.h"

namespace bg {

constexpr int kStackSize = 64;     // entries per ray, 4-wide; the builder checks max_stack against it
constexpr int kStackSize8 = 96;    // entries per ray, 8-wide (up to 7 pushes per level)
// stack entries per ray kept in shared memory: 8 for the 4-wide traversal
// (measured: +6 % incoherent / +3 % coherent ray casts), none for the 8-wide one
template <int WIDTH>
__host__ __device__ constexpr int smem_stack_entries() { return WIDTH == 4 ? 8 : 0; }
template <int WIDTH>
__host__ __device__ constexpr int stack_entries() { return WIDTH == 8 ? kStackSize8 : kStackSize; }
// traversal steps between warp refill points (measured on passes of 2^24 paths:
// closest hit 24 > 16 > 12 by about 1 % of the frame; any hit 16 > 8, 32).
// (Measured and rejected: each lane's next ray prefetched into shared memory by
// cp.async from a per-warp pool of 32 indices, refilling every 24 / 12 / 8 / 4
// steps: C3 567 -> 528 / 519 / 511 / 280 Msamples/s with 4-wide nodes; and
// registers capped at 48 or 40 for 40 or 48 resident warps per SM: spills,
// 559 -> 544 / 495 Msamples/s.)
constexpr int kRefillStepsClosest = 24;
constexpr int kRefillStepsAny = 16;
constexpr float kBoxSlack = 4e-7f;
// The slack is applied as one fused multiply-add, t1 + |t1| * kBoxSlack rounded
// once: the same half-ulp guarantee as a multiply and an add (whose product
// term is exact to far below an ulp of t1), one instruction fewer per child
// box (measured: C3 extension and shadow traversal 1 % shorter, C2 coherent
// casts 1.2-1.6 % faster, hits unchanged).
// (Measured and rejected: slab distances as one fmaf(P, 1/d, -o/d) each, with a
// per-ray absolute error bound added to the slack.  The bound, 2^-24 max|o/d|,
// is huge for rays nearly parallel to an axis, so such rays visited most of the
// tree: C3 ran at 8 instead of 500 Msamples/s.)

struct Ray {
    v3 o, d, inv;
    float tmin, tmax;
    uint32_t oct;    // bit k set: direction component k is negative (sign of 1/d)
};

__device__ __forceinline__ Ray make_ray(float4 a, float4 b) {
    Ray r;
    r.o = mk(a.x, a.y, a.z); r.tmin = a.w;
    r.d = mk(b.x, b.y, b.z); r.tmax = b.w;
    r.inv = mk(1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z);
    r.oct = (signbit(r.inv.x) ? 1u : 0u) | (signbit(r.inv.y) ? 2u : 0u) | (signbit(r.inv.z) ? 4u : 0u);
    return r;
}

// Mesh::IntersectFace (primitive/mesh.cpp:7-45), bit-exact.
__device__ __forceinline__ bool mt_test(v3 o, v3 d, v3 p1, v3 e1, v3 e2, float tmin, float tmax,
                                        float& t, float& a, float& b) {
    v3 s1 = cross(d, e2);
    float invd = 1.f / dot(s1, e1);
    v3 dd = sub(o, p1);
    float b1 = dot(dd, s1) * invd;
    if (b1 < 0.f || b1 > 1.f) return false;
    v3 s2 = cross(dd, e1);
    float b2 = dot(d, s2) * invd;
    if (b2 < 0.f || b1 + b2 > 1.f) return false;
    float tmp = dot(e2, s2) * invd;
    if (tmp > tmin && tmp <= tmax) {
        t = tmp; a = b1; b = b2;
        return true;
    }
    return false;
}

// ray in the object space of bundle `bundle`; with WT also the watertight
// test's shear (Woop, Benthin and Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013): kz = the axis of the largest |d|, kx, ky
// the next two (swapped when d[kz] < 0, keeping the winding), sx = d[kx] /
// d[kz], sy = d[ky] / d[kz], sz = 1 / d[kz]
struct ObjRay {
    int bundle;
    v3 o, d;
};
struct ObjRayWT : ObjRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float comp(v3 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : v.z; }

__device__ __forceinline__ void shear(ObjRay&) {}
__device__ __forceinline__ void shear(ObjRayWT& c) {
    const float ax = fabsf(c.d.x), ay = fabsf(c.d.y), az = fabsf(c.d.z);
    c.kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    c.kx = c.kz == 2 ? 0 : c.kz + 1;
    c.ky = c.kx == 2 ? 0 : c.kx + 1;
    const float dz = comp(c.d, c.kz);
    if (dz < 0.f) { const int t = c.kx; c.kx = c.ky; c.ky = t; }
    c.sx = comp(c.d, c.kx) / dz;
    c.sy = comp(c.d, c.ky) / dz;
    c.sz = 1.f / dz;
}

template <class OR>
__device__ __forceinline__ void obj_ray(const DevScene& S, const Ray& r, int b, OR& c) {
    if (b == c.bundle) return;
    c.bundle = b;
    if (b < 0) {
        c.o = r.o; c.d = r.d;
    } else {
        const float* mi = S.bundles[b].minv;
        float m[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) m[k] = __ldg(mi + k);
        c.o = xf_point(m, r.o);
        c.d = xf_vector(m, r.d);
    }
    shear(c);
}

// Watertight ray / triangle test (Woop, Benthin and Wald 2013) on the exact
// vertices: the edge functions U, V, W of an edge are computed from the same
// sheared vertex coordinates in both triangles that share it (and are exact
// negatives of each other there), so no ray passes between them.  Edges are
// inclusive; an edge function that comes out exactly 0 is recomputed in double
// precision.  Returns t and the barycentrics of p2 (a) and p3 (b), as
// Moller-Trumbore's b1, b2.
__device__ __forceinline__ bool wt_test(const ObjRayWT& c, v3 p1, v3 p2, v3 p3, float tmin, float tmax, float& t,
                                        float& a, float& b) {
    const v3 A = sub(p1, c.o), B = sub(p2, c.o), C = sub(p3, c.o);
    const float az = comp(A, c.kz), bz = comp(B, c.kz), cz = comp(C, c.kz);
    const float ax = comp(A, c.kx) - c.sx * az, ay = comp(A, c.ky) - c.sy * az;
    const float bx = comp(B, c.kx) - c.sx * bz, by = comp(B, c.ky) - c.sy * bz;
    const float cx = comp(C, c.kx) - c.sx * cz, cy = comp(C, c.ky) - c.sy * cz;
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = float(double(cx) * double(by) - double(cy) * double(bx));
        V = float(double(ax) * double(cy) - double(ay) * double(cx));
        W = float(double(bx) * double(ay) - double(by) * double(ax));
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = U + V + W;
    if (det == 0.f) return false;
    const float T = U * (c.sz * az) + V * (c.sz * bz) + W * (c.sz * cz);
    const float rcp = 1.f / det;
    const float tt = T * rcp;
    if (!(tt > tmin && tt <= tmax)) return false;
    t = tt;
    a = V * rcp;
    b = W * rcp;
    return true;
}

// Test the 4 children of node `ni`; returns a hit mask and entry distances.
__device__ __forceinline__ uint32_t box4(const WideNode4* __restrict__ nodes, int ni, const Ray& r, float best,
                                         float tn[4], int32_t ch[4]) {
    // the near / far planes of each axis are picked by load address (the node
    // stores lo and hi of an axis in adjacent float4s), not by per-plane selects
    const float4* p = reinterpret_cast<const float4*>(nodes + ni);
    const int fx = int(r.oct & 1u), fy = int((r.oct >> 1) & 1u), fz = int((r.oct >> 2) & 1u);
    const float4 nx4 = __ldg(p + fx), fx4 = __ldg(p + (1 - fx));
    const float4 ny4 = __ldg(p + 2 + fy), fy4 = __ldg(p + 3 - fy);
    const float4 nz4 = __ldg(p + 4 + fz), fz4 = __ldg(p + 5 - fz);
    int4 c = __ldg(reinterpret_cast<const int4*>(p + 6));
    const float nxa[4] = {nx4.x, nx4.y, nx4.z, nx4.w}, fxa[4] = {fx4.x, fx4.y, fx4.z, fx4.w};
    const float nya[4] = {ny4.x, ny4.y, ny4.z, ny4.w}, fya[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
    const float nza[4] = {nz4.x, nz4.y, nz4.z, nz4.w}, fza[4] = {fz4.x, fz4.y, fz4.z, fz4.w};
    ch[0] = c.x; ch[1] = c.y; ch[2] = c.z; ch[3] = c.w;
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float ax = (nxa[i] - r.o.x) * r.inv.x;
        float bx = (fxa[i] - r.o.x) * r.inv.x;
        float ay = (nya[i] - r.o.y) * r.inv.y;
        float by = (fya[i] - r.o.y) * r.inv.y;
        float az = (nza[i] - r.o.z) * r.inv.z;
        float bz = (fza[i] - r.o.z) * r.inv.z;
        float t0 = fmaxf(fmaxf(ax, ay), fmaxf(az, r.tmin));
        float t1 = fminf(fminf(bx, by), fminf(bz, best));
        t1 = fmaf(fabsf(t1), kBoxSlack, t1);
        tn[i] = t0;
        if (t0 <= t1) mask |= 1u << i;
    }
    return mask;
}

// Test the 8 children of compressed node `ni`.  Each plane is dequantised
// exactly (P = fmaf(2^23 + q, s, o2), see QNode8) and then tested exactly as in
// box4, so the same slack argument holds.  Returns the hit mask over slots.
__device__ __forceinline__ uint32_t box8(const QNode8* __restrict__ nodes, int ni, const Ray& r, float best,
                                         float tn[8], int32_t ch[8]) {
    const float4* p = reinterpret_cast<const float4*>(nodes + ni);
    const float4 hd = __ldg(p);
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(p + 1));
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(p + 2));
    const uint4 qx = __ldg(reinterpret_cast<const uint4*>(p + 3));
    const uint4 qy = __ldg(reinterpret_cast<const uint4*>(p + 4));
    const uint4 qz = __ldg(reinterpret_cast<const uint4*>(p + 5));
    const uint32_t meta = __float_as_uint(hd.w);
    const float sx = __uint_as_float((meta & 0xffu) << 23);
    const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
    const uint32_t valid = meta >> 24;
    // near / far plane bytes of slots 0-3 (.x) and 4-7 (.y) for this ray's octant
    const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
    const uint2 qnx = nx ? make_uint2(qx.z, qx.w) : make_uint2(qx.x, qx.y);
    const uint2 qfx = nx ? make_uint2(qx.x, qx.y) : make_uint2(qx.z, qx.w);
    const uint2 qny = ny ? make_uint2(qy.z, qy.w) : make_uint2(qy.x, qy.y);
    const uint2 qfy = ny ? make_uint2(qy.x, qy.y) : make_uint2(qy.z, qy.w);
    const uint2 qnz = nz ? make_uint2(qz.z, qz.w) : make_uint2(qz.x, qz.y);
    const uint2 qfz = nz ? make_uint2(qz.x, qz.y) : make_uint2(qz.z, qz.w);
    ch[0] = c0.x; ch[1] = c0.y; ch[2] = c0.z; ch[3] = c0.w;
    ch[4] = c1.x; ch[5] = c1.y; ch[6] = c1.z; ch[7] = c1.w;
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        // byte (i & 3) of the word as the float 2^23 + q
        const uint32_t sel = 0x7540u | uint32_t(i & 3);
        const float nqx = __uint_as_float(__byte_perm(i < 4 ? qnx.x : qnx.y, 0x4B000000u, sel));
        const float fqx = __uint_as_float(__byte_perm(i < 4 ? qfx.x : qfx.y, 0x4B000000u, sel));
        const float nqy = __uint_as_float(__byte_perm(i < 4 ? qny.x : qny.y, 0x4B000000u, sel));
        const float fqy = __uint_as_float(__byte_perm(i < 4 ? qfy.x : qfy.y, 0x4B000000u, sel));
        const float nqz = __uint_as_float(__byte_perm(i < 4 ? qnz.x : qnz.y, 0x4B000000u, sel));
        const float fqz = __uint_as_float(__byte_perm(i < 4 ? qfz.x : qfz.y, 0x4B000000u, sel));
        const float ax = (fmaf(nqx, sx, hd.x) - r.o.x) * r.inv.x;
        const float bx = (fmaf(fqx, sx, hd.x) - r.o.x) * r.inv.x;
        const float ay = (fmaf(nqy, sy, hd.y) - r.o.y) * r.inv.y;
        const float by = (fmaf(fqy, sy, hd.y) - r.o.y) * r.inv.y;
        const float az = (fmaf(nqz, sz, hd.z) - r.o.z) * r.inv.z;
        const float bz = (fmaf(fqz, sz, hd.z) - r.o.z) * r.inv.z;
        float t0 = fmaxf(fmaxf(ax, ay), fmaxf(az, r.tmin));
        float t1 = fminf(fminf(bx, by), fminf(bz, best));
        t1 = fmaf(fabsf(t1), kBoxSlack, t1);
        tn[i] = t0;
        if (t0 <= t1) mask |= 1u << i;
    }
    return mask & valid;
}

// Slot permutation s -> s ^ oct applied to an 8-bit mask.
__device__ __forceinline__ uint32_t octant_order(uint32_t m, uint32_t oct) {
    if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
    return m;
}

// Traversal stack: the first SM entries of each ray live in shared memory
// (entry-major, one column per thread), deeper entries in local memory.
template <int SM>
struct RayStack {
    int2* sm;        // &shared[0][threadIdx.x]; entry i at sm[i * stride]
    int2* lm;        // local array; entry i >= SM at lm[i - SM]
    int stride;
    __device__ __forceinline__ void put(int i, int2 v) const {
        if (SM > 0 && i < SM) sm[i * stride] = v;
        else lm[i - SM] = v;
    }
    __device__ __forceinline__ int2 get(int i) const {
        if (SM > 0 && i < SM) return sm[i * stride];
        return lm[i - SM];
    }
};

struct Counters {
    unsigned long long rays, nodes, tris;
};

// Per-lane traversal state kept across refill points.
template <bool WT>
struct TravState {
    Ray r;
    typename std::conditional<WT, ObjRayWT, ObjRay>::type cache;
    float best, u, v;
    int prim;
    int cls;        // material class of the closest hit so far (TriRec e2.w)
    int item;       // current node / leaf code; kNone when the stack must be popped
    int sp;
};
constexpr int kNone = 0x7fffffff;   // == kEmptyChild

template <class TS>
__device__ __forceinline__ void trav_init(TS& s, float4 a, float4 b) {
    s.r = make_ray(a, b);
    s.cache.bundle = -2;
    s.best = s.r.tmax;
    s.prim = -1;
    s.cls = 0;
    s.u = s.v = 0.f;
    s.item = 0;      // root
    s.sp = 0;
}

// Runs at most `steps` node / leaf visits.  Returns true when the ray is done.
// Pops the next stack entry, skipping entries that start beyond the closest
// hit; false when the stack is empty.
template <bool ANY, class STACK, class TS>
__device__ __forceinline__ bool trav_pop(TS& s, const STACK& stack, int& item) {
    while (s.sp > 0) {
        const int2 e = stack.get(--s.sp);
        // the entry distance carries the box test's rounding: cull with its slack
        if (!ANY && __int_as_float(e.y) > fmaf(fabsf(s.best), kBoxSlack, s.best)) continue;
        item = e.x;
        return true;
    }
    return false;
}

// Visits internal node `item`: continues with the nearest hit child (s.item),
// pushes the others.  False on stack overflow (error flag raised).
template <bool COUNT, int WIDTH, class STACK, class TS>
__device__ __forceinline__ bool trav_node(const DevScene& S, TS& s, const STACK& stack, int item,
                                          Counters& cnt) {
    if (COUNT) ++cnt.nodes;
    if (WIDTH == 8) {
        float tn[8];
        int32_t ch[8];
        const uint32_t mask = box8(S.nodes8, item, s.r, s.best, tn, ch);
        if (mask == 0) { s.item = kNone; return true; }
        // visit order i = slot ^ octant: continue with the first hit, push the
        // others so that they pop in visit order
        const uint32_t om = octant_order(mask, s.r.oct);
        const uint32_t rest = om & (om - 1u);
        const int first = __ffs(om) - 1;
        const int nrest = __popc(rest);
        if (s.sp + nrest > kStackSize8) {
            atomicOr(S.errflags, BG_FLAG_STACK_OVERFLOW);
            return false;
        }
        int next = kNone;
#pragma unroll
        for (int sl = 0; sl < 8; ++sl) {
            const int i = sl ^ int(s.r.oct);
            if ((rest >> i) & 1u) stack.put(s.sp + __popc(rest >> (i + 1)), make_int2(ch[sl], __float_as_int(tn[sl])));
            if (i == first) next = ch[sl];
        }
        s.sp += nrest;
        s.item = next;
        return true;
    }
    float tn[4];
    int32_t ch[4];
    const uint32_t mask = box4(S.nodes, item, s.r, s.best, tn, ch);
    // order the children by entry distance with a 4-input sorting network on
    // registers (missed children get +inf and sort last)
    const int nh = __popc(mask);
    if (nh == 0) { s.item = kNone; return true; }
    float ht[4];
    int hc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        ht[i] = (mask & (1u << i)) ? tn[i] : __int_as_float(0x7f800000);
        hc[i] = ch[i];
    }
    auto cex = [&](int a, int b) {
        const bool sw = ht[a] > ht[b];
        const float ta = ht[a], tb = ht[b];
        const int ca = hc[a], cb = hc[b];
        ht[a] = sw ? tb : ta; ht[b] = sw ? ta : tb;
        hc[a] = sw ? cb : ca; hc[b] = sw ? ca : cb;
    };
    cex(0, 1); cex(2, 3); cex(0, 2); cex(1, 3); cex(1, 2);
    // push the farther ones (farthest first), continue with the nearest
    if (s.sp + nh - 1 > kStackSize) {
        atomicOr(S.errflags, BG_FLAG_STACK_OVERFLOW);
        return false;
    }
#pragma unroll
    for (int i = 3; i >= 1; --i)
        if (i < nh) stack.put(s.sp++, make_int2(hc[i], __float_as_int(ht[i])));
    s.item = hc[0];
    return true;
}

// Tests the first triangle of leaf code `item` (bit 31 set, count-1 in bits
// 27..30, first triangle in bits 0..26) and sets the lane's next item: the
// rest of the leaf, or a pop.  True when an any-hit query found its hit.  One
// triangle per traversal step keeps lanes that are in a leaf in step with
// lanes that are in a node (measured against the whole leaf in one step: C2
// incoherent closest hits +4 %, any hits +3.5 %, C3 frame +1-2 %).
// WT: the scene's records hold the vertices (p1, p2, p3) and the test is the
// watertight one; otherwise they hold (p1, e1, e2) for Moller-Trumbore.
template <bool ANY, bool COUNT, bool WT>
__device__ __forceinline__ bool trav_leaf(const DevScene& S, TravState<WT>& s, int item, Counters& cnt) {
    const uint32_t code = uint32_t(item);
    const int count = int((code >> kLeafStartBits) & 15u) + 1;
    const int start = int(code & uint32_t(kMaxLeafStart));
    // the rest of the leaf: one triangle fewer, starting one later
    s.item = count > 1 ? int(code - (1u << kLeafStartBits) + 1u) : kNone;
    const float4* tp = reinterpret_cast<const float4*>(S.tris + start);
    float4 v0 = __ldg(tp), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
    if (COUNT) ++cnt.tris;
    obj_ray(S, s.r, __float_as_int(v0.w), s.cache);
    float t, a, b;
    bool hit;
    if constexpr (WT)
        hit = wt_test(s.cache, mk(v0.x, v0.y, v0.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z), s.r.tmin,
                      ANY ? s.r.tmax : s.best, t, a, b);
    else
        hit = mt_test(s.cache.o, s.cache.d, mk(v0.x, v0.y, v0.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z),
                      s.r.tmin, ANY ? s.r.tmax : s.best, t, a, b);
    if (hit) {
        s.prim = __float_as_int(e1.w);
        if (ANY) return true;
        s.best = t; s.u = a; s.v = b;
        s.cls = __float_as_int(e2.w);
    }
    return false;
}

// Runs at most `steps` node / leaf visits.  Returns true when the ray is done.
// (Measured and rejected: node and leaf visits in two warp-wide phases,
// with or without postponing a lane's leaf while others still descend: the
// votes and the longer loops cost 2.5-4x on C2 and C3.)
template <bool ANY, bool COUNT, int WIDTH, class STACK, bool WT>
__device__ __forceinline__ bool trav_steps(const DevScene& S, TravState<WT>& s, const STACK& stack, int steps,
                                           Counters& cnt) {
    for (int it = 0; it < steps; ++it) {
        int item = s.item;
        if (item == kNone && !trav_pop<ANY>(s, stack, item)) return true;
        if (item >= 0) {
            if (!trav_node<COUNT, WIDTH>(S, s, stack, item, cnt)) return true;
        } else {
            if (trav_leaf<ANY, COUNT>(S, s, item, cnt)) return true;
        }
    }
    return false;
}

}  // namespace bg
