// Quantisation of one 8-wide compressed node (QNode8), shared by the host
// builder (bvh_build.cpp) and the device collapse (gpu_build.cu) so that both
// emit the same bytes for the same children.  Only exact arithmetic is used:
// exponents come from frexp, planes from ldexp / floor / ceil, and the
// self-check evaluates the traversal's own dequantisation fmaf(2^23 + q, 2^e, o2).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "bvh_build.h"

#if defined(__CUDACC__)
#define BG_HD __host__ __device__ __forceinline__
#else
#define BG_HD inline
#endif

namespace bg {

// std::min / std::max semantics (the first argument wins ties and NaNs)
BG_HD float qmin(float a, float b) { return b < a ? b : a; }
BG_HD float qmax(float a, float b) { return a < b ? b : a; }

// floor(log2(x)) and ceil(log2(x)) for finite x > 0, exactly
BG_HD int floor_log2(double x) {
    int ex = 0;
    ::frexp(x, &ex);            // x = m 2^ex, m in [0.5, 1)
    return ex - 1;
}
BG_HD int ceil_log2(double x) {
    int ex = 0;
    const double m = ::frexp(x, &ex);
    return m == 0.5 ? ex - 1 : ex;
}

// Grid of one axis for children spanning [L, H]: the smallest exponent e
// (step 2^e) and origin index k (|k| < 2^23 - 256) with k 2^e <= L and
// (k + 255) 2^e >= H; returns kQMaxExp + 1 when none exists.
BG_HD int qnode_axis_exact(float L, float H, double* k) {
    int e = -120;
    const double ext = double(H) - double(L);
    if (ext > 0.0) {
        const int c = ceil_log2(ext / 255.0) - 1;
        e = c > e ? c : e;
    }
    const double aL = ::fabs(double(L));
    if (aL > 0.0) {
        const int c = floor_log2(aL) - 23;
        e = c > e ? c : e;
    }
    for (; e <= kQMaxExp; ++e) {
        const double kk = ::floor(::ldexp(double(L), -e));
        if (::fabs(kk) > 8388608.0 - 257.0) continue;
        if (::ldexp(kk + 255.0, e) < double(H)) continue;
        *k = kk;
        return e;
    }
    *k = 0.0;
    return kQMaxExp + 1;
}

// Fills q from nk (2..8) children: kb[i] = {lo x, y, z, hi x, y, z}, codes[i]
// the child encoding.  Slot assignment: greedy over (child, slot) by the
// child's centroid offset projected on the slot's octant signs, so that slot
// (i ^ octant) is roughly the i-th child met by a ray of that octant.  Returns
// false when a plane cannot be made conservative (coordinates too large).
BG_HD bool fill_qnode8(QNode8& q, const float (*kb)[6], const int32_t* codes, int nk) {
    bool ok = true;
    float ulo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, uhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < nk; ++i)
        for (int a = 0; a < 3; ++a) { ulo[a] = qmin(ulo[a], kb[i][a]); uhi[a] = qmax(uhi[a], kb[i][3 + a]); }
    double cen[8][3];
    for (int i = 0; i < nk; ++i)
        for (int a = 0; a < 3; ++a)
            cen[i][a] = 0.5 * (double(kb[i][a]) + double(kb[i][3 + a])) - 0.5 * (double(ulo[a]) + double(uhi[a]));
    int slot_of[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool cused[8] = {false, false, false, false, false, false, false, false};
    bool sused[8] = {false, false, false, false, false, false, false, false};
    for (int r = 0; r < nk; ++r) {
        double best = 1e300;
        int bc = -1, bs = -1;
        for (int c = 0; c < nk; ++c) {
            if (cused[c]) continue;
            for (int sl = 0; sl < 8; ++sl) {
                if (sused[sl]) continue;
                double cost = 0.0;
                for (int a = 0; a < 3; ++a) cost += ((sl >> a) & 1 ? -cen[c][a] : cen[c][a]);
                if (cost < best) { best = cost; bc = c; bs = sl; }
            }
        }
        if (bc < 0) {               // NaN centroids: take the first free pair
            for (int c = 0; c < nk && bc < 0; ++c) if (!cused[c]) bc = c;
            for (int sl = 0; sl < 8 && bs < 0; ++sl) if (!sused[sl]) bs = sl;
        }
        cused[bc] = true; sused[bs] = true; slot_of[bc] = bs;
    }
    int e[3];
    double k[3];
    for (int a = 0; a < 3; ++a) {
        e[a] = qnode_axis_exact(ulo[a], uhi[a], &k[a]);
        if (e[a] > kQMaxExp) { ok = false; e[a] = kQMaxExp; }
    }
    float o2[3];
    for (int a = 0; a < 3; ++a) o2[a] = float(::ldexp(k[a] - 8388608.0, e[a]));
    q.o2x = o2[0]; q.o2y = o2[1]; q.o2z = o2[2];
    uint32_t valid = 0;
    uint8_t qb[3][2][8];
    for (int a = 0; a < 3; ++a)
        for (int sl = 0; sl < 8; ++sl) { qb[a][0][sl] = 255; qb[a][1][sl] = 0; }   // unused slot: inverted box
    for (int sl = 0; sl < 8; ++sl) q.child[sl] = kEmptyChild;
    for (int c = 0; c < nk; ++c) {
        const int sl = slot_of[c];
        valid |= 1u << sl;
        q.child[sl] = codes[c];
        for (int a = 0; a < 3; ++a) {
            const double lo = ::floor(::ldexp(double(kb[c][a]), -e[a])) - k[a];
            const double hi = ::ceil(::ldexp(double(kb[c][3 + a]), -e[a])) - k[a];
            double cl = 0.0 < lo ? lo : 0.0, ch = 0.0 < hi ? hi : 0.0;   // clamp to [0, 255]; NaN -> 0
            cl = cl < 255.0 ? cl : 255.0;
            ch = ch < 255.0 ? ch : 255.0;
            qb[a][0][sl] = uint8_t(cl);
            qb[a][1][sl] = uint8_t(ch);
        }
    }
    q.meta = uint32_t(e[0] + 127) | (uint32_t(e[1] + 127) << 8) | (uint32_t(e[2] + 127) << 16) | (valid << 24);
    for (int c = 0; c < nk; ++c) {      // self-check against the traversal's dequantisation
        const int sl = slot_of[c];
        for (int a = 0; a < 3; ++a) {
            const float st = ::ldexpf(1.0f, e[a]);
            const float plo = ::fmaf(8388608.0f + float(qb[a][0][sl]), st, o2[a]);
            const float phi = ::fmaf(8388608.0f + float(qb[a][1][sl]), st, o2[a]);
            if (!(plo <= kb[c][a] && phi >= kb[c][3 + a])) ok = false;
        }
    }
    uint32_t* w[3] = {q.qx, q.qy, q.qz};
    for (int a = 0; a < 3; ++a)
        for (int h = 0; h < 2; ++h)
            for (int half = 0; half < 2; ++half) {
                uint32_t v = 0;
                for (int j = 0; j < 4; ++j) v |= uint32_t(qb[a][h][4 * half + j]) << (8 * j);
                w[a][2 * h + half] = v;
            }
    return ok;
}

}  // namespace bg
