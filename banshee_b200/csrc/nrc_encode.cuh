// Radiance-cache input encoding (shared by the encode kernel and the fused
// tcgen05 inference kernel): multiresolution hash grid of the normalised
// position (16 levels x 2 features, trilinear; Mueller et al., "Instant Neural
// Graphics Primitives", 2022) and one-blob encodings of the direction and
// normal in spherical coordinates (Mueller et al., "Neural Importance
// Sampling", 2019), packed as 128 bf16 values (64 words).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "cache.h"
#include "device_common.cuh"

namespace bg {

// two floats -> bf16 pair (round to nearest even), low half first
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// ------------------------------------------------------------- encoding
__device__ __forceinline__ uint32_t grid_index(const NrcDev& C, int level, int x, int y, int z) {
    const uint32_t T = 1u << C.log2_T;
    const uint32_t n1 = uint32_t(C.res[level]) + 1u;
    if (uint64_t(n1) * n1 * n1 <= T) return uint32_t(x) + n1 * (uint32_t(y) + n1 * uint32_t(z));
    return (uint32_t(x) * 1u ^ uint32_t(y) * 2654435761u ^ uint32_t(z) * 805459861u) & (T - 1u);
}

struct GridCorner {
    int x0, y0, z0;
    float fx, fy, fz;
};
__device__ __forceinline__ GridCorner grid_cell(const NrcDev& C, int level, const float* u) {
    GridCorner g;
    const float N = float(C.res[level]);
    float x = u[0] * N, y = u[1] * N, z = u[2] * N;
    float fx0 = fminf(floorf(x), N - 1.f), fy0 = fminf(floorf(y), N - 1.f), fz0 = fminf(floorf(z), N - 1.f);
    g.x0 = int(fx0); g.y0 = int(fy0); g.z0 = int(fz0);
    g.fx = x - fx0; g.fy = y - fy0; g.fz = z - fz0;
    return g;
}

__device__ __forceinline__ void norm_pos(const NrcDev& C, const float* f, float* u) {
#pragma unroll
    for (int k = 0; k < 3; ++k) u[k] = fminf(fmaxf((f[k] - C.bmin[k]) * C.bscale[k], 0.f), 1.f);
}

// one-blob encoding of v in [0,1] into 16 bf16 values, packed two per word
__device__ __forceinline__ void one_blob(float v, uint32_t* w) {
#pragma unroll
    for (int b = 0; b < 16; b += 2) {
        const float d0 = v - (b + 0.5f) * (1.f / 16.f), d1 = v - (b + 1.5f) * (1.f / 16.f);
        w[b / 2] = pack_bf16(__expf(-d0 * d0 * 128.f), __expf(-d1 * d1 * 128.f));
    }
}

__device__ __forceinline__ void sph(float x, float y, float z, float& th, float& ph) {
    th = acosf(fminf(fmaxf(z, -1.f), 1.f)) * (1.f / BG_PI);
    ph = atan2f(y, x) * (0.5f / BG_PI) + 0.5f;
}

// The encoded row of one raw query record (16 floats: position, outgoing
// direction, shading normal, roughness, albedo): words 0-15 the grid features,
// 16-47 the four one-blobs, 48-49 roughness and albedo, 50 a constant 1, the
// rest 0.
__device__ __forceinline__ void encode_row(const NrcDev& C, const float* __restrict__ f, uint32_t (&w)[kNrcIn / 2]) {
    const float4* f4 = reinterpret_cast<const float4*>(f);
    const float4 q0 = f4[0], q1 = f4[1], q2 = f4[2], q3 = f4[3];
    const float fr[13] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, q3.x};
    float u[3];
    norm_pos(C, fr, u);
#pragma unroll
    for (int l = 0; l < kNrcLevels; ++l) {
        GridCorner g = grid_cell(C, l, u);
        float a0 = 0.f, a1 = 0.f;
#pragma unroll
        for (int cidx = 0; cidx < 8; ++cidx) {
            const int dx = cidx & 1, dy = (cidx >> 1) & 1, dz = (cidx >> 2) & 1;
            const float wt = (dx ? g.fx : 1.f - g.fx) * (dy ? g.fy : 1.f - g.fy) * (dz ? g.fz : 1.f - g.fz);
            const uint32_t idx = grid_index(C, l, g.x0 + dx, g.y0 + dy, g.z0 + dz);
            const float2 v = __ldg(reinterpret_cast<const float2*>(C.grid + (size_t(l) << C.log2_T) * 2 + size_t(idx) * 2));
            a0 += wt * v.x;
            a1 += wt * v.y;
        }
        w[l] = pack_bf16(a0, a1);
    }
    float th, ph;
    sph(fr[3], fr[4], fr[5], th, ph);
    one_blob(th, w + 16);
    one_blob(ph, w + 24);
    sph(fr[6], fr[7], fr[8], th, ph);
    one_blob(th, w + 32);
    one_blob(ph, w + 40);
    w[48] = pack_bf16(fr[9], fr[10]);
    w[49] = pack_bf16(fr[11], fr[12]);
    w[50] = pack_bf16(1.f, 0.f);
#pragma unroll
    for (int k = 51; k < kNrcIn / 2; ++k) w[k] = 0u;
}

}  // namespace bg
