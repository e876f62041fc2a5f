// Image samplers of the sampler plugin surface (sampler/sampler.h:57-66),
// evaluated per camera sample (pixel p, sample index s) without sequential
// state, so every wavefront lane computes its own sample:
//   * SobolSampler (sampler/sobol_sampler.cpp:3-49): x = scrambled base-2
//     radical inverse of s, y = scrambled Sobol (0,2) point s, top 24 bits of
//     each; the two scrambles are the first two NextUint of a McRng seeded by
//     the keyed rand() of (p, 0xFFFFFFFF) (the sampler's constructor draws);
//   * CmjSampler (sampler/cmj_sampler.cpp:3-73; Kensler, "Correlated
//     Multi-Jittered Sampling", 2013): sample s mod g^2 of pattern j = s / g^2,
//     whose index is the first NextUint of a McRng seeded by the keyed rand()
//     of (p, 0x80000000 + j) (the sampler draws one per pattern).
// The integer hashes and the float expressions are the reference's, so the
// samples are bit-identical to the reference classes under the same keys.
#pragma once

#include "device_common.cuh"
#include "../../include/banshee_gpu.h"

namespace bg {

__device__ __forceinline__ float sobol_radical_inverse(uint32_t n, uint32_t scramble) {
    const uint32_t r = __brev(n) ^ scramble;
    return float((r >> 8) & 0xffffffu) / float(1 << 24);
}

__device__ __forceinline__ float sobol_02(uint32_t n, uint32_t scramble) {
    uint32_t col = 0x80000000u;
    while (n) {
        if (n & 1u) scramble ^= col;
        n >>= 1;
        col ^= col >> 1;
    }
    return float((scramble >> 8) & 0xffffffu) / float(1 << 24);
}

__device__ __forceinline__ uint32_t cmj_permute(uint32_t i, uint32_t l, uint32_t p) {
    uint32_t w = l - 1;
    w |= w >> 1; w |= w >> 2; w |= w >> 4; w |= w >> 8; w |= w >> 16;
    do {
        i ^= p;             i *= 0xe170893du;
        i ^= p >> 16;       i ^= (i & w) >> 4;
        i ^= p >> 8;        i *= 0x0929eb3fu;
        i ^= p >> 23;       i ^= (i & w) >> 1;
        i *= 1u | p >> 27;  i *= 0x6935fa69u;
        i ^= (i & w) >> 11; i *= 0x74dcb303u;
        i ^= (i & w) >> 2;  i *= 0x9e501cc3u;
        i ^= (i & w) >> 2;  i *= 0xc860a3dfu;
        i &= w;
        i ^= i >> 5;
    } while (i >= l);
    return (i + p) % l;
}

__device__ __forceinline__ float cmj_jitter(uint32_t i, uint32_t p) {
    i ^= p;
    i ^= i >> 17; i ^= i >> 10; i *= 0xb36534e5u;
    i ^= i >> 12; i ^= i >> 21; i *= 0x93fc4795u;
    i ^= 0xdf6e307fu; i ^= i >> 17; i *= 1u | p >> 18;
    return float(i) * (1.0f / 4294967808.0f);
}

// Image sample of camera sample (pixel, s); img is the sample's keyed McRng
// (used by BG_SAMPLER_RANDOM only).
__device__ __forceinline__ void image_sample(int kind, int grid, uint64_t seed, uint32_t pixel, uint32_t s,
                                             McRng& img, float& x, float& y) {
    if (kind == BG_SAMPLER_SOBOL) {
        const uint64_t k = keyed_key(seed, pixel, 0xFFFFFFFFu);
        McRng m{keyed_rand(k, 0), keyed_rand(k, 1)};
        const uint32_t sc0 = mc_next_uint(m);
        const uint32_t sc1 = mc_next_uint(m);
        x = sobol_radical_inverse(s, sc0);
        y = sobol_02(s, sc1);
    } else if (kind == BG_SAMPLER_CMJ) {
        const uint32_t g2 = uint32_t(grid * grid);
        const uint64_t k = keyed_key(seed, pixel, 0x80000000u + s / g2);
        McRng m{keyed_rand(k, 0), keyed_rand(k, 1)};
        const uint32_t p = mc_next_uint(m);
        const int si = int(s % g2);
        const int sx = int(cmj_permute(uint32_t(si % grid), uint32_t(grid), p * 0xa511e9b3u));
        const int sy = int(cmj_permute(uint32_t(si / grid), uint32_t(grid), p * 0x63d83595u));
        const float jx = cmj_jitter(uint32_t(si), p * 0xa399d265u);
        const float jy = cmj_jitter(uint32_t(si), p * 0x711ad6a5u);
        const float g = float(grid);
        x = (float(si % grid) + (float(sy) + jx) / g) / g;
        y = (float(si / grid) + (float(sx) + jy) / g) / g;
    } else {
        sample2d(img, x, y);
    }
}

}  // namespace bg
