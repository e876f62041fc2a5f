// Device math shared by the traversal and shading kernels.
//
// Every translation unit of the library is compiled with -fmad=false and IEEE
// division / square root, so each operator below is one correctly rounded
// float operation, in the same order as Banshee's float3 / matrix code
// (math/float3.h, math/matrix.h, math/mathutils.h).  That makes ray
// generation, ray transforms and the Moller-Trumbore test bit-identical to the
// reference on the same inputs; only the transcendental functions
// (sinf/cosf/powf/atanf) differ from libm by a few ulp.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bg {

#define BG_PI 3.14159265358979323846f
#define BG_MINPDF 0.05f
#define BG_MAXRADIANCE 4.f

struct v3 { float x, y, z; };

__host__ __device__ __forceinline__ v3 mk(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
__host__ __device__ __forceinline__ v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ v3 muls(v3 a, float c) { return mk(a.x * c, a.y * c, a.z * c); }
__host__ __device__ __forceinline__ v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float sqnorm(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// float3::normalize: v * (1 / sqrt(|v|^2)), math/float3.h:50,57
__host__ __device__ __forceinline__ v3 normalize(v3 v) {
    float s = sqnorm(v);
    if (s > 0.f) {
        float cinv = 1.f / sqrtf(s);
        v.x *= cinv; v.y *= cinv; v.z *= cinv;
    }
    return v;
}
// math/float3.h:103-109
__host__ __device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - b.y * a.z, b.x * a.z - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float fmin_std(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float fmax_std(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float clamp_ref(float x, float a, float b) { return x < a ? a : (x > b ? b : x); }

// 3x4 row-major affine transform (the top three rows of Banshee's matrix).
struct Xform { float m[12]; };

// matrix * float3 (math/matrix.h:208-220): r_i = ((0 + m_i0 v0) + m_i1 v1) + m_i2 v2
__host__ __device__ __forceinline__ v3 xf_vector(const float* m, v3 v) {
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    r0 += m[0] * v.x; r0 += m[1] * v.y; r0 += m[2] * v.z;
    r1 += m[4] * v.x; r1 += m[5] * v.y; r1 += m[6] * v.z;
    r2 += m[8] * v.x; r2 += m[9] * v.y; r2 += m[10] * v.z;
    return mk(r0, r1, r2);
}
// transform_point (math/mathutils.h:129-137)
__host__ __device__ __forceinline__ v3 xf_point(const float* m, v3 p) {
    v3 r = xf_vector(m, p);
    r.x += m[3]; r.y += m[7]; r.z += m[11];
    return r;
}
// transform_normal = minv^T * n (math/mathutils.h:148-151)
__host__ __device__ __forceinline__ v3 xf_normal(const float* minv, v3 n) {
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    r0 += minv[0] * n.x; r0 += minv[4] * n.y; r0 += minv[8] * n.z;
    r1 += minv[1] * n.x; r1 += minv[5] * n.y; r1 += minv[9] * n.z;
    r2 += minv[2] * n.x; r2 += minv[6] * n.y; r2 += minv[10] * n.z;
    return mk(r0, r1, r2);
}

// ------------------------------------------------------------------ RNG
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Keyed stand-in for the global rand() (math/mathutils.h:62-65): 31-bit draws
// keyed by (seed, pixel, sample) and a per-sample call counter.
__host__ __device__ __forceinline__ uint64_t keyed_key(uint64_t seed, uint32_t pixel, uint32_t sample) {
    return splitmix64(seed ^ splitmix64((uint64_t(pixel) << 32) | sample));
}
__host__ __device__ __forceinline__ uint32_t keyed_rand(uint64_t key, uint32_t counter) {
    return uint32_t(splitmix64(key ^ (uint64_t(counter) * 0xD1B54A32D192ED03ull)) >> 33);
}
// rand_float: (float)rand() / RAND_MAX, RAND_MAX -> 2147483648.0f
__host__ __device__ __forceinline__ float rand_float(uint32_t r) { return float(int(r)) / float(2147483647); }

// McRng (rng/mcrng.h:54-65)
struct McRng { uint32_t z, w; };
__host__ __device__ __forceinline__ uint32_t mc_next_uint(McRng& r) {
    r.z = 36969u * (r.z & 65535u) + (r.z >> 16);
    r.w = 18000u * (r.w & 65535u) + (r.w >> 16);
    return (r.z << 16) + r.w;
}
__host__ __device__ __forceinline__ float mc_next_float(McRng& r) { return float(mc_next_uint(r)) * 2.328306e-10f; }
// RandomSampler::Sample2D (sampler/random_sampler.h:58-61).  g++ evaluates the
// two NextFloat() arguments right to left: x is the second draw, y the first.
__host__ __device__ __forceinline__ void sample2d(McRng& r, float& x, float& y) {
    float first = mc_next_float(r);
    float second = mc_next_float(r);
    x = second;
    y = first;
}

}  // namespace bg
