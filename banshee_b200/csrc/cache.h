// Neural radiance cache: device-side types shared by cache.cu and render.cu.
//
// No counterpart in the reference (Banshee has no learned component).  The
// encoding and network follow the published neural radiance caching design
// (Mueller et al., "Real-time Neural Radiance Caching for Path Tracing", 2021)
// with a multiresolution hash-grid position encoding (Mueller et al., "Instant
// Neural Graphics Primitives", 2022):
//   input  = hash grid (16 levels x 2 features) of the normalised position
//          + one-blob(16) of the outgoing direction and of the normal in
//            spherical coordinates (4 x 16) + roughness + albedo (3) + 1
//          -> 101 values, zero-padded to 128 bf16
//   MLP    = 128 -> 64 -> 64 -> 64 -> 64 -> 64 -> 16 (5 hidden ReLU layers,
//            3 outputs used), no biases, bf16 weights and activations, fp32
//            accumulation
//   loss   = relative L2: (pred - target)^2 / (pred^2 + 0.01), pred^2 not
//            differentiated
//   optim  = Adam (beta1 0.9, beta2 0.99, eps 1e-15) on fp32 master weights
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace bg {

constexpr int kNrcIn = 128;
constexpr int kNrcH = 64;
constexpr int kNrcOut = 16;
constexpr int kNrcLevels = 16;
constexpr int kNrcFeat = 2;
constexpr int kNrcGridDims = kNrcLevels * kNrcFeat;     // 32
// packed weight offsets (elements), row-major [out][in]
constexpr int kNrcW0 = 0;                               // [64][128]
constexpr int kNrcW1 = kNrcW0 + kNrcH * kNrcIn;         // [64][64] x 4
constexpr int kNrcW5 = kNrcW1 + 4 * kNrcH * kNrcH;      // [16][64]
constexpr int kNrcParams = kNrcW5 + kNrcOut * kNrcH;    // 25,600
constexpr int kNrcFeatFloats = 16;                      // raw query record

// Raw query record (16 floats): position (3), outgoing direction (3, unit),
// shading normal (3), roughness, albedo (3), 3 unused.
struct NrcDev {
    // hash grid
    float* grid;               // [levels][T][2] fp32 parameters
    float* grid_grad;
    float* grid_m;
    float* grid_v;
    int log2_T;
    int res[kNrcLevels];       // per-level resolution
    float bmin[3], bscale[3];  // position normalisation to [0,1]^3
    // MLP
    float* w;                  // fp32 master [kNrcParams]
    float* w_grad;
    float* w_m;
    float* w_v;
    __nv_bfloat16* wb;         // bf16 copy used by the kernels
    float lr, beta1, beta2, eps;
    int* step;                 // Adam step counter (device)
    uint32_t wait_polls;       // tcgen05 mbarrier wait budget (0 = default)
};

}  // namespace bg
