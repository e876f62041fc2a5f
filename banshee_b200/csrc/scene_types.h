// Device-resident scene layout (HBM), shared by host upload code and kernels.
//
//   nodes    WideNode4[nnodes]   128 B, one L2 line per 4-wide node
//   nodes8   QNode8[nnodes8]      96 B, three 32-byte sectors per 8-wide compressed node
//   tris     TriRec[ntris]        48 B, leaf order; what traversal streams
//   shade    ShadeRec[ntris]     112 B, global primitive order; read once per hit
//   bundles  BundleRec[nmeshes]   per-mesh transform, identity flag, area-light owner
//   mats     MatRec[nmats], lights LightRec[nlights]
#pragma once

#include <cstdint>
#include <vector_types.h>

#include "bvh_build.h"

namespace bg {

// Moller-Trumbore operands in object space: v0 = p1, e1 = p2 - p1, e2 = p3 - p1
// (computed once with the same float subtraction as primitive/mesh.cpp:13-14).
// v0.w = bundle index (int bits), e1.w = global primitive id (int bits), e2.w
// = material class of the face (int bits: 0 emissive, 1 Lambert, 2 GGX; what
// the renderer splits its shading by).  A scene committed with the watertight
// test holds the vertices themselves: v0 = p1, e1 = p2, e2 = p3 (same .w fields).
struct alignas(16) TriRec {
    float4 v0, e1, e2;
};
static_assert(sizeof(TriRec) == 48, "TriRec is 48 bytes");

// Everything Mesh::FillHit needs (primitive/mesh.cpp:47-97) for one face.
//   a = (p1, bundle)   b = (p2, material)   c = (p3, uv1.x)
//   d = (n1, uv1.y)    e = (n2, uv2.x)      f = (n3, uv2.y)   g = (uv3, 0, 0)
struct alignas(16) ShadeRec {
    float4 a, b, c, d, e, f, g;
};
static_assert(sizeof(ShadeRec) == 112, "ShadeRec is 112 bytes");

struct alignas(16) BundleRec {
    float m[12];        // world transform, rows 0..2
    float minv[12];     // inverse, rows 0..2
    int32_t identity;   // m and minv are exactly the identity
    int32_t arealight;  // ShapeBundle::arealight_ (last AreaLight made on it), -1 if none
    int32_t nfaces;
    int32_t pad;
    int64_t start;      // global id of face 0
    int64_t pad2;
};

struct MatRec {
    int32_t type;       // BG_MAT_*
    float kd[3];
    float ks[3];
    float eta;
    float a;            // GGX roughness
    float e[3];
};

struct LightRec {
    int32_t type;       // BG_LIGHT_*
    int32_t mesh, face, matidx;
    float dir[3];       // directional: normalize(d) (light/directional_light.h:44)
    float e[3];         // directional radiance / area: emission of the material
    float env[3];       // environment: scale * pow(texel, 1/gamma), precomputed on the host
    float area_world;   // area: Mesh::GetShapeSurfaceArea (world space, mesh.cpp:304-321)
    float pdf_obj;      // area: FillSample's 1 / area in object space (mesh.cpp:121)
    float pad;
};

struct DevScene {
    const WideNode4* nodes;
    const QNode8* nodes8;
    const TriRec* tris;
    const ShadeRec* shade;
    const BundleRec* bundles;
    const MatRec* mats;
    const LightRec* lights;
    unsigned int* errflags;
    int64_t ntris;
    int32_t nbundles, nmats, nlights;
    int32_t width;          // node layout traversed: 4 (nodes) or 8 (nodes8)
    float bg[3];
    int32_t has_area;       // some light is an AreaLight (selects the shading variant)
    int32_t watertight;     // tris hold (p1, p2, p3) for the watertight test, not (p1, e1, e2)
    int32_t pad3;
};

}  // namespace bg
