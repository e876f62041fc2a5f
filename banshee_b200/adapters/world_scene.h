// gpu_scene_from_world: the geometry of a committed Banshee World as a B200
// library scene, for GpuAccelerator.  Header-only; same build requirements as
// gpu_accelerator.h.
//
//   world.Commit();
//   bg_scene* s = gpu_scene_from_world(ctx, world);     // committed
//   world.accel_.reset(new GpuAccelerator(world, s));   // World::Intersect on the GPU
//   ...
//   bg_scene_destroy(s);                                // after the accelerator is gone
//
// One library mesh per Mesh bundle, in World::shapebundles_ order, built from
// the bundles' public accessors: Mesh::GetVertices / GetNumVertices /
// GetFaces / GetNumFaces (primitive/mesh.h:83-89) and ShapeBundle::GetTransform
// (primitive/shapebundle.h:142).  Ray casts on it find the same primitive,
// t, u and v as the World's own Bvh: the same vertices, the same transforms,
// the reference's Moller-Trumbore arithmetic.  GpuAccelerator fills each hit
// with the owning Mesh's FillHit on the host, so a ray-casting drop-in needs
// nothing else.
//
// Shading normals, uvs, materials and lights are private to the reference's
// Mesh, Material and Light classes, so a scene that the library shades itself
// (GpuRenderer, bg_render) is described through bg_scene_add_mesh /
// bg_scene_add_material / bg_scene_add_light from the data the World was built
// from.  Here the vertex positions stand in for the shading normals and every
// face refers to one placeholder Lambert material: ray casts read neither.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "primitive/mesh.h"
#include "world/world.h"
#include "banshee_gpu.h"

inline bg_scene* gpu_scene_from_world(bg_ctx* ctx, World const& world, bg_build_opts const* opts = nullptr) {
    bg_scene* s = nullptr;
    if (bg_scene_create(ctx, &s) != BG_OK) throw std::runtime_error(bg_last_error());
    try {
        std::vector<int32_t> vidx;
        const int32_t material0 = 0;   // every face: material 0 (stride 0)
        for (auto const& b : world.shapebundles_) {
            const Mesh* m = dynamic_cast<const Mesh*>(b.get());
            if (!m) throw std::runtime_error("gpu_scene_from_world: only Mesh bundles are supported");
            const Mesh::Face* faces = m->GetFaces();
            const int nf = int(m->GetNumFaces());
            // the library reads vertex indices with one stride per index; a Face
            // holds them among its other indices, so they are gathered here
            vidx.resize(3 * size_t(nf));
            for (int f = 0; f < nf; ++f) {
                vidx[3 * size_t(f)] = faces[f].vi0;
                vidx[3 * size_t(f) + 1] = faces[f].vi1;
                vidx[3 * size_t(f) + 2] = faces[f].vi2;
            }
            bg_mesh_desc d = {};
            d.vertices = m->GetNumVertices() ? &m->GetVertices()[0].x : nullptr;
            d.nvertices = int32_t(m->GetNumVertices());
            d.vstride = int32_t(sizeof(float3));
            d.normals = d.vertices;
            d.nnormals = d.nvertices;
            d.nstride = d.vstride;
            d.vidx = vidx.data();
            d.nidx = vidx.data();
            d.materials = &material0;
            d.mstride = 0;
            d.nfaces = nf;
            matrix xf, xfinv;
            m->GetTransform(xf, xfinv);
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) {
                    d.m[4 * r + c] = xf.m[r][c];
                    d.minv[4 * r + c] = xfinv.m[r][c];
                }
            if (bg_scene_add_mesh(s, &d, nullptr) != BG_OK) throw std::runtime_error(bg_last_error());
        }
        bg_material_desc placeholder = {};
        placeholder.type = BG_MAT_LAMBERT;
        placeholder.kd[0] = placeholder.kd[1] = placeholder.kd[2] = 0.5f;
        if (bg_scene_add_material(s, &placeholder, nullptr) != BG_OK) throw std::runtime_error(bg_last_error());
        if (bg_scene_commit(s, opts) != BG_OK) throw std::runtime_error(bg_last_error());
    } catch (...) {
        bg_scene_destroy(s);
        throw;
    }
    return s;
}
