// GpuAccelerator: Banshee's Intersectable (accelerator/intersectable.h:41-50)
// answered by the B200 library.  Header-only; include it in a Banshee build
// that also has include/banshee_gpu.h on its include path and links
// libbanshee_gpu.so.
//
//   world.Commit();                                    // World::accel_ = Bvh
//   bg_scene* s = ...;                                 // same meshes, same order (bg_scene_add_mesh)
//   world.accel_.reset(new GpuAccelerator(world, s));  // from now on World::Intersect runs on the GPU
//
// Closest hit: bg_intersect_closest_host finds (primitive, t, u, v) with the
// reference's own Moller-Trumbore arithmetic, then the owning Mesh's FillHit
// (primitive/mesh.cpp:47-97) fills the ShapeBundle::Hit exactly as
// Mesh::IntersectShape does, so tracers see the same hits as with Bvh.
// Per-ray calls exist for compatibility with code that calls
// World::Intersect one ray at a time; batches belong on bg_intersect_closest.
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "accelerator/intersectable.h"
#include "primitive/mesh.h"
#include "world/world.h"
#include "banshee_gpu.h"

class GpuAccelerator : public Intersectable {
public:
    GpuAccelerator(World const& world, bg_scene* scene) : scene_(scene) {
        int64_t base = 0;
        for (auto const& b : world.shapebundles_) {
            const Mesh* m = dynamic_cast<const Mesh*>(b.get());
            if (!m) throw std::runtime_error("GpuAccelerator: only Mesh bundles are supported");
            meshes_.push_back(m);
            first_.push_back(base);
            base += int64_t(m->GetNumShapes());
        }
    }

    // World::Intersect has set hit.t = r.t.y (world/world.cpp:21)
    bool Intersect(ray const& r, ShapeBundle::Hit& hit) const override {
        bg_ray q = {{r.o.x, r.o.y, r.o.z}, r.t.x, {r.d.x, r.d.y, r.d.z}, hit.t};
        bg_hit h;
        if (bg_intersect_closest_host(scene_, &q, &h, 1) != BG_OK) throw std::runtime_error(bg_last_error());
        if (h.primid < 0) return false;
        const size_t b = size_t(std::upper_bound(first_.begin(), first_.end(), int64_t(h.primid)) - first_.begin()) - 1;
        meshes_[b]->FillHit(size_t(h.primid - first_[b]), h.t, h.u, h.v, hit);
        return true;
    }

    bool Intersect(ray const& r) const override {
        bg_ray q = {{r.o.x, r.o.y, r.o.z}, r.t.x, {r.d.x, r.d.y, r.d.z}, r.t.y};
        uint8_t occluded = 0;
        if (bg_intersect_any_host(scene_, &q, &occluded, 1) != BG_OK) throw std::runtime_error(bg_last_error());
        return occluded != 0;
    }

private:
    bg_scene* scene_;
    std::vector<const Mesh*> meshes_;
    std::vector<int64_t> first_;    // global id of each mesh's face 0
};
