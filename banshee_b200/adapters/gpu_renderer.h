// GpuRenderer: Banshee's Renderer (renderer/renderer.h:42-54) that renders the
// whole frame with the B200 library's wavefront tracer.  Header-only; same
// build requirements as gpu_accelerator.h.
//
//   GpuRenderer r(scene, camera_desc, tracer_desc, sampler_desc, w, h, rgbw);
//   r.Render(world);          // rgbw (w*h*4 floats, host) += the frame's samples
//
// rgbw has FileImagePlane's layout (sum r, g, b, sample count; rows
// bottom-up, imageplane/fileimageplane.cpp:29-34), so FileImagePlane::Finalize's
// (c / w)^(1/2.2) applies unchanged (bg_image_finalize / bg_image_write).
// The scene must hold the World's meshes, materials and lights in the World's
// order; the camera descriptor carries PerscpectiveCamera's constructor
// arguments (camera/perspective_camera.cpp:5).  Each Render call advances the
// sample offset, so repeated calls accumulate new samples (progressive).
// Render checks that the scene describes the World it is given (as many
// bundles, faces, materials and lights) and throws if not: shading normals,
// uvs, materials and lights are private to the reference's classes, so the
// scene cannot be read back from the World itself (world_scene.h builds the
// geometry-only scene GpuAccelerator needs).
#pragma once

#include <stdexcept>

#include "renderer/renderer.h"
#include "world/world.h"
#include "banshee_gpu.h"

class GpuRenderer : public Renderer {
public:
    GpuRenderer(bg_scene* scene, bg_camera_desc const& camera, bg_tracer_desc const& tracer,
                bg_sampler_desc const& sampler, int width, int height, float* rgbw)
        : scene_(scene), camera_(camera), tracer_(tracer), sampler_(sampler), w_(width), h_(height), out_(rgbw) {}

    void Render(World const& world) const override {
        check_world(world);
        bg_sampler_desc s = sampler_;
        s.sample_offset = next_;
        if (bg_render_host(scene_, &camera_, &tracer_, &s, w_, h_, out_, nullptr) != BG_OK)
            throw std::runtime_error(bg_last_error());
        next_ += s.spp;
    }

private:
    void check_world(World const& world) const {
        bg_scene_info info;
        if (bg_scene_info_get(scene_, &info) != BG_OK) throw std::runtime_error(bg_last_error());
        int64_t faces = 0;
        for (auto const& b : world.shapebundles_) faces += int64_t(b->GetNumShapes());
        if (int64_t(world.shapebundles_.size()) != info.nmeshes || faces != info.ntriangles ||
            int64_t(world.materials_.size()) != info.nmaterials || int64_t(world.lights_.size()) != info.nlights)
            throw std::runtime_error("GpuRenderer: the device scene does not describe this World");
    }

    bg_scene* scene_;
    bg_camera_desc camera_;
    bg_tracer_desc tracer_;
    bg_sampler_desc sampler_;
    int w_, h_;
    float* out_;
    mutable int next_ = 0;
};
