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
#pragma once

#include <stdexcept>

#include "renderer/renderer.h"
#include "banshee_gpu.h"

class GpuRenderer : public Renderer {
public:
    GpuRenderer(bg_scene* scene, bg_camera_desc const& camera, bg_tracer_desc const& tracer,
                bg_sampler_desc const& sampler, int width, int height, float* rgbw)
        : scene_(scene), camera_(camera), tracer_(tracer), sampler_(sampler), w_(width), h_(height), out_(rgbw) {}

    void Render(World const&) const override {
        bg_sampler_desc s = sampler_;
        s.sample_offset = next_;
        if (bg_render_host(scene_, &camera_, &tracer_, &s, w_, h_, out_, nullptr) != BG_OK)
            throw std::runtime_error(bg_last_error());
        next_ += s.spp;
    }

private:
    bg_scene* scene_;
    bg_camera_desc camera_;
    bg_tracer_desc tracer_;
    bg_sampler_desc sampler_;
    int w_, h_;
    float* out_;
    mutable int next_ = 0;
};
