// Wavefront GI / DI renderer (filled in below).
#include "internal.h"

namespace bg {
struct RenderState {};
void render_state_free(RenderState* rs) { delete rs; }
}  // namespace bg

extern "C" int bg_render(bg_scene*, const bg_camera_desc*, const bg_tracer_desc*, const bg_sampler_desc*, int32_t,
                         int32_t, float*, bg_render_stats*, void*) {
    return bg::set_error(BG_ERR_UNSUPPORTED, "not built yet");
}
extern "C" int bg_render_host(bg_scene*, const bg_camera_desc*, const bg_tracer_desc*, const bg_sampler_desc*,
                              int32_t, int32_t, float*, bg_render_stats*) {
    return bg::set_error(BG_ERR_UNSUPPORTED, "not built yet");
}
