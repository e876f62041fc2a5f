// Render jobs: shared by the single-scene renderer and the multi-scene batch.
#pragma once

#include <cstdint>
#include <vector>
#include <vector_types.h>

#include "../../include/banshee_gpu.h"

namespace bg {

struct CamDev {        // PerscpectiveCamera frame, computed on the host (perspective_camera.cpp:5-23)
    float fwd[3], right[3], up[3], p[3];
    float znear, zfar, dimx, dimy;
};

// A render job: one scene (root node, light range, background) seen by one
// camera.  A single-scene render is one job; a batch merges several scenes into
// one device scene and renders many jobs through the same queues.
struct JobRec {
    int root, light0, nlights, pad;
    float bg[4];
};

struct JobSpec {       // host-side job description
    JobRec rec;
    CamDev cam;
    int W, H, spp, soff;
    uint64_t seed;
    float4* accum;
    int skind = 0, grid = 0;   // image sampler (BG_SAMPLER_*), CMJ grid size
};

// Paths-per-pass candidates of the autotuners: 2^19 .. 2^24.  Larger passes
// amortise the deep bounces, which hold few paths and take about the same time
// whatever the pass size (2^24 paths hold about 20 GB of state with 2 lights).  A candidate
// is skipped when the probe fits in half of it: it would run the same passes
// as the one before.
constexpr int kPassCandidates = 6;
inline int64_t pass_candidate(int i) { return int64_t(1) << (19 + i); }
inline bool pass_candidate_needed(int i, int64_t probe_samples) {
    return i == 0 || pass_candidate(i) / 2 < probe_samples;
}

CamDev make_camera(const bg_camera_desc* c);
int render_jobs(bg_scene* s, bg_cache* cache, const std::vector<JobSpec>& jobs, const bg_tracer_desc* tr,
                bg_render_stats* stats, cudaStream_t st, bool batched);

}  // namespace bg
