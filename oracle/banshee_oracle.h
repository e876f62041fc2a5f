/*
 * banshee_oracle.h -- CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C restatement of Banshee's ray-casting and path-tracing hot path,
 * used by tests/, the smoke check and bench.py's CPU-baseline leg as the
 * checker.  Nothing in the product library links or calls it.  Every function
 * cites the reference file:line it restates (paths relative to
 * FireRays/Banshee/).  Parity of this restatement is pinned against the
 * reference's own sources compiled unmodified (oracle/Makefile -> oracle/_ref)
 * through the golden fixtures under tests/golden/.
 */
#ifndef BANSHEE_ORACLE_H
#define BANSHEE_ORACLE_H

#include <stdint.h>
#include "../include/banshee_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_world or_world;

/* World assembly + World::Commit (world/world.cpp:5-16): builds the reference
 * binary SAH BVH (accelerator/bvh.cpp:16-496) over the world-space triangle
 * bounds.  Returns NULL on invalid input. */
or_world* or_world_create(const bg_mesh_desc* meshes, int32_t nmeshes,
                          const bg_material_desc* mats, int32_t nmats,
                          const bg_light_desc* lights, int32_t nlights,
                          const float* bgcolor);
void or_world_destroy(or_world* w);
int64_t or_world_ntriangles(const or_world* w);
int64_t or_world_nnodes(const or_world* w);

/* World::Intersect(ray, Hit&) / World::Intersect(ray) over n rays,
 * parallel over nthreads host threads (0 = all cores). */
void or_intersect_closest(const or_world* w, const bg_ray* rays, bg_hit* hits,
                          int64_t n, int32_t nthreads);
void or_intersect_any(const or_world* w, const bg_ray* rays, uint8_t* occluded,
                      int64_t n, int32_t nthreads);
/* Nodes visited and triangles tested by the reference traversal. */
void or_traversal_counts(const or_world* w, const bg_ray* rays, int64_t n, int32_t any_hit,
                         uint64_t* nodes, uint64_t* triangles);
/* Mesh::IntersectShape for one global triangle id against one ray with
 * hit.t = tmax; returns 1 and the hit t (u, v) if accepted. */
int32_t or_triangle_test(const or_world* w, int64_t primid, const bg_ray* ray,
                         float* t, float* u, float* v);

/* ImageRenderer-style render of pixels [x0,x1) x [y0,y1) with the keyed
 * sampler contract of banshee_gpu.h into accum_rgbw (W*H float4, rows flipped
 * as in imageplane/fileimageplane.cpp:29-34). */
void or_render(const or_world* w, const bg_camera_desc* cam, int32_t tracer_kind,
               int32_t maxdepth, int32_t width, int32_t height, int32_t spp,
               int32_t sample_offset, uint64_t seed, float* accum_rgbw,
               int32_t x0, int32_t y0, int32_t x1, int32_t y1, int32_t nthreads,
               int32_t sampler_kind, int32_t sampler_grid, float ao_radius);

/* Primary rays of PerscpectiveCamera::GenerateRay for an image-plane sample
 * (camera/perspective_camera.cpp:25-38). */
void or_camera_rays(const bg_camera_desc* cam, const float* samples, bg_ray* rays, int64_t n);

/* The keyed rand() of the sampler contract. */
uint32_t or_keyed_rand(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t counter);

#ifdef __cplusplus
}
#endif

#endif
