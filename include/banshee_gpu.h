/*
 * banshee_gpu.h -- C ABI of the B200 (sm_100a) ray-casting and path-tracing
 * library that drops in behind Banshee's intersection and tracer plugin
 * surfaces.
 *
 * Every entry point returns an int status: BG_OK (0) on success, a negative
 * BG_ERR_* code otherwise; bg_last_error() returns a thread-local message for
 * the last failure.  No C++ exception crosses this boundary.  Pointers named
 * *_dev are device pointers (cudaMalloc'd or managed) and calls taking them are
 * asynchronous on the given CUDA stream (a cudaStream_t passed as void*, NULL
 * for the legacy default stream).  Calls named *_host take host pointers and
 * are synchronous; the host<->device copies happen inside the call.
 *
 * Reference interfaces replaced (paths relative to FireRays/Banshee/):
 *   Intersectable::Intersect(ray const&, Hit&)   accelerator/intersectable.h:46
 *   Intersectable::Intersect(ray const&)         accelerator/intersectable.h:48
 *   World::Commit / World::Intersect             world/world.cpp:5-29
 *   Mesh::Mesh(...) + ShapeBundle::SetTransform  primitive/mesh.h:69-76,
 *                                                primitive/shapebundle.h:139
 *   Renderer::Render(World const&)               renderer/renderer.h:49
 *   Tracer::GetLi (GiTracer / DiTracer)          tracer/tracer.h:53,
 *                                                tracer/gitracer.cpp:13,
 *                                                tracer/ditracer.cpp:19
 *   Sampler / Camera plugins                     sampler/sampler.h:57-66,
 *                                                camera/camera.h:53
 */
#ifndef BANSHEE_GPU_H
#define BANSHEE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define BG_OK                  0
#define BG_ERR_INVALID_ARG    -1  /* bad pointer, size or descriptor field   */
#define BG_ERR_CUDA           -2  /* a CUDA runtime call failed              */
#define BG_ERR_OOM            -3  /* device or host allocation failed        */
#define BG_ERR_STATE          -4  /* call order (e.g. intersect before commit)*/
#define BG_ERR_OVERFLOW       -5  /* a device-side bound was hit (stack, queue)*/
#define BG_ERR_TIMEOUT        -6  /* a bounded device wait gave up           */
#define BG_ERR_UNSUPPORTED    -7  /* valid in Banshee, not on this path      */
#define BG_ERR_NO_DEVICE      -8  /* no CUDA device / extension not usable   */

/* Device-side error word bits, read with bg_scene_error_flags(). */
#define BG_FLAG_STACK_OVERFLOW 0x1u
#define BG_FLAG_QUEUE_OVERFLOW 0x2u
#define BG_FLAG_BAD_INDEX      0x4u
#define BG_FLAG_TIMEOUT        0x8u

typedef struct bg_ctx bg_ctx;
typedef struct bg_scene bg_scene;

/* -------------------------------------------------------------- rays/hits */
/* 32 bytes: float4(o, tmin), float4(d, tmax).  Mirrors class ray
 * (math/ray.h:42-62): o, d and the interval t = (tmin, tmax).  Arrays must be
 * 16-byte aligned. */
typedef struct bg_ray {
    float o[3];
    float tmin;
    float d[3];
    float tmax;
} bg_ray;

/* 16 bytes.  primid is the global triangle index (faces numbered mesh by mesh
 * in the order meshes were added), -1 on a miss; (u, v) are the Moller-Trumbore
 * barycentrics (b1, b2) of mesh.cpp:20-26, t the hit distance.  Banshee's Hit
 * (primitive/shapebundle.h:156-176) carries no primitive id; the shading
 * fields it does carry are recomputed from (primid, u, v) by the shade stage. */
typedef struct bg_hit {
    float t;
    int32_t primid;
    float u;
    float v;
} bg_hit;

/* ------------------------------------------------------------------ scene */
/* Mirrors the Mesh constructor (primitive/mesh.h:69-76, mesh.cpp:126-214):
 * separately indexed vertices/normals/uvs with byte strides (0 = packed for
 * vertex, normal, uv and the three index arrays) and one material index per
 * face.  As in mesh.cpp:212, mstride is NOT defaulted: 0 makes every face read
 * materials[0].  uvs may be NULL (all uvs (0,0), mesh.cpp:165-181).  m/minv is
 * the row-major bundle transform of ShapeBundle::SetTransform. */
typedef struct bg_mesh_desc {
    const float*   vertices; int32_t nvertices; int32_t vstride;
    const float*   normals;  int32_t nnormals;  int32_t nstride;
    const float*   uvs;      int32_t nuvs;      int32_t ustride;
    const int32_t* vidx;     int32_t vistride;
    const int32_t* nidx;     int32_t nistride;
    const int32_t* uidx;     int32_t uistride;
    const int32_t* materials; int32_t mstride;
    int32_t nfaces;
    float m[16];
    float minv[16];
} bg_mesh_desc;

enum {
    BG_MAT_LAMBERT        = 0, /* SimpleMaterial(Lambert(kd))          bsdf/lambert.h       */
    BG_MAT_MICROFACET_GGX = 1, /* SimpleMaterial(Microfacet(eta, ks, FresnelDielectric,
                                  GgxDistribution(roughness)))       bsdf/microfacet.h    */
    BG_MAT_EMISSIVE       = 2  /* Emissive(e)                         material/emissive.h  */
};

typedef struct bg_material_desc {
    int32_t type;
    float kd[3];
    float ks[3];
    float eta;
    float roughness;
    float e[3];
} bg_material_desc;

enum {
    BG_LIGHT_AREA        = 0, /* AreaLight(face, mesh, material of that face) light/arealight.cpp:11 */
    BG_LIGHT_DIRECTIONAL = 1, /* DirectionalLight(d, e)      light/directional_light.h:42        */
    BG_LIGHT_ENVIRONMENT = 2  /* EnvironmentLight over a constant texture e, (scale, gamma)
                                 light/environment_light.h:45                                   */
};

typedef struct bg_light_desc {
    int32_t type;
    int32_t mesh;   /* area: mesh index        */
    int32_t face;   /* area: face within mesh  */
    float d[3];     /* directional: direction  */
    float e[3];     /* directional: radiance; environment: constant texel */
    float scale;    /* environment: radiance scale */
    float gamma;    /* environment: gamma applied as pow(texel, 1/gamma) */
} bg_light_desc;

/* PerscpectiveCamera(eye, at, up, zcap=(znear,zfar), fovy, aspect),
 * camera/perspective_camera.cpp:5-23.  As in the reference, "fovy" sets the
 * image-plane WIDTH: dim.x = 2 tan(fovy/2) znear, dim.y = dim.x / aspect. */
typedef struct bg_camera_desc {
    float eye[3];
    float at[3];
    float up[3];
    float znear, zfar;
    float fovy;
    float aspect;
} bg_camera_desc;

typedef struct bg_build_opts {
    int32_t node_width;     /* BVH layout: 4 (128-byte nodes), 8 (96-byte
                               compressed nodes) or 0 = build both, the
                               active one switchable (bg_scene_set_node_width) */
    int32_t max_leaf_size;  /* triangles per leaf, 1..16 (0 = default 4)*/
    int32_t sah_bins;       /* binned-SAH bins (0 = default 32)         */
    int32_t builder;        /* 0 = host binned SAH; 1 = device LBVH
                               (Morton order, faster build, looser tree);
                               2 = device PLOC (nearest-neighbour
                               clustering over the Morton order, radius 16);
                               3 = device binned SAH (top-down, 32 bins) */
    int32_t intersect;      /* ray / triangle test of every cast and render:
                               BG_INTERSECT_REFERENCE (0) = Moller-Trumbore in
                               the reference's operation order (primitive/
                               mesh.cpp:7-45): hits bit-exact with Bvh::Intersect;
                               BG_INTERSECT_WATERTIGHT (1) = watertight test
                               (Woop, Benthin and Wald 2013): no ray passes
                               between triangles that share an edge or a
                               vertex; not in the reference, hits differ from
                               Moller-Trumbore only at edges */
} bg_build_opts;

#define BG_INTERSECT_REFERENCE  0
#define BG_INTERSECT_WATERTIGHT 1

typedef struct bg_scene_info {
    int64_t ntriangles;
    int64_t nnodes;
    int64_t node_bytes;     /* device bytes of the node array            */
    int64_t tri_bytes;      /* device bytes of the traversal triangles   */
    int64_t shade_bytes;    /* device bytes of the shading records       */
    int32_t node_stride;    /* bytes per node                             */
    int32_t max_depth;      /* deepest node level                         */
    int32_t max_stack;      /* traversal stack entries a ray may need     */
    int32_t nmeshes;
    int32_t nmaterials;
    int32_t nlights;
    double  build_ms;       /* whole commit (wall time)                   */
    int32_t node_width;     /* active node layout: 4 or 8                  */
    int32_t node_widths;    /* layouts built: 4 | 8                        */
    double  bvh_ms;         /* of build_ms: world boxes, tree build and
                               wide collapses                             */
    double  records_ms;     /*   triangle / shading records (device)      */
    double  upload_ms;      /*   validation and mesh-array upload         */
} bg_scene_info;

/* ---------------------------------------------------------------- tracing */
enum {
    BG_TRACER_GI = 0,       /* GiTracer(maxdepth), tracer/gitracer.cpp    */
    BG_TRACER_DI = 1,       /* DiTracer, tracer/ditracer.cpp:19-55        */
    BG_TRACER_AO = 2        /* AoTracer(radius), tracer/aotracer.cpp:9-49 */
};

#define BG_RENDER_TIME_PHASES   0x1  /* per-phase CUDA-event timing into bg_render_stats */
#define BG_RENDER_COUNT_TRAVERSAL 0x2 /* instrumented replay of every 64th traced ray    */

typedef struct bg_tracer_desc {
    int32_t kind;
    int32_t maxdepth;
    int32_t flags;          /* BG_RENDER_* instrumentation bits (0 = none)   */
    float ao_radius;        /* BG_TRACER_AO: occlusion radius (AoTracer ctor) */
} bg_tracer_desc;

/* Sampler plugin: every camera sample (pixel p, sample index s) gets fresh
 * RandomSampler(McRng) image, light and BSDF samplers
 * (sampler/random_sampler.h:48-80, rng/mcrng.h:45-76) whose McRng seeds, and
 * the global rand() draws of GiTracer (light pick, Russian roulette,
 * gitracer.cpp:75,119), come from a counter-keyed generator:
 *   rand() = splitmix64(k ^ (counter * 0xD1B54A32D192ED03)) >> 33,
 *   k = splitmix64(seed ^ splitmix64(p << 32 | s)),
 * counter = 0, 1, 2, ... within that camera sample.  This is the determinism
 * contract shared with the CPU oracle. */
/* Image-sampler kinds.  The light and BSDF samplers are always the keyed
 * RandomSampler(McRng) above; the image (camera) sample of (pixel p, sample s)
 * comes from:
 *   BG_SAMPLER_RANDOM  the keyed RandomSampler(McRng) above;
 *   BG_SAMPLER_SOBOL   SobolSampler (sampler/sobol_sampler.cpp:3-49): point s
 *                      of the pixel's scrambled (0,2) sequence, scrambles =
 *                      the first two NextUint of a McRng seeded by the keyed
 *                      rand() of (p, 0xFFFFFFFF);
 *   BG_SAMPLER_CMJ     CmjSampler(grid) (sampler/cmj_sampler.cpp:3-73): sample
 *                      s mod grid^2 of pattern j = s / grid^2, the pattern
 *                      index being the first NextUint of a McRng seeded by
 *                      the keyed rand() of (p, 0x80000000 + j).
 * Sample indices s must stay below 2^31. */
enum {
    BG_SAMPLER_RANDOM = 0,
    BG_SAMPLER_SOBOL = 1,
    BG_SAMPLER_CMJ = 2
};

typedef struct bg_sampler_desc {
    int32_t kind;           /* BG_SAMPLER_* image sampler                 */
    int32_t spp;            /* camera samples per pixel in this call      */
    uint64_t seed;
    int32_t sample_offset;  /* index of the first sample of this call     */
    int32_t grid;           /* BG_SAMPLER_CMJ: grid size (1..16)          */
} bg_sampler_desc;

typedef struct bg_render_stats {
    int64_t camera_samples;
    int64_t rays_extension; /* extension (camera + bounce) closest-hit rays */
    int64_t rays_closest;   /* extension + MIS closest-hit rays           */
    int64_t rays_any;       /* shadow rays                                */
    int64_t kernel_launches;/* library kernels launched by the call       */
    float   ms_total;
    float   ms_extend;      /* extension closest-hit traversal            */
    float   ms_mis;         /* MIS closest-hit traversal                  */
    float   ms_shadow;      /* any-hit traversal                          */
    float   ms_shade;       /* generate + shade + resolve + accumulate    */
    int32_t launches_extend;/* extension traversal launches               */
    float   ms_cache_query; /* radiance cache: encode + inference + resolve */
    float   ms_cache_train; /* radiance cache: training steps             */
    /* BG_RENDER_COUNT_TRAVERSAL: replay of every 64th ray of each queue:
     * rays replayed, nodes fetched, triangles tested                      */
    int64_t sub_rays_extension, sub_nodes_extension, sub_tris_extension;
    int64_t sub_rays_any, sub_nodes_any, sub_tris_any;
    int64_t sub_rays_mis, sub_nodes_mis, sub_tris_mis;
} bg_render_stats;

/* ------------------------------------------------------------------- API */
const char* bg_last_error(void);
int bg_version(int32_t* major, int32_t* minor);

/* Allocation accounting.  Every device allocation the library makes (scene,
 * tree, wavefront state, cache, build scratch) and its pinned host staging is
 * counted, and may be capped: bg_alloc_limit(bytes) allows `bytes` more bytes
 * from this call on, process-wide (bytes < 0 removes the cap).  An allocation
 * past the cap fails without calling CUDA, exactly as a failed cudaMalloc does:
 * the entry point returns BG_ERR_OOM and keeps no partial state (a scene whose
 * commit failed stays uncommitted and holds no device memory; a render whose
 * path state could not be allocated holds none either).  For out-of-memory
 * tests and for applications that give the library a fixed budget.  No
 * counterpart in the reference. */
typedef struct bg_alloc_stats {
    int64_t calls;          /* allocations made since load                 */
    int64_t bytes;          /* bytes of those allocations                   */
    int64_t refused;        /* allocations refused by the cap               */
    int64_t budget;         /* bytes still allowed, -1 = no cap             */
} bg_alloc_stats;
int bg_alloc_limit(int64_t bytes);
int bg_alloc_stats_get(bg_alloc_stats* out);

int bg_ctx_create(int32_t device, bg_ctx** out);
int bg_ctx_destroy(bg_ctx* ctx);
int bg_ctx_sync(bg_ctx* ctx);

/* World assembly.  Mirrors World::shapebundles_/materials_/lights_/bgcolor_
 * (world/world.h:75-87) and World::Commit (world/world.cpp:5-16). */
int bg_scene_create(bg_ctx* ctx, bg_scene** out);
int bg_scene_destroy(bg_scene* scene);
int bg_scene_add_mesh(bg_scene* scene, const bg_mesh_desc* mesh, int32_t* index);
int bg_scene_add_material(bg_scene* scene, const bg_material_desc* mat, int32_t* index);
int bg_scene_add_light(bg_scene* scene, const bg_light_desc* light, int32_t* index);
int bg_scene_set_background(bg_scene* scene, const float rgb[3]);
int bg_scene_commit(bg_scene* scene, const bg_build_opts* opts);
int bg_scene_info_get(bg_scene* scene, bg_scene_info* info);
int bg_scene_error_flags(bg_scene* scene, uint32_t* flags, int32_t clear);
/* Selects the node layout traversal uses (4 or 8; it must have been built).
 * No counterpart in the reference, whose Bvh has one binary layout. */
int bg_scene_set_node_width(bg_scene* scene, int32_t width);

/* Closest hit: replaces World::Intersect(ray, Hit&) -> Bvh::Intersect
 * (world/world.cpp:19-23, accelerator/bvh.cpp:499-573).  A triangle is
 * accepted when its Moller-Trumbore t lies in (tmin, tmax] (mesh.cpp:33). */
int bg_intersect_closest(bg_scene* scene, const bg_ray* rays_dev, bg_hit* hits_dev,
                         int64_t n, void* stream);
/* Any hit: replaces World::Intersect(ray) -> Bvh::Intersect(ray)
 * (world/world.cpp:26-29, accelerator/bvh.cpp:575-647).  occluded_dev[i] = 1
 * if some triangle has t in (tmin, tmax]. */
int bg_intersect_any(bg_scene* scene, const bg_ray* rays_dev, uint8_t* occluded_dev,
                     int64_t n, void* stream);
int bg_intersect_closest_host(bg_scene* scene, const bg_ray* rays, bg_hit* hits, int64_t n);
int bg_intersect_any_host(bg_scene* scene, const bg_ray* rays, uint8_t* occluded, int64_t n);

/* Instrumented replay of the same traversal: total nodes fetched and
 * triangles tested over the n rays (the per-ray byte model of the roofline).
 * Runs on the scene's device and gives the calling thread's current device
 * back; synchronous on `stream`.  A replay whose traversal stack overflowed
 * returns BG_ERR_OVERFLOW (the counts would be short). */
int bg_traversal_counts(bg_scene* scene, const bg_ray* rays_dev, int64_t n, int32_t any_hit,
                        uint64_t* nodes, uint64_t* triangles, void* stream);
/* Same counts as bg_traversal_counts, for callers that cannot let the library
 * allocate device memory (an application that reserves the device's memory for
 * its own pool; a profiling harness that cudaFree's implicit synchronisation
 * would disturb).  No counterpart in the reference.  Allocates nothing: its
 * scratch is a 16 MiB static device array, held by every GPU that loads the
 * library until exit, so n is limited to 1,048,560 rays for closest hit and
 * 16,776,960 for any hit (larger n returns BG_ERR_INVALID_ARG).  The first
 * call on a device looks up the array's address; make it before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race.
 * Like bg_traversal_counts it runs on the scene's device, gives the calling
 * thread's current device back, is synchronous on `stream` and returns
 * BG_ERR_OVERFLOW when the replay's traversal stack overflowed. */
int bg_traversal_counts_noalloc(bg_scene* scene, const bg_ray* rays_dev, int64_t n, int32_t any_hit,
                                uint64_t* nodes, uint64_t* triangles, void* stream);

/* Renderer::Render for ImageRenderer/MtImageRenderer + the tracer plugin
 * (renderer/imagerenderer.cpp:9-59).  Adds spp samples per pixel into
 * accum_rgbw_dev (width*height float4: rgb sum and sample count in w), rows
 * flipped as FileImagePlane::WriteSample does (imageplane/fileimageplane.cpp:29-34).
 * The caller zeroes the buffer once and may call repeatedly with increasing
 * sample_offset to accumulate progressively.  stats may be NULL. */
int bg_render(bg_scene* scene, const bg_camera_desc* camera, const bg_tracer_desc* tracer,
              const bg_sampler_desc* sampler, int32_t width, int32_t height,
              float* accum_rgbw_dev, bg_render_stats* stats, void* stream);
/* Same, with the accumulation buffer in host memory: it is copied in, the
 * samples are added on the device and the result is copied back. */
int bg_render_host(bg_scene* scene, const bg_camera_desc* camera, const bg_tracer_desc* tracer,
                   const bg_sampler_desc* sampler, int32_t width, int32_t height,
                   float* accum_rgbw, bg_render_stats* stats);

/* ----------------------------------------------------- multi-scene batch */
/* Many independent scenes, cameras, resolutions and sample counts traced
 * together: the committed scenes are merged into one device scene, and every
 * job's camera samples share the same wavefront queues, persistent kernels and
 * per-pass CUDA graph.  No counterpart in the reference (one World per
 * Renderer::Render call, renderer/renderer.h:49).  Each job's image is
 * bit-identical to rendering its scene alone with the same sampler. */
typedef struct bg_batch bg_batch;

typedef struct bg_batch_job {
    int32_t scene;             /* index from bg_batch_add_scene              */
    int32_t width, height;
    int32_t reserved;
    bg_camera_desc camera;
    bg_sampler_desc sampler;   /* spp, seed, sample_offset                   */
    float* accum_rgbw_dev;     /* width*height float4, as bg_render          */
} bg_batch_job;

typedef struct bg_tune_result {
    int32_t trace_threads;     /* traversal block size chosen                */
    int32_t paths_per_pass;    /* wavefront size chosen                      */
    int32_t candidates;        /* configurations timed                       */
    float ms;                  /* time of the best probe render              */
    float msamples_per_s;      /* its throughput                             */
    int32_t node_width;        /* node layout chosen (4 or 8)                */
} bg_tune_result;

int bg_batch_create(bg_ctx* ctx, bg_batch** out);
/* The scene must be committed; its device data is copied at bg_batch_commit,
 * after which the scene may be destroyed. */
int bg_batch_add_scene(bg_batch* batch, bg_scene* scene, int32_t* index);
int bg_batch_commit(bg_batch* batch);
int bg_batch_info(bg_batch* batch, bg_scene_info* info);
int bg_batch_render(bg_batch* batch, const bg_batch_job* jobs, int32_t njobs, const bg_tracer_desc* tracer,
                    bg_render_stats* stats, void* stream);
/* Times node layouts {4-wide, 8-wide compressed} (those every scene built) x
 * traversal block sizes {128, 256} x paths per pass {2^19 .. 2^24} on
 * the jobs with spp capped at probe_spp and keeps the fastest for later
 * bg_batch_render calls.  A pass size is skipped when the probe's samples fit
 * in half of it (it would run the same passes as the size before), and the
 * sizes end at the first one whose buffers do not fit in device memory.
 * result->candidates counts the configurations timed.  The jobs'
 * accumulation buffers receive the probe samples: clear them before the real
 * render.  Synchronises. */
int bg_batch_autotune(bg_batch* batch, const bg_batch_job* jobs, int32_t njobs, const bg_tracer_desc* tracer,
                      int32_t probe_spp, bg_tune_result* result, void* stream);
int bg_batch_destroy(bg_batch* batch);
/* Autotuner for one scene and camera: the same candidates as
 * bg_batch_autotune, each probed with probe_spp samples per pixel rendered
 * into accum_rgbw_dev (clear it before the real render); the fastest is kept
 * for later bg_render / bg_render_host calls of this scene.  Passes are sized
 * for the probe: calls with more samples than probe_spp use the same pass
 * size.  The path state and queues of a pass stay allocated with the scene,
 * about 1.2 KB per path with 2 lights (20 GB at 2^24 paths).  No counterpart
 * in the reference.  Synchronises. */
int bg_scene_autotune(bg_scene* scene, const bg_camera_desc* camera, const bg_tracer_desc* tracer,
                      int32_t probe_spp, int32_t width, int32_t height, float* accum_rgbw_dev,
                      bg_tune_result* result, void* stream);

/* ------------------------------------------------------------ images */
/* FileImagePlane::Finalize (imageplane/fileimageplane.cpp:13-27): rgb[i] =
 * (sum / samples)^(1/2.2) per channel of the W*H RGBW accumulation buffer
 * (rows bottom-up, as WriteSample stores them).  Host buffers. */
int bg_image_finalize(const float* rgbw, int32_t width, int32_t height, float* rgb);
/* Finalize + write, replacing OiioImageIo::Write (imageio/oiioimageio.cpp:
 * 40-56) for headless use: ".ppm" = 8-bit (clamped to [0,1], rounded), ".pfm"
 * = 32-bit float.  Host buffer. */
int bg_image_write(const char* path, const float* rgbw, int32_t width, int32_t height);

/* ------------------------------------------------------ radiance cache */
/* Neural radiance cache.  No counterpart in the reference: Banshee has no
 * learned component.  A hash-grid + one-blob encoded, 64-wide, 5-hidden-layer
 * BF16 MLP (fp32 accumulation) predicts the outgoing radiance at a path
 * vertex; it is trained online (Adam, relative L2 loss) on radiance that
 * training paths of the tracer itself produce, and rendering paths end into it
 * after cache_depth bounces (bg_render_cached). */
typedef struct bg_cache bg_cache;

typedef struct bg_cache_desc {
    int32_t levels;            /* hash-grid levels: 16 (0 = 16)                */
    int32_t log2_table_size;   /* entries per level = 2^this (19 in C5)        */
    int32_t base_resolution;   /* coarsest grid resolution (16)                */
    int32_t max_resolution;    /* finest grid resolution (2048)                */
    int32_t train_paths;       /* training paths per frame (65536)             */
    int32_t cache_depth;       /* rendering paths end into the cache here (2)  */
    int32_t train_batch;       /* rows per Adam step (16384)                   */
    int32_t train_steps;       /* Adam steps per frame at most (4)             */
    float learning_rate;       /* Adam learning rate (1e-2)                    */
    float bbox_min[3];         /* position normalisation; all zero = scene     */
    float bbox_max[3];         /* bounds                                       */
    uint64_t seed;             /* parameter initialisation                     */
    int32_t mlp_kernel;        /* inference and training: 0 = tcgen05 (TMEM
                                  accumulators), 1 = mma.sync (registers)      */
    int32_t train_suffix;      /* 0: training paths run to maxdepth (unbiased
                                  targets); k > 0: they end into the cache k
                                  bounces after cache_depth (self-training, the
                                  pass stops there)                             */
    int32_t wait_polls;        /* mlp_kernel 0: polls of each bounded mbarrier
                                  wait before the kernel gives up, raises
                                  BG_FLAG_TIMEOUT and returns (0 = 2^24).  A
                                  budget of 1 makes every wait give up at once:
                                  a test of the timeout path.                   */
} bg_cache_desc;

/* Query record: 16 floats per row = position (3), outgoing direction (3),
 * shading normal (3), roughness, albedo (3), 3 unused.  Outputs / targets are
 * 4 floats per row (rgb, unused). */
int bg_cache_create(bg_scene* scene, const bg_cache_desc* desc, bg_cache** out);
int bg_cache_destroy(bg_cache* cache);
/* resolutions: 16 ints; norm6: position normalisation u = (p - norm6[0:3]) * norm6[3:6]. */
int bg_cache_info(bg_cache* cache, int32_t* nparams_mlp, int64_t* nparams_grid, int32_t* resolutions, float* norm6);
int bg_cache_query(bg_cache* cache, const float* features_dev, float* out_rgba_dev, int64_t n, void* stream);
/* One training step on n rows: loss, gradients and (apply != 0) an Adam
 * update.  loss (may be NULL) receives the mean relative L2 loss; passing it
 * synchronises. */
int bg_cache_train(bg_cache* cache, const float* features_dev, const float* target_rgba_dev, int64_t n,
                   int32_t apply, float* loss, void* stream);
/* Host copies of the fp32 parameters / last gradients (any may be NULL):
 * MLP packed as [64][128], 4 x [64][64], [16][64] row-major ([out][in]);
 * grid as [levels][2^log2_table_size][2]. */
int bg_cache_params(bg_cache* cache, float* mlp, float* grid, float* mlp_grad, float* grid_grad);
int bg_cache_set_params(bg_cache* cache, const float* mlp, const float* grid);
/* Renders like bg_render with GiTracer(tracer->maxdepth), except that
 * rendering paths end into the cache at vertex desc.cache_depth, and
 * desc.train_paths paths per call are traced in full and train the cache
 * (desc.train_steps Adam steps) after the frame: at the start of the cache's
 * next call, beside its first bounces.  When calls of several caches of one
 * scene interleave, a call that finds another cache's rows pending trains
 * them into that cache first (synchronously), so every cache trains on each
 * of its frames once; destroying a cache drops its pending rows. */
int bg_render_cached(bg_scene* scene, bg_cache* cache, const bg_camera_desc* camera, const bg_tracer_desc* tracer,
                     const bg_sampler_desc* sampler, int32_t width, int32_t height, float* accum_rgbw_dev,
                     bg_render_stats* stats, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BANSHEE_GPU_H */
