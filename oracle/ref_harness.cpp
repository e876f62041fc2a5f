/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives Banshee's own, unmodified C++ (compiled from the reference tree by
 * oracle/Makefile into oracle/_ref/libbanshee_ref.so) through its public
 * plugin surfaces, to pin the CPU restatement and to time the reference CPU
 * tracer.  Only the pieces the reference leaves to its host application are
 * written here:
 *   - a constant TextureSystem (texture/texturesystem.h:56) so that
 *     EnvironmentLight reads a constant texel (OpenImageIO is absent);
 *   - an ImagePlane with FileImagePlane's accumulation
 *     (imageplane/fileimageplane.cpp:29-34) into a caller buffer;
 *   - a Renderer (renderer/renderer.h:49) with ImageRenderer's per-sample body
 *     (renderer/imagerenderer.cpp:25-43) that keys the global rand() and seeds
 *     fresh RandomSampler(McRng) samplers per camera sample (the determinism
 *     contract documented in include/banshee_gpu.h);
 *   - rand(), interposed (the .so is linked -Bsymbolic), so that
 *     rand_float/rand_uint (math/mathutils.h:62-65) and the McRng seeds
 *     (rng/mcrng.h:48-51) draw from the keyed generator.
 * World assembly mirrors World's public fields (world/world.h:75-87) and the
 * Mesh / AreaLight constructors.  For ray casting the world is built with
 * per-face material index = global triangle id and per-face uvs
 * (0,0),(1,0),(0,1), so that Hit::m is the primitive id and Hit::uv the
 * Moller-Trumbore barycentrics (primitive/mesh.cpp:94-95).
 */
#include <atomic>
#include <functional>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "world/world.h"
#include "primitive/mesh.h"
#include "material/simplematerial.h"
#include "material/emissive.h"
#include "bsdf/lambert.h"
#include "bsdf/microfacet.h"
#include "bsdf/fresnel.h"
#include "bsdf/microfacet_distribution.h"
#include "light/arealight.h"
#include "light/directional_light.h"
#include "light/environment_light.h"
#include "camera/perspective_camera.h"
#include "tracer/gitracer.h"
#include "tracer/ditracer.h"
#ifdef BANSHEE_GPU_ADAPTER
#include "adapters/gpu_accelerator.h"
#include "adapters/gpu_renderer.h"
#include "adapters/world_scene.h"
#endif
#include "tracer/aotracer.h"
#include "sampler/sobol_sampler.h"
#include "sampler/cmj_sampler.h"
#include "sampler/random_sampler.h"
#include "rng/mcrng.h"
#include "renderer/renderer.h"
#include "imageplane/imageplane.h"
#include "texture/texturesystem.h"

#include "../include/banshee_gpu.h"

/* ----------------------------------------------------------- keyed rand */
namespace {
struct KeyState {
    uint64_t key = 0;
    uint32_t counter = 0;
};
thread_local KeyState g_key;

inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
void set_key(uint64_t seed, uint32_t pixel, uint32_t sample) {
    g_key.key = splitmix64(seed ^ splitmix64((static_cast<uint64_t>(pixel) << 32) | sample));
    g_key.counter = 0;
}
}  // namespace

extern "C" int rand(void) {
    uint64_t c = g_key.counter++;
    return static_cast<int>(splitmix64(g_key.key ^ (c * 0xD1B54A32D192ED03ull)) >> 33);
}

/* ------------------------------------------------------------ plugins */
namespace {
class ConstTextureSystem : public TextureSystem {
public:
    float3 Sample(std::string const& name, float2 const&, float2 const&, Options const&) const override {
        auto it = values_.find(name);
        return it == values_.end() ? float3(0, 0, 0) : it->second;
    }
    void GetTextureInfo(std::string const&, TextureDesc& d) const override { d.width = 1; d.height = 1; }
    std::map<std::string, float3> values_;
};

class BufferImagePlane : public ImagePlane {
public:
    BufferImagePlane(int w, int h, float* buf) : ImagePlane(int2(w, h), nullptr), buf_(buf) {}
protected:
    void WriteSample(int2 const& pos, float3 const& value) override {
        int2 res = resolution();
        float* px = buf_ + 4 * (static_cast<size_t>(res.x) * (res.y - 1 - pos.y) + pos.x);
        px[0] += value.x; px[1] += value.y; px[2] += value.z; px[3] += 1.f;
    }
private:
    float* buf_;
};

// Rng whose NextUint is the first NextUint of a McRng seeded under a fixed
// key: the CMJ pattern index of pattern j of a pixel (the sampler contract).
class PatternRng : public Rng {
public:
    PatternRng(uint64_t seed, uint32_t pixel, uint32_t j) : seed_(seed), pixel_(pixel), j_(j) {}
    float NextFloat() const override { return NextUint() * 2.328306e-10f; }
    unsigned NextUint() const override {
        set_key(seed_, pixel_, 0x80000000u + j_);
        McRng m;
        return m.NextUint();
    }
    Rng* Clone() const override { return new PatternRng(seed_, pixel_, j_); }
private:
    uint64_t seed_;
    uint32_t pixel_, j_;
};

class KeyedRenderer : public Renderer {
public:
    KeyedRenderer(ImagePlane& plane, Tracer const& tracer, uint64_t seed, int spp, int soff,
                  int x0, int y0, int x1, int y1, int nthreads, int skind = BG_SAMPLER_RANDOM, int grid = 0)
        : plane_(plane), tracer_(tracer), seed_(seed), spp_(spp), soff_(soff),
          x0_(x0), y0_(y0), x1_(x1), y1_(y1), nthreads_(nthreads), skind_(skind), grid_(grid) {}

    void Render(World const& world) const override {
        int nt = nthreads_ > 0 ? nthreads_ : static_cast<int>(std::thread::hardware_concurrency());
        if (nt < 1) nt = 1;
        std::atomic<int> next(y0_);
        auto work = [&]() {
            for (;;) {
                int y = next++;
                if (y >= y1_) break;
                RenderRow(world, y);
            }
        };
        std::vector<std::thread> th;
        for (int i = 1; i < nt; ++i) th.emplace_back(work);
        work();
        for (auto& t : th) t.join();
    }

private:
    void RenderRow(World const& world, int y) const {
        int2 imgres = plane_.resolution();
        Camera const& cam(*world.camera_.get());
        for (int x = x0_; x < x1_; ++x) {
            const uint32_t pixel = static_cast<uint32_t>(y * imgres.x + x);
            // Sobol: one sampler per pixel, scrambled from the key (pixel, 0xFFFFFFFF),
            // advanced to the first sample index of this call
            std::unique_ptr<SobolSampler> sobol;
            if (skind_ == BG_SAMPLER_SOBOL) {
                set_key(seed_, pixel, 0xFFFFFFFFu);
                sobol.reset(new SobolSampler(1, new McRng()));
                for (int k = 0; k < soff_; ++k) sobol->Sample2D();
            }
            for (int s = 0; s < spp_; ++s) {
                const uint32_t si = static_cast<uint32_t>(soff_ + s);
                float2 cmj;
                if (skind_ == BG_SAMPLER_CMJ) {
                    const uint32_t g2 = static_cast<uint32_t>(grid_ * grid_);
                    CmjSampler c(grid_, new PatternRng(seed_, pixel, si / g2));
                    for (uint32_t k = 0; k <= si % g2; ++k) cmj = c.Sample2D();
                }
                set_key(seed_, pixel, si);
                RandomSampler imgsampler(1, new McRng());
                RandomSampler lightsampler(1, new McRng());
                RandomSampler brdfsampler(1, new McRng());
                float2 sample = imgsampler.Sample2D();
                if (skind_ == BG_SAMPLER_SOBOL) sample = sobol->Sample2D();
                if (skind_ == BG_SAMPLER_CMJ) sample = cmj;
                float2 imgsample((float)x / imgres.x + (1.f / imgres.x) * sample.x,
                                 (float)y / imgres.y + (1.f / imgres.y) * sample.y);
                ray r;
                cam.GenerateRay(imgsample, r);
                plane_.AddSample(int2(x, y), tracer_.GetLi(r, world, lightsampler, brdfsampler));
            }
        }
    }

    ImagePlane& plane_;
    Tracer const& tracer_;
    uint64_t seed_;
    int spp_, soff_, x0_, y0_, x1_, y1_, nthreads_, skind_, grid_;
};

matrix mat_from(const float* a) {
    return matrix(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7],
                  a[8], a[9], a[10], a[11], a[12], a[13], a[14], a[15]);
}

struct RefWorld {
    World world;
    ConstTextureSystem texsys;
    int64_t ntris = 0;
};
}  // namespace

extern "C" {

/* raycast != 0: per-face material = global triangle id, per-face uvs = the
 * barycentric frame; materials and lights are ignored. */
void* ref_world_create(const bg_mesh_desc* meshes, int32_t nmeshes,
                       const bg_material_desc* mats, int32_t nmats,
                       const bg_light_desc* lights, int32_t nlights,
                       const float* bgcolor, int32_t raycast) {
    RefWorld* rw = new RefWorld();
    try {
        int64_t base = 0;
        static const float bary_uv[6] = {0.f, 0.f, 1.f, 0.f, 0.f, 1.f};
        for (int i = 0; i < nmeshes; ++i) {
            const bg_mesh_desc& d = meshes[i];
            Mesh* m;
            if (raycast) {
                std::vector<int> ids(d.nfaces), uidx(3 * static_cast<size_t>(d.nfaces));
                for (int f = 0; f < d.nfaces; ++f) {
                    ids[f] = static_cast<int>(base + f);
                    uidx[3 * f] = 0; uidx[3 * f + 1] = 1; uidx[3 * f + 2] = 2;
                }
                m = new Mesh(d.vertices, d.nvertices, d.vstride, d.normals, d.nnormals, d.nstride,
                             bary_uv, 3, 0, d.vidx, d.vistride, d.nidx, d.nistride,
                             uidx.data(), 0, ids.data(), sizeof(int), d.nfaces);
            } else {
                m = new Mesh(d.vertices, d.nvertices, d.vstride, d.normals, d.nnormals, d.nstride,
                             d.uvs, d.nuvs, d.ustride, d.vidx, d.vistride, d.nidx, d.nistride,
                             d.uidx, d.uistride, d.materials, d.mstride, d.nfaces);
            }
            m->SetTransform(mat_from(d.m), mat_from(d.minv));
            rw->world.shapebundles_.push_back(std::unique_ptr<ShapeBundle>(m));
            base += d.nfaces;
        }
        rw->ntris = base;
        if (!raycast) {
            for (int i = 0; i < nmats; ++i) {
                const bg_material_desc& md = mats[i];
                Material* mat = nullptr;
                if (md.type == BG_MAT_LAMBERT) {
                    mat = new SimpleMaterial(new Lambert(rw->texsys, float3(md.kd[0], md.kd[1], md.kd[2])));
                } else if (md.type == BG_MAT_MICROFACET_GGX) {
                    mat = new SimpleMaterial(new Microfacet(rw->texsys, md.eta, float3(md.ks[0], md.ks[1], md.ks[2]),
                                                            "", "", new FresnelDielectric(),
                                                            new GgxDistribution(md.roughness)));
                } else {
                    mat = new Emissive(float3(md.e[0], md.e[1], md.e[2]));
                }
                rw->world.materials_.push_back(std::unique_ptr<Material>(mat));
            }
            for (int i = 0; i < nlights; ++i) {
                const bg_light_desc& ld = lights[i];
                Light* l = nullptr;
                if (ld.type == BG_LIGHT_AREA) {
                    Mesh* mesh = static_cast<Mesh*>(rw->world.shapebundles_[ld.mesh].get());
                    int mi = mesh->GetFaces()[ld.face].m;
                    l = new AreaLight(ld.face, *mesh, *rw->world.materials_[mi]);
                } else if (ld.type == BG_LIGHT_DIRECTIONAL) {
                    l = new DirectionalLight(float3(ld.d[0], ld.d[1], ld.d[2]), float3(ld.e[0], ld.e[1], ld.e[2]));
                } else {
                    std::string name = "const" + std::to_string(i);
                    rw->texsys.values_[name] = float3(ld.e[0], ld.e[1], ld.e[2]);
                    l = new EnvironmentLight(rw->texsys, name, ld.scale, ld.gamma);
                }
                rw->world.lights_.push_back(std::unique_ptr<Light>(l));
            }
            if (bgcolor) rw->world.bgcolor_ = float3(bgcolor[0], bgcolor[1], bgcolor[2]);
        }
        rw->world.Commit();
    } catch (...) {
        delete rw;
        return nullptr;
    }
    return rw;
}

void ref_world_destroy(void* w) { delete static_cast<RefWorld*>(w); }

#ifdef BANSHEE_GPU_ADAPTER
/* Replaces the committed World's Bvh by the B200 library's scene through the
 * GpuAccelerator adapter (the drop-in the integration guide describes). */
int ref_world_use_gpu(void* w, void* gpu_scene) {
    RefWorld* rw = static_cast<RefWorld*>(w);
    try {
        rw->world.accel_.reset(new GpuAccelerator(rw->world, static_cast<bg_scene*>(gpu_scene)));
    } catch (...) {
        return -1;
    }
    return 0;
}

/* Builds the device scene from the committed World itself
 * (gpu_scene_from_world: the bundles' public accessors) and installs
 * GpuAccelerator over it.  *scene_out receives that scene; the caller destroys
 * it (bg_scene_destroy) after the world. */
int ref_world_use_gpu_world(void* w, void* gpu_ctx, void** scene_out) {
    RefWorld* rw = static_cast<RefWorld*>(w);
    try {
        bg_scene* s = gpu_scene_from_world(static_cast<bg_ctx*>(gpu_ctx), rw->world);
        *scene_out = s;
        rw->world.accel_.reset(new GpuAccelerator(rw->world, s));
    } catch (...) {
        return -1;
    }
    return 0;
}

/* Renders `frames` progressive frames of spp samples each through the
 * GpuRenderer adapter (Renderer::Render) into accum_rgbw. */
int ref_gpu_renderer(void* w, void* gpu_scene, const bg_camera_desc* c, int32_t tracer_kind, int32_t maxdepth,
                     int32_t width, int32_t height, int32_t spp, int32_t frames, uint64_t seed, float* accum_rgbw) {
    RefWorld* rw = static_cast<RefWorld*>(w);
    bg_tracer_desc t = {tracer_kind, maxdepth, 0, 0.f};
    bg_sampler_desc smp = {BG_SAMPLER_RANDOM, spp, seed, 0, 0};
    try {
        GpuRenderer r(static_cast<bg_scene*>(gpu_scene), *c, t, smp, width, height, accum_rgbw);
        for (int f = 0; f < frames; ++f) r.Render(rw->world);
    } catch (...) {
        return -1;
    }
    return 0;
}
#endif

static void parallel_rays(int64_t n, int nthreads, const std::function<void(int64_t)>& fn) {
    int nt = nthreads > 0 ? nthreads : static_cast<int>(std::thread::hardware_concurrency());
    if (nt < 1) nt = 1;
    std::atomic<int64_t> next(0);
    const int64_t chunk = 1024;
    auto work = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            int64_t e = b + chunk < n ? b + chunk : n;
            for (int64_t i = b; i < e; ++i) fn(i);
        }
    };
    std::vector<std::thread> th;
    for (int i = 1; i < nt; ++i) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

void ref_intersect_closest(void* w, const bg_ray* rays, bg_hit* hits, int64_t n, int32_t nthreads) {
    World const& world = static_cast<RefWorld*>(w)->world;
    parallel_rays(n, nthreads, [&](int64_t i) {
        const bg_ray& q = rays[i];
        ray r(float3(q.o[0], q.o[1], q.o[2]), float3(q.d[0], q.d[1], q.d[2]), float2(q.tmin, q.tmax));
        ShapeBundle::Hit hit;
        bool b = world.Intersect(r, hit);
        hits[i].t = b ? hit.t : q.tmax;
        hits[i].primid = b ? hit.m : -1;
        hits[i].u = b ? hit.uv.x : 0.f;
        hits[i].v = b ? hit.uv.y : 0.f;
    });
}

void ref_intersect_any(void* w, const bg_ray* rays, uint8_t* occ, int64_t n, int32_t nthreads) {
    World const& world = static_cast<RefWorld*>(w)->world;
    parallel_rays(n, nthreads, [&](int64_t i) {
        const bg_ray& q = rays[i];
        ray r(float3(q.o[0], q.o[1], q.o[2]), float3(q.d[0], q.d[1], q.d[2]), float2(q.tmin, q.tmax));
        occ[i] = world.Intersect(r) ? 1 : 0;
    });
}

void ref_render(void* w, const bg_camera_desc* c, int32_t tracer_kind, int32_t maxdepth,
                int32_t width, int32_t height, int32_t spp, int32_t sample_offset, uint64_t seed,
                float* accum_rgbw, int32_t x0, int32_t y0, int32_t x1, int32_t y1, int32_t nthreads,
                int32_t sampler_kind, int32_t sampler_grid, float ao_radius) {
    RefWorld* rw = static_cast<RefWorld*>(w);
    rw->world.camera_.reset(new PerscpectiveCamera(float3(c->eye[0], c->eye[1], c->eye[2]),
                                                   float3(c->at[0], c->at[1], c->at[2]),
                                                   float3(c->up[0], c->up[1], c->up[2]),
                                                   float2(c->znear, c->zfar), c->fovy, c->aspect));
    BufferImagePlane plane(width, height, accum_rgbw);
    std::unique_ptr<Tracer> tracer;
    if (tracer_kind == BG_TRACER_DI) tracer.reset(new DiTracer());
    else if (tracer_kind == BG_TRACER_AO) tracer.reset(new AoTracer(ao_radius));
    else tracer.reset(new GiTracer(maxdepth));
    KeyedRenderer renderer(plane, *tracer, seed, spp, sample_offset, x0, y0, x1, y1, nthreads, sampler_kind,
                           sampler_grid);
    renderer.Render(rw->world);
}

/* McRng draws under a key, to check the interposed rand() is the one used. */
void ref_mcrng_draws(uint64_t seed, uint32_t pixel, uint32_t sample, int32_t n, float* out) {
    set_key(seed, pixel, sample);
    RandomSampler s(1, new McRng());
    for (int i = 0; i < n; ++i) {
        float2 v = s.Sample2D();
        out[2 * i] = v.x;
        out[2 * i + 1] = v.y;
    }
}

int64_t ref_world_ntriangles(void* w) { return static_cast<RefWorld*>(w)->ntris; }

}  // extern "C"
