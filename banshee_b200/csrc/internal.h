// Host-side library internals shared by the API and render translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/banshee_gpu.h"
#include "device_common.cuh"
#include "scene_types.h"

namespace bg {

int set_error(int code, const char* fmt, ...);

#define BG_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::bg::set_error(e_ == cudaErrorMemoryAllocation ? BG_ERR_OOM : BG_ERR_CUDA, \
                                   "%s failed: %s", #call, cudaGetErrorString(e_));      \
    } while (0)

struct MeshHost {
    std::vector<v3> verts, normals;
    std::vector<float> uvs;              // 2 per uv
    std::vector<int32_t> vi, ni, ti, m;  // 3, 3, 3, 1 per face
    float xf[16], xfinv[16];
    int nfaces = 0;
};

// Charges an allocation against the library's optional cap (bg_alloc_limit)
// and counts it; false = refused (report BG_ERR_OOM without calling CUDA).
bool alloc_charge(size_t bytes);

// Device buffer that grows on demand (never shrinks until freed).
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Scratch of one synchronous call (a commit's build buffers): drawn from a
// per-device memory pool on the legacy default stream, so repeated commits
// reuse memory instead of calling cudaMalloc / cudaFree each time.  Every use
// must be on the legacy stream; the pool keeps up to kScratchKeepBytes.
struct ScratchBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
    ~ScratchBuf() { release(); }
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};
constexpr size_t kScratchKeepBytes = size_t(4) << 30;

// Makes `device` current for the lifetime of the guard and gives the caller's
// current device back afterwards (entry points that must run on the scene's
// device whatever the calling thread had selected).
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
        else if (err == cudaSuccess) prev = -1;   // already current: nothing to restore
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

struct RenderState;   // render.cu
void render_state_free(RenderState* rs);

}  // namespace bg

// A context lives until bg_ctx_destroy has been called AND every scene and
// batch created on it is destroyed (each holds a reference), so objects may be
// destroyed in any order.
struct bg_ctx {
    int device = 0;
    int num_sms = 0;
    size_t l2_bytes = 0;
    std::atomic<int> refs{1};   // the creator's reference + one per live scene / batch
};

namespace bg {
inline void ctx_retain(bg_ctx* c) { c->refs.fetch_add(1); }
inline void ctx_release(bg_ctx* c) {
    if (c && c->refs.fetch_sub(1) == 1) delete c;
}
}  // namespace bg

struct bg_scene {
    bg_ctx* ctx = nullptr;
    std::mutex mu;
    std::vector<bg::MeshHost> meshes;
    std::vector<bg_material_desc> mats;
    std::vector<bg_light_desc> lights;
    float bg[3] = {0.f, 0.f, 0.f};
    float bbox_lo[3] = {0.f, 0.f, 0.f}, bbox_hi[3] = {0.f, 0.f, 0.f};   // world bounds of all triangles
    bool committed = false;

    bg::DevBuf nodes, tris, shade, bundles, mats_d, lights_d, err;
    bg::DevBuf work;          // persistent-kernel work counters (scratch)
    std::atomic<unsigned> work_slot{0};
    bg::DevBuf host_rays, host_out;   // staging of bg_render_host
    uint64_t uid = 0;                 // unique over the process (per-thread ray-cast staging keys on it)
    bg::DevScene dev{};
    bg_scene_info info{};
    bg::RenderState* render = nullptr;
    int trace_blocks[2][2][2][2] = {};   // [width 4/8][any][count][128/256 threads]: persistent grid sizes
    int64_t tune_paths = 0;   // autotuned paths per pass (0 = default)
    int tune_threads = 0;     // autotuned traversal block size (0 = default 128)
    bg::DevBuf nodes8;        // 8-wide compressed tree (empty if not built)
    int64_t nnodes4 = 0, nnodes8 = 0;
    int max_stack4 = 0, max_stack8 = 0, max_depth4 = 0, max_depth8 = 0;
    bool owns_buffers = true;
    // bg_render_host: the accumulation buffer's upload runs on copy_stream and
    // overlaps the pass; the pass's accumulate waits for ev_accum
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_accum = nullptr;
};

namespace bg {
// Launch helpers (api.cu)
constexpr int kTraceThreads = 128;
constexpr int kDefaultNodeWidth = 4;   // active layout when both are built
void set_width_info(bg_scene* s);
// Device BVH build (gpu_build.cu) from device world boxes lo/hi (3 floats per
// triangle): builder 1 = LBVH, 2 = PLOC.  Writes the leaf order (n entries,
// device) and the node arrays the params ask for, grown to their exact sizes.
struct DeviceBvh {
    int64_t nnodes4 = 0, nnodes8 = 0;
    int max_depth4 = 0, max_stack4 = 0, max_depth8 = 0, max_stack8 = 0;
    bool quant_ok = true;     // false: 8-wide planes could not be made conservative
};
int gpu_build_bvh(const float* lo, const float* hi, int64_t n, int builder, const BuildParams& bp, int32_t* order,
                  DevBuf& nodes4, DevBuf& nodes8, DeviceBvh& out);
// Top-down binned-SAH binary tree on the device (sah_build.cu), in gpu_build.cu's
// numbering: sorted[p] = triangle at final position p (leaf p), internal nodes
// n .. 2n-2 with the root n; left / right / parent of 2n - 1 entries.
int sah_binary_tree(const float* lo, const float* hi, int64_t n, int32_t* sorted, int32_t* left, int32_t* right,
                    int32_t* parent);

// One commit's mesh arrays on the device (scene_records.cu): the meshes'
// vertex, normal and uv arrays and per-face index arrays concatenated, with
// each face's bundle, and the world-space triangle boxes.
struct MeshArrays {
    ScratchBuf verts, normals, uvs, vi, ni, ti, mat, offs, bundle, lo, hi, bbox;
};
// material class of a hit (bits 28-29 of a packed primid): 0 misses / emissive,
// 1 Lambert, 2 GGX; primids stay below 2^27
constexpr int kPrimMask = (1 << 28) - 1;
constexpr int kClassShift = 28;

int upload_mesh_arrays(const std::vector<MeshHost>& meshes, int64_t ntris, MeshArrays& A);
// world boxes into A.lo / A.hi (Mesh::GetShapeWorldBounds) and the scene bounds of their finite values
int device_world_boxes(MeshArrays& A, const BundleRec* bundles, int64_t ntris, float bbox_lo[3], float bbox_hi[3]);
// traversal records in leaf order (order: device) and shading records in primitive order
// vertices: the watertight test's records (p1, p2, p3) instead of (p1, e1, e2)
// mat_class: class per material index (0 other, 1 Lambert, 2 GGX), stored in TriRec e2.w
int device_records(const MeshArrays& A, const BundleRec* bundles, const int32_t* order, int64_t ntris,
                   TriRec* tris, ShadeRec* shade, bool vertices, const int32_t* mat_class, int nmat);
constexpr int kWorkSlots = 256;
unsigned long long* next_work_counter(bg_scene* s);
void scene_launch_setup(bg_scene* s);
// Extras of a traversal launch.  Any hit: the shadow-ray resolve fused into the
// trace (a ray that finds no occluder stores contrib[i] into slots[slot_of[i]]
// instead of writing an occlusion byte).  Closest hit: hit_class != 0 packs the
// material class of the hit triangle into bits 28-29 of the written primid
// (the renderer's extension queues; see kPrimMask).
struct ShadowResolve {
    const float4* contrib;
    const int* slot_of;
    float4* slots;
    int hit_class;
};
int launch_trace(bg_scene* s, bool any_hit, const float4* rays, int64_t n_static, const int* n_dev,
                 bg_hit* hits, uint8_t* occ, cudaStream_t st, unsigned long long* counters = nullptr,
                 int stride = 1, unsigned long long* work = nullptr, const int* roots = nullptr,
                 const ShadowResolve* resolve = nullptr);
}  // namespace bg
