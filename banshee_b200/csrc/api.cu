// C ABI (include/banshee_gpu.h): context, scene assembly and commit, ray casts.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>

#include "bvh_build.h"
#include "internal.h"
#include "traverse.cuh"

namespace bg {

static thread_local std::string g_error;

int set_error(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

// Allocation accounting and the optional cap (bg_alloc_limit): every device
// and pinned-host allocation the library makes is charged here first.
static std::mutex g_alloc_mu;
static int64_t g_alloc_budget = -1;   // bytes still allowed; < 0 = no cap
static int64_t g_alloc_calls = 0, g_alloc_bytes = 0, g_alloc_refused = 0;

bool alloc_charge(size_t bytes) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    if (g_alloc_budget >= 0) {
        if (int64_t(bytes) > g_alloc_budget) {
            ++g_alloc_refused;
            return false;
        }
        g_alloc_budget -= int64_t(bytes);
    }
    ++g_alloc_calls;
    g_alloc_bytes += int64_t(bytes);
    return true;
}

int DevBuf::ensure(size_t need) {
    if (need <= bytes && ptr) return BG_OK;
    release();
    size_t want = std::max<size_t>(need, 256);
    if (!alloc_charge(want))
        return set_error(BG_ERR_OOM, "device allocation of %zu bytes refused: over the library's allocation limit", want);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        cudaGetLastError();
        return set_error(BG_ERR_OOM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    bytes = want;
    return BG_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

static cudaMemPool_t scratch_pool(int device) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0) return nullptr;
    if (size_t(device) >= pools.size()) pools.resize(size_t(device) + 1, nullptr);
    if (!pools[size_t(device)]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        uint64_t keep = kScratchKeepBytes;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[size_t(device)] = p;
    }
    return pools[size_t(device)];
}

int ScratchBuf::ensure(size_t need) {
    if (need <= bytes && ptr) return BG_OK;
    release();
    int dev = 0;
    BG_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool = scratch_pool(dev);
    if (!pool) return set_error(BG_ERR_CUDA, "scratch memory pool unavailable on device %d", dev);
    const size_t want = std::max<size_t>(need, 256);
    if (!alloc_charge(want))
        return set_error(BG_ERR_OOM, "scratch allocation of %zu bytes refused: over the library's allocation limit", want);
    cudaError_t e = cudaMallocFromPoolAsync(&ptr, want, pool, 0);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return set_error(BG_ERR_OOM, "scratch allocation (%zu bytes) failed: %s", want, cudaGetErrorString(e));
    }
    bytes = want;
    return BG_OK;
}

void ScratchBuf::release() {
    if (ptr) cudaFreeAsync(ptr, 0);
    ptr = nullptr;
    bytes = 0;
}

// ------------------------------------------------------------ trace kernel
// Persistent threads with per-lane dynamic fetch: lanes whose ray finished
// take new ray indices from one global counter with a single warp-aggregated
// atomicAdd, every kRefillStepsClosest / kRefillStepsAny traversal steps.
// Termination: the counter is monotone and every ray finishes after at most
// one visit per node.
template <bool ANY, bool COUNT, int THREADS = kTraceThreads, int WIDTH = 4, bool WT = false>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
k_trace(DevScene S, const float4* __restrict__ rays, int64_t n_static, const int* __restrict__ n_dev,
        bg_hit* __restrict__ hits, uint8_t* __restrict__ occ, unsigned long long* __restrict__ work,
        unsigned long long* __restrict__ counters, int stride, const int* __restrict__ roots, ShadowResolve res) {
    // roots (optional): per-ray root node, for rays of several scenes merged into one
    // res.slots (any hit, optional): visible rays store their contribution in their slot
    // COUNT: instrumented replay of rays 0, stride, 2*stride, ... (outputs compacted)
    const int64_t n_all = n_dev ? int64_t(*n_dev) : n_static;
    const int64_t n = COUNT ? (n_all + stride - 1) / stride : n_all;
    const unsigned lane = threadIdx.x & 31u;
    constexpr int kSm = smem_stack_entries<WIDTH>();
    int2 lstack[stack_entries<WIDTH>() - kSm];
    __shared__ int2 sstack[kSm > 0 ? kSm : 1][THREADS];
    const RayStack<kSm> stack{&sstack[0][threadIdx.x], lstack, THREADS};
    TravState<WT> s;
    Counters cnt{0ull, 0ull, 0ull};
    int64_t ridx = -1;
    bool active = false, exhausted = false;
    for (;;) {
        if (!exhausted) {
            unsigned need = __ballot_sync(0xffffffffu, !active);
            if (need) {
                int c = __popc(need);
                int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if (lane == unsigned(leader)) base = atomicAdd(work, (unsigned long long)c);
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + c >= (unsigned long long)n) exhausted = true;
                if (!active) {
                    int64_t my = int64_t(base) + __popc(need & ((1u << lane) - 1u));
                    if (my < n) {
                        ridx = my;
                        const int64_t src = COUNT ? my * stride : my;
                        float4 a = __ldg(rays + 2 * src), b = __ldg(rays + 2 * src + 1);
                        trav_init(s, a, b);
                        if (roots) s.item = __ldg(roots + src);
                        if (COUNT) ++cnt.rays;
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            if (trav_steps<ANY, COUNT, WIDTH>(S, s, stack, ANY ? kRefillStepsAny : kRefillStepsClosest, cnt)) {
                if (ANY) {
                    if (!res.slots) occ[ridx] = s.prim >= 0 ? 1 : 0;
                    else if (s.prim < 0) res.slots[__ldg(res.slot_of + ridx)] = __ldg(res.contrib + ridx);
                } else {
                    bg_hit h;
                    h.t = s.prim >= 0 ? s.best : s.r.tmax;
                    h.primid = s.prim;
                    h.u = s.u;
                    h.v = s.v;
                    if (res.hit_class && s.prim >= 0) h.primid = s.prim | (s.cls << kClassShift);
                    reinterpret_cast<float4*>(hits)[ridx] = *reinterpret_cast<float4*>(&h);
                }
                active = false;
            }
        }
    }
    if (COUNT) {
        for (int off = 16; off > 0; off >>= 1) {
            cnt.rays += __shfl_down_sync(0xffffffffu, cnt.rays, off);
            cnt.nodes += __shfl_down_sync(0xffffffffu, cnt.nodes, off);
            cnt.tris += __shfl_down_sync(0xffffffffu, cnt.tris, off);
        }
        if (lane == 0) {
            atomicAdd(counters, cnt.rays);
            atomicAdd(counters + 1, cnt.nodes);
            atomicAdd(counters + 2, cnt.tris);
        }
    }
}

template <bool ANY, bool COUNT, int THREADS, int WIDTH, bool WT>
static int trace_blocks(bg_scene* s) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace<ANY, COUNT, THREADS, WIDTH, WT>, THREADS, 0);
    if (nb < 1) nb = 1;
    return nb * s->ctx->num_sms;
}

// Grid sizes of every traversal variant of the scene's intersection test:
// [width 4/8][any][count][128/256 threads].
template <int WIDTH, bool WT>
static void setup_width(bg_scene* s, int w) {
    s->trace_blocks[w][0][0][0] = trace_blocks<false, false, 128, WIDTH, WT>(s);
    s->trace_blocks[w][1][0][0] = trace_blocks<true, false, 128, WIDTH, WT>(s);
    s->trace_blocks[w][0][1][0] = trace_blocks<false, true, 128, WIDTH, WT>(s);
    s->trace_blocks[w][1][1][0] = trace_blocks<true, true, 128, WIDTH, WT>(s);
    s->trace_blocks[w][0][0][1] = trace_blocks<false, false, 256, WIDTH, WT>(s);
    s->trace_blocks[w][1][0][1] = trace_blocks<true, false, 256, WIDTH, WT>(s);
}

void scene_launch_setup(bg_scene* s) {
    if (s->dev.watertight) {
        setup_width<4, true>(s, 0);
        setup_width<8, true>(s, 1);
    } else {
        setup_width<4, false>(s, 0);
        setup_width<8, false>(s, 1);
    }
}

unsigned long long* next_work_counter(bg_scene* s) {
    unsigned slot = s->work_slot.fetch_add(1) % kWorkSlots;
    return s->work.as<unsigned long long>() + slot;
}

template <int WIDTH, bool WT>
static void launch_width(bg_scene* s, bool any_hit, const float4* rays, int64_t n_static, const int* n_dev,
                         bg_hit* hits, uint8_t* occ, cudaStream_t st, unsigned long long* counters, int stride,
                         unsigned long long* w, const int* roots,
                         ShadowResolve res = ShadowResolve{nullptr, nullptr, nullptr, 0}) {
    const int wi = WIDTH == 8 ? 1 : 0;
    const DevScene& d = s->dev;
    // a static count smaller than the persistent grid (a few rays of a *_host
    // call) gets only the blocks it can use
    auto grid = [&](int blocks, int threads) {
        if (n_dev || n_static <= 0) return blocks;
        const int64_t rays_n = counters ? (n_static + stride - 1) / stride : n_static;
        return int(std::max<int64_t>(1, std::min<int64_t>(blocks, (rays_n + threads - 1) / threads)));
    };
    if (counters) {
        if (any_hit)
            k_trace<true, true, 128, WIDTH, WT><<<grid(s->trace_blocks[wi][1][1][0], 128), 128, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, counters, stride, roots, res);
        else
            k_trace<false, true, 128, WIDTH, WT><<<grid(s->trace_blocks[wi][0][1][0], 128), 128, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, counters, stride, roots, res);
    } else if (s->tune_threads == 256) {
        if (any_hit)
            k_trace<true, false, 256, WIDTH, WT><<<grid(s->trace_blocks[wi][1][0][1], 256), 256, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, nullptr, 1, roots, res);
        else
            k_trace<false, false, 256, WIDTH, WT><<<grid(s->trace_blocks[wi][0][0][1], 256), 256, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, nullptr, 1, roots, res);
    } else if (any_hit) {
        k_trace<true, false, 128, WIDTH, WT><<<grid(s->trace_blocks[wi][1][0][0], 128), 128, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, nullptr, 1, roots, res);
    } else {
        k_trace<false, false, 128, WIDTH, WT><<<grid(s->trace_blocks[wi][0][0][0], 128), 128, 0, st>>>(d, rays, n_static, n_dev, hits, occ, w, nullptr, 1, roots, res);
    }
}

// The traversal kernel of the scene's node layout and intersection test.
static void launch_layout(bg_scene* s, bool any_hit, const float4* rays, int64_t n_static, const int* n_dev,
                          bg_hit* hits, uint8_t* occ, cudaStream_t st, unsigned long long* counters, int stride,
                          unsigned long long* w, const int* roots, ShadowResolve res) {
    // (Measured and rejected: any-hit rays on the 8-wide nodes while closest-hit
    // rays use the 4-wide ones: the C3 shadow traversal took 16.6 instead of 13.6 ms.)
    const bool w8 = s->dev.width == 8, wt = s->dev.watertight != 0;
    if (w8 && wt) launch_width<8, true>(s, any_hit, rays, n_static, n_dev, hits, occ, st, counters, stride, w, roots, res);
    else if (w8) launch_width<8, false>(s, any_hit, rays, n_static, n_dev, hits, occ, st, counters, stride, w, roots, res);
    else if (wt) launch_width<4, true>(s, any_hit, rays, n_static, n_dev, hits, occ, st, counters, stride, w, roots, res);
    else launch_width<4, false>(s, any_hit, rays, n_static, n_dev, hits, occ, st, counters, stride, w, roots, res);
}

int launch_trace(bg_scene* s, bool any_hit, const float4* rays, int64_t n_static, const int* n_dev,
                 bg_hit* hits, uint8_t* occ, cudaStream_t st, unsigned long long* counters, int stride,
                 unsigned long long* work, const int* roots, const ShadowResolve* resolve) {
    unsigned long long* w = work ? work : next_work_counter(s);
    BG_CUDA(cudaMemsetAsync(w, 0, sizeof(unsigned long long), st));
    ShadowResolve res{nullptr, nullptr, nullptr, 0};
    if (resolve && !counters) {
        if (any_hit) res = *resolve;
        else res.hit_class = resolve->hit_class;
    }
    launch_layout(s, any_hit, rays, n_static, n_dev, hits, occ, st, counters, stride, w, roots, res);
    BG_CUDA(cudaGetLastError());
    return BG_OK;
}

// Node-layout fields of bg_scene_info for the active width.
void set_width_info(bg_scene* s) {
    bg_scene_info& info = s->info;
    const bool w8 = s->dev.width == 8;
    info.node_width = s->dev.width;
    info.nnodes = w8 ? s->nnodes8 : s->nnodes4;
    info.node_stride = int32_t(w8 ? sizeof(QNode8) : sizeof(WideNode4));
    info.node_bytes = info.nnodes * info.node_stride;
    info.max_depth = w8 ? s->max_depth8 : s->max_depth4;
    info.max_stack = w8 ? s->max_stack8 : s->max_stack4;
    info.node_widths = (s->dev.nodes ? 4 : 0) | (s->dev.nodes8 ? 8 : 0);
}

// ------------------------------------------------------------ commit
static bool is_identity(const float* m) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            if (m[4 * i + j] != (i == j ? 1.f : 0.f)) return false;
    return true;
}

static int commit_scene(bg_scene* s, const bg_build_opts* opts) {
    auto t0 = std::chrono::steady_clock::now();
    const int nm = int(s->meshes.size());
    if (nm == 0) return set_error(BG_ERR_STATE, "bg_scene_commit: the scene has no meshes");
    int64_t ntris = 0;
    std::vector<int64_t> start(nm);
    for (int i = 0; i < nm; ++i) { start[i] = ntris; ntris += s->meshes[i].nfaces; }
    if (ntris == 0) return set_error(BG_ERR_STATE, "bg_scene_commit: the scene has no triangles");
    if (ntris > int64_t(kMaxLeafStart)) return set_error(BG_ERR_UNSUPPORTED, "bg_scene_commit: %lld triangles exceed %d", (long long)ntris, kMaxLeafStart);
    const int nmat = int(s->mats.size());
    // validate materials per face and lights (AreaLight ctor, light/arealight.cpp:15-19)
    for (int i = 0; i < nm; ++i)
        for (int f = 0; f < s->meshes[i].nfaces; ++f)
            if (s->meshes[i].m[f] < 0 || s->meshes[i].m[f] >= std::max(nmat, 1))
                if (nmat > 0) return set_error(BG_ERR_INVALID_ARG, "mesh %d face %d: material %d out of range", i, f, s->meshes[i].m[f]);
    std::vector<BundleRec> bundles(nm);
    for (int i = 0; i < nm; ++i) {
        const MeshHost& mh = s->meshes[i];
        BundleRec& b = bundles[i];
        memcpy(b.m, mh.xf, sizeof(b.m));
        memcpy(b.minv, mh.xfinv, sizeof(b.minv));
        b.identity = is_identity(mh.xf) && is_identity(mh.xfinv);
        b.arealight = -1;
        b.nfaces = mh.nfaces;
        b.pad = 0;
        b.start = start[i];
        b.pad2 = 0;
    }
    std::vector<LightRec> lights(s->lights.size());
    for (size_t li = 0; li < s->lights.size(); ++li) {
        const bg_light_desc& d = s->lights[li];
        LightRec& L = lights[li];
        memset(&L, 0, sizeof(L));
        L.type = d.type;
        L.mesh = d.mesh;
        L.face = d.face;
        L.matidx = -1;
        if (d.type == BG_LIGHT_AREA) {
            if (d.mesh < 0 || d.mesh >= nm || d.face < 0 || d.face >= s->meshes[d.mesh].nfaces)
                return set_error(BG_ERR_INVALID_ARG, "light %zu: mesh/face out of range", li);
            int mi = s->meshes[d.mesh].m[d.face];
            if (mi < 0 || mi >= nmat || s->mats[mi].type != BG_MAT_EMISSIVE)
                return set_error(BG_ERR_INVALID_ARG, "AreaLight: The material passed is not an emissive one (light %zu)", li);
            L.matidx = mi;
            for (int k = 0; k < 3; ++k) L.e[k] = s->mats[mi].e[k];
            const MeshHost& mh = s->meshes[d.mesh];
            const int f = d.face;
            v3 p1 = mh.verts[mh.vi[3 * f]], p2 = mh.verts[mh.vi[3 * f + 1]], p3 = mh.verts[mh.vi[3 * f + 2]];
            L.pdf_obj = 1.f / (sqrtf(fabsf(sqnorm(cross(sub(p3, p1), sub(p3, p2))))) * 0.5f);
            float m12[12];
            memcpy(m12, mh.xf, sizeof(m12));
            v3 w1 = xf_point(m12, p1), w2 = xf_point(m12, p2), w3 = xf_point(m12, p3);
            L.area_world = sqrtf(fabsf(sqnorm(cross(sub(w3, w1), sub(w3, w2))))) * 0.5f;
            bundles[d.mesh].arealight = int(li);   // last one wins, light/arealight.cpp:22
        } else if (d.type == BG_LIGHT_DIRECTIONAL) {
            v3 n = normalize(mk(d.d[0], d.d[1], d.d[2]));
            L.dir[0] = n.x; L.dir[1] = n.y; L.dir[2] = n.z;
            for (int k = 0; k < 3; ++k) L.e[k] = d.e[k];
        } else if (d.type == BG_LIGHT_ENVIRONMENT) {
            // scale * pow(texel, 1/gamma) with the double ::pow of environment_light.cpp:27,48
            float invgamma = 1.f / d.gamma;
            for (int k = 0; k < 3; ++k) L.env[k] = float(std::pow(double(d.e[k]), double(invgamma))) * d.scale;
        } else {
            return set_error(BG_ERR_INVALID_ARG, "light %zu: unknown type %d", li, d.type);
        }
    }
    std::vector<MatRec> mats(std::max(nmat, 1));
    for (int i = 0; i < nmat; ++i) {
        const bg_material_desc& d = s->mats[i];
        if (d.type < BG_MAT_LAMBERT || d.type > BG_MAT_EMISSIVE)
            return set_error(BG_ERR_INVALID_ARG, "material %d: unknown type %d", i, d.type);
        MatRec& m = mats[i];
        m.type = d.type;
        for (int k = 0; k < 3; ++k) { m.kd[k] = d.kd[k]; m.ks[k] = d.ks[k]; m.e[k] = d.e[k]; }
        m.eta = d.eta;
        m.a = d.roughness;
    }
    BuildParams bp;
    int want_width = 0;
    if (opts) {
        want_width = opts->node_width;
        if (want_width != 0 && want_width != 4 && want_width != 8)
            return set_error(BG_ERR_UNSUPPORTED, "node_width %d: supported widths are 4 and 8 (0: both)", want_width);
        if (opts->max_leaf_size) bp.max_leaf = opts->max_leaf_size;
        if (opts->sah_bins) bp.bins = opts->sah_bins;
        if (opts->intersect != BG_INTERSECT_REFERENCE && opts->intersect != BG_INTERSECT_WATERTIGHT)
            return set_error(BG_ERR_INVALID_ARG, "intersect %d: 0 (reference Moller-Trumbore) or 1 (watertight)",
                             opts->intersect);
        if (opts->builder < 0 || opts->builder > 3)
            return set_error(BG_ERR_INVALID_ARG,
                             "builder %d: 0 (host SAH), 1 (device LBVH), 2 (device PLOC) or 3 (device SAH)",
                             opts->builder);
    }
    const int device_build = (opts && ntris >= 2) ? opts->builder : 0;
    if (bp.max_leaf < 1 || bp.max_leaf > 16 || bp.bins < 2 || bp.bins > 256)
        return set_error(BG_ERR_INVALID_ARG, "build options out of range (leaf 1..16, bins 2..256)");
    bp.wide4 = want_width != 8;
    bp.wide8 = want_width != 4;
    int rc;
    // mesh arrays to the device; boxes, tree and records are built there
    MeshArrays A;
    if ((rc = upload_mesh_arrays(s->meshes, ntris, A))) return rc;
    if ((rc = s->bundles.ensure(bundles.size() * sizeof(BundleRec)))) return rc;
    BG_CUDA(cudaMemcpy(s->bundles.ptr, bundles.data(), bundles.size() * sizeof(BundleRec), cudaMemcpyHostToDevice));
    const auto tb0 = std::chrono::steady_clock::now();
    // world-space triangle bounds (Mesh::GetShapeWorldBounds, primitive/mesh.cpp:263-283)
    if ((rc = device_world_boxes(A, s->bundles.as<BundleRec>(), ntris, s->bbox_lo, s->bbox_hi))) return rc;
    ScratchBuf order_d;
    if ((rc = order_d.ensure(size_t(ntris) * 4))) return rc;
    int64_t nn4 = 0, nn8 = 0;
    int ms4 = 0, md4 = 0, ms8 = 0, md8 = 0;
    if (device_build) {
        DeviceBvh db;
        if ((rc = gpu_build_bvh(A.lo.as<float>(), A.hi.as<float>(), ntris, device_build, bp, order_d.as<int32_t>(),
                                s->nodes, s->nodes8, db)))
            return rc;
        nn4 = db.nnodes4; ms4 = db.max_stack4; md4 = db.max_depth4;
        nn8 = db.nnodes8; ms8 = db.max_stack8; md8 = db.max_depth8;
    } else {
        std::vector<float> lo(3 * size_t(ntris)), hi(3 * size_t(ntris));
        BG_CUDA(cudaMemcpy(lo.data(), A.lo.ptr, lo.size() * 4, cudaMemcpyDeviceToHost));
        BG_CUDA(cudaMemcpy(hi.data(), A.hi.ptr, hi.size() * 4, cudaMemcpyDeviceToHost));
        BuildResult br = build_wide_bvh(lo.data(), hi.data(), ntris, bp);
        nn4 = int64_t(br.nodes.size()); ms4 = br.max_stack; md4 = br.max_depth;
        nn8 = int64_t(br.nodes8.size()); ms8 = br.max_stack8; md8 = br.max_depth8;
        if ((rc = s->nodes.ensure(std::max<size_t>(1, br.nodes.size()) * sizeof(WideNode4))) ||
            (rc = s->nodes8.ensure(std::max<size_t>(1, br.nodes8.size()) * sizeof(QNode8))))
            return rc;
        if (nn4)
            BG_CUDA(cudaMemcpy(s->nodes.ptr, br.nodes.data(), size_t(nn4) * sizeof(WideNode4), cudaMemcpyHostToDevice));
        if (nn8)
            BG_CUDA(cudaMemcpy(s->nodes8.ptr, br.nodes8.data(), size_t(nn8) * sizeof(QNode8), cudaMemcpyHostToDevice));
        BG_CUDA(cudaMemcpy(order_d.ptr, br.order.data(), size_t(ntris) * 4, cudaMemcpyHostToDevice));
    }
    if (want_width == 8 && nn8 == 0)
        return set_error(BG_ERR_UNSUPPORTED, "scene coordinates too large for the 8-wide compressed nodes");
    if (bp.wide4 && ms4 > kStackSize)
        return set_error(BG_ERR_UNSUPPORTED, "BVH needs a %d-entry traversal stack (> %d)", ms4, kStackSize);
    if (nn8 && ms8 > kStackSize8) {
        if (want_width == 8)
            return set_error(BG_ERR_UNSUPPORTED, "8-wide BVH needs a %d-entry traversal stack (> %d)", ms8, kStackSize8);
        nn8 = 0;
    }
    const auto tb1 = std::chrono::steady_clock::now();
    // traversal records in leaf order, shading records in primitive order
    if ((rc = s->tris.ensure(size_t(ntris) * sizeof(TriRec))) || (rc = s->shade.ensure(size_t(ntris) * sizeof(ShadeRec))))
        return rc;
    const bool watertight = opts && opts->intersect == BG_INTERSECT_WATERTIGHT;
    // material class per material (the renderer's shading split), stored with each triangle
    std::vector<int32_t> mclass(std::max(nmat, 1), 0);
    for (int i = 0; i < nmat; ++i)
        mclass[i] = s->mats[i].type == BG_MAT_LAMBERT ? 1 : s->mats[i].type == BG_MAT_MICROFACET_GGX ? 2 : 0;
    ScratchBuf mclass_d;
    if ((rc = mclass_d.ensure(mclass.size() * 4))) return rc;
    BG_CUDA(cudaMemcpy(mclass_d.ptr, mclass.data(), mclass.size() * 4, cudaMemcpyHostToDevice));
    if ((rc = device_records(A, s->bundles.as<BundleRec>(), order_d.as<int32_t>(), ntris, s->tris.as<TriRec>(),
                             s->shade.as<ShadeRec>(), watertight, mclass_d.as<int32_t>(), nmat)))
        return rc;
    const auto tb2 = std::chrono::steady_clock::now();
    if ((rc = s->mats_d.ensure(mats.size() * sizeof(MatRec))) ||
        (rc = s->lights_d.ensure(std::max<size_t>(1, lights.size()) * sizeof(LightRec))) ||
        (rc = s->err.ensure(sizeof(unsigned))) ||
        (rc = s->work.ensure(kWorkSlots * sizeof(unsigned long long))))
        return rc;
    BG_CUDA(cudaMemcpy(s->mats_d.ptr, mats.data(), mats.size() * sizeof(MatRec), cudaMemcpyHostToDevice));
    if (!lights.empty())
        BG_CUDA(cudaMemcpy(s->lights_d.ptr, lights.data(), lights.size() * sizeof(LightRec), cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemset(s->err.ptr, 0, sizeof(unsigned)));
    BG_CUDA(cudaMemset(s->work.ptr, 0, kWorkSlots * sizeof(unsigned long long)));
    DevScene& d = s->dev;
    d.nodes = nn4 ? s->nodes.as<WideNode4>() : nullptr;
    d.nodes8 = nn8 ? s->nodes8.as<QNode8>() : nullptr;
    s->nnodes4 = nn4;
    s->nnodes8 = nn8;
    s->max_stack4 = ms4; s->max_depth4 = md4;
    s->max_stack8 = ms8; s->max_depth8 = md8;
    d.width = d.nodes ? (want_width == 0 && d.nodes8 ? kDefaultNodeWidth : 4) : 8;
    d.tris = s->tris.as<TriRec>();
    d.shade = s->shade.as<ShadeRec>();
    d.bundles = s->bundles.as<BundleRec>();
    d.mats = s->mats_d.as<MatRec>();
    d.lights = s->lights_d.as<LightRec>();
    d.errflags = s->err.as<unsigned>();
    d.ntris = ntris;
    d.nbundles = nm;
    d.nmats = nmat;
    d.nlights = int(lights.size());
    d.has_area = 0;
    for (const LightRec& L : lights) d.has_area |= L.type == BG_LIGHT_AREA ? 1 : 0;
    d.watertight = watertight ? 1 : 0;
    d.bg[0] = s->bg[0]; d.bg[1] = s->bg[1]; d.bg[2] = s->bg[2];
    scene_launch_setup(s);
    auto t1 = std::chrono::steady_clock::now();
    bg_scene_info& info = s->info;
    info.ntriangles = ntris;
    info.tri_bytes = ntris * int64_t(sizeof(TriRec));
    info.shade_bytes = ntris * int64_t(sizeof(ShadeRec));
    set_width_info(s);
    info.nmeshes = nm;
    info.nmaterials = nmat;
    info.nlights = int(lights.size());
    info.build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    info.bvh_ms = std::chrono::duration<double, std::milli>(tb1 - tb0).count();
    info.records_ms = std::chrono::duration<double, std::milli>(tb2 - tb1).count();
    info.upload_ms = std::chrono::duration<double, std::milli>(tb0 - t0).count();
    s->committed = true;
    return BG_OK;
}

static int check_scene(bg_scene* s) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed (call bg_scene_commit first)");
    return BG_OK;
}

static int check_rays(const void* rays, const void* out, int64_t n) {
    if (n < 0) return set_error(BG_ERR_INVALID_ARG, "negative ray count");
    if (n > 0 && (!rays || !out)) return set_error(BG_ERR_INVALID_ARG, "NULL ray or output pointer");
    if (n > 0 && (reinterpret_cast<uintptr_t>(rays) & 15u)) return set_error(BG_ERR_INVALID_ARG, "ray array must be 16-byte aligned");
    if (n > (int64_t(1) << 40)) return set_error(BG_ERR_INVALID_ARG, "ray count too large");
    return BG_OK;
}

}  // namespace bg

using namespace bg;

extern "C" {

const char* bg_last_error(void) { return g_error.c_str(); }

int bg_version(int32_t* major, int32_t* minor) {
    if (major) *major = 1;
    if (minor) *minor = 0;
    return BG_OK;
}

int bg_alloc_limit(int64_t bytes) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_alloc_budget = bytes < 0 ? -1 : bytes;
    return BG_OK;
}

int bg_alloc_stats_get(bg_alloc_stats* out) {
    if (!out) return set_error(BG_ERR_INVALID_ARG, "out is NULL");
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    out->calls = g_alloc_calls;
    out->bytes = g_alloc_bytes;
    out->refused = g_alloc_refused;
    out->budget = g_alloc_budget;
    return BG_OK;
}

int bg_ctx_create(int32_t device, bg_ctx** out) {
    if (!out) return set_error(BG_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(BG_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= n) return set_error(BG_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, n);
    BG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    BG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return set_error(BG_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    bg_ctx* c = new (std::nothrow) bg_ctx();
    if (!c) return set_error(BG_ERR_OOM, "host allocation failed");
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    c->l2_bytes = size_t(prop.l2CacheSize);
    *out = c;
    return BG_OK;
}

int bg_ctx_destroy(bg_ctx* ctx) {
    ctx_release(ctx);   // freed once its scenes and batches are gone too
    return BG_OK;
}

int bg_ctx_sync(bg_ctx* ctx) {
    if (!ctx) return set_error(BG_ERR_INVALID_ARG, "ctx is NULL");
    BG_CUDA(cudaSetDevice(ctx->device));
    BG_CUDA(cudaDeviceSynchronize());
    return BG_OK;
}

int bg_scene_create(bg_ctx* ctx, bg_scene** out) {
    if (!ctx || !out) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    bg_scene* s = new (std::nothrow) bg_scene();
    if (!s) return set_error(BG_ERR_OOM, "host allocation failed");
    s->ctx = ctx;
    ctx_retain(ctx);
    static std::atomic<uint64_t> next_uid{1};
    s->uid = next_uid.fetch_add(1);
    *out = s;
    return BG_OK;
}

int bg_scene_destroy(bg_scene* s) {
    if (!s) return BG_OK;
    bg_ctx* ctx = s->ctx;
    {
        DeviceGuard dg(ctx->device);
        cudaDeviceSynchronize();
        for (DevBuf* b : {&s->nodes, &s->nodes8, &s->tris, &s->shade, &s->bundles, &s->mats_d, &s->lights_d, &s->err,
                          &s->work, &s->host_rays, &s->host_out})
            b->release();
        if (s->render) render_state_free(s->render);
        if (s->ev_accum) cudaEventDestroy(s->ev_accum);
        if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
        delete s;
    }
    ctx_release(ctx);
    return BG_OK;
}

// Mesh::Mesh, primitive/mesh.cpp:126-214 (strided reads; mstride not defaulted)
int bg_scene_add_mesh(bg_scene* s, const bg_mesh_desc* d, int32_t* index) {
    if (!s || !d) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->committed) return set_error(BG_ERR_STATE, "scene already committed");
    if (d->nfaces < 0 || d->nvertices < 0 || d->nnormals < 0 || d->nuvs < 0)
        return set_error(BG_ERR_INVALID_ARG, "negative count in mesh descriptor");
    if (d->nfaces > 0 && (!d->vertices || !d->normals || !d->vidx || !d->nidx || !d->materials))
        return set_error(BG_ERR_INVALID_ARG, "mesh descriptor has NULL arrays");
    MeshHost mh;
    const int vs = d->vstride ? d->vstride : int(3 * sizeof(float));
    const int ns = d->nstride ? d->nstride : int(3 * sizeof(float));
    mh.verts.resize(size_t(d->nvertices));
    for (int i = 0; i < d->nvertices; ++i) {
        const float* c = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->vertices) + size_t(i) * vs);
        mh.verts[i] = mk(c[0], c[1], c[2]);
    }
    mh.normals.resize(size_t(d->nnormals));
    for (int i = 0; i < d->nnormals; ++i) {
        const float* c = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->normals) + size_t(i) * ns);
        mh.normals[i] = mk(c[0], c[1], c[2]);
    }
    const bool hasuv = d->uvs && d->nuvs > 0;
    if (hasuv) {
        const int us = d->ustride ? d->ustride : int(2 * sizeof(float));
        mh.uvs.resize(2 * size_t(d->nuvs));
        for (int i = 0; i < d->nuvs; ++i) {
            const float* c = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d->uvs) + size_t(i) * us);
            mh.uvs[2 * i] = c[0];
            mh.uvs[2 * i + 1] = c[1];
        }
    } else {
        mh.uvs.assign(2, 0.f);
    }
    const int vis = d->vistride ? d->vistride : int(sizeof(int));
    const int nis = d->nistride ? d->nistride : int(sizeof(int));
    const int uis = d->uistride ? d->uistride : int(sizeof(int));
    auto rd = [](const int32_t* p, size_t k, int stride) {
        return *reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(p) + k * size_t(stride));
    };
    const int nuv = hasuv ? d->nuvs : 1;
    mh.nfaces = d->nfaces;
    mh.vi.resize(3 * size_t(d->nfaces));
    mh.ni.resize(3 * size_t(d->nfaces));
    mh.ti.resize(3 * size_t(d->nfaces));
    mh.m.resize(size_t(d->nfaces));
    for (int f = 0; f < d->nfaces; ++f) {
        for (int k = 0; k < 3; ++k) {
            int v = rd(d->vidx, 3 * size_t(f) + k, vis);
            int nn = rd(d->nidx, 3 * size_t(f) + k, nis);
            int t = hasuv ? rd(d->uidx, 3 * size_t(f) + k, uis) : 0;
            if (v < 0 || v >= d->nvertices || nn < 0 || nn >= d->nnormals || t < 0 || t >= nuv)
                return set_error(BG_ERR_INVALID_ARG, "face %d: index out of range", f);
            mh.vi[3 * f + k] = v;
            mh.ni[3 * f + k] = nn;
            mh.ti[3 * f + k] = t;
        }
        mh.m[f] = rd(d->materials, size_t(f), d->mstride);
    }
    memcpy(mh.xf, d->m, sizeof(mh.xf));
    memcpy(mh.xfinv, d->minv, sizeof(mh.xfinv));
    s->meshes.push_back(std::move(mh));
    if (index) *index = int32_t(s->meshes.size() - 1);
    return BG_OK;
}

int bg_scene_add_material(bg_scene* s, const bg_material_desc* m, int32_t* index) {
    if (!s || !m) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->committed) return set_error(BG_ERR_STATE, "scene already committed");
    s->mats.push_back(*m);
    if (index) *index = int32_t(s->mats.size() - 1);
    return BG_OK;
}

int bg_scene_add_light(bg_scene* s, const bg_light_desc* l, int32_t* index) {
    if (!s || !l) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->committed) return set_error(BG_ERR_STATE, "scene already committed");
    s->lights.push_back(*l);
    if (index) *index = int32_t(s->lights.size() - 1);
    return BG_OK;
}

int bg_scene_set_background(bg_scene* s, const float rgb[3]) {
    if (!s || !rgb) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    s->bg[0] = rgb[0]; s->bg[1] = rgb[1]; s->bg[2] = rgb[2];
    s->dev.bg[0] = rgb[0]; s->dev.bg[1] = rgb[1]; s->dev.bg[2] = rgb[2];
    return BG_OK;
}

int bg_scene_commit(bg_scene* s, const bg_build_opts* opts) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->committed) return set_error(BG_ERR_STATE, "scene already committed");
    BG_CUDA(cudaSetDevice(s->ctx->device));
    const int rc = commit_scene(s, opts);
    if (rc != BG_OK) {
        // a failed commit keeps nothing on the device: the scene stays
        // uncommitted and may be committed again (e.g. after memory is freed)
        for (DevBuf* b : {&s->nodes, &s->nodes8, &s->tris, &s->shade, &s->bundles, &s->mats_d, &s->lights_d, &s->err,
                          &s->work})
            b->release();
        s->dev = DevScene{};
        s->nnodes4 = s->nnodes8 = 0;
    }
    return rc;
}

int bg_scene_info_get(bg_scene* s, bg_scene_info* info) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (!info) return set_error(BG_ERR_INVALID_ARG, "info is NULL");
    *info = s->info;
    return BG_OK;
}

int bg_scene_error_flags(bg_scene* s, uint32_t* flags, int32_t clear) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (!flags) return set_error(BG_ERR_INVALID_ARG, "flags is NULL");
    unsigned v = 0;
    BG_CUDA(cudaMemcpy(&v, s->err.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (clear) BG_CUDA(cudaMemset(s->err.ptr, 0, sizeof(unsigned)));
    *flags = v;
    return BG_OK;
}

int bg_scene_set_node_width(bg_scene* s, int32_t width) {
    int rc = check_scene(s);
    if (rc) return rc;
    if (width != 4 && width != 8) return set_error(BG_ERR_INVALID_ARG, "node width %d: 4 or 8", width);
    if ((width == 4 && !s->dev.nodes) || (width == 8 && !s->dev.nodes8))
        return set_error(BG_ERR_UNSUPPORTED, "the %d-wide layout of this scene was not built", width);
    std::lock_guard<std::mutex> lk(s->mu);
    s->dev.width = width;
    set_width_info(s);
    return BG_OK;
}

int bg_intersect_closest(bg_scene* s, const bg_ray* rays, bg_hit* hits, int64_t n, void* stream) {
    int rc;
    if ((rc = check_scene(s)) || (rc = check_rays(rays, hits, n))) return rc;
    if (n == 0) return BG_OK;
    if (reinterpret_cast<uintptr_t>(hits) & 15u) return set_error(BG_ERR_INVALID_ARG, "hit array must be 16-byte aligned");
    return launch_trace(s, false, reinterpret_cast<const float4*>(rays), n, nullptr, hits, nullptr,
                        static_cast<cudaStream_t>(stream));
}

int bg_intersect_any(bg_scene* s, const bg_ray* rays, uint8_t* occ, int64_t n, void* stream) {
    int rc;
    if ((rc = check_scene(s)) || (rc = check_rays(rays, occ, n))) return rc;
    if (n == 0) return BG_OK;
    return launch_trace(s, true, reinterpret_cast<const float4*>(rays), n, nullptr, nullptr, occ,
                        static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// Per-thread staging of the *_host ray casts.  Banshee's renderers call
// World::Intersect from every thread of their pool (async/thread_pool.h:
// 136-150, renderer/mt_imagerenderer.cpp:86), one ray at a time.  Each calling
// thread gets its own stream, pinned host staging, device buffers and
// persistent-kernel work counter per scene, so concurrent calls run side by
// side on the GPU instead of queueing on the scene lock; a thread keeps the
// staging of its last kStages scenes (least recently used replaced).
namespace {
struct CastStage {
    uint64_t scene_uid = 0;
    int device = -1;
    uint64_t used = 0;
    cudaStream_t st = nullptr;
    DevBuf dev;                      // work counter (256 B) | rays | results
    void* pinned = nullptr;          // rays | results | error word
    size_t pinned_bytes = 0;
    void release() {
        if (st) cudaStreamSynchronize(st);
        dev.release();
        if (pinned) cudaFreeHost(pinned);
        if (st) cudaStreamDestroy(st);
        st = nullptr; pinned = nullptr; pinned_bytes = 0; scene_uid = 0; device = -1;
    }
    ~CastStage() { release(); }
};
constexpr int kStages = 4;
thread_local CastStage t_stage[kStages];
thread_local uint64_t t_stage_clock = 0;
}  // namespace

static CastStage* cast_stage(bg_scene* s) {
    CastStage* pick = &t_stage[0];
    for (CastStage& c : t_stage) {
        if (c.scene_uid == s->uid && c.device == s->ctx->device) { pick = &c; break; }
        if (c.used < pick->used) pick = &c;
    }
    if (pick->scene_uid != s->uid || pick->device != s->ctx->device) {
        pick->release();
        pick->scene_uid = s->uid;
        pick->device = s->ctx->device;
    }
    pick->used = ++t_stage_clock;
    return pick;
}

static int host_cast(bg_scene* s, const bg_ray* rays, void* out, int64_t n, bool any) {
    int rc;
    if ((rc = check_scene(s)) || (rc = check_rays(rays, out, n))) return rc;
    if (n == 0) return BG_OK;
    DeviceGuard dg(s->ctx->device);
    if (dg.err != cudaSuccess) return set_error(BG_ERR_CUDA, "ray cast: %s", cudaGetErrorString(dg.err));
    CastStage* c = cast_stage(s);
    if (!c->st) BG_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    const size_t rb = size_t(n) * sizeof(bg_ray), ob = size_t(n) * (any ? 1 : sizeof(bg_hit));
    const size_t ob16 = (ob + 15) & ~size_t(15);
    if ((rc = c->dev.ensure(256 + rb + ob16))) return rc;
    if (c->pinned_bytes < rb + ob16 + 16) {
        if (c->pinned) cudaFreeHost(c->pinned);
        c->pinned = nullptr;
        c->pinned_bytes = 0;
        const size_t want = std::max<size_t>(rb + ob16 + 16, 4096);
        if (!alloc_charge(want))
            return set_error(BG_ERR_OOM, "pinned staging of %zu bytes refused: over the library's allocation limit", want);
        BG_CUDA(cudaMallocHost(&c->pinned, want));
        c->pinned_bytes = want;
    }
    char* hp = static_cast<char*>(c->pinned);
    char* dp = c->dev.as<char>();
    memcpy(hp, rays, rb);
    BG_CUDA(cudaMemcpyAsync(dp + 256, hp, rb, cudaMemcpyHostToDevice, c->st));
    rc = launch_trace(s, any, reinterpret_cast<const float4*>(dp + 256), n, nullptr,
                      any ? nullptr : reinterpret_cast<bg_hit*>(dp + 256 + rb), any ? reinterpret_cast<uint8_t*>(dp + 256 + rb) : nullptr,
                      c->st, nullptr, 1, reinterpret_cast<unsigned long long*>(dp));
    if (rc) return rc;
    BG_CUDA(cudaMemcpyAsync(hp + rb, dp + 256 + rb, ob, cudaMemcpyDeviceToHost, c->st));
    BG_CUDA(cudaMemcpyAsync(hp + rb + ob16, s->err.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    BG_CUDA(cudaStreamSynchronize(c->st));
    memcpy(out, hp + rb, ob);
    unsigned flags = 0;
    memcpy(&flags, hp + rb + ob16, sizeof(unsigned));
    if (flags & BG_FLAG_STACK_OVERFLOW) return set_error(BG_ERR_OVERFLOW, "traversal stack overflow");
    return BG_OK;
}

extern "C" {

int bg_intersect_closest_host(bg_scene* s, const bg_ray* rays, bg_hit* hits, int64_t n) {
    return host_cast(s, rays, hits, n, false);
}

int bg_intersect_any_host(bg_scene* s, const bg_ray* rays, uint8_t* occ, int64_t n) {
    return host_cast(s, rays, occ, n, true);
}

}  // extern "C"

// A replay whose traversal stack overflowed undercounts: report it as the
// *_host casts do (the scene's device error word, read synchronously).
static int counts_overflow_check(bg_scene* s) {
    unsigned flags = 0;
    BG_CUDA(cudaMemcpy(&flags, s->err.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flags & BG_FLAG_STACK_OVERFLOW) return set_error(BG_ERR_OVERFLOW, "traversal stack overflow during the replay");
    return BG_OK;
}

extern "C" {

int bg_traversal_counts(bg_scene* s, const bg_ray* rays, int64_t n, int32_t any_hit, uint64_t* nodes,
                        uint64_t* triangles, void* stream) {
    int rc;
    if ((rc = check_scene(s)) || (rc = check_rays(rays, nodes, n))) return rc;
    if (!triangles) return set_error(BG_ERR_INVALID_ARG, "triangles is NULL");
    DeviceGuard dg(s->ctx->device);
    if (dg.err != cudaSuccess) return set_error(BG_ERR_CUDA, "traversal counts: %s", cudaGetErrorString(dg.err));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DevBuf tmp;
    if ((rc = tmp.ensure(256 + (any_hit ? size_t(n) : size_t(n) * sizeof(bg_hit))))) return rc;
    unsigned long long* cnt = tmp.as<unsigned long long>();
    bg_hit* hits = reinterpret_cast<bg_hit*>(tmp.as<char>() + 256);
    uint8_t* occ = tmp.as<uint8_t>() + 256;
    cudaError_t e = cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), st);
    if (e == cudaSuccess && n > 0) {
        rc = launch_trace(s, any_hit != 0, reinterpret_cast<const float4*>(rays), n, nullptr, hits, occ, st, cnt, 1);
        if (rc) { tmp.release(); return rc; }
    }
    unsigned long long h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    tmp.release();
    if (e != cudaSuccess) return set_error(BG_ERR_CUDA, "traversal counts: %s", cudaGetErrorString(e));
    *nodes = h[1];
    *triangles = h[2];
    return counts_overflow_check(s);
}

}  // extern "C"

// ------------------------------------------------------------------------
// Allocation-free traversal counts.
//
// bg_traversal_counts() allocates a temporary device buffer on every call (for
// the counters and for the hits the replay writes and throws away).  Some
// callers cannot let a library allocate: an application that reserves all of
// the device's memory up front for its own pool, where a cudaMalloc at run time
// may fail or fragment that pool; and a profiling harness, where cudaFree's
// implicit device synchronisation would disturb the timing it is measuring.
// bg_traversal_counts_noalloc() does the same replay with its scratch in the
// fixed-size array below, so it calls no cudaMalloc, cudaFree or allocating
// library routine.
//
// The array lives in every CUDA context that loads this library, from module
// load until exit.  Its device address is looked up once per device with
// cudaGetSymbolAddress, by the first call on that device, with that device
// current; make that first call before any stream capture.  Every call makes
// the scene's device current for its own work and gives the calling thread's
// current device back before it returns.  All calls share the
// array and it keeps the last call's contents: each call clears the counters it
// uses, and calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the same memory.
namespace bg {
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;   // 16 MiB
constexpr size_t kNoAllocHeader = 256;                       // counters + work counter
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {nullptr};

static int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= 64) return set_error(BG_ERR_INVALID_ARG, "device %d out of range for the static scratch", device);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        // the caller has made `device` current (DeviceGuard)
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(BG_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed: %s", cudaGetErrorString(e));
        }
        g_noalloc_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
    return BG_OK;
}
}  // namespace bg

extern "C" int bg_traversal_counts_noalloc(bg_scene* s, const bg_ray* rays, int64_t n, int32_t any_hit,
                                           uint64_t* nodes, uint64_t* triangles, void* stream) {
    using namespace bg;
    int rc;
    if ((rc = check_scene(s)) || (rc = check_rays(rays, nodes, n))) return rc;
    if (!triangles) return set_error(BG_ERR_INVALID_ARG, "triangles is NULL");
    const size_t per_ray = any_hit ? 1 : sizeof(bg_hit);
    const int64_t max_rays = int64_t((kNoAllocScratchBytes - kNoAllocHeader) / per_ray);
    if (n > max_rays)
        return set_error(BG_ERR_INVALID_ARG,
                         "bg_traversal_counts_noalloc: %lld rays exceed the %lld-ray limit of its %zu-byte static "
                         "scratch (%s); split the rays or use bg_traversal_counts",
                         (long long)n, (long long)max_rays, kNoAllocScratchBytes, any_hit ? "any hit" : "closest hit");
    DeviceGuard dg(s->ctx->device);   // the scene's device for this call; the caller's comes back after
    if (dg.err != cudaSuccess)
        return set_error(BG_ERR_CUDA, "bg_traversal_counts_noalloc: %s", cudaGetErrorString(dg.err));
    unsigned char* base = nullptr;
    if ((rc = noalloc_scratch(s->ctx->device, &base))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base);        // rays, nodes, triangles
    unsigned long long* work = cnt + 4;                                            // persistent-kernel work counter
    bg_hit* hits = reinterpret_cast<bg_hit*>(base + kNoAllocHeader);
    uint8_t* occ = base + kNoAllocHeader;
    cudaError_t e = cudaMemsetAsync(base, 0, kNoAllocHeader, st);   // counters and work counter start at zero
    if (e == cudaSuccess && n > 0) {
        const float4* r4 = reinterpret_cast<const float4*>(rays);
        launch_layout(s, any_hit != 0, r4, n, nullptr, any_hit ? nullptr : hits, any_hit ? occ : nullptr, st, cnt, 1,
                      work, nullptr, ShadowResolve{nullptr, nullptr, nullptr, 0});
        e = cudaGetLastError();
    }
    unsigned long long h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(BG_ERR_CUDA, "bg_traversal_counts_noalloc: %s", cudaGetErrorString(e));
    *nodes = h[1];
    *triangles = h[2];
    return counts_overflow_check(s);
}
