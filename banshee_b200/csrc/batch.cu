// Multi-scene batches: many independent scenes, cameras, resolutions and
// sample counts traced together from one global set of wavefront queues by the
// same persistent kernels, each pass replayed from one CUDA graph.
//
// bg_batch_commit merges the committed scenes into one device scene: node,
// triangle, shading-record, bundle, material and light arrays are concatenated
// and their cross indices offset on the device; every ray carries the root node
// of its scene.  Banshee renders one World at a time (renderer/renderer.h:49);
// the batch has no counterpart there.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "internal.h"
#include "render.h"

namespace bg {

__global__ void k_fix_nodes(WideNode4* nodes, int64_t n, int node_off, int tri_off) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        WideNode4& w = nodes[i];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int32_t c = w.child[k];
            if (c == kEmptyChild) continue;
            if (c >= 0) {
                w.child[k] = c + node_off;
            } else {
                uint32_t code = uint32_t(c);
                uint32_t start = (code & uint32_t(kMaxLeafStart)) + uint32_t(tri_off);
                w.child[k] = int32_t((code & ~uint32_t(kMaxLeafStart)) | start);
            }
        }
    }
}

__global__ void k_fix_nodes8(QNode8* nodes, int64_t n, int node_off, int tri_off) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        QNode8& w = nodes[i];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            int32_t c = w.child[k];
            if (c == kEmptyChild) continue;
            if (c >= 0) {
                w.child[k] = c + node_off;
            } else {
                uint32_t code = uint32_t(c);
                uint32_t start = (code & uint32_t(kMaxLeafStart)) + uint32_t(tri_off);
                w.child[k] = int32_t((code & ~uint32_t(kMaxLeafStart)) | start);
            }
        }
    }
}

__global__ void k_fix_tris(TriRec* tris, int64_t n, int bundle_off, int prim_off) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        TriRec& t = tris[i];
        int b = __float_as_int(t.v0.w);
        if (b >= 0) t.v0.w = __int_as_float(b + bundle_off);
        t.e1.w = __int_as_float(__float_as_int(t.e1.w) + prim_off);
    }
}

__global__ void k_fix_shade(ShadeRec* sh, int64_t n, int bundle_off, int mat_off) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        ShadeRec& r = sh[i];
        r.a.w = __int_as_float(__float_as_int(r.a.w) + bundle_off);
        r.b.w = __int_as_float(__float_as_int(r.b.w) + mat_off);
    }
}

}  // namespace bg

struct bg_batch {
    bg_ctx* ctx = nullptr;
    std::vector<bg_scene*> scenes;
    bg_scene merged;
    std::vector<bg::JobRec> rec;    // per scene: root (4-wide), light range, background
    std::vector<int> root8;         // per scene: root of its 8-wide tree in the merged array
    bool committed = false;
};

using namespace bg;

extern "C" {

int bg_batch_create(bg_ctx* ctx, bg_batch** out) {
    if (!ctx || !out) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    bg_batch* b = new bg_batch();
    b->ctx = ctx;
    b->merged.ctx = ctx;
    ctx_retain(ctx);
    *out = b;
    return BG_OK;
}

int bg_batch_add_scene(bg_batch* b, bg_scene* s, int32_t* index) {
    if (!b || !s) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (b->committed) return set_error(BG_ERR_STATE, "batch already committed");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    if (s->ctx != b->ctx) return set_error(BG_ERR_INVALID_ARG, "scene belongs to another context");
    b->scenes.push_back(s);
    if (index) *index = int32_t(b->scenes.size() - 1);
    return BG_OK;
}

int bg_batch_commit(bg_batch* b) {
    if (!b) return set_error(BG_ERR_INVALID_ARG, "batch is NULL");
    if (b->committed) return set_error(BG_ERR_STATE, "batch already committed");
    if (b->scenes.empty()) return set_error(BG_ERR_STATE, "batch has no scenes");
    auto t0 = std::chrono::steady_clock::now();
    BG_CUDA(cudaSetDevice(b->ctx->device));
    int64_t nn = 0, nn8 = 0, nt = 0, nb = 0, nm = 0, nl = 0;
    bool all4 = true, all8 = true;
    for (bg_scene* s : b->scenes) {
        nn += s->nnodes4; nn8 += s->nnodes8; nt += s->info.ntriangles; nb += s->info.nmeshes;
        nm += std::max(1, s->info.nmaterials); nl += s->info.nlights;
        all4 = all4 && s->dev.nodes; all8 = all8 && s->dev.nodes8;
    }
    if (!all4 && !all8) return set_error(BG_ERR_UNSUPPORTED, "the batch's scenes share no node layout");
    for (bg_scene* s : b->scenes)
        if (s->dev.watertight != b->scenes[0]->dev.watertight)
            return set_error(BG_ERR_UNSUPPORTED, "the batch's scenes use different ray / triangle tests");
    if (!all4) nn = 0;
    if (!all8) nn8 = 0;
    if (nt > int64_t(kMaxLeafStart)) return set_error(BG_ERR_UNSUPPORTED, "batch of %lld triangles exceeds %d", (long long)nt, kMaxLeafStart);
    if (std::max(nn, nn8) > (int64_t(1) << 31) - 2) return set_error(BG_ERR_UNSUPPORTED, "batch has too many nodes");
    bg_scene& M = b->merged;
    int rc;
    if ((rc = M.nodes.ensure(size_t(std::max<int64_t>(nn, 1)) * sizeof(WideNode4))) ||
        (rc = M.nodes8.ensure(size_t(std::max<int64_t>(nn8, 1)) * sizeof(QNode8))) ||
        (rc = M.tris.ensure(size_t(nt) * sizeof(TriRec))) ||
        (rc = M.shade.ensure(size_t(nt) * sizeof(ShadeRec))) || (rc = M.bundles.ensure(size_t(nb) * sizeof(BundleRec))) ||
        (rc = M.mats_d.ensure(size_t(nm) * sizeof(MatRec))) ||
        (rc = M.lights_d.ensure(size_t(std::max<int64_t>(nl, 1)) * sizeof(LightRec))) ||
        (rc = M.err.ensure(sizeof(unsigned))) || (rc = M.work.ensure(kWorkSlots * sizeof(unsigned long long))))
        return rc;
    int64_t no = 0, no8 = 0, to = 0, bo = 0, mo = 0, lo = 0;
    b->rec.clear();
    b->root8.clear();
    for (bg_scene* s : b->scenes) {
        const bg_scene_info& I = s->info;
        const int64_t nmat = std::max(1, I.nmaterials);
        if (all4) {
            BG_CUDA(cudaMemcpy(M.nodes.as<WideNode4>() + no, s->nodes.ptr, size_t(s->nnodes4) * sizeof(WideNode4),
                               cudaMemcpyDeviceToDevice));
            k_fix_nodes<<<1024, 256>>>(M.nodes.as<WideNode4>() + no, s->nnodes4, int(no), int(to));
        }
        if (all8) {
            BG_CUDA(cudaMemcpy(M.nodes8.as<QNode8>() + no8, s->nodes8.ptr, size_t(s->nnodes8) * sizeof(QNode8),
                               cudaMemcpyDeviceToDevice));
            k_fix_nodes8<<<1024, 256>>>(M.nodes8.as<QNode8>() + no8, s->nnodes8, int(no8), int(to));
        }
        BG_CUDA(cudaMemcpy(M.tris.as<TriRec>() + to, s->tris.ptr, size_t(I.ntriangles) * sizeof(TriRec), cudaMemcpyDeviceToDevice));
        BG_CUDA(cudaMemcpy(M.shade.as<ShadeRec>() + to, s->shade.ptr, size_t(I.ntriangles) * sizeof(ShadeRec), cudaMemcpyDeviceToDevice));
        BG_CUDA(cudaMemcpy(M.mats_d.as<MatRec>() + mo, s->mats_d.ptr, size_t(nmat) * sizeof(MatRec), cudaMemcpyDeviceToDevice));
        k_fix_tris<<<1024, 256>>>(M.tris.as<TriRec>() + to, I.ntriangles, int(bo), int(to));
        k_fix_shade<<<1024, 256>>>(M.shade.as<ShadeRec>() + to, I.ntriangles, int(bo), int(mo));
        BG_CUDA(cudaGetLastError());
        std::vector<BundleRec> bun(size_t(I.nmeshes));
        BG_CUDA(cudaMemcpy(bun.data(), s->bundles.ptr, bun.size() * sizeof(BundleRec), cudaMemcpyDeviceToHost));
        for (BundleRec& r : bun) {
            r.start += to;
            if (r.arealight >= 0) r.arealight += int32_t(lo);
        }
        BG_CUDA(cudaMemcpy(M.bundles.as<BundleRec>() + bo, bun.data(), bun.size() * sizeof(BundleRec), cudaMemcpyHostToDevice));
        if (I.nlights > 0) {
            std::vector<LightRec> li(size_t(I.nlights));
            BG_CUDA(cudaMemcpy(li.data(), s->lights_d.ptr, li.size() * sizeof(LightRec), cudaMemcpyDeviceToHost));
            for (LightRec& r : li) {
                if (r.mesh >= 0) r.mesh += int32_t(bo);
                if (r.matidx >= 0) r.matidx += int32_t(mo);
            }
            BG_CUDA(cudaMemcpy(M.lights_d.as<LightRec>() + lo, li.data(), li.size() * sizeof(LightRec), cudaMemcpyHostToDevice));
        }
        JobRec jr;
        jr.root = int(no);
        jr.light0 = int(lo);
        jr.nlights = I.nlights;
        jr.pad = 0;
        jr.bg[0] = s->bg[0]; jr.bg[1] = s->bg[1]; jr.bg[2] = s->bg[2]; jr.bg[3] = 0.f;
        b->rec.push_back(jr);
        b->root8.push_back(int(no8));
        no += all4 ? s->nnodes4 : 0; no8 += all8 ? s->nnodes8 : 0;
        to += I.ntriangles; bo += I.nmeshes; mo += nmat; lo += I.nlights;
    }
    BG_CUDA(cudaMemset(M.err.ptr, 0, sizeof(unsigned)));
    BG_CUDA(cudaMemset(M.work.ptr, 0, kWorkSlots * sizeof(unsigned long long)));
    BG_CUDA(cudaDeviceSynchronize());
    DevScene& d = M.dev;
    d.nodes = all4 ? M.nodes.as<WideNode4>() : nullptr;
    d.nodes8 = all8 ? M.nodes8.as<QNode8>() : nullptr;
    d.width = all4 ? (all8 ? kDefaultNodeWidth : 4) : 8;
    M.nnodes4 = nn; M.nnodes8 = nn8;
    d.tris = M.tris.as<TriRec>();
    d.shade = M.shade.as<ShadeRec>();
    d.bundles = M.bundles.as<BundleRec>();
    d.mats = M.mats_d.as<MatRec>();
    d.lights = M.lights_d.as<LightRec>();
    d.errflags = M.err.as<unsigned>();
    d.ntris = nt;
    d.nbundles = int(nb);
    d.nmats = int(nm);
    d.nlights = int(nl);
    d.has_area = 0;
    for (bg_scene* s : b->scenes) d.has_area |= s->dev.has_area;
    d.watertight = b->scenes[0]->dev.watertight;
    scene_launch_setup(&M);
    bg_scene_info& info = M.info;
    info.ntriangles = nt;
    info.tri_bytes = nt * int64_t(sizeof(TriRec));
    info.shade_bytes = nt * int64_t(sizeof(ShadeRec));
    info.nmeshes = int(nb);
    info.nmaterials = int(nm);
    info.nlights = int(nl);
    for (bg_scene* s : b->scenes) {
        M.max_depth4 = std::max(M.max_depth4, s->max_depth4);
        M.max_stack4 = std::max(M.max_stack4, s->max_stack4);
        M.max_depth8 = std::max(M.max_depth8, s->max_depth8);
        M.max_stack8 = std::max(M.max_stack8, s->max_stack8);
    }
    set_width_info(&M);
    info.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    M.committed = true;
    b->committed = true;
    return BG_OK;
}

int bg_batch_info(bg_batch* b, bg_scene_info* info) {
    if (!b || !info) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (!b->committed) return set_error(BG_ERR_STATE, "batch not committed");
    *info = b->merged.info;
    return BG_OK;
}

static int batch_jobs(bg_batch* b, const bg_batch_job* jobs, int32_t njobs, std::vector<JobSpec>& out, int spp_cap) {
    if (!b || (njobs > 0 && !jobs)) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (!b->committed) return set_error(BG_ERR_STATE, "batch not committed");
    if (njobs < 0) return set_error(BG_ERR_INVALID_ARG, "negative job count");
    out.resize(size_t(njobs));
    for (int32_t i = 0; i < njobs; ++i) {
        const bg_batch_job& j = jobs[i];
        if (j.scene < 0 || j.scene >= int32_t(b->scenes.size())) return set_error(BG_ERR_INVALID_ARG, "job %d: scene %d out of range", i, j.scene);

        JobSpec& J = out[size_t(i)];
        J.rec = b->rec[size_t(j.scene)];
        if (b->merged.dev.width == 8) J.rec.root = b->root8[size_t(j.scene)];
        J.cam = make_camera(&j.camera);
        J.W = j.width;
        J.H = j.height;
        J.spp = spp_cap > 0 ? std::min(j.sampler.spp, spp_cap) : j.sampler.spp;
        J.soff = j.sampler.sample_offset;
        J.seed = j.sampler.seed;
        J.accum = reinterpret_cast<float4*>(j.accum_rgbw_dev);
        J.skind = j.sampler.kind;
        J.grid = j.sampler.grid;
    }
    return BG_OK;
}

int bg_batch_render(bg_batch* b, const bg_batch_job* jobs, int32_t njobs, const bg_tracer_desc* tracer,
                    bg_render_stats* stats, void* stream) {
    std::vector<JobSpec> js;
    int rc = batch_jobs(b, jobs, njobs, js, 0);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(b->merged.mu);
    return render_jobs(&b->merged, nullptr, js, tracer, stats, static_cast<cudaStream_t>(stream), true);
}

// Autotuner: times every (node layout, traversal block size, paths per pass)
// candidate on the given jobs with spp capped to `probe_spp` (their
// accumulation buffers receive those samples), keeps the fastest.
int bg_batch_autotune(bg_batch* b, const bg_batch_job* jobs, int32_t njobs, const bg_tracer_desc* tracer,
                      int32_t probe_spp, bg_tune_result* result, void* stream) {
    if (!b) return set_error(BG_ERR_INVALID_ARG, "batch is NULL");
    if (!b->committed) return set_error(BG_ERR_STATE, "batch not committed");
    std::vector<JobSpec> js;
    std::lock_guard<std::mutex> lk(b->merged.mu);
    bg_scene& M = b->merged;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<int> widths;
    if (M.dev.nodes) widths.push_back(4);
    if (M.dev.nodes8) widths.push_back(8);
    const int threads[2] = {128, 256};
    float best = 1e30f;
    int best_t = 128, best_w = M.dev.width;
    int64_t best_p = int64_t(1) << 21;
    int tried = 0;
    int rc = BG_OK;
    cudaEvent_t e0, e1;
    BG_CUDA(cudaEventCreate(&e0));
    BG_CUDA(cudaEventCreate(&e1));
    for (int w : widths) {
        M.dev.width = w;
        if ((rc = batch_jobs(b, jobs, njobs, js, std::max(1, probe_spp)))) break;   // roots of this layout
        int64_t probe_samples = 0;
        for (const JobSpec& J : js) probe_samples += int64_t(J.W) * J.H * J.spp;
        for (int t : threads) {
            for (int pi = 0; pi < kPassCandidates && pass_candidate_needed(pi, probe_samples); ++pi) {
                const int64_t p = pass_candidate(pi);
                M.tune_threads = t;
                M.tune_paths = p;
                // first call warms the graph and buffers for this candidate, the second is timed
                if ((rc = render_jobs(&M, nullptr, js, tracer, nullptr, st, true))) {
                    if (rc == BG_ERR_OOM && pi > 0) {   // no room for passes this large: keep the smaller
                        cudaGetLastError();
                        rc = BG_OK;
                    }
                    break;
                }
                BG_CUDA(cudaEventRecord(e0, st));
                if ((rc = render_jobs(&M, nullptr, js, tracer, nullptr, st, true))) break;
                BG_CUDA(cudaEventRecord(e1, st));
                BG_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                BG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                ++tried;
                if (ms < best) { best = ms; best_t = t; best_p = p; best_w = w; }
            }
            if (rc) break;
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    M.dev.width = best_w;
    set_width_info(&M);
    if (rc) return rc;
    M.tune_threads = best_t;
    M.tune_paths = best_p;
    int64_t samples = 0;
    for (const JobSpec& J : js) samples += int64_t(J.W) * J.H * J.spp;
    if (result) {
        result->trace_threads = best_t;
        result->paths_per_pass = int32_t(best_p);
        result->candidates = tried;
        result->ms = best;
        result->msamples_per_s = best > 0.f ? float(double(samples) / (double(best) * 1e3)) : 0.f;
        result->node_width = best_w;
    }
    return BG_OK;
}

int bg_batch_destroy(bg_batch* b) {
    if (!b) return BG_OK;
    bg_ctx* ctx = b->ctx;
    {
        bg_scene& M = b->merged;
        DeviceGuard dg(ctx->device);
        cudaDeviceSynchronize();
        for (DevBuf* d : {&M.nodes, &M.nodes8, &M.tris, &M.shade, &M.bundles, &M.mats_d, &M.lights_d, &M.err, &M.work,
                          &M.host_rays, &M.host_out})
            d->release();
        if (M.render) { render_state_free(M.render); M.render = nullptr; }
        delete b;
    }
    ctx_release(ctx);
    return BG_OK;
}

}  // extern "C"
