// Wavefront GI / DI renderer: Renderer::Render + GiTracer / DiTracer on the GPU.
//
// The recursive per-sample GiTracer::GetLi (tracer/gitracer.cpp:13-140) and
// DiTracer::GetDi (tracer/ditracer.cpp:57-239) become one wave of paths per
// bounce:
//   generate  camera rays + per-sample samplers           (renderer/imagerenderer.cpp:25-38)
//   extend    closest hit of the extension rays           (persistent k_trace)
//   shade     gather last bounce's direct light, FillHit, light sampling and
//             BSDF sampling for MIS, BSDF continuation, Russian roulette;
//             pushes shadow / MIS / extension rays through warp-aggregated
//             atomics (ballot + prefix count, one atomic per warp)
//   shadow    any hit of light-sample and environment-MIS rays
//   mis       closest hit of BSDF-sampled rays towards area lights
//   resolve   write each visible contribution to its path's fixed DI slot
//   finalize  gather pending slots, clamp (gitracer.cpp:139), per-sample radiance
//   accumulate per pixel, samples in order: FileImagePlane::WriteSample
//             (imageplane/fileimageplane.cpp:29-34), rows flipped
// Each path owns 2 * nlights DI slots (light-sample and BSDF-sample term per
// light), summed in light order like GetDi, so images are deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cache.h"
#include "internal.h"
#include "render.h"
#include "samplers.cuh"
#include "shading.cuh"

namespace bg {

// cache.cu
int nrc_prepare(bg_cache* c, int64_t train_rows, int64_t query_rows);
int nrc_encode(bg_cache* c, const float* feat, const int* n_dev, int64_t n_static, int offset, int limit, cudaStream_t st);
int nrc_infer(bg_cache* c, const int* n_dev, int64_t n_static, float4* out, cudaStream_t st);
int nrc_query(bg_cache* c, const float* feat, const int* n_dev, int64_t n_static, float4* out, cudaStream_t st);
int nrc_train_step(bg_cache* c, const float* feat, const float4* target, const int* n_dev, int offset, int B, bool apply,
                   cudaStream_t st);
const bg_cache_desc* nrc_desc(const bg_cache* c);
int64_t nrc_next_frame(bg_cache* c);
int64_t nrc_frame(const bg_cache* c);   // frames rendered so far
uint64_t nrc_id(const bg_cache* c);          // unique over the process, never reused
uint64_t nrc_buf_epoch(const bg_cache* c);   // changes whenever the cache's scratch is reallocated
int nrc_graph_node(bg_cache* c, cudaGraphExec_t exec, cudaGraphNode_t node, bool* is_cache);
bg_scene* nrc_scene(const bg_cache* c);

__global__ void k_clamp_count(int* n, int cap) {
    if (*n > cap) *n = cap;
}

constexpr int kShadeThreads = 128;
constexpr int kMaxBounceCounters = 6 * 1024;   // 6 work counters per bounce, maxdepth <= 1024
constexpr int kGraphKey = 15;                    // int64 fields identifying a captured pass


// A pass segment: `ns` samples of pixels [p0, p0 + np) of job `job`, as paths
// [path0, path0 + np * ns) of the pass.
struct SegRec {
    CamDev cam;
    float4* accum;
    uint64_t seed;
    int job, np, ns, p0, s0, W, H, path0, pix0;   // pix0: prefix sum of np over earlier segments
    int skind, grid;                               // image sampler of the job
};
constexpr int kMaxSegs = 1024;



struct RenderState {
    int64_t cap = 0;   // paths per pass
    int kmax = 0;      // DI slots per path
    int nlights = 0;
    DevBuf ext_rays[2], ext_path[2], ext_hits;
    DevBuf sh_rays, sh_contrib, sh_slot;
    DevBuf mis_rays, mis_a, mis_b, mis_c, mis_hits;
    DevBuf end_path;
    DevBuf cls;        // material-class lists of the extension queue: 3 x cap queue indices
    DevBuf counts;     // int: ext[0], ext[1], sh, mis, end ; u64 totals at +64 bytes
    DevBuf st_key, st_cnt, st_rng, st_bs, st_thr, st_rad, st_dithr, st_flags;
    DevBuf slots, sample_rad;
    DevBuf cnt_out;    // outputs of the instrumented 1/64 replays
    DevBuf work;       // persistent-kernel work counters of the pass (6 per bounce)
    // radiance-cache mode: cache queries, training-path vertex records, training samples
    DevBuf q_feat, q_path, q_thr, q_out, rec, tr_feat, tr_target;
    int64_t q_cap = 0, tr_cap = 0;       // tr_cap: rows per training set
    int tr_set = 0;                      // training set this frame writes
    // rows of the other set wait to be trained at the start of the next frame
    // of the same cache (pending_frame: that cache's frame index which wrote them)
    uint64_t pending_cache = 0;         // id (nrc_id) of the cache whose training rows are pending
    bg_cache* pending_ptr = nullptr;    // that cache (cleared when it is destroyed)
    // bumped whenever a buffer that captured passes bake in is reallocated
    // (segment / job tables, cache-mode queues and training sets): graphs
    // captured before then hold stale pointers and must not be replayed
    uint64_t buf_epoch = 0;
    int64_t pending_frame = -1;
    cudaStream_t tstream = nullptr;      // training of the previous frame's rows
    cudaEvent_t ev_tstart = nullptr, ev_train = nullptr;
    // segment table of the pass in flight: int header {nseg, total} + SegRec[kMaxSegs]
    DevBuf segs, jobs;
    int njobs_cap = 0;
    void* host_tab[2] = {nullptr, nullptr};     // pinned staging of the segment + job tables
    size_t host_tab_bytes[2] = {0, 0};
    cudaEvent_t tab_ev[2] = {nullptr, nullptr};
    int tab_i = 0;
    DevBuf ext_root[2], sh_root, mis_root;   // per-ray root node (batched renders)
    int blocks = 0;
    int blocks_class = 0;   // grid of the material-class shading kernels
    // CUDA graph of one pass, replayed on an internal stream
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // side streams of a pass: the next bounce's extension trace (fstream) and
    // this bounce's MIS trace + resolve (mstream), with fork / join events
    cudaStream_t fstream = nullptr, mstream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_mjoin = nullptr;
    // captured passes, eight kept, least recently used replaced (a cached
    // render alternates between two training-row sets, and the training-path
    // stride, which a captured pass bakes in, follows the frame's size)
    struct PassGraph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t gen_node = nullptr, acc_node = nullptr;
        std::vector<cudaGraphNode_t> cache_nodes;   // kernels whose arguments belong to the cache
        int64_t key[kGraphKey] = {};
        uint64_t used = 0;
    } graphs[8];
    uint64_t graph_clock = 0;
};

void render_state_free(RenderState* rs) {
    for (int i = 0; i < 2; ++i) {
        if (rs->tab_ev[i]) { cudaEventSynchronize(rs->tab_ev[i]); cudaEventDestroy(rs->tab_ev[i]); }
        if (rs->host_tab[i]) cudaFreeHost(rs->host_tab[i]);
    }
    for (auto& pg : rs->graphs) {
        if (pg.exec) cudaGraphExecDestroy(pg.exec);
        if (pg.graph) cudaGraphDestroy(pg.graph);
    }
    if (rs->ev_in) cudaEventDestroy(rs->ev_in);
    if (rs->ev_out) cudaEventDestroy(rs->ev_out);
    if (rs->gstream) cudaStreamDestroy(rs->gstream);
    if (rs->ev_fork) cudaEventDestroy(rs->ev_fork);
    if (rs->ev_join) cudaEventDestroy(rs->ev_join);
    if (rs->fstream) cudaStreamDestroy(rs->fstream);
    if (rs->ev_tstart) cudaEventDestroy(rs->ev_tstart);
    if (rs->ev_train) cudaEventDestroy(rs->ev_train);
    if (rs->tstream) cudaStreamDestroy(rs->tstream);
    if (rs->ev_mjoin) cudaEventDestroy(rs->ev_mjoin);
    if (rs->mstream) cudaStreamDestroy(rs->mstream);
    for (DevBuf* b : {&rs->ext_rays[0], &rs->ext_rays[1], &rs->ext_path[0], &rs->ext_path[1], &rs->ext_hits,
                      &rs->sh_rays, &rs->sh_contrib, &rs->sh_slot, &rs->mis_rays, &rs->mis_a, &rs->mis_b,
                      &rs->mis_c, &rs->mis_hits, &rs->end_path, &rs->counts, &rs->st_key, &rs->st_cnt, &rs->st_rng,
                      &rs->st_bs, &rs->st_thr, &rs->st_rad, &rs->st_dithr, &rs->st_flags, &rs->slots,
                      &rs->sample_rad, &rs->cnt_out, &rs->work, &rs->q_feat, &rs->q_path, &rs->q_thr,
                      &rs->q_out, &rs->rec, &rs->tr_feat, &rs->tr_target, &rs->segs, &rs->jobs,
                      &rs->ext_root[0], &rs->ext_root[1], &rs->sh_root, &rs->mis_root, &rs->cls})
        b->release();
    delete rs;
}

enum : int { kCntExt0 = 0, kCntExt1 = 1, kCntSh = 2, kCntMis = 3, kCntEnd = 4, kCntQuery = 5, kCntTrain = 6 };
constexpr int kCntCls = 12;   // three material-class counters (k_classify)
// extension traces write the material class of each hit into its primid
static const ShadowResolve kExtTrace{nullptr, nullptr, nullptr, 1};
// shadow / MIS / ended-path counters of the odd bounces when direct light is
// resolved one bounce late (the even bounces use kCntSh..kCntEnd)
constexpr int kCntSh1 = 8;
// training rows alternate between two halves of tr_feat / tr_target (counters
// kCntTrain + set): a frame writes one while the previous frame's are trained on
constexpr int kCntTrainSets = 2;
enum : unsigned { kFlagNoClamp = 1u, kFlagTrain = 2u };   // bits 8..15: recorded vertices of a training path

struct PathState {
    unsigned long long* key;
    unsigned* cnt;
    uint4* rng;        // light McRng (z,w), BSDF McRng (z,w)
    float2* bs;        // GiTracer's BSDF sample, reused at every bounce (gitracer.cpp:36-41,88)
    float4* thr;       // throughput
    float4* rad;       // radiance; w = pending DI slots (int bits)
    float4* dithr;     // throughput of the bounce whose DI is pending; w = light-count multiplier
    unsigned* flags;
    float4* slots;     // cap * kmax
    float4* sample_rad;
    float4* rec;       // training paths: per vertex feat[4], throughput, radiance before the vertex
};

struct Queues {
    float4* ext_rays_in; int* ext_path_in; bg_hit* ext_hits;
    float4* ext_rays_out; int* ext_path_out;
    float4* sh_rays; float4* sh_contrib; int* sh_slot;
    float4* mis_rays; float4* mis_a; float4* mis_b; int4* mis_c; bg_hit* mis_hits;
    int* end_path;
    int* n_ext_in; int* n_ext_out; int* n_sh; int* n_mis; int* n_end;
    unsigned long long* totals;   // [0] closest rays, [1] any rays
    float4* q_feat; int* q_path; float4* q_thr; int* n_query;        // cache queries
    float4* tr_feat; float4* tr_target; int* n_train; int tr_cap;   // training samples
    int* ext_root_in; int* ext_root_out; int* sh_root; int* mis_root; // per-ray roots, batched only
    const JobRec* jobs;
    int* n_cls; int* cls;                                            // material-class lists (k_classify)
};

// With direct light resolved one bounce late, a path's DI slots and DI
// throughput alternate between two halves by bounce parity, and rad.w packs the
// pending slot counts of both (bits 0-15: even bounces, 16-31: odd bounces).
__device__ __forceinline__ int pend_get(int packed, int h) { return (packed >> (16 * h)) & 0xffff; }
__device__ __forceinline__ int pend_set(int packed, int h, int v) {
    return int((unsigned(packed) & ~(0xffffu << (16 * h))) | (unsigned(v) << (16 * h)));
}

// Warp-aggregated slot allocation: one atomicAdd per converged group of lanes.
__device__ __forceinline__ int warp_push(int* counter) {
    unsigned m = __activemask();
    int leader = __ffs(m) - 1;
    unsigned lane = threadIdx.x & 31u;
    int base = 0;
    if (lane == unsigned(leader)) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ void put_ray(float4* rays, int i, v3 o, float tmin, v3 d, float tmax) {
    rays[2 * i] = make_float4(o.x, o.y, o.z, tmin);
    rays[2 * i + 1] = make_float4(d.x, d.y, d.z, tmax);
}

// ------------------------------------------------------------- generate
__device__ __forceinline__ int find_seg(const SegRec* segs, int nseg, int i) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {                 // last segment with path0 <= i
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].path0 <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kShadeThreads)
k_generate(const SegRec* __restrict__ segs, int nseg, int total, PathState P, Queues Q, int train_stride,
           int train_phase) {
    const int nthreads = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += nthreads) {
        const SegRec& G = segs[find_seg(segs, nseg, i)];
        const CamDev& cam = G.cam;
        const int W = G.W, H = G.H;
        const int li = i - G.path0;
        const int sl = li / G.np;
        // queue slot i holds the sample of pixel offset `off` of its slice: slices of
        // whole rows are laid out in 8 x 4 pixel tiles (one warp's 32 rays), row
        // groups of 4 in turn, rows beyond the last full group in row order; the
        // path index stays the pixel's, so only the ray order changes
        int off = li - sl * G.np;
        if (W % 8 == 0 && G.p0 % W == 0 && G.np % W == 0 && off < (G.np / (4 * W)) * 4 * W) {
            const int rg = off / (4 * W), rem = off - rg * 4 * W;
            const int tc = rem >> 5, w = rem & 31;
            off = (4 * rg + (w >> 3)) * W + 8 * tc + (w & 7);
        }
        const int pix = G.p0 + off;
        const int path = G.path0 + sl * G.np + off;
        const uint32_t s = uint32_t(G.s0 + sl);
        const uint64_t key = keyed_key(G.seed, uint32_t(pix), s);
        McRng img{keyed_rand(key, 0), keyed_rand(key, 1)};
        McRng lr{keyed_rand(key, 2), keyed_rand(key, 3)};
        McRng br{keyed_rand(key, 4), keyed_rand(key, 5)};
        float sx, sy;
        image_sample(G.skind, G.grid, G.seed, uint32_t(pix), s, img, sx, sy);
        const int x = pix % W, y = pix / W;
        float ix = (float)x / W + (1.f / W) * sx;
        float iy = (float)y / H + (1.f / H) * sy;
        // PerscpectiveCamera::GenerateRay (perspective_camera.cpp:25-38)
        float cx = (ix - 0.5f) * cam.dimx, cy = (iy - 0.5f) * cam.dimy;
        v3 d = normalize(add(add(muls(mk(cam.fwd[0], cam.fwd[1], cam.fwd[2]), cam.znear),
                                 muls(mk(cam.right[0], cam.right[1], cam.right[2]), cx)),
                             muls(mk(cam.up[0], cam.up[1], cam.up[2]), cy)));
        put_ray(Q.ext_rays_in, i, mk(cam.p[0], cam.p[1], cam.p[2]), cam.znear, d, cam.zfar);
        Q.ext_path_in[i] = path;
        if (Q.ext_root_in) Q.ext_root_in[i] = Q.jobs[G.job].root;
        P.key[path] = key;
        P.cnt[path] = 6u;
        P.rng[path] = make_uint4(lr.z, lr.w, br.z, br.w);
        P.thr[path] = make_float4(1.f, 1.f, 1.f, 0.f);
        P.rad[path] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
        P.flags[path] = ((train_stride > 0 && (path + train_phase) % train_stride == 0) ? kFlagTrain : 0u) |
                        (unsigned(G.job) << 16);
        P.sample_rad[path] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *Q.n_ext_in = total;
}

// Adds the pending direct-light slots of a path (slots from `slot0`, DI
// throughput at `di`) into its radiance in light order: di = ls + bs per light
// (GetDi), radiance += (throughput * di) * mult.
__device__ __forceinline__ v3 gather_pending(const PathState& P, size_t slot0, size_t di, v3 rad, int pending) {
    if (pending == 0) return rad;
    float4 dt = P.dithr[di];
    v3 thr = mk(dt.x, dt.y, dt.z);
    const float4* sl = P.slots + slot0;
    for (int j = 0; j < pending; j += 2) {
        float4 a = sl[j], b = sl[j + 1];
        v3 di = add(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
        rad = add(rad, muls(mulv(thr, di), dt.w));
    }
    return rad;
}

struct ShadeArgs {
    int bounce, maxdepth, kind, kmax, batched;
    int cache_depth;              // -1: plain tracer
    int train_end;                // training paths end into the cache here (-1: they run to maxdepth)
    int train_stride;
    float ao_radius;              // BG_TRACER_AO
    int defer;                    // direct light resolved one bounce late (slot halves by bounce parity)
    int cap;                      // paths per pass (size of one slot half / 2 kmax)
};

// Radiance-cache query record of a surface point: position, outgoing
// direction, shading normal, roughness, albedo (layout of bg_cache_query).
__device__ __forceinline__ void cache_features(const SHit& h, v3 wo, const MatRec& M, float4 (&f)[4]) {
    float rough = 0.f, ar = 0.f, ag = 0.f, ab = 0.f;
    if (M.type == BG_MAT_LAMBERT) {
        rough = 1.f; ar = M.kd[0]; ag = M.kd[1]; ab = M.kd[2];
    } else if (M.type == BG_MAT_MICROFACET_GGX) {
        float r0 = (M.eta - 1.f) / (M.eta + 1.f);
        r0 *= r0;
        rough = M.a; ar = r0 * M.ks[0]; ag = r0 * M.ks[1]; ab = r0 * M.ks[2];
    }
    f[0] = make_float4(h.p.x, h.p.y, h.p.z, wo.x);
    f[1] = make_float4(wo.y, wo.z, h.n.x, h.n.y);
    f[2] = make_float4(h.n.z, rough, ar, ag);
    f[3] = make_float4(ab, 0.f, 0.f, 0.f);
}

// One light's DirectIllumination terms (DiTracer::GetDi, ditracer.cpp:57-239, n = 1).
// AREA = false: no light of the scene is an area light.  INL: BSDF and light
// sampling inline (the material-class kernels) instead of out of line.
template <bool AREA, bool INL>
__device__ __forceinline__ void emit_di(const DevScene& S, const Queues& Q, int li, const SHit& h, const MatRec& M, v3 wo,
                                        McRng& lr, McRng& br, int slot0, int path, int root) {
    const LightRec L = load_light(S, li);
    float lx, ly, bx, by;
    sample2d(lr, lx, ly);
    sample2d(br, bx, by);
    const bool singular = light_singular(L);
    float lightpdf = 0.f, bsdfpdf = 0.f;
    v3 ldir;
    v3 le = light_getsample<AREA, INL>(S, L, h, lx, ly, ldir, lightpdf);
    if (lightpdf > BG_MINPDF && sqnorm(le) > 0.f) {
        v3 wi = normalize(ldir);
        float dist = sqrtf(sqnorm(ldir));
        v3 bsdf = mat_eval<INL>(M, h, wi, wo);
        float c = fabsf(dot(h.n, wi));
        v3 ls;
        if (singular) {
            ls = muls(muls(mulv(le, bsdf), c), (1.f / lightpdf));
        } else {
            bsdfpdf = mat_pdf<INL>(M, h, wi, wo);
            float w = power_heuristic(lightpdf, bsdfpdf);
            ls = muls(muls(muls(mulv(le, bsdf), c), w), (1.f / lightpdf));
        }
        if (sqnorm(ls) > 0.f) {
            int e = warp_push(Q.n_sh);
            put_ray(Q.sh_rays, e, h.p, 0.01f, wi, dist - 0.01f);
            Q.sh_contrib[e] = make_float4(ls.x, ls.y, ls.z, 0.f);
            Q.sh_slot[e] = slot0;
            if (root >= 0) Q.sh_root[e] = root;
        }
    }
    if (!singular) {
        int type = 0;
        v3 wi;
        v3 f = mat_sample<INL>(M, h, bx, by, wo, wi, bsdfpdf, type);
        wi = normalize(wi);
        if (sqnorm(f) > 0.f && bsdfpdf > BG_MINPDF) {
            float w = 1.f;
            bool skip = false;
            if (!(type & kBsdfSpecular)) {
                float lp = light_getpdf<AREA>(S, L, h, wi);
                if (lp < BG_MINPDF) skip = true;
                else w = power_heuristic(bsdfpdf, lp);
            }
            if (!skip) {
                float c = fabsf(dot(h.n, wi));
                if (!AREA || L.type == BG_LIGHT_ENVIRONMENT) {
                    // a hit anywhere gives 0 (no bundle points at this light); a miss gives GetLe
                    v3 lev = mk(L.env[0], L.env[1], L.env[2]);
                    v3 bs = muls(muls(muls(mulv(lev, f), c), w), (1.f / bsdfpdf));
                    if (sqnorm(bs) > 0.f) {
                        int e = warp_push(Q.n_sh);
                        put_ray(Q.sh_rays, e, h.p, 0.01f, wi, 10000000.f);
                        Q.sh_contrib[e] = make_float4(bs.x, bs.y, bs.z, 0.f);
                        Q.sh_slot[e] = slot0 + 1;
                        if (root >= 0) Q.sh_root[e] = root;
                    }
                } else {
                    int e = warp_push(Q.n_mis);
                    put_ray(Q.mis_rays, e, h.p, 0.01f, wi, 10000000.f);
                    Q.mis_a[e] = make_float4(f.x, f.y, f.z, c);
                    Q.mis_b[e] = make_float4(h.p.x, h.p.y, h.p.z, w);
                    Q.mis_c[e] = make_int4(path, slot0 + 1, li, __float_as_int(1.f / bsdfpdf));
                    if (root >= 0) Q.mis_root[e] = root;
                }
            }
        }
    }
}

// One instantiation per tracer kind, cache mode and area-light presence keeps
// each kernel's code (and its instruction-cache footprint and registers) to
// what that configuration runs.
//
// MAT: the material class of the hits this kernel shades (kMatAny: any, the
// type read per hit; BG_MAT_LAMBERT / BG_MAT_MICROFACET_GGX: only hits on that
// material; kMatOther: misses and emissive hits).  A class kernel compiles
// only its own BSDF, inline, so it needs fewer registers and no call frame.
constexpr int kMatAny = -1;
constexpr int kMatOther = BG_MAT_EMISSIVE;

template <int KIND, bool CACHE, bool AREA, int MAT>
__device__ __forceinline__ void shade_path(const DevScene& S, const ShadeArgs& A, const PathState& P, const Queues& Q,
                                           int e) {
    // deferred mode: this bounce's DI goes to half h, which held the DI of bounce
    // - 2 (gathered first); half 1 - h (bounce - 1) is still being resolved
    const int h = A.bounce & 1;
    const size_t shalf = A.defer ? size_t(h) * size_t(A.cap) * size_t(A.kmax) : 0;
    const size_t dhalf = A.defer ? size_t(h) * size_t(A.cap) : 0;
    {
        const int path = Q.ext_path_in[e];
        bg_hit hit = Q.ext_hits[e];
        if (hit.primid >= 0) hit.primid &= kPrimMask;   // the material class rides in bits 28-29
        const float4 rd = Q.ext_rays_in[2 * e + 1];
        const v3 d = mk(rd.x, rd.y, rd.z);
        float4 r4 = P.rad[path];
        v3 rad = mk(r4.x, r4.y, r4.z);
        const int packed = __float_as_int(r4.w);
        rad = gather_pending(P, shalf + size_t(path) * A.kmax, dhalf + path, rad,
                             A.defer ? pend_get(packed, h) : packed);
        const JobRec J = Q.jobs[P.flags[path] >> 16];
        const int root = A.batched ? J.root : -1;
        unsigned flags = 0u;
        int pending = 0;
        bool end = false;
        if (hit.primid < 0) {
            if (KIND == BG_TRACER_AO) {
                flags |= kFlagNoClamp;  // AoTracer: a miss is black (aotracer.cpp:47)
            } else if (A.bounce == 0) { // primary miss: bgcolor + sum of GetLe, unclamped (gitracer.cpp:22-33)
                rad = add(rad, mk(J.bg[0], J.bg[1], J.bg[2]));
                for (int i = J.light0; i < J.light0 + J.nlights; ++i) {
                    LightRec L = load_light(S, i);
                    if (L.type == BG_LIGHT_ENVIRONMENT) rad = add(rad, mk(L.env[0], L.env[1], L.env[2]));
                }
                flags |= kFlagNoClamp;
            }
            end = true;
        } else {
            SHit h;
            fill_hit(S, hit.primid, hit.u, hit.v, h);
            uint4 rg = P.rng[path];
            McRng lr{rg.x, rg.y}, br{rg.z, rg.w};
            float2 bs;
            if (A.bounce == 0 && KIND == BG_TRACER_GI) {
                sample2d(br, bs.x, bs.y);
                P.bs[path] = bs;
            } else {
                bs = P.bs[path];
            }
            MatRec M = load_mat(S, h.m);
            if (MAT != kMatAny) M.type = MAT;   // a class kernel: the material type is a constant
            const v3 wo = neg(d);
            float4 t4 = P.thr[path];
            v3 thr = mk(t4.x, t4.y, t4.z);
            const unsigned pflags = P.flags[path];
            const bool train = (pflags & kFlagTrain) != 0;
            flags = pflags;
            if (KIND == BG_TRACER_AO) {
                // AoTracer::GetLi (aotracer.cpp:9-49), one light-sampler sample:
                // a cosine ray about the shading normal, t in (0.00002, radius);
                // the visibility 1 lands in the first slot unless the ray is occluded
                float ax, ay;
                sample2d(lr, ax, ay);
                const v3 dir = map_to_hemisphere(h.n, ax, ay, 1.f);
                const int base = int(shalf) + path * A.kmax;
                P.slots[size_t(base)] = make_float4(0.f, 0.f, 0.f, 0.f);
                P.slots[size_t(base) + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
                const int k = warp_push(Q.n_sh);
                put_ray(Q.sh_rays, k, h.p, 0.00002f, dir, A.ao_radius);
                Q.sh_contrib[k] = make_float4(1.f, 1.f, 1.f, 0.f);
                Q.sh_slot[k] = base;
                if (root >= 0) Q.sh_root[k] = root;
                P.dithr[dhalf + path] = make_float4(1.f, 1.f, 1.f, 1.f);
                pending = 2;
                flags |= kFlagNoClamp;
                P.rng[path] = make_uint4(lr.z, lr.w, br.z, br.w);
                end = true;
            } else if (A.bounce == 0 && M.type == BG_MAT_EMISSIVE) {
                if (KIND == BG_TRACER_GI) rad = add(rad, emissive_le(M, h.n, wo));   // gitracer.cpp:61-68
                if (KIND == BG_TRACER_DI) flags |= kFlagNoClamp;                    // ditracer.cpp:29-32
                end = true;
            } else if ((CACHE && A.cache_depth >= 0) &&
                       ((!train && A.bounce == A.cache_depth) || (train && A.bounce == A.train_end))) {
                // the rendering path ends into the radiance cache at this vertex; so
                // does a training path at the end of its suffix (self-training: its
                // recorded vertices learn from the cache's own prediction here)
                float4 f[4];
                cache_features(h, wo, M, f);
                int q = warp_push(Q.n_query);
#pragma unroll
                for (int k = 0; k < 4; ++k) Q.q_feat[4 * q + k] = f[k];
                Q.q_path[q] = path;
                Q.q_thr[q] = make_float4(thr.x, thr.y, thr.z, 0.f);
                end = true;
            } else {
                if ((CACHE && A.cache_depth >= 0) && train && A.bounce >= A.cache_depth) {
                    // training path: remember the vertex, its throughput and the radiance so far
                    // (from cache_depth on: the depths at which the cache is queried)
                    const int t = path / A.train_stride;   // training paths are train_stride apart
                    float4* rr = P.rec + (size_t(t) * A.maxdepth + A.bounce) * 6;
                    float4 f[4];
                    cache_features(h, wo, M, f);
#pragma unroll
                    for (int k = 0; k < 4; ++k) rr[k] = f[k];
                    rr[4] = make_float4(thr.x, thr.y, thr.z, 0.f);
                    rr[5] = make_float4(rad.x, rad.y, rad.z, 0.f);
                    flags = (flags & ~0xff00u) | (unsigned(A.bounce + 1) << 8);
                }
                unsigned cnt = P.cnt[path];
                const int base = int(shalf) + path * A.kmax;
                // bounce 0: every light, weight 1; later: one light picked by rand(), weight L
                // (gitracer.cpp:72-84)
                int first = J.light0, nl = J.nlights;
                float mult = 1.f;
                if (A.bounce != 0) {
                    first = J.light0 + int(keyed_rand(P.key[path], cnt++) % unsigned(J.nlights));
                    nl = 1;
                    mult = (float)J.nlights;
                }
                pending = 2 * nl;
                for (int j = 0; j < pending; ++j) P.slots[size_t(base) + j] = make_float4(0.f, 0.f, 0.f, 0.f);
                for (int i = 0; i < nl; ++i)
                    emit_di<AREA, MAT != kMatAny>(S, Q, first + i, h, M, wo, lr, br, base + 2 * i, path, root);
                P.dithr[dhalf + path] = make_float4(thr.x, thr.y, thr.z, mult);
                if (KIND == BG_TRACER_DI) {
                    flags |= kFlagNoClamp;
                    end = true;
                } else {
                    // continue the path with the reused BSDF sample (gitracer.cpp:87-134)
                    int type = 0;
                    float pdf = 0.f;
                    v3 wi;
                    v3 f = mat_sample<MAT != kMatAny>(M, h, bs.x, bs.y, wo, wi, pdf, type);
                    if (sqnorm(f) == 0.f || pdf < BG_MINPDF) {
                        end = true;
                    } else {
                        v3 nd = normalize(wi);
                        thr = mulv(thr, muls(f, (fabsf(dot(h.n, wi)) / pdf)));
                        if (A.bounce > 3) {
                            float rnd = rand_float(keyed_rand(P.key[path], cnt++));
                            float lum = 0.2126f * thr.x + 0.7152f * thr.y + 0.0722f * thr.z;
                            float q = fmin_std(0.5f, lum);
                            if (rnd > q) end = true;
                            else thr = muls(thr, (1.f / q));
                        }
                        if (!end && A.bounce + 1 >= A.maxdepth) end = true;   // loop ends before the next hit is used
                        if (!end) {
                            int k = warp_push(Q.n_ext_out);
                            put_ray(Q.ext_rays_out, k, h.p, 0.01f, nd, 1000000.f);
                            Q.ext_path_out[k] = path;
                            if (root >= 0) Q.ext_root_out[k] = root;
                        }
                        P.thr[path] = make_float4(thr.x, thr.y, thr.z, 0.f);
                    }
                }
                P.cnt[path] = cnt;
                P.rng[path] = make_uint4(lr.z, lr.w, br.z, br.w);
            }
        }
        P.rad[path] = make_float4(rad.x, rad.y, rad.z, __int_as_float(A.defer ? pend_set(packed, h, pending) : pending));
        if (hit.primid < 0) flags |= P.flags[path];
        P.flags[path] = flags;
        if (end) {
            int k = warp_push(Q.n_end);
            Q.end_path[k] = path;
        }
    }
}

// Every hit of the extension queue, material read per hit.
template <int KIND, bool CACHE, bool AREA>
__global__ void __launch_bounds__(kShadeThreads, 8)   // 64 registers (measured: 8 > 7 > 10 > 6 blocks / SM)
k_shade(DevScene S, ShadeArgs A, PathState P, Queues Q) {
    const int n = *Q.n_ext_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) Q.totals[0] += (unsigned long long)n;
    const int nthreads = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += nthreads)
        shade_path<KIND, CACHE, AREA, kMatAny>(S, A, P, Q, e);
}

// (Measured and rejected: tracing the secondary extension and shadow queues in
// the order of their rays' direction octants, a counting sort in 256-entry
// blocks: every k_trace launch of a C3 frame got 4-7 % slower, as a lane refill
// then draws its rays from an 8 times wider stretch of the queue, i.e. of the
// image, and the sort cost 3 % of the frame besides.)

// Splits the extension queue by material class: list c of Q.cls (entries
// c * cap ..) receives the queue indices of the hits of class c (0 = misses and
// emissive, 1 = Lambert, 2 = GGX), in queue order within a block.  The class
// comes with the hit (bits 28-29 of primid, written by the extension trace
// from TriRec e2.w), so this reads 16 bytes per ray and makes three atomics
// per block of kClassifyThreads rays.
constexpr int kClassifyThreads = 512;
__global__ void __launch_bounds__(kClassifyThreads)
k_classify(Queues Q, int cap) {
    __shared__ int wcount[kClassifyThreads / 32][3];
    __shared__ int base[3];
    const int n = *Q.n_ext_in;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (int start = blockIdx.x * kClassifyThreads; start < n; start += gridDim.x * kClassifyThreads) {
        const int e = start + int(threadIdx.x);
        int cls = -1;
        if (e < n) {
            const int prim = Q.ext_hits[e].primid;
            cls = prim < 0 ? 0 : (prim >> kClassShift) & 3;
        }
        unsigned m[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            m[c] = __ballot_sync(0xffffffffu, cls == c);
            if (lane == 0) wcount[warp][c] = __popc(m[c]);
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            const int c = int(threadIdx.x);
            int tot = 0;
            for (int w = 0; w < kClassifyThreads / 32; ++w) {
                const int k = wcount[w][c];
                wcount[w][c] = tot;                       // exclusive offset of warp w
                tot += k;
            }
            base[c] = tot ? atomicAdd(Q.n_cls + c, tot) : 0;
        }
        __syncthreads();
        if (cls >= 0) {
            const unsigned mine = cls == 0 ? m[0] : cls == 1 ? m[1] : m[2];
            Q.cls[size_t(cls) * cap + base[cls] + wcount[warp][cls] + __popc(mine & ((1u << lane) - 1u))] = e;
        }
        __syncthreads();
    }
}

// The hits of one material class (list MAT of k_classify).
// 5 blocks of 128 threads per SM: 96 registers; no spills in the Lambert
// kernel, 4 bytes in the GGX one (measured per step of C3: 8 blocks 9.6 ms of
// shading, 6 blocks 9.3 ms, 5 blocks 8.8 ms, 4 blocks 0.3 ms slower than 5).
// The area-light instantiations spill 140-200 bytes at 96 registers, but the
// same 5 blocks serve them best (C1 GiTracer: 4 blocks with 128 registers
// 587 Msamples/s, 5 blocks 699, 6 blocks 685, 8 blocks 665).
constexpr int kShadeClassBlocks = 5;
// (Measured and rejected: the misses-and-emissive kernel at 8 blocks / SM on
// the full grid, 0.15 ms per C3 step slower in the serial phase timing.)
template <int KIND, bool CACHE, bool AREA, int MAT>
__global__ void __launch_bounds__(kShadeThreads, kShadeClassBlocks)
k_shade_class(DevScene S, ShadeArgs A, PathState P, Queues Q) {
    constexpr int c = MAT == BG_MAT_LAMBERT ? 1 : MAT == BG_MAT_MICROFACET_GGX ? 2 : 0;
    const int n = Q.n_cls[c];
    if (MAT == kMatOther && blockIdx.x == 0 && threadIdx.x == 0) Q.totals[0] += (unsigned long long)*Q.n_ext_in;
    const int nthreads = gridDim.x * blockDim.x;
    const int* list = Q.cls + size_t(c) * A.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nthreads)
        shade_path<KIND, CACHE, AREA, MAT>(S, A, P, Q, list[i]);
}

// Material-class kernels of one configuration: classify, then misses and
// emissive hits, Lambert hits and GGX hits, each by its own kernel.
// (Measured: one kernel for every material, 64 registers and out-of-line BSDF
// calls, shaded a C3 step in 11.6 ms; the class kernels take 6.3 ms.)
template <int KIND, bool CACHE, bool AREA>
static int launch_shade_split(const DevScene& d, int nb, int nbc, cudaStream_t st, const ShadeArgs& A,
                              const PathState& P, const Queues& Q) {
    BG_CUDA(cudaMemsetAsync(Q.n_cls, 0, 3 * sizeof(int), st));
    k_classify<<<nb, kClassifyThreads, 0, st>>>(Q, A.cap);
    k_shade_class<KIND, CACHE, AREA, kMatOther><<<nbc, kShadeThreads, 0, st>>>(d, A, P, Q);
    k_shade_class<KIND, CACHE, AREA, BG_MAT_LAMBERT><<<nbc, kShadeThreads, 0, st>>>(d, A, P, Q);
    k_shade_class<KIND, CACHE, AREA, BG_MAT_MICROFACET_GGX><<<nbc, kShadeThreads, 0, st>>>(d, A, P, Q);
    return BG_OK;
}

// The shading kernels for a tracer kind, cache mode and the scene's lights.
// Returns the number of kernels launched (< 0: an error code).  AoTracer has no
// BSDF: its paths are shaded by one kernel.
static int launch_shade(const DevScene& d, int kind, bool cache, int nb, int nbc, cudaStream_t st,
                        const ShadeArgs& A, const PathState& P, const Queues& Q) {
    const bool area = d.has_area != 0;
    if (kind == BG_TRACER_AO) {
        k_shade<BG_TRACER_AO, false, false><<<nb, kShadeThreads, 0, st>>>(d, A, P, Q);
        return 1;
    }
    int rc;
    if (kind == BG_TRACER_DI)
        rc = area ? launch_shade_split<BG_TRACER_DI, false, true>(d, nb, nbc, st, A, P, Q)
                  : launch_shade_split<BG_TRACER_DI, false, false>(d, nb, nbc, st, A, P, Q);
    else if (cache)
        rc = area ? launch_shade_split<BG_TRACER_GI, true, true>(d, nb, nbc, st, A, P, Q)
                  : launch_shade_split<BG_TRACER_GI, true, false>(d, nb, nbc, st, A, P, Q);
    else
        rc = area ? launch_shade_split<BG_TRACER_GI, false, true>(d, nb, nbc, st, A, P, Q)
                  : launch_shade_split<BG_TRACER_GI, false, false>(d, nb, nbc, st, A, P, Q);
    return rc ? rc : 4;
}

// BSDF-sampled rays towards area lights: the closest hit must be on a bundle
// whose (last registered) area light is this one, front facing
// (ditracer.cpp:199-220).
__global__ void __launch_bounds__(kShadeThreads)
k_resolve_mis(DevScene S, PathState P, Queues Q) {
    const int n = *Q.n_mis;
    const int nthreads = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += nthreads) {
        const bg_hit hit = Q.mis_hits[e];
        if (hit.primid < 0) continue;   // area lights emit nothing on a miss
        const int4 c = Q.mis_c[e];
        const int bundle = __float_as_int(__ldg(&S.shade[hit.primid].a.w));
        if (__ldg(&S.bundles[bundle].arealight) != c.z) continue;
        SHit h;
        fill_hit(S, hit.primid, hit.u, hit.v, h);
        const float4 rd = Q.mis_rays[2 * e + 1];
        const v3 wi = mk(rd.x, rd.y, rd.z);
        const float4 a = Q.mis_a[e], b = Q.mis_b[e];
        v3 dd = sub(h.p, mk(b.x, b.y, b.z));
        if (!(dot(h.n, neg(wi)) > 0.f)) continue;
        float d2inv = 1.f / sqnorm(dd);
        const MatRec M = load_mat(S, h.m);
        if (M.type != BG_MAT_EMISSIVE) continue;
        v3 le = muls(emissive_le(M, h.n, neg(wi)), d2inv);
        if (!(sqnorm(le) > 0.f)) continue;
        v3 bs = muls(muls(muls(mulv(le, mk(a.x, a.y, a.z)), a.w), b.w), __int_as_float(c.w));
        P.slots[c.y] = make_float4(bs.x, bs.y, bs.z, 0.f);
    }
}

__global__ void __launch_bounds__(kShadeThreads)
k_finalize(PathState P, Queues Q, int kmax, int maxdepth, int train_stride, int train_from, int bounce, int defer,
           int cap) {
    const int n = *Q.n_end;
    const int nthreads = gridDim.x * blockDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) {   // the bounce's shadow and MIS rays (statistics)
        Q.totals[1] += (unsigned long long)*Q.n_sh;
        Q.totals[2] += (unsigned long long)*Q.n_mis;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += nthreads) {
        const int path = Q.end_path[e];
        float4 r4 = P.rad[path];
        const int packed = __float_as_int(r4.w);
        v3 rad = mk(r4.x, r4.y, r4.z);
        if (defer) {   // the previous bounce's DI, then this bounce's
            const int h = bounce & 1, g = h ^ 1;
            rad = gather_pending(P, size_t(g) * cap * kmax + size_t(path) * kmax, size_t(g) * cap + path, rad,
                                 pend_get(packed, g));
            rad = gather_pending(P, size_t(h) * cap * kmax + size_t(path) * kmax, size_t(h) * cap + path, rad,
                                 pend_get(packed, h));
        } else {
            rad = gather_pending(P, size_t(path) * kmax, size_t(path), rad, packed);
        }
        const unsigned fl = P.flags[path];
        const int nv = int((fl >> 8) & 0xffu);
        if ((fl & kFlagTrain) && nv > 0 && train_stride > 0) {
            // one training sample per recorded vertex: radiance gathered from that
            // vertex on, divided by the throughput that reached it
            const int t = path / train_stride;
            for (int k = train_from; k < nv; ++k) {
                const float4* rr = P.rec + (size_t(t) * maxdepth + k) * 6;
                const float4 tk = rr[4], rb = rr[5];
                if (!(tk.x > 1e-6f && tk.y > 1e-6f && tk.z > 1e-6f)) continue;
                int q = warp_push(Q.n_train);
                if (q >= Q.tr_cap) continue;
#pragma unroll
                for (int j = 0; j < 4; ++j) Q.tr_feat[4 * q + j] = rr[j];
                Q.tr_target[q] = make_float4((rad.x - rb.x) / tk.x, (rad.y - rb.y) / tk.y, (rad.z - rb.z) / tk.z, 0.f);
            }
        }
        if (!(fl & kFlagNoClamp)) {
            v3 r = muls(rad, (1.f / 1));
            rad = mk(clamp_ref(r.x, 0.f, BG_MAXRADIANCE), clamp_ref(r.y, 0.f, BG_MAXRADIANCE), clamp_ref(r.z, 0.f, BG_MAXRADIANCE));
        }
        P.sample_rad[path] = make_float4(rad.x, rad.y, rad.z, 1.f);
    }
}

// rendering paths that ended into the cache: radiance += throughput * max(prediction, 0)
__global__ void __launch_bounds__(kShadeThreads)
k_cache_resolve(PathState P, Queues Q, const float4* __restrict__ pred) {
    const int n = *Q.n_query;
    const int nthreads = gridDim.x * blockDim.x;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += nthreads) {
        const int path = Q.q_path[q];
        const float4 p = pred[q], t = Q.q_thr[q];
        float4 r = P.rad[path];
        r.x += t.x * fmaxf(p.x, 0.f);
        r.y += t.y * fmaxf(p.y, 0.f);
        r.z += t.z * fmaxf(p.z, 0.f);
        P.rad[path] = r;
    }
}

// FileImagePlane::WriteSample per pixel, samples in order (rows flipped).
__global__ void __launch_bounds__(kShadeThreads)
k_accumulate(PathState P, const SegRec* __restrict__ segs, int nseg, int npix) {
    const int nthreads = gridDim.x * blockDim.x;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npix; t += nthreads) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (segs[mid].pix0 <= t) lo = mid; else hi = mid - 1;
        }
        const SegRec& G = segs[lo];
        const int i = t - G.pix0;
        const int pix = G.p0 + i;
        const int x = pix % G.W, y = pix / G.W;
        float4* px = G.accum + size_t(G.W) * size_t(G.H - 1 - y) + x;
        float4 acc = *px;
        for (int s = 0; s < G.ns; ++s) {
            float4 v = P.sample_rad[size_t(G.path0) + size_t(s) * G.np + i];
            acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += 1.f;
        }
        *px = acc;
    }
}

CamDev make_camera(const bg_camera_desc* c) {
    CamDev k;
    v3 eye = mk(c->eye[0], c->eye[1], c->eye[2]), at = mk(c->at[0], c->at[1], c->at[2]), up = mk(c->up[0], c->up[1], c->up[2]);
    v3 fwd = normalize(sub(at, eye));
    v3 right = cross(fwd, normalize(up));
    v3 u = cross(right, fwd);
    k.fwd[0] = fwd.x; k.fwd[1] = fwd.y; k.fwd[2] = fwd.z;
    k.right[0] = right.x; k.right[1] = right.y; k.right[2] = right.z;
    k.up[0] = u.x; k.up[1] = u.y; k.up[2] = u.z;
    k.p[0] = eye.x; k.p[1] = eye.y; k.p[2] = eye.z;
    k.znear = c->znear;
    k.zfar = c->zfar;
    k.dimx = 2 * tanf(c->fovy * 0.5f) * c->znear;
    k.dimy = k.dimx / c->aspect;
    return k;
}

// DevBuf::ensure that bumps the render state's buffer epoch when the buffer
// moves, so no captured pass is replayed with the old address.
static int ensure_tracked(RenderState* rs, DevBuf& b, size_t need) {
    const void* before = b.ptr;
    const int rc = b.ensure(need);
    if (b.ptr != before) ++rs->buf_epoch;
    return rc;
}

static int alloc_state(bg_scene* s, RenderState* rs, int64_t cap, int L) {
    rs->cap = cap;
    rs->nlights = L;
    rs->kmax = 2 * L;
    const size_t C = size_t(cap);
    int rc;
    for (int k = 0; k < 2; ++k) {
        if ((rc = rs->ext_rays[k].ensure(C * 32)) || (rc = rs->ext_path[k].ensure(C * 4)) ||
            (rc = rs->ext_root[k].ensure(C * 4)))
            return rc;
    }
    // shadow / MIS / ended-path queues, DI slots and DI throughput come in two
    // halves (bounce parity) for passes that resolve direct light one bounce late
    if (C * size_t(rs->kmax) * 2 >= (size_t(1) << 31))
        return set_error(BG_ERR_UNSUPPORTED, "paths per pass x light slots too large (%zu x %d)", C, rs->kmax);
    if ((rc = rs->ext_hits.ensure(C * 16)) ||
        (rc = rs->sh_rays.ensure(2 * C * 2 * L * 32)) || (rc = rs->sh_contrib.ensure(2 * C * 2 * L * 16)) ||
        (rc = rs->sh_slot.ensure(2 * C * 2 * L * 4)) ||
        (rc = rs->sh_root.ensure(2 * C * 2 * L * 4)) ||
        (rc = rs->mis_rays.ensure(2 * C * L * 32)) || (rc = rs->mis_a.ensure(2 * C * L * 16)) ||
        (rc = rs->mis_b.ensure(2 * C * L * 16)) || (rc = rs->mis_c.ensure(2 * C * L * 16)) ||
        (rc = rs->mis_hits.ensure(2 * C * L * 16)) || (rc = rs->mis_root.ensure(2 * C * L * 4)) ||
        (rc = rs->end_path.ensure(2 * C * 4)) || (rc = rs->cls.ensure(3 * C * 4)) ||
        (rc = rs->counts.ensure(256)) ||
        (rc = rs->st_key.ensure(C * 8)) || (rc = rs->st_cnt.ensure(C * 4)) || (rc = rs->st_rng.ensure(C * 16)) ||
        (rc = rs->st_bs.ensure(C * 8)) || (rc = rs->st_thr.ensure(C * 16)) || (rc = rs->st_rad.ensure(C * 16)) ||
        (rc = rs->st_dithr.ensure(2 * C * 16)) || (rc = rs->st_flags.ensure(C * 4)) ||
        (rc = rs->slots.ensure(2 * C * rs->kmax * 16)) || (rc = rs->sample_rad.ensure(C * 16)) ||
        (rc = rs->cnt_out.ensure((C * 2 * L / 64 + 64) * 16)) ||
        (rc = rs->work.ensure(size_t(kMaxBounceCounters) * 8)))
        return rc;
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade<BG_TRACER_AO, false, false>, kShadeThreads, 0);
    rs->blocks = std::max(1, nb) * s->ctx->num_sms;
    nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade_class<BG_TRACER_GI, false, false, BG_MAT_MICROFACET_GGX>,
                                                  kShadeThreads, 0);
    rs->blocks_class = std::max(1, nb) * s->ctx->num_sms;
    BG_CUDA(cudaStreamCreateWithFlags(&rs->gstream, cudaStreamNonBlocking));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_in, cudaEventDisableTiming));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_out, cudaEventDisableTiming));
    BG_CUDA(cudaStreamCreateWithFlags(&rs->fstream, cudaStreamNonBlocking));
    BG_CUDA(cudaStreamCreateWithFlags(&rs->tstream, cudaStreamNonBlocking));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_tstart, cudaEventDisableTiming));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_train, cudaEventDisableTiming));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_fork, cudaEventDisableTiming));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_join, cudaEventDisableTiming));
    BG_CUDA(cudaStreamCreateWithFlags(&rs->mstream, cudaStreamNonBlocking));
    BG_CUDA(cudaEventCreateWithFlags(&rs->ev_mjoin, cudaEventDisableTiming));
    return BG_OK;
}

// Path state and queues for passes of `cap` paths with up to maxL lights per
// job; a failed allocation leaves no state behind (the next call starts over).
static int ensure_state(bg_scene* s, int64_t cap, int maxL) {
    const int L = std::max(1, maxL);
    if (s->render && s->render->cap >= cap && s->render->nlights == L) return BG_OK;
    if (s->render) render_state_free(s->render);
    s->render = new RenderState();
    const int rc = alloc_state(s, s->render, cap, L);
    if (rc) {
        render_state_free(s->render);
        s->render = nullptr;
    }
    return rc;
}

struct Instr {
    bool time_phases = false, count_trav = false;
    cudaStream_t st = nullptr;
    std::vector<cudaEvent_t> evs;   // begin/end pairs; phase tag in tags
    std::vector<int> tags;
    int64_t launches = 0;
    int launches_extend = 0;
    void mark(int tag) {
        if (!time_phases) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        evs.push_back(e);
        tags.push_back(tag);
    }
};

// One pass: a slice of the device segment table plus the bounce-loop settings.
struct PassCfg {
    const SegRec* segs;        // device pointer to this pass's segments
    int nseg, total, npix;
    int maxdepth, kind;
    bool batched;
    bg_cache* cache;           // radiance-cache mode when non-null
    int cache_depth, train_end, train_stride, train_phase;
    bool wait_train;           // the first query stage waits for RenderState::ev_train
    float ao_radius;
};

// Queue pointers of a bounce: extension queue `c` in, 1 - c out; shadow, MIS
// and ended-path queues and their counters of parity `par`.
static void pass_queues(RenderState* rs, int c, bool batched, Queues& Q, int par = 0) {
    int* cnt = rs->counts.as<int>();
    const size_t C = size_t(rs->cap), L = size_t(rs->nlights);
    const size_t sh = par ? C * 2 * L : 0, mi = par ? C * L : 0;   // entries before this parity's half
    Q.ext_hits = rs->ext_hits.as<bg_hit>();
    Q.sh_rays = rs->sh_rays.as<float4>() + 2 * sh; Q.sh_contrib = rs->sh_contrib.as<float4>() + sh;
    Q.sh_slot = rs->sh_slot.as<int>() + sh;
    Q.mis_rays = rs->mis_rays.as<float4>() + 2 * mi; Q.mis_a = rs->mis_a.as<float4>() + mi;
    Q.mis_b = rs->mis_b.as<float4>() + mi;
    Q.mis_c = rs->mis_c.as<int4>() + mi; Q.mis_hits = rs->mis_hits.as<bg_hit>() + mi;
    Q.end_path = rs->end_path.as<int>() + (par ? C : 0);
    const int c0 = par ? kCntSh1 : kCntSh;
    Q.n_sh = cnt + c0; Q.n_mis = cnt + c0 + 1; Q.n_end = cnt + c0 + 2;
    Q.totals = reinterpret_cast<unsigned long long*>(rs->counts.as<char>() + 64);
    Q.ext_rays_in = rs->ext_rays[c].as<float4>(); Q.ext_path_in = rs->ext_path[c].as<int>();
    Q.ext_rays_out = rs->ext_rays[1 - c].as<float4>(); Q.ext_path_out = rs->ext_path[1 - c].as<int>();
    Q.n_ext_in = cnt + (c ? kCntExt1 : kCntExt0);
    Q.n_ext_out = cnt + (c ? kCntExt0 : kCntExt1);
    Q.q_feat = rs->q_feat.as<float4>(); Q.q_path = rs->q_path.as<int>(); Q.q_thr = rs->q_thr.as<float4>();
    Q.n_query = cnt + kCntQuery;
    Q.tr_feat = rs->tr_feat.as<float4>() + size_t(rs->tr_set) * rs->tr_cap * 4;
    Q.tr_target = rs->tr_target.as<float4>() + size_t(rs->tr_set) * rs->tr_cap;
    Q.n_train = cnt + kCntTrain + rs->tr_set;
    Q.tr_cap = int(rs->tr_cap);
    Q.ext_root_in = batched ? rs->ext_root[c].as<int>() : nullptr;
    Q.ext_root_out = batched ? rs->ext_root[1 - c].as<int>() : nullptr;
    Q.sh_root = batched ? rs->sh_root.as<int>() + sh : nullptr;
    Q.mis_root = batched ? rs->mis_root.as<int>() + mi : nullptr;
    Q.jobs = rs->jobs.as<JobRec>();
    Q.n_cls = cnt + kCntCls;
    Q.cls = rs->cls.as<int>();
}

static PathState path_state(RenderState* rs) {
    PathState P;
    P.key = rs->st_key.as<unsigned long long>();
    P.cnt = rs->st_cnt.as<unsigned>();
    P.rng = rs->st_rng.as<uint4>();
    P.bs = rs->st_bs.as<float2>();
    P.thr = rs->st_thr.as<float4>();
    P.rad = rs->st_rad.as<float4>();
    P.dithr = rs->st_dithr.as<float4>();
    P.flags = rs->st_flags.as<unsigned>();
    P.slots = rs->slots.as<float4>();
    P.sample_rad = rs->sample_rad.as<float4>();
    P.rec = rs->rec.as<float4>();
    return P;
}

// Enqueues one pass on `st`: generate, maxdepth bounces of extend / shade /
// shadow / MIS / resolve / finalize, accumulate.
static int enqueue_pass(bg_scene* s, RenderState* rs, cudaStream_t st, const PassCfg& c, Instr* ins) {
    const int nb = rs->blocks;
    PathState P = path_state(rs);
    Queues Q;
    int cur = 0;
    pass_queues(rs, cur, c.batched, Q);
    int* cnt = rs->counts.as<int>();
    int rc;
    k_generate<<<nb, kShadeThreads, 0, st>>>(c.segs, c.nseg, c.total, P, Q, c.cache ? c.train_stride : 0, c.train_phase);
    if (ins) ++ins->launches;
    bg_hit* cnt_hits = rs->cnt_out.as<bg_hit>();
    uint8_t* cnt_occ = rs->cnt_out.as<uint8_t>();
    // Without phase timing or traversal counting, the extension trace of bounce b + 1 runs on a
    // second stream beside bounce b's shadow and MIS traces, resolves and
    // finalize: it reads only the queue that shade(b) wrote and the hit buffer
    // shade(b) has finished with; the MIS trace and its resolve run on a third
    // stream beside the shadow trace.  The deep, nearly empty bounces are latency
    // chains (one ray's traversal is dozens of dependent node loads), so
    // running two chains side by side shortens the pass.
    const bool fork = (ins == nullptr || (!ins->time_phases && !ins->count_trav)) && rs->fstream != nullptr &&
                      rs->mstream != nullptr;
    const int depth = std::max(1, c.maxdepth);
    if (fork && !c.cache) {
        // Direct light resolved one bounce late.  Shade(b) gathers the DI of
        // bounce b - 2 and writes its own into the slot half of parity b, so the
        // main stream runs extension trace -> shade -> extension trace -> ...
        // while a side stream traces bounce b's shadow and MIS rays, resolves
        // them and finalizes the paths that ended at b; shade(b + 2) waits for
        // that.  Radiance is summed in the same order (every bounce's DI in turn,
        // and nothing else is added after bounce 0), so images are unchanged.
        cudaStream_t ds = rs->mstream;
        cudaEvent_t evd[2] = {rs->ev_join, rs->ev_mjoin};
        for (int b = 0; b < depth; ++b) {
            const int par = b & 1;
            unsigned long long* wk = rs->work.as<unsigned long long>() + 6 * b;
            pass_queues(rs, cur, c.batched, Q, par);
            if (b >= 2) BG_CUDA(cudaStreamWaitEvent(st, evd[par], 0));   // bounce b - 2's side work is done
            BG_CUDA(cudaMemsetAsync(Q.n_ext_out, 0, sizeof(int), st));
            BG_CUDA(cudaMemsetAsync(cnt + (par ? kCntSh1 : kCntSh), 0, 3 * sizeof(int), st));
            if (b == 0) {
                if ((rc = launch_trace(s, false, Q.ext_rays_in, 0, Q.n_ext_in, Q.ext_hits, nullptr, st, nullptr, 1, wk,
                                       Q.ext_root_in, &kExtTrace)))
                    return rc;
                if (ins) { ++ins->launches; ++ins->launches_extend; }
            }
            ShadeArgs A{b, c.maxdepth, c.kind, rs->kmax, c.batched ? 1 : 0, -1, -1, 0, c.ao_radius, 1, int(rs->cap)};
            const int nsh = launch_shade(s->dev, c.kind, false, nb, rs->blocks_class, st, A, P, Q);
            if (nsh < 0) return nsh;
            if (ins) ins->launches += nsh - 1;
            BG_CUDA(cudaEventRecord(rs->ev_fork, st));
            BG_CUDA(cudaStreamWaitEvent(ds, rs->ev_fork, 0));
            const ShadowResolve sr{Q.sh_contrib, Q.sh_slot, P.slots};
            if ((rc = launch_trace(s, true, Q.sh_rays, 0, Q.n_sh, nullptr, nullptr, ds, nullptr, 1, wk + 2, Q.sh_root,
                                   &sr)))
                return rc;
            if (s->dev.has_area) {   // MIS rays go to area lights only (the queue is empty otherwise)
                if ((rc = launch_trace(s, false, Q.mis_rays, 0, Q.n_mis, Q.mis_hits, nullptr, ds, nullptr, 1, wk + 3,
                                       Q.mis_root)))
                    return rc;
                k_resolve_mis<<<nb, kShadeThreads, 0, ds>>>(s->dev, P, Q);
                if (ins) ins->launches += 2;
            }
            k_finalize<<<nb, kShadeThreads, 0, ds>>>(P, Q, rs->kmax, c.maxdepth, 0, 0, b, 1, int(rs->cap));
            BG_CUDA(cudaEventRecord(evd[par], ds));
            if (ins) ins->launches += 3;
            if (b + 1 < depth) {
                cur = 1 - cur;
                Queues Qn;
                pass_queues(rs, cur, c.batched, Qn, par ^ 1);
                if ((rc = launch_trace(s, false, Qn.ext_rays_in, 0, Qn.n_ext_in, Qn.ext_hits, nullptr, st, nullptr, 1,
                                       wk + 6, Qn.ext_root_in, &kExtTrace)))
                    return rc;
                if (ins) { ++ins->launches; ++ins->launches_extend; }
            }
        }
        BG_CUDA(cudaStreamWaitEvent(st, evd[(depth - 1) & 1], 0));   // the side stream is in bounce order
    }
    for (int b = 0; b < depth && !(fork && !c.cache); ++b) {
        unsigned long long* wk = rs->work.as<unsigned long long>() + 6 * b;
        BG_CUDA(cudaMemsetAsync(Q.n_ext_out, 0, sizeof(int), st));
        BG_CUDA(cudaMemsetAsync(cnt + kCntSh, 0, 3 * sizeof(int), st));
        if (!fork || b == 0) {
            if (ins) ins->mark(0);
            if ((rc = launch_trace(s, false, Q.ext_rays_in, 0, Q.n_ext_in, Q.ext_hits, nullptr, st, nullptr, 1, wk, Q.ext_root_in, &kExtTrace))) return rc;
            if (ins) { ins->mark(0); ++ins->launches; ++ins->launches_extend; }
        }
        if (ins && ins->count_trav) {
            if ((rc = launch_trace(s, false, Q.ext_rays_in, 0, Q.n_ext_in, cnt_hits, nullptr, st, Q.totals + 3, 64, wk + 1, Q.ext_root_in))) return rc;
            ++ins->launches;
        }
        ShadeArgs A{b, c.maxdepth, c.kind, rs->kmax, c.batched ? 1 : 0, c.cache ? c.cache_depth : -1,
                    c.cache ? c.train_end : -1, c.cache ? c.train_stride : 0, c.ao_radius, 0, int(rs->cap)};
        const bool query_here = c.cache && (b == c.cache_depth || b == c.train_end);
        if (query_here) BG_CUDA(cudaMemsetAsync(Q.n_query, 0, sizeof(int), st));
        // the network the queries read is the one the previous frame's rows trained
        // (with side streams the wait sits on the query's own stream, below)
        const bool wait_here = c.cache && (c.wait_train || !ins) && b == c.cache_depth;
        if (wait_here && !fork)
            BG_CUDA(cudaStreamWaitEvent(st, rs->ev_train, ins ? 0u : unsigned(cudaEventWaitExternal)));
        const int nsh = launch_shade(s->dev, c.kind, c.cache != nullptr, nb, rs->blocks_class, st, A, P, Q);
        if (nsh < 0) return nsh;
        if (ins) { ins->launches += nsh; ins->mark(1); }
        const bool forked = fork && b + 1 < depth;
        if (forked) {
            Queues Qn;
            pass_queues(rs, 1 - cur, c.batched, Qn);
            BG_CUDA(cudaEventRecord(rs->ev_fork, st));
            BG_CUDA(cudaStreamWaitEvent(rs->fstream, rs->ev_fork, 0));
            if ((rc = launch_trace(s, false, Qn.ext_rays_in, 0, Qn.n_ext_in, Qn.ext_hits, nullptr, rs->fstream, nullptr, 1,
                                   wk + 6, Qn.ext_root_in, &kExtTrace)))
                return rc;
            BG_CUDA(cudaEventRecord(rs->ev_join, rs->fstream));
            if (ins) { ++ins->launches; ++ins->launches_extend; }
        }
        if (fork) {   // MIS trace and its resolve beside the shadow trace (they write different slots)
            if (!forked) BG_CUDA(cudaEventRecord(rs->ev_fork, st));
            BG_CUDA(cudaStreamWaitEvent(rs->mstream, rs->ev_fork, 0));
            if (s->dev.has_area) {   // MIS rays go to area lights only (the queue is empty otherwise)
                if ((rc = launch_trace(s, false, Q.mis_rays, 0, Q.n_mis, Q.mis_hits, nullptr, rs->mstream, nullptr, 1,
                                       wk + 3, Q.mis_root)))
                    return rc;
                k_resolve_mis<<<nb, kShadeThreads, 0, rs->mstream>>>(s->dev, P, Q);
            }
            if (query_here) {   // the cache query too: it adds to P.rad of ended paths, the resolves write P.slots
                if (wait_here)
                    BG_CUDA(cudaStreamWaitEvent(rs->mstream, rs->ev_train, ins ? 0u : unsigned(cudaEventWaitExternal)));
                float4* qo = rs->q_out.as<float4>();
                if ((rc = nrc_query(c.cache, rs->q_feat.as<float>(), Q.n_query, 0, qo, rs->mstream))) return rc;
                k_cache_resolve<<<nb, kShadeThreads, 0, rs->mstream>>>(P, Q, qo);
                if (ins) ins->launches += nrc_desc(c.cache)->mlp_kernel == 0 ? 2 : 3;
            }
            BG_CUDA(cudaEventRecord(rs->ev_mjoin, rs->mstream));
        }
        const ShadowResolve sr{Q.sh_contrib, Q.sh_slot, P.slots};   // visible rays land in their slot
        if ((rc = launch_trace(s, true, Q.sh_rays, 0, Q.n_sh, nullptr, nullptr, st, nullptr, 1, wk + 2, Q.sh_root, &sr)))
            return rc;
        if (ins) { ins->mark(1); ins->mark(2); }
        if (!fork && s->dev.has_area &&
            (rc = launch_trace(s, false, Q.mis_rays, 0, Q.n_mis, Q.mis_hits, nullptr, st, nullptr, 1, wk + 3, Q.mis_root)))
            return rc;
        if (ins) { ins->mark(2); ins->launches += s->dev.has_area ? 2 : 1; }
        if (ins && ins->count_trav) {
            if ((rc = launch_trace(s, true, Q.sh_rays, 0, Q.n_sh, nullptr, cnt_occ, st, Q.totals + 6, 64, wk + 4, Q.sh_root))) return rc;
            if ((rc = launch_trace(s, false, Q.mis_rays, 0, Q.n_mis, cnt_hits, nullptr, st, Q.totals + 9, 64, wk + 5, Q.mis_root))) return rc;
            ins->launches += 2;
        }
        if (fork) BG_CUDA(cudaStreamWaitEvent(st, rs->ev_mjoin, 0));
        else if (s->dev.has_area) k_resolve_mis<<<nb, kShadeThreads, 0, st>>>(s->dev, P, Q);
        if (query_here && !fork) {
            // paths that ended into the cache here: encode, infer, add throughput * prediction
            if (ins) ins->mark(3);
            float4* qo = rs->q_out.as<float4>();
            if ((rc = nrc_query(c.cache, rs->q_feat.as<float>(), Q.n_query, 0, qo, st))) return rc;
            k_cache_resolve<<<nb, kShadeThreads, 0, st>>>(P, Q, qo);
            if (ins) { ins->launches += nrc_desc(c.cache)->mlp_kernel == 0 ? 2 : 3; ins->mark(3); }
        }
        k_finalize<<<nb, kShadeThreads, 0, st>>>(P, Q, rs->kmax, c.maxdepth, c.cache ? c.train_stride : 0,
                                                 c.cache ? c.cache_depth : 0, b, 0, int(rs->cap));
        if (ins) ins->launches += s->dev.has_area ? 2 : 1;
        if (forked) BG_CUDA(cudaStreamWaitEvent(st, rs->ev_join, 0));
        cur = 1 - cur;
        pass_queues(rs, cur, c.batched, Q);
    }
    // the accumulation buffer may still be arriving from the host (bg_render_host)
    // (captured into the pass graph as an event-wait node; a plain wait otherwise)
    if (s->ev_accum) BG_CUDA(cudaStreamWaitEvent(st, s->ev_accum, ins ? 0u : unsigned(cudaEventWaitExternal)));
    k_accumulate<<<nb, kShadeThreads, 0, st>>>(P, c.segs, c.nseg, c.npix);
    if (ins) ++ins->launches;
    BG_CUDA(cudaGetLastError());
    return BG_OK;
}

// Captures one pass into a CUDA graph (once per bounce-loop shape) and finds
// the two kernel nodes whose arguments (the segment slice, the training-path
// phase) change per pass, and the radiance-cache kernel nodes, which are
// pointed at the rendering cache on every replay (a cache of the same
// configuration replays the same graph).
static int pass_graph(bg_scene* s, RenderState* rs, const PassCfg& c, RenderState::PassGraph*& out) {
    uint32_t aob;
    memcpy(&aob, &c.ao_radius, sizeof(aob));
    const int64_t key[kGraphKey] = {c.maxdepth, c.kind, c.batched ? 1 : 0, rs->kmax, int64_t(rs->cap), s->tune_threads,
                                    s->dev.width, int64_t(aob), s->ev_accum ? 1 : 0,
                                    c.cache ? int64_t(nrc_desc(c.cache)->mlp_kernel) + 1 : 0,
                                    c.cache ? c.cache_depth : -1, c.cache ? c.train_end : -1,
                                    c.cache ? c.train_stride : 0, c.cache ? rs->tr_set : 0,
                                    int64_t(rs->buf_epoch)};
    ++rs->graph_clock;
    for (auto& pg : rs->graphs)
        if (pg.exec && memcmp(key, pg.key, sizeof(key)) == 0) { pg.used = rs->graph_clock; out = &pg; return BG_OK; }
    RenderState::PassGraph* pg = &rs->graphs[0];
    for (auto& q : rs->graphs)
        if (!q.exec || q.used < pg->used) pg = &q;       // an empty slot or the least recently used
    if (pg->exec) { cudaGraphExecDestroy(pg->exec); pg->exec = nullptr; }
    if (pg->graph) { cudaGraphDestroy(pg->graph); pg->graph = nullptr; }
    BG_CUDA(cudaStreamBeginCapture(rs->gstream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_pass(s, rs, rs->gstream, c, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(rs->gstream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return set_error(BG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    pg->graph = g;
    size_t nn = 0;
    BG_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    BG_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    pg->gen_node = pg->acc_node = nullptr;
    pg->cache_nodes.clear();
    for (cudaGraphNode_t n : nodes) {
        cudaGraphNodeType t;
        BG_CUDA(cudaGraphNodeGetType(n, &t));
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        BG_CUDA(cudaGraphKernelNodeGetParams(n, &kp));
        if (kp.func == reinterpret_cast<void*>(k_generate)) pg->gen_node = n;
        if (kp.func == reinterpret_cast<void*>(k_accumulate)) pg->acc_node = n;
        if (c.cache) {
            bool is_cache = false;
            if ((rc = nrc_graph_node(c.cache, nullptr, n, &is_cache))) return rc;
            if (is_cache) pg->cache_nodes.push_back(n);
        }
    }
    if (!pg->gen_node || !pg->acc_node) return set_error(BG_ERR_STATE, "pass graph: kernel nodes not found");
    BG_CUDA(cudaGraphInstantiate(&pg->exec, g, 0));
    memcpy(pg->key, key, sizeof(key));
    pg->used = rs->graph_clock;
    out = pg;
    return BG_OK;
}

static int launch_pass_graph(bg_scene* s, RenderState* rs, const PassCfg& c) {
    RenderState::PassGraph* pg = nullptr;
    int rc = pass_graph(s, rs, c, pg);
    if (rc) return rc;
    PathState P = path_state(rs);
    Queues Q;
    pass_queues(rs, 0, c.batched, Q);
    const SegRec* segs = c.segs;
    int nseg = c.nseg, total = c.total, npix = c.npix;
    int tstride = c.cache ? c.train_stride : 0, tphase = c.cache ? c.train_phase : 0;
    void* gargs[] = {&segs, &nseg, &total, &P, &Q, &tstride, &tphase};
    cudaKernelNodeParams kp;
    BG_CUDA(cudaGraphKernelNodeGetParams(pg->gen_node, &kp));
    kp.kernelParams = gargs;
    kp.extra = nullptr;
    BG_CUDA(cudaGraphExecKernelNodeSetParams(pg->exec, pg->gen_node, &kp));
    void* aargs[] = {&P, &segs, &nseg, &npix};
    BG_CUDA(cudaGraphKernelNodeGetParams(pg->acc_node, &kp));
    kp.kernelParams = aargs;
    kp.extra = nullptr;
    BG_CUDA(cudaGraphExecKernelNodeSetParams(pg->exec, pg->acc_node, &kp));
    // the cache's kernels read the cache this render uses (graphs are keyed by
    // the cache's configuration, not by the cache)
    for (cudaGraphNode_t n : pg->cache_nodes) {
        bool is_cache = false;
        if ((rc = nrc_graph_node(c.cache, pg->exec, n, &is_cache))) return rc;
    }
    BG_CUDA(cudaGraphLaunch(pg->exec, rs->gstream));
    return BG_OK;
}

// Splits jobs into sample chunks and packs them into passes of at most `cap`
// paths; two chunks of one job whose pixels overlap never share a pass (their
// per-pixel sums must stay ordered by sample).
static void plan_passes(const std::vector<JobSpec>& jobs, int64_t cap, std::vector<SegRec>& segs,
                        std::vector<int>& pass_begin) {
    std::vector<SegRec> all;
    for (size_t j = 0; j < jobs.size(); ++j) {
        const JobSpec& J = jobs[j];
        const int64_t npix = int64_t(J.W) * J.H;
        if (npix <= cap) {
            for (int s0 = 0; s0 < J.spp;) {
                int ns = int(std::max<int64_t>(1, std::min<int64_t>(J.spp - s0, cap / npix)));
                SegRec g{};
                g.cam = J.cam; g.accum = J.accum; g.seed = J.seed; g.job = int(j);
                g.skind = J.skind; g.grid = J.grid;
                g.np = int(npix); g.ns = ns; g.p0 = 0; g.s0 = J.soff + s0; g.W = J.W; g.H = J.H;
                all.push_back(g);
                s0 += ns;
            }
        } else {
            for (int s = 0; s < J.spp; ++s)
                for (int64_t p0 = 0; p0 < npix; p0 += cap) {
                    SegRec g{};
                    g.cam = J.cam; g.accum = J.accum; g.seed = J.seed; g.job = int(j);
                    g.skind = J.skind; g.grid = J.grid;
                    g.np = int(std::min<int64_t>(cap, npix - p0)); g.ns = 1; g.p0 = int(p0); g.s0 = J.soff + s;
                    g.W = J.W; g.H = J.H;
                    all.push_back(g);
                }
        }
    }
    int64_t used = 0;
    int first = 0;
    pass_begin.clear();
    segs.clear();
    for (size_t k = 0; k < all.size(); ++k) {
        SegRec g = all[k];
        const int64_t size = int64_t(g.np) * g.ns;
        bool conflict = used + size > cap || int(segs.size()) - first >= kMaxSegs;
        for (int q = first; q < int(segs.size()) && !conflict; ++q) {
            const SegRec& o = segs[size_t(q)];
            if (o.job == g.job && o.p0 < g.p0 + g.np && g.p0 < o.p0 + o.np) conflict = true;
        }
        if (segs.empty() || conflict) {
            pass_begin.push_back(int(segs.size()));
            first = int(segs.size());
            used = 0;
        }
        int pix0 = 0;
        for (int q = first; q < int(segs.size()); ++q) pix0 += segs[size_t(q)].np;
        g.path0 = int(used);
        g.pix0 = pix0;
        segs.push_back(g);
        used += size;
    }
    pass_begin.push_back(int(segs.size()));
}

int render_jobs(bg_scene* s, bg_cache* cache, const std::vector<JobSpec>& jobs, const bg_tracer_desc* tr,
                bg_render_stats* stats, cudaStream_t st, bool batched) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    if (!tr) return set_error(BG_ERR_INVALID_ARG, "NULL tracer");
    if (tr->kind != BG_TRACER_GI && tr->kind != BG_TRACER_DI && tr->kind != BG_TRACER_AO)
        return set_error(BG_ERR_UNSUPPORTED, "tracer kind %d", tr->kind);
    if (tr->kind == BG_TRACER_AO && !std::isfinite(tr->ao_radius))
        return set_error(BG_ERR_INVALID_ARG, "AO radius must be finite");
    if (tr->kind == BG_TRACER_GI && (tr->maxdepth < 0 || tr->maxdepth > 1024)) return set_error(BG_ERR_INVALID_ARG, "maxdepth %d", tr->maxdepth);
    if (jobs.empty()) return BG_OK;
    if (jobs.size() > 65535) return set_error(BG_ERR_INVALID_ARG, "too many jobs (%zu > 65535)", jobs.size());
    int maxL = 1;
    int64_t total_samples = 0, max_job = 0;
    for (const JobSpec& J : jobs) {
        if (J.W <= 0 || J.H <= 0 || int64_t(J.W) * J.H > (int64_t(1) << 28)) return set_error(BG_ERR_INVALID_ARG, "bad resolution %dx%d", J.W, J.H);
        if (J.spp < 0 || J.soff < 0) return set_error(BG_ERR_INVALID_ARG, "negative spp / sample offset");
        if (int64_t(J.soff) + J.spp > (int64_t(1) << 31)) return set_error(BG_ERR_INVALID_ARG, "sample indices must stay below 2^31");
        if (J.skind != BG_SAMPLER_RANDOM && J.skind != BG_SAMPLER_SOBOL && J.skind != BG_SAMPLER_CMJ)
            return set_error(BG_ERR_UNSUPPORTED, "sampler kind %d", J.skind);
        if (J.skind == BG_SAMPLER_CMJ && (J.grid < 1 || J.grid > 16))
            return set_error(BG_ERR_INVALID_ARG, "CMJ grid %d outside 1..16", J.grid);
        if (!J.accum || (reinterpret_cast<uintptr_t>(J.accum) & 15u)) return set_error(BG_ERR_INVALID_ARG, "accumulation buffer must be non-NULL and 16-byte aligned");
        if (J.rec.nlights <= 0) return set_error(BG_ERR_UNSUPPORTED, "a scene without lights (GiTracer divides by the light count)");
        maxL = std::max(maxL, J.rec.nlights);
        total_samples += int64_t(J.W) * J.H * J.spp;
        max_job = std::max(max_job, int64_t(J.W) * J.H * std::max(1, J.spp));
    }
    const int64_t target = s->tune_paths > 0 ? s->tune_paths : (int64_t(1) << 21);   // paths per pass
    int64_t cap = std::max<int64_t>(1, std::min<int64_t>(target, std::max<int64_t>(total_samples, 1)));
    // at most 2^26 DI slots (2 per light) per pass, which bounds the shadow / MIS
    // queues too (about 16 GB at the bound): scenes with many lights get smaller passes
    cap = std::max<int64_t>(1, std::min<int64_t>(cap, (int64_t(1) << 26) / (2 * std::max(1, maxL))));
    int rc = ensure_state(s, cap, maxL);
    if (rc) return rc;
    RenderState* rs = s->render;   // buffers may be larger than this call's pass size
    const int maxdepth = tr->kind == BG_TRACER_GI ? tr->maxdepth : 1;
    unsigned long long* totals = reinterpret_cast<unsigned long long*>(rs->counts.as<char>() + 64);

    std::vector<SegRec> segs;
    std::vector<int> pass_begin;
    plan_passes(jobs, cap, segs, pass_begin);
    const int npass = int(pass_begin.size()) - 1;
    if ((rc = ensure_tracked(rs, rs->segs, std::max<size_t>(1, segs.size()) * sizeof(SegRec))) ||
        (rc = ensure_tracked(rs, rs->jobs, jobs.size() * sizeof(JobRec))))
        return rc;
    std::vector<JobRec> jrec(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) jrec[j] = jobs[j].rec;

    // Graph replay unless statistics were asked for or the caller's stream is
    // capturing (cached renders too: the frame's training-path phase is a
    // parameter of the generate node, the rest of the pass is frame-invariant).
    cudaStreamCaptureStatus cap_st = cudaStreamCaptureStatusNone;
    BG_CUDA(cudaStreamIsCapturing(st, &cap_st));
    const bool use_graph = !stats && cap_st == cudaStreamCaptureStatusNone;
    cudaStream_t ws = use_graph ? rs->gstream : st;
    if (use_graph) {
        BG_CUDA(cudaEventRecord(rs->ev_in, st));
        BG_CUDA(cudaStreamWaitEvent(rs->gstream, rs->ev_in, 0));
    }
    {
        // tables go through pinned, double-buffered staging so the upload stays asynchronous
        const int i = rs->tab_i ^= 1;
        const size_t sb = segs.size() * sizeof(SegRec), jb = jrec.size() * sizeof(JobRec);
        if (rs->tab_ev[i]) BG_CUDA(cudaEventSynchronize(rs->tab_ev[i]));
        else BG_CUDA(cudaEventCreateWithFlags(&rs->tab_ev[i], cudaEventDisableTiming));
        if (rs->host_tab_bytes[i] < sb + jb) {
            if (rs->host_tab[i]) cudaFreeHost(rs->host_tab[i]);
            rs->host_tab[i] = nullptr;
            rs->host_tab_bytes[i] = 0;
            if (!alloc_charge((sb + jb) * 2))
                return set_error(BG_ERR_OOM, "pinned staging of %zu bytes refused: over the library's allocation limit",
                                 (sb + jb) * 2);
            BG_CUDA(cudaMallocHost(&rs->host_tab[i], (sb + jb) * 2));
            rs->host_tab_bytes[i] = (sb + jb) * 2;
        }
        char* h = static_cast<char*>(rs->host_tab[i]);
        memcpy(h, segs.data(), sb);
        memcpy(h + sb, jrec.data(), jb);
        BG_CUDA(cudaMemcpyAsync(rs->segs.ptr, h, sb, cudaMemcpyHostToDevice, ws));
        BG_CUDA(cudaMemcpyAsync(rs->jobs.ptr, h + sb, jb, cudaMemcpyHostToDevice, ws));
        BG_CUDA(cudaEventRecord(rs->tab_ev[i], ws));
    }
    Instr ins;
    ins.st = st;
    ins.time_phases = stats && (tr->flags & BG_RENDER_TIME_PHASES);
    ins.count_trav = stats && (tr->flags & BG_RENDER_COUNT_TRAVERSAL);
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (stats) {
        // totals: [0] extension rays, [1] any rays, [2] MIS rays, replays (rays, nodes, tris):
        // [3..5] extension, [6..8] any, [9..11] MIS
        BG_CUDA(cudaMemsetAsync(totals, 0, 12 * sizeof(unsigned long long), st));
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, st);
    }
    // radiance-cache mode: training-path selection and buffers
    int cache_depth = -1, train_end = -1, stride = 0, phase = 0, tsteps = 0, tbatch = 0;
    bool train_prev = false, wait_train = false;
    if (cache) {
        const bg_cache_desc* cd = nrc_desc(cache);
        if (tr->kind != BG_TRACER_GI) return set_error(BG_ERR_UNSUPPORTED, "the radiance cache serves GiTracer only");
        cache_depth = cd->cache_depth;
        if (cache_depth < 0 || cache_depth >= std::max(1, maxdepth)) return set_error(BG_ERR_INVALID_ARG, "cache_depth %d outside [0, maxdepth)", cache_depth);
        if (cd->train_suffix < 0) return set_error(BG_ERR_INVALID_ARG, "train_suffix %d < 0", cd->train_suffix);
        if (cd->train_suffix > 0 && cache_depth + cd->train_suffix < std::max(1, maxdepth))
            train_end = cache_depth + cd->train_suffix;
        const int64_t tp = std::max<int64_t>(1, cd->train_paths);
        stride = int(std::max<int64_t>(1, std::min<int64_t>(total_samples / tp, int64_t(1) << 24)));
        phase = int(nrc_next_frame(cache) % stride);
        tsteps = std::max(0, cd->train_steps);
        tbatch = std::max(1, cd->train_batch);
        const int64_t tpaths_pass = cap / stride + 2;
        const int64_t tr_cap = (total_samples / stride + 2 * npass + 2) * maxdepth;
        if (rs->q_cap < cap) {
            if ((rc = ensure_tracked(rs, rs->q_feat, size_t(cap) * 64)) ||
                (rc = ensure_tracked(rs, rs->q_path, size_t(cap) * 4)) ||
                (rc = ensure_tracked(rs, rs->q_thr, size_t(cap) * 16)) ||
                (rc = ensure_tracked(rs, rs->q_out, size_t(cap) * 16)))
                return rc;
            rs->q_cap = cap;
        }
        if ((rc = ensure_tracked(rs, rs->rec, size_t(tpaths_pass) * maxdepth * 6 * 16))) return rc;
        if (rs->tr_cap < tr_cap) {
            if ((rc = ensure_tracked(rs, rs->tr_feat, size_t(tr_cap) * 64 * kCntTrainSets)) ||
                (rc = ensure_tracked(rs, rs->tr_target, size_t(tr_cap) * 16 * kCntTrainSets)))
                return rc;
            rs->tr_cap = tr_cap;
            rs->pending_cache = 0;                   // the sets were reallocated
            rs->pending_ptr = nullptr;
        }
        if ((rc = nrc_prepare(cache, tbatch, cap))) return rc;
        // Online training is one frame behind: this frame's training rows go to
        // one set while the previous frame's rows (the other set) are trained on
        // a side stream, beside this frame's first bounces, which do not read
        // the cache; the first query stage waits for that training.
        const int64_t frame = nrc_frame(cache) - 1;
        if (rs->pending_cache != 0 && rs->pending_cache != nrc_id(cache) && rs->pending_ptr) {
            // Rows another cache of this scene left pending (renders of several
            // caches interleaved): train them into that cache now, so that every
            // cache trains on each of its frames once.  Synchronous, as that
            // cache's next render may come on another stream.
            bg_cache* other = rs->pending_ptr;
            const bg_cache_desc* od = nrc_desc(other);
            const int oset = rs->tr_set;             // the set its last render wrote
            int* ntr = rs->counts.as<int>() + kCntTrain + oset;
            const float* feat = rs->tr_feat.as<float>() + size_t(oset) * rs->tr_cap * 16;
            const float4* target = rs->tr_target.as<float4>() + size_t(oset) * rs->tr_cap;
            k_clamp_count<<<1, 1, 0, st>>>(ntr, int(rs->tr_cap));
            for (int i = 0; i < std::max(0, od->train_steps); ++i)
                if ((rc = nrc_train_step(other, feat, target, ntr, i * std::max(1, od->train_batch),
                                         std::max(1, od->train_batch), true, st)))
                    return rc;
            BG_CUDA(cudaStreamSynchronize(st));
            rs->pending_cache = 0;
            rs->pending_ptr = nullptr;
        }
        train_prev = tsteps > 0 && rs->pending_cache == nrc_id(cache) && rs->pending_frame == frame - 1;
        rs->tr_set ^= 1;
        int* ntr_prev = rs->counts.as<int>() + kCntTrain + (rs->tr_set ^ 1);
        if (train_prev) {
            const float* feat = rs->tr_feat.as<float>() + size_t(rs->tr_set ^ 1) * rs->tr_cap * 16;
            const float4* target = rs->tr_target.as<float4>() + size_t(rs->tr_set ^ 1) * rs->tr_cap;
            const bool side = !ins.time_phases;
            cudaStream_t ts = side ? rs->tstream : st;
            if (side) {
                BG_CUDA(cudaEventRecord(rs->ev_tstart, st));
                BG_CUDA(cudaStreamWaitEvent(ts, rs->ev_tstart, 0));
            }
            ins.mark(4);
            k_clamp_count<<<1, 1, 0, ts>>>(ntr_prev, int(rs->tr_cap));
            for (int i = 0; i < tsteps; ++i)
                if ((rc = nrc_train_step(cache, feat, target, ntr_prev, i * tbatch, tbatch, true, ts))) return rc;
            // per step: encode, forward + backward, weight gradients (one tcgen05 kernel or six
            // mma.sync ones), grid backward, step counter, two Adam kernels
            ins.launches += 1 + (cd->mlp_kernel == 0 ? 7 : 12) * tsteps;
            ins.mark(4);
            if (side) BG_CUDA(cudaEventRecord(rs->ev_train, ts));
            wait_train = side;
        }
        // a replayed pass always holds the wait on ev_train: without training this frame it waits on nothing new
        if (use_graph && !wait_train) BG_CUDA(cudaEventRecord(rs->ev_train, st));
        BG_CUDA(cudaMemsetAsync(rs->counts.as<int>() + kCntTrain + rs->tr_set, 0, sizeof(int), st));
        rs->pending_cache = nrc_id(cache);
        rs->pending_ptr = cache;
        rs->pending_frame = frame;
    }
    int64_t done_samples = 0;
    for (int p = 0; p < npass; ++p) {
        PassCfg c;
        c.segs = rs->segs.as<SegRec>() + pass_begin[size_t(p)];
        c.nseg = pass_begin[size_t(p) + 1] - pass_begin[size_t(p)];
        c.total = 0;
        c.npix = 0;
        for (int q = pass_begin[size_t(p)]; q < pass_begin[size_t(p) + 1]; ++q) {
            c.total += segs[size_t(q)].np * segs[size_t(q)].ns;
            c.npix += segs[size_t(q)].np;
        }
        // with a training suffix no path continues past train_end
        c.maxdepth = train_end >= 0 ? train_end + 1 : maxdepth;
        c.kind = tr->kind;
        c.ao_radius = tr->kind == BG_TRACER_AO ? tr->ao_radius : 0.f;
        c.batched = batched;
        c.cache = cache;
        c.cache_depth = cache_depth;
        c.train_end = train_end;
        c.wait_train = wait_train && p == 0;
        c.train_stride = stride;
        c.train_phase = phase;
        rc = use_graph ? launch_pass_graph(s, rs, c) : enqueue_pass(s, rs, st, c, &ins);
        if (rc) return rc;
        done_samples += c.total;
    }
    if (wait_train) BG_CUDA(cudaStreamWaitEvent(st, rs->ev_train, 0));   // the call's work ends with the training
    if (use_graph) {
        BG_CUDA(cudaEventRecord(rs->ev_out, rs->gstream));
        BG_CUDA(cudaStreamWaitEvent(st, rs->ev_out, 0));
    }
    if (stats) {
        cudaEventRecord(ev1, st);
        BG_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        unsigned long long t[12];
        BG_CUDA(cudaMemcpy(t, totals, sizeof(t), cudaMemcpyDeviceToHost));
        memset(stats, 0, sizeof(*stats));
        stats->camera_samples = done_samples;
        stats->rays_extension = int64_t(t[0]);
        stats->rays_closest = int64_t(t[0] + t[2]);
        stats->rays_any = int64_t(t[1]);
        stats->kernel_launches = ins.launches;
        stats->launches_extend = ins.launches_extend;
        stats->ms_total = ms;
        float phase_ms[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (size_t i = 0; i + 1 < ins.evs.size(); i += 2) {
            float m = 0.f;
            cudaEventElapsedTime(&m, ins.evs[i], ins.evs[i + 1]);
            phase_ms[ins.tags[i]] += m;
        }
        for (cudaEvent_t e : ins.evs) cudaEventDestroy(e);
        stats->ms_extend = phase_ms[0];
        stats->ms_shadow = phase_ms[1];
        stats->ms_mis = phase_ms[2];
        stats->ms_cache_query = phase_ms[3];
        stats->ms_cache_train = phase_ms[4];
        stats->ms_shade = ins.time_phases ? ms - phase_ms[0] - phase_ms[1] - phase_ms[2] - phase_ms[3] - phase_ms[4] : 0.f;
        stats->sub_rays_extension = int64_t(t[3]);
        stats->sub_nodes_extension = int64_t(t[4]);
        stats->sub_tris_extension = int64_t(t[5]);
        stats->sub_rays_any = int64_t(t[6]);
        stats->sub_nodes_any = int64_t(t[7]);
        stats->sub_tris_any = int64_t(t[8]);
        stats->sub_rays_mis = int64_t(t[9]);
        stats->sub_nodes_mis = int64_t(t[10]);
        stats->sub_tris_mis = int64_t(t[11]);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    return BG_OK;
}

static int render_impl(bg_scene* s, bg_cache* cache, const bg_camera_desc* cam, const bg_tracer_desc* tr,
                       const bg_sampler_desc* sm, int W, int H, float4* accum, bg_render_stats* stats, cudaStream_t st) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    if (!cam || !tr || !sm || !accum) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::vector<JobSpec> jobs(1);
    JobSpec& J = jobs[0];
    J.rec.root = 0;
    J.rec.light0 = 0;
    J.rec.nlights = s->dev.nlights;
    J.rec.pad = 0;
    J.rec.bg[0] = s->dev.bg[0]; J.rec.bg[1] = s->dev.bg[1]; J.rec.bg[2] = s->dev.bg[2]; J.rec.bg[3] = 0.f;
    J.cam = make_camera(cam);
    J.W = W; J.H = H; J.spp = sm->spp; J.soff = sm->sample_offset; J.seed = sm->seed; J.accum = accum;
    J.skind = sm->kind; J.grid = sm->grid;
    return render_jobs(s, cache, jobs, tr, stats, st, false);
}

// Times every (node layout, traversal block size, paths per pass) candidate
// on this scene with `probe_spp` samples per pixel into accum (which receives
// them), keeps the fastest for later renders of the scene.
static int scene_autotune(bg_scene* s, const bg_camera_desc* cam, const bg_tracer_desc* tr, int32_t probe_spp,
                          int W, int H, float4* accum, bg_tune_result* result, cudaStream_t st) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    if (!cam || !tr || !accum) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    std::vector<int> widths;
    if (s->dev.nodes) widths.push_back(4);
    if (s->dev.nodes8) widths.push_back(8);
    const int threads[2] = {128, 256};
    const int64_t probe_samples = int64_t(W) * H * std::max(1, probe_spp);
    bg_sampler_desc sm = {BG_SAMPLER_RANDOM, std::max(1, probe_spp), 1, 0, 0};
    float best = 1e30f;
    int best_t = 128, best_w = s->dev.width, tried = 0, rc = BG_OK;
    int64_t best_p = int64_t(1) << 21;
    cudaEvent_t e0, e1;
    BG_CUDA(cudaEventCreate(&e0));
    BG_CUDA(cudaEventCreate(&e1));
    for (int w : widths) {
        s->dev.width = w;
        for (int t : threads) {
            for (int pi = 0; pi < kPassCandidates && pass_candidate_needed(pi, probe_samples); ++pi) {
                const int64_t p = pass_candidate(pi);
                s->tune_threads = t;
                s->tune_paths = p;
                // the first render warms the graph and buffers of this candidate, the second is timed
                if ((rc = render_impl(s, nullptr, cam, tr, &sm, W, H, accum, nullptr, st))) {
                    if (rc == BG_ERR_OOM && pi > 0) {   // no room for passes this large: keep the smaller
                        cudaGetLastError();
                        rc = BG_OK;
                    }
                    break;
                }
                BG_CUDA(cudaEventRecord(e0, st));
                if ((rc = render_impl(s, nullptr, cam, tr, &sm, W, H, accum, nullptr, st))) break;
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
    s->dev.width = best_w;
    set_width_info(s);
    if (rc) return rc;
    s->tune_threads = best_t;
    s->tune_paths = best_p;
    if (result) {
        result->trace_threads = best_t;
        result->paths_per_pass = int32_t(best_p);
        result->candidates = tried;
        result->ms = best;
        result->msamples_per_s = best > 0.f ? float(double(W) * H * sm.spp / (double(best) * 1e3)) : 0.f;
        result->node_width = best_w;
    }
    return BG_OK;
}

// A destroyed cache's pending training rows are dropped (bg_cache_destroy).
void render_forget_cache(bg_scene* s, const bg_cache* c) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    RenderState* rs = s->render;
    if (rs && rs->pending_ptr == c) {
        rs->pending_ptr = nullptr;
        rs->pending_cache = 0;
    }
}

}  // namespace bg

using namespace bg;

extern "C" int bg_scene_autotune(bg_scene* s, const bg_camera_desc* cam, const bg_tracer_desc* tr, int32_t probe_spp,
                                 int32_t W, int32_t H, float* accum, bg_tune_result* result, void* stream) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    return scene_autotune(s, cam, tr, probe_spp, W, H, reinterpret_cast<float4*>(accum), result,
                          static_cast<cudaStream_t>(stream));
}

extern "C" int bg_render(bg_scene* s, const bg_camera_desc* cam, const bg_tracer_desc* tr, const bg_sampler_desc* sm,
                         int32_t W, int32_t H, float* accum, bg_render_stats* stats, void* stream) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    return render_impl(s, nullptr, cam, tr, sm, W, H, reinterpret_cast<float4*>(accum), stats, static_cast<cudaStream_t>(stream));
}

extern "C" int bg_render_cached(bg_scene* s, bg_cache* cache, const bg_camera_desc* cam, const bg_tracer_desc* tr,
                                const bg_sampler_desc* sm, int32_t W, int32_t H, float* accum, bg_render_stats* stats,
                                void* stream) {
    if (!s || !cache) return set_error(BG_ERR_INVALID_ARG, "scene or cache is NULL");
    if (nrc_scene(cache) != s) return set_error(BG_ERR_INVALID_ARG, "the cache was created for another scene");
    std::lock_guard<std::mutex> lk(s->mu);
    return render_impl(s, cache, cam, tr, sm, W, H, reinterpret_cast<float4*>(accum), stats, static_cast<cudaStream_t>(stream));
}

extern "C" int bg_render_host(bg_scene* s, const bg_camera_desc* cam, const bg_tracer_desc* tr, const bg_sampler_desc* sm,
                              int32_t W, int32_t H, float* accum, bg_render_stats* stats) {
    if (!s) return set_error(BG_ERR_INVALID_ARG, "scene is NULL");
    if (!accum) return set_error(BG_ERR_INVALID_ARG, "accum is NULL");
    if (W <= 0 || H <= 0) return set_error(BG_ERR_INVALID_ARG, "bad resolution");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    const size_t bytes = size_t(W) * H * 16;
    int rc = s->host_out.ensure(bytes);   // staging shared with the host ray casts (both hold the scene lock)
    if (rc) return rc;
    float4* d = s->host_out.as<float4>();
    if (!s->copy_stream) {
        BG_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        BG_CUDA(cudaEventCreateWithFlags(&s->ev_accum, cudaEventDisableTiming));
    }
    // upload on the copy stream, overlapping the pass; only accumulate waits for it
    BG_CUDA(cudaMemcpyAsync(d, accum, bytes, cudaMemcpyHostToDevice, s->copy_stream));
    BG_CUDA(cudaEventRecord(s->ev_accum, s->copy_stream));
    rc = render_impl(s, nullptr, cam, tr, sm, W, H, d, stats, 0);
    if (rc) { cudaStreamSynchronize(s->copy_stream); return rc; }
    BG_CUDA(cudaMemcpy(accum, d, bytes, cudaMemcpyDeviceToHost));
    unsigned flags = 0;
    BG_CUDA(cudaMemcpy(&flags, s->err.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flags & BG_FLAG_STACK_OVERFLOW) return set_error(BG_ERR_OVERFLOW, "traversal stack overflow");
    return BG_OK;
}
