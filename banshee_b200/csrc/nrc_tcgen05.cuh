// Radiance-cache MLP inference on the 5th-generation tensor cores (tcgen05).
//
// Persistent CTAs; each group of 128 threads works on one tile of 128 query
// rows at a time (the inference kernel's layout is described above it):
//   * the six weight matrices live in shared memory for the whole kernel, in
//     the K-major no-swizzle canonical layout of the UMMA shared-memory
//     descriptors: 8x8 bf16 core matrices of 128 contiguous bytes, core
//     matrices adjacent in K 128 bytes apart (LBO), 8-row groups K/8 * 128
//     bytes apart (SBO);
//   * the activation tile (A operand, 128 x K bf16) is in the same layout;
//   * the fp32 accumulator (128 lanes x 64 columns) is in tensor memory;
//   * thread 0 issues tcgen05.mma (M = 128, N = 64 or 16, K = 16 per
//     instruction) and commits to an mbarrier; every thread then reads its own
//     accumulator row (TMEM lane = tile row) with tcgen05.ld, applies ReLU,
//     rounds to bf16 and writes the next layer's A row.
// Waits on the mbarrier are bounded (NrcDev::wait_polls polls, 0 = the
// default of 2^24): on timeout the kernel raises BG_FLAG_TIMEOUT, stops, gives
// its outstanding MMA group one more wait with the default bound, releases
// its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "cache.h"
#include "nrc_encode.cuh"

namespace bg {

constexpr int kTcRows = 128;                               // rows per tile (UMMA M)
constexpr int kTcW0 = 0;                                   // [64 x 128]
constexpr int kTcW1 = kTcW0 + 64 * 128 * 2;                // 4 x [64 x 64]
constexpr int kTcW5 = kTcW1 + 4 * 64 * 64 * 2;             // [16 x 64]
constexpr int kTcA0 = kTcW5 + 16 * 64 * 2;                 // [128 x 128]
constexpr int kTcA1 = kTcA0 + kTcRows * 128 * 2;           // [128 x 64]
constexpr int kTcBar = kTcA1 + kTcRows * 64 * 2;           // mbarrier (8 B) + TMEM base (4 B)
constexpr int kTcSmem = kTcBar + 16;
constexpr uint32_t kTcCols = 64;                           // TMEM columns allocated
constexpr uint32_t kTcWaitLimit = 1u << 24;                // mbarrier polls before giving up

// byte offset of core-matrix row `r`, 16-byte chunk `kc` in a K-major tile with KC chunks per row
__host__ __device__ constexpr uint32_t tc_off(int r, int kc, int KC) {
    return uint32_t((r >> 3) * (KC * 128) + kc * 128 + (r & 7) * 16);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);   // version 1, no swizzle
}

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, A K-major, B K-major
// (b_mn = false) or MN-major (b_mn = true), M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int N, bool b_mn = false) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (b_mn ? (1u << 16) : 0u) | (uint32_t(N >> 3) << 17) |
           (uint32_t(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// true once the phase of parity `phase` of the mbarrier has completed; false
// after `polls` polls (0 = kTcWaitLimit).  The first poll is a non-blocking
// test_wait, the rest are try_wait (which may suspend the thread briefly), so
// a budget of one poll gives up at once unless the phase is already complete.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase, uint32_t polls = 0) {
    const uint32_t limit = polls ? polls : kTcWaitLimit;
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(bar), "r"(phase) : "memory");
    if (done) return true;
    for (uint32_t it = 1; it < limit; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(bar), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tc_pack(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// weight matrix [N][K] (row-major bf16 in global memory) -> canonical K-major smem tile
__device__ __forceinline__ void tc_load_weights(const __nv_bfloat16* __restrict__ w, int N, int K, unsigned char* dst) {
    const int KC = K / 8;
    for (int i = threadIdx.x; i < N * KC; i += blockDim.x) {
        const int n = i / KC, kc = i % KC;
        *reinterpret_cast<uint4*>(dst + tc_off(n, kc, KC)) = *reinterpret_cast<const uint4*>(w + size_t(n) * K + kc * 8);
    }
}

// Inference: CTAs of kTiGroups x 128 threads.  Each group of four warps runs
// its own 128-row tiles through the six layers with its own mbarrier, its own
// 64 TMEM columns and its own 32 KB activation slot: the 128-wide input tile,
// whose first 16 KB the 64-wide hidden tiles reuse once the layer-0 MMA has
// completed (82 KB of shared memory per group with the weights, against
// 100 KB with a separate hidden tile).  Groups synchronise on named barriers
// (ids 1..kTiGroups), the CTA only at start and end.  The kernel is bound by
// the encoding's hash-grid gathers, not by the MMA chain: measured on the C3
// frame's queries, one group per CTA at two CTAs per SM (the smaller shared
// footprint leaves more L1 to the gathers) took 103 us per launch, four groups
// in one CTA per SM 126 us; the previous layout (separate hidden tile) 1.07 ms
// per 8-spp frame against 0.68 ms now.
// feat != nullptr: the input rows are encoded here from the raw query records
// (16 floats each; thread r of a group encodes row r of its tile straight into
// the A tile), so no encoded row goes through global memory; otherwise they
// are read from X.
constexpr int kTiGroups = 1;
constexpr int kTiCtasPerSm = 2;                            // CTAs per SM in the grid
constexpr int kTiThreads = 128 * kTiGroups;
constexpr int kTiSlot0 = kTcA0;                            // group g's slot at kTiSlot0 + g * kTiSlotBytes
constexpr int kTiSlotBytes = kTcRows * 128 * 2;            // 32 KB: the [128 x 128] input tile
constexpr int kTiBar = kTiSlot0 + kTiGroups * kTiSlotBytes;   // kTiGroups mbarriers + TMEM base
constexpr int kTiSmem = kTiBar + 8 * kTiGroups + 16;
constexpr uint32_t kTiCols = 64 * kTiGroups;               // TMEM columns (a power of two >= 32)
static_assert(kTiSmem <= 227 * 1024, "inference shared memory");
static_assert((kTiCols & (kTiCols - 1)) == 0 && kTiCols <= 512, "TMEM allocation");

__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory");
}

__global__ void __launch_bounds__(kTiThreads, kTiCtasPerSm) k_nrc_infer_tc(NrcDev C, const __nv_bfloat16* __restrict__ X,
                                                                const int* n_dev, int64_t n_static,
                                                                float4* __restrict__ out,
                                                                unsigned* __restrict__ errflags,
                                                                const float* __restrict__ feat) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char* smem = tc_smem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = warp >> 2;              // tile group
    const int gt = tid & 127;             // thread within the group = tile row = TMEM lane
    const int gw = warp & 3;              // warp within the group (TMEM lanes 32 gw .. 32 gw + 31)
    const uint32_t sbase = uint32_t(__cvta_generic_to_shared(smem));
    const uint32_t bar = sbase + kTiBar + 8 * g;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTiBar + 8 * kTiGroups);
    __shared__ int abort_flag[kTiGroups];
    unsigned char* slot = smem + kTiSlot0 + g * kTiSlotBytes;
    const uint32_t sslot = sbase + kTiSlot0 + g * kTiSlotBytes;

    tc_load_weights(C.wb + kNrcW0, 64, 128, smem + kTcW0);
    for (int l = 0; l < 4; ++l) tc_load_weights(C.wb + kNrcW1 + l * 4096, 64, 64, smem + kTcW1 + l * 8192);
    tc_load_weights(C.wb + kNrcW5, 16, 64, smem + kTcW5);
    if (tid < kTiGroups) {
        abort_flag[tid] = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbase + kTiBar + 8 * tid) : "memory");
    }
    if (tid == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sbase + kTiBar + 8 * kTiGroups), "r"(kTiCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + uint32_t(64 * g);           // this group's accumulator columns
    const uint32_t trow = tmem + (uint32_t(gw * 32) << 16);        // this warp's 32 lanes

    const int64_t n = n_dev ? int64_t(*n_dev) : n_static;
    const int64_t ntiles = (n + kTcRows - 1) / kTcRows;
    uint32_t phase = 0;
    for (int64_t tile = int64_t(blockIdx.x) * kTiGroups + g; tile < ntiles; tile += int64_t(gridDim.x) * kTiGroups) {
        const int64_t row0 = tile * kTcRows;
        if (feat) {
            // thread gt encodes row gt of the tile into the input tile (16 chunks of 16 bytes)
            uint32_t w[kNrcIn / 2];
            const int64_t gr = row0 + gt;
            if (gr < n) {
                encode_row(C, feat + size_t(gr) * kNrcFeatFloats, w);
            } else {
#pragma unroll
                for (int k = 0; k < kNrcIn / 2; ++k) w[k] = 0u;
            }
#pragma unroll
            for (int kc = 0; kc < 16; ++kc)
                *reinterpret_cast<uint4*>(slot + tc_off(gt, kc, 16)) =
                    make_uint4(w[4 * kc], w[4 * kc + 1], w[4 * kc + 2], w[4 * kc + 3]);
        } else {
            // input rows -> input tile; 8 lanes write 8 rows of one chunk (conflict-free), 4 chunks per warp
            for (int j = 0; j < 16; ++j) {
                const int u = j * 4 + gw, rg = u >> 2, kq4 = u & 3;
                const int r = rg * 8 + (lane & 7), kc = kq4 * 4 + (lane >> 3);
                const int64_t gr = row0 + r;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (gr < n) v = *reinterpret_cast<const uint4*>(X + size_t(gr) * kNrcIn + kc * 8);
                *reinterpret_cast<uint4*>(slot + tc_off(r, kc, 16)) = v;
            }
        }
        tc_fence_async_smem();
        tc_fence_before();
        group_sync(g);
        for (int layer = 0; layer < 6; ++layer) {
            if (gt == 0) {
                tc_fence_after();
                const int KC = layer == 0 ? 16 : 8;
                const uint32_t b = sbase + (layer == 0 ? kTcW0 : layer < 5 ? kTcW1 + (layer - 1) * 8192 : kTcW5);
                const uint32_t idesc = tc_idesc(layer < 5 ? 64 : 16);
                for (int s = 0; s < KC / 2; ++s)
                    tc_mma(tmem, tc_desc(sslot + s * 256, 128, KC * 128), tc_desc(b + s * 256, 128, KC * 128), idesc,
                           s > 0 ? 1u : 0u);
                tc_commit(bar);
            }
            if (!tc_wait(bar, phase, C.wait_polls)) {
                atomicOr(errflags, BG_FLAG_TIMEOUT);
                abort_flag[g] = 1;
            }
            phase ^= 1u;
            tc_fence_after();
            group_sync(g);
            if (abort_flag[g]) break;
            if (layer < 5) {
                // ReLU, bf16, into the hidden tile (the slot's first 16 KB: the MMA that read them is done)
#pragma unroll
                for (int c4 = 0; c4 < 4; ++c4) {
                    float v[16];
                    tc_ld16(trow + uint32_t(c4 * 16), v);
                    uint4 p0, p1;
                    p0.x = tc_pack(fmaxf(v[0], 0.f), fmaxf(v[1], 0.f));
                    p0.y = tc_pack(fmaxf(v[2], 0.f), fmaxf(v[3], 0.f));
                    p0.z = tc_pack(fmaxf(v[4], 0.f), fmaxf(v[5], 0.f));
                    p0.w = tc_pack(fmaxf(v[6], 0.f), fmaxf(v[7], 0.f));
                    p1.x = tc_pack(fmaxf(v[8], 0.f), fmaxf(v[9], 0.f));
                    p1.y = tc_pack(fmaxf(v[10], 0.f), fmaxf(v[11], 0.f));
                    p1.z = tc_pack(fmaxf(v[12], 0.f), fmaxf(v[13], 0.f));
                    p1.w = tc_pack(fmaxf(v[14], 0.f), fmaxf(v[15], 0.f));
                    *reinterpret_cast<uint4*>(slot + tc_off(gt, 2 * c4, 8)) = p0;
                    *reinterpret_cast<uint4*>(slot + tc_off(gt, 2 * c4 + 1, 8)) = p1;
                }
                tc_fence_async_smem();
            } else {
                float v[16];
                tc_ld16(trow, v);
                if (row0 + gt < n) out[row0 + gt] = make_float4(v[0], v[1], v[2], 0.f);
            }
            tc_fence_before();
            group_sync(g);
        }
        if (abort_flag[g]) break;
    }
    // after a timeout, give the group's outstanding MMA one more bounded wait before the TMEM is freed
    if (abort_flag[g] && gt == 0) tc_wait(bar, phase ^ 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(*tmem_slot), "r"(kTiCols) : "memory");
    }
}


// ------------------------------------------------------------- training
// Fused forward + backward of one Adam step's rows on tcgen05, same outputs as
// the mma.sync k_nrc_train: hidden activations H[l] and layer-output gradients
// DZ[l] (bf16, for the weight-gradient kernels), DZ5, the hash-grid feature
// gradient dX (fp32, 32 columns) and the summed relative-L2 loss.
//
// The backward products dH = dZ * W need B = W with the layer's input features
// as N: the forward weight tiles already hold W[out][in] in 8x8 core matrices
// of 8 rows (out) x 16 contiguous bytes (in), which is exactly an MN-major B
// core matrix (8 K-rows x 8 contiguous N elements), so the backward reads the
// same shared memory through MN-major descriptors (SBO = 128 bytes between
// groups of 8 inputs, LBO = KC * 128 bytes between groups of 8 outputs).
// Each thread keeps its row's ReLU masks (64 bits per hidden layer) in registers.
constexpr int kTtA0 = kTcA0;                 // input tile; reused for the dZ5 tile after layer 0
constexpr int kTtSmem = kTcSmem;

struct TcTrainArgs {
    const __nv_bfloat16* X;      // encoded inputs of this step's rows [B][128]
    const float4* target;        // this step's targets [B] (already offset)
    __nv_bfloat16* H;            // [5][B][64]
    __nv_bfloat16* DZ;           // [5][B][64]
    __nv_bfloat16* DZ5;          // [B][16]
    float* dX;                   // [B][32]
    float* loss;
    int B;
};

__global__ void __launch_bounds__(128, 2) k_nrc_train_tc(NrcDev C, TcTrainArgs T, const int* n_dev, int offset,
                                                         int limit, unsigned* __restrict__ errflags) {
    extern __shared__ __align__(1024) unsigned char tt_smem[];
    unsigned char* smem = tt_smem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = uint32_t(__cvta_generic_to_shared(smem));
    const uint32_t bar = sbase + kTcBar;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTcBar + 8);
    __shared__ int abort_flag;

    tc_load_weights(C.wb + kNrcW0, 64, 128, smem + kTcW0);
    for (int l = 0; l < 4; ++l) tc_load_weights(C.wb + kNrcW1 + l * 4096, 64, 64, smem + kTcW1 + l * 8192);
    tc_load_weights(C.wb + kNrcW5, 16, 64, smem + kTcW5);
    if (tid == 0) {
        abort_flag = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sbase + kTcBar + 8), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);

    int n = n_dev ? *n_dev - offset : T.B;
    if (limit > 0 && n > limit) n = limit;
    if (n < 0) n = 0;
    const float invn = n > 0 ? 1.f / (3.f * float(n)) : 0.f;
    const int ntiles = (n + kTcRows - 1) / kTcRows;
    uint32_t phase = 0;
    float lsum = 0.f;

    // one MMA group on the tile in `a` (K-major, KC chunks) with weights at `b`
    auto run = [&](uint32_t a, int KC, uint32_t b, uint32_t b_lbo, uint32_t b_sbo, uint32_t b_kstep, uint32_t idesc) {
        if (tid == 0) {
            tc_fence_after();
            for (int s = 0; s < KC / 2; ++s)
                tc_mma(tmem, tc_desc(a + s * 256, 128, KC * 128), tc_desc(b + s * b_kstep, b_lbo, b_sbo), idesc,
                       s > 0 ? 1u : 0u);
            tc_commit(bar);
        }
        if (!tc_wait(bar, phase, C.wait_polls)) {
            atomicOr(errflags, BG_FLAG_TIMEOUT);
            abort_flag = 1;
        }
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();
        return abort_flag == 0;
    };
    // this thread's accumulator row (64 columns) -> 8 bf16 chunks, optionally masked / rectified
    auto row64 = [&](uint32_t (&packed)[32], uint32_t (&mask)[2], bool relu, bool apply_mask) {
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
            float v[16];
            tc_ld16(trow + uint32_t(c4 * 16), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = c4 * 16 + j;
                if (relu) {
                    if (v[j] > 0.f) mask[col >> 5] |= 1u << (col & 31);
                    v[j] = fmaxf(v[j], 0.f);
                }
                if (apply_mask && !((mask[col >> 5] >> (col & 31)) & 1u)) v[j] = 0.f;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) packed[c4 * 8 + j] = tc_pack(v[2 * j], v[2 * j + 1]);
        }
    };
    auto store_row = [&](const uint32_t (&packed)[32], __nv_bfloat16* g, int64_t grow, bool to_global) {
        const int r = tid;
#pragma unroll
        for (int kc = 0; kc < 8; ++kc) {
            const uint4 v = make_uint4(packed[4 * kc], packed[4 * kc + 1], packed[4 * kc + 2], packed[4 * kc + 3]);
            *reinterpret_cast<uint4*>(smem + kTcA1 + tc_off(r, kc, 8)) = v;
            if (to_global) reinterpret_cast<uint4*>(g + size_t(grow) * 64)[kc] = v;
        }
    };

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t row0 = int64_t(tile) * kTcRows;
        const int64_t grow = row0 + tid;
        const bool live = grow < n;
        for (int j = 0; j < 16; ++j) {
            const int u = j * 4 + warp, rg = u >> 2, kq4 = u & 3;
            const int r = rg * 8 + (lane & 7), kc = kq4 * 4 + (lane >> 3);
            const int64_t g = row0 + r;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (g < n) v = *reinterpret_cast<const uint4*>(T.X + size_t(g) * kNrcIn + kc * 8);
            *reinterpret_cast<uint4*>(smem + kTtA0 + tc_off(r, kc, 16)) = v;
        }
        tc_fence_async_smem();
        tc_fence_before();
        __syncthreads();
        uint32_t masks[5][2];
#pragma unroll
        for (int l = 0; l < 5; ++l) masks[l][0] = masks[l][1] = 0u;
        bool ok = true;
        // ---- forward: hidden layers
#pragma unroll
        for (int l = 0; l < 5 && ok; ++l) {
            ok = l == 0 ? run(sbase + kTtA0, 16, sbase + kTcW0, 128, 16 * 128, 256, tc_idesc(64))
                        : run(sbase + kTcA1, 8, sbase + kTcW1 + (l - 1) * 8192, 128, 8 * 128, 256, tc_idesc(64));
            if (!ok) break;
            uint32_t packed[32];
            row64(packed, masks[l], true, false);
            store_row(packed, T.H + size_t(l) * T.B * 64, grow, live);
            tc_fence_async_smem();
            tc_fence_before();
            __syncthreads();
        }
        if (!ok) break;
        // ---- output layer and the loss gradient (columns 0..2 of 16)
        if (!run(sbase + kTcA1, 8, sbase + kTcW5, 128, 8 * 128, 256, tc_idesc(16))) break;
        {
            float v[16];
            tc_ld16(trow, v);
            float g[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) g[j] = 0.f;
            if (live) {
                const float* y = reinterpret_cast<const float*>(T.target + grow);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float p = v[j], den = p * p + 0.01f, d = p - y[j];
                    lsum += d * d / den;
                    g[j] = 2.f * d / den * invn;
                }
            }
            uint4 z0, z1;
            z0.x = tc_pack(g[0], g[1]); z0.y = tc_pack(g[2], g[3]); z0.z = tc_pack(g[4], g[5]); z0.w = tc_pack(g[6], g[7]);
            z1.x = tc_pack(g[8], g[9]); z1.y = tc_pack(g[10], g[11]); z1.z = tc_pack(g[12], g[13]); z1.w = tc_pack(g[14], g[15]);
            // dZ5 tile [128 x 16] (K-major, 2 chunks) in the free input-tile space
            *reinterpret_cast<uint4*>(smem + kTtA0 + tc_off(tid, 0, 2)) = z0;
            *reinterpret_cast<uint4*>(smem + kTtA0 + tc_off(tid, 1, 2)) = z1;
            if (live) {
                reinterpret_cast<uint4*>(T.DZ5 + size_t(grow) * 16)[0] = z0;
                reinterpret_cast<uint4*>(T.DZ5 + size_t(grow) * 16)[1] = z1;
            }
        }
        tc_fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // ---- backward: dH4 = dZ5 W5 (K = 16 outputs, N = 64 inputs), then dH_{l-1} = dZ_l W_l
        if (!run(sbase + kTtA0, 2, sbase + kTcW5, 8 * 128, 128, 2 * 8 * 128, tc_idesc(64, true))) break;
#pragma unroll
        for (int l = 4; l >= 0 && ok; --l) {
            uint32_t packed[32];
            row64(packed, masks[l], false, true);              // dZ_l = dH_l masked by ReLU'(z_l)
            store_row(packed, T.DZ + size_t(l) * T.B * 64, grow, live);
            tc_fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (l > 0) {
                ok = run(sbase + kTcA1, 8, sbase + kTcW1 + (l - 1) * 8192, 8 * 128, 128, 2 * 8 * 128,
                         tc_idesc(64, true));
            } else {
                // dX = dZ0 W0, hash-grid columns 0..31 only
                ok = run(sbase + kTcA1, 8, sbase + kTcW0, 16 * 128, 128, 2 * 16 * 128, tc_idesc(32, true));
                if (ok) {
                    float v0[16], v1[16];
                    tc_ld16(trow, v0);
                    tc_ld16(trow + 16u, v1);
                    if (live) {
                        float4* dst = reinterpret_cast<float4*>(T.dX + size_t(grow) * 32);
#pragma unroll
                        for (int q = 0; q < 4; ++q) dst[q] = make_float4(v0[4 * q], v0[4 * q + 1], v0[4 * q + 2], v0[4 * q + 3]);
#pragma unroll
                        for (int q = 0; q < 4; ++q) dst[4 + q] = make_float4(v1[4 * q], v1[4 * q + 1], v1[4 * q + 2], v1[4 * q + 3]);
                    }
                    tc_fence_before();
                    __syncthreads();
                }
            }
        }
        if (!ok || abort_flag) break;
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if (lane == 0 && lsum != 0.f) atomicAdd(T.loss, lsum);
    if (abort_flag && tid == 0) tc_wait(bar, phase ^ 1u);
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTcCols) : "memory");
    }
}


// ------------------------------------------------------------- weight gradients
// The six weight-gradient GEMMs of one Adam step, dW_l[o][i] = sum_s dZ_l[s][o]
// A_l[s][i] (A_0 = the encoded rows X, A_l = H_{l-1}), on tcgen05 in one kernel.
// The samples s are the reduction dimension K: a CTA stages kWgS samples of
// every operand as plain row copies (row s of an operand at tc_off(s, chunk,
// width / 8)), which read as MN-major operands (8 K-rows of 8 contiguous
// M / N elements per core matrix: LBO = the stride between groups of 8
// samples, SBO = 128 bytes between groups of 8 features), exactly as the
// training backward reads its weights.  Every MMA has M = 128: layer 0's A is
// X (128 features); the 64-wide inputs of two layers are stacked into one
// 128-wide A (P1 = [H0 | H1], P2 = [H2 | H3], P3 = [H4 | 0]), and each of them
// is multiplied by the two layers' dZ in turn, so the products needed sit in
// the accumulator's top or bottom 64 lanes (the other half of each product is
// not used).  Accumulators (transposed, D[i][o]) stay in TMEM over the CTA's
// chunks: cols 0-63 dW0^T, 64-127 dW1^T (lanes 0-63), 128-191 dW2^T (lanes
// 64-127), 192-255 dW3^T (0-63), 256-319 dW4^T (64-127), 320-335 dW5^T (0-63);
// at the end each CTA adds them into dW with coalesced float atomics (split K
// over CTAs, as the mma.sync kernels do).
constexpr int kWgS = 128;                                  // samples per staged chunk
constexpr int kWgThreads = 256;
constexpr int kWgX = 0;                                    // [kWgS x 128] A tiles: X, P1, P2, P3
constexpr int kWgA = kWgS * 128 * 2;                       // bytes per A tile
constexpr int kWgDz = 4 * kWgA;                            // [kWgS x 64] x 5: dZ0..dZ4
constexpr int kWgDzB = kWgS * 64 * 2;
constexpr int kWgDz5 = kWgDz + 5 * kWgDzB;                 // [kWgS x 16]
constexpr int kWgBar = kWgDz5 + kWgS * 16 * 2;
constexpr int kWgSmem = kWgBar + 16;
constexpr uint32_t kWgCols = 512;
static_assert(kWgSmem <= 227 * 1024, "weight-gradient shared memory");

struct TcWgradArgs {
    const __nv_bfloat16* X;      // [B][128] encoded rows
    const __nv_bfloat16* H;      // [5][B][64]
    const __nv_bfloat16* DZ;     // [5][B][64]
    const __nv_bfloat16* DZ5;    // [B][16]
    float* dW;                   // [kNrcParams], accumulated
    int B;
};

__global__ void __launch_bounds__(kWgThreads, 1) k_nrc_wgrad_tc(NrcDev C, TcWgradArgs T, const int* n_dev, int offset,
                                                                int limit, unsigned* __restrict__ errflags) {
    extern __shared__ __align__(1024) unsigned char wg_smem[];
    unsigned char* smem = wg_smem;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = uint32_t(__cvta_generic_to_shared(smem));
    const uint32_t bar = sbase + kWgBar;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kWgBar + 8);
    __shared__ int abort_flag;

    int n = n_dev ? *n_dev - offset : T.B;
    if (limit > 0 && n > limit) n = limit;
    if (n < 0) n = 0;
    const int nchunks = (n + kWgS - 1) / kWgS;
    if (int(blockIdx.x) >= nchunks) return;   // (uniform per CTA, before any TMEM allocation)

    // the zero half of P3 is written once
    for (int v = tid; v < kWgS * 8; v += kWgThreads) {
        const int sl = v >> 3, kc = 8 + (v & 7);
        *reinterpret_cast<uint4*>(smem + kWgX + 3 * kWgA + tc_off(sl, kc, 16)) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid == 0) {
        abort_flag = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sbase + kWgBar + 8), "r"(kWgCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const size_t L = size_t(T.B) * 64;
    uint32_t phase = 0;
    bool first = true;
    for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const int s0 = chunk * kWgS;
        // stage: 16-byte pieces of sample rows; rows past n are zero
        for (int v = tid; v < kWgS * 16; v += kWgThreads) {              // X: 16 chunks per row
            const int sl = v >> 4, kc = v & 15;
            uint4 x = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) x = *reinterpret_cast<const uint4*>(T.X + size_t(s0 + sl) * 128 + kc * 8);
            *reinterpret_cast<uint4*>(smem + kWgX + tc_off(sl, kc, 16)) = x;
        }
        for (int v = tid; v < kWgS * 8 * 5; v += kWgThreads) {           // H0..H4 into P1, P2, P3
            const int l = v / (kWgS * 8), r = v % (kWgS * 8), sl = r >> 3, kc = r & 7;
            uint4 x = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) x = *reinterpret_cast<const uint4*>(T.H + size_t(l) * L + size_t(s0 + sl) * 64 + kc * 8);
            const int tile = 1 + (l >> 1), half = l & 1;
            *reinterpret_cast<uint4*>(smem + kWgX + tile * kWgA + tc_off(sl, kc + 8 * half, 16)) = x;
        }
        for (int v = tid; v < kWgS * 8 * 5; v += kWgThreads) {           // dZ0..dZ4
            const int l = v / (kWgS * 8), r = v % (kWgS * 8), sl = r >> 3, kc = r & 7;
            uint4 x = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) x = *reinterpret_cast<const uint4*>(T.DZ + size_t(l) * L + size_t(s0 + sl) * 64 + kc * 8);
            *reinterpret_cast<uint4*>(smem + kWgDz + l * kWgDzB + tc_off(sl, kc, 8)) = x;
        }
        for (int v = tid; v < kWgS * 2; v += kWgThreads) {               // dZ5
            const int sl = v >> 1, kc = v & 1;
            uint4 x = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) x = *reinterpret_cast<const uint4*>(T.DZ5 + size_t(s0 + sl) * 16 + kc * 8);
            *reinterpret_cast<uint4*>(smem + kWgDz5 + tc_off(sl, kc, 2)) = x;
        }
        tc_fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            // (A tile, its LBO) x (B tile, its LBO, N) -> TMEM columns
            auto gemm = [&](uint32_t a, uint32_t b, uint32_t b_lbo, int N, uint32_t col) {
                const uint32_t idesc = tc_idesc(N, true) | (1u << 15);   // A and B MN-major
                for (int k = 0; k < kWgS / 16; ++k)
                    tc_mma(tmem + col, tc_desc(a + k * 2 * 2048, 2048, 128), tc_desc(b + k * 2 * b_lbo, b_lbo, 128),
                           idesc, (first && k == 0) ? 0u : 1u);
            };
            const uint32_t A0 = sbase + kWgX, P1 = A0 + kWgA, P2 = A0 + 2 * kWgA, P3 = A0 + 3 * kWgA;
            const uint32_t Z = sbase + kWgDz;
            gemm(A0, Z + 0 * kWgDzB, 1024, 64, 0);
            gemm(P1, Z + 1 * kWgDzB, 1024, 64, 64);
            gemm(P1, Z + 2 * kWgDzB, 1024, 64, 128);
            gemm(P2, Z + 3 * kWgDzB, 1024, 64, 192);
            gemm(P2, Z + 4 * kWgDzB, 1024, 64, 256);
            gemm(P3, sbase + kWgDz5, 256, 16, 320);
            tc_commit(bar);
        }
        first = false;
        if (!tc_wait(bar, phase, C.wait_polls)) {
            atomicOr(errflags, BG_FLAG_TIMEOUT);
            abort_flag = 1;
        }
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();   // the MMAs have read this chunk's tiles before they are overwritten
        if (abort_flag) break;
    }
    if (!abort_flag) {
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (lane = feature i); warps w and w + 4
        // split the columns
        const int q = warp & 3, half = warp >> 2;
        const int i = q * 32 + (tid & 31);
        const uint32_t trow = tmem + (uint32_t(q * 32) << 16);
        auto out = [&](uint32_t col0, int ncols, float* dst, int ld, int ioff) {
            for (int c = 0; c < ncols; c += 16) {
                float v[16];
                tc_ld16(trow + col0 + uint32_t(c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) atomicAdd(dst + size_t(c + j) * ld + (i - ioff), v[j]);
            }
        };
        float* dW = T.dW;
        if (half == 0) {
            out(0, 64, dW + kNrcW0, 128, 0);                                   // dW0[o][i], i = 0..127
            if (i < 64) out(64, 64, dW + kNrcW1, 64, 0);                       // dW1 = H0^T dZ1
            else out(128, 64, dW + kNrcW1 + 4096, 64, 64);                     // dW2 = H1^T dZ2
        } else {
            if (i < 64) {
                out(192, 64, dW + kNrcW1 + 2 * 4096, 64, 0);                   // dW3 = H2^T dZ3
                out(320, 16, dW + kNrcW5, 64, 0);                              // dW5 = H4^T dZ5
            } else {
                out(256, 64, dW + kNrcW1 + 3 * 4096, 64, 64);                  // dW4 = H3^T dZ4
            }
        }
    }
    // after a timeout, give the outstanding MMA group one more bounded wait before freeing its TMEM
    if (abort_flag && tid == 0) tc_wait(bar, phase ^ 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kWgCols) : "memory");
    }
}

}  // namespace bg
