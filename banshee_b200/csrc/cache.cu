// Neural radiance cache (see cache.h): encoding, fused BF16 tensor-core MLP
// inference and training, hash-grid backward, Adam, and its C ABI.
//
// The MLP kernels keep a warp's 16 rows in registers through all six layers:
// the fp32 accumulator fragment of mma.m16n8k16 for output columns 16j..16j+15
// is, after ReLU and bf16 packing, exactly the A fragment of k-tile j of the
// next layer, so activations never leave the register file.  Weights live in
// shared memory with rows padded by 8 elements (conflict-free fragment loads);
// the backward pass uses a transposed copy.
#include <cmath>
#include <cstring>
#include <vector>

#include "cache.h"
#include "internal.h"
#include "nrc_encode.cuh"
#include "nrc_tcgen05.cuh"

namespace bg {

// ------------------------------------------------------------- helpers
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float lo_f(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float hi_f(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// shared-memory layouts (bf16 elements): forward W[out][in], backward W^T[in][out]
constexpr int kS0 = 136, kS1 = 72, kS5 = 72;           // forward row strides
constexpr int kFwW0 = 0, kFwW1 = kFwW0 + 64 * kS0, kFwW5 = kFwW1 + 4 * 64 * kS1, kFwTotal = kFwW5 + 16 * kS5;
constexpr int kT0 = 72, kT1 = 72, kT5 = 24;            // backward row strides
constexpr int kBwW0 = 0, kBwW1 = kBwW0 + 128 * kT0, kBwW5 = kBwW1 + 4 * 64 * kT1, kBwTotal = kBwW5 + 64 * kT5;

__device__ void load_weights_fwd(const __nv_bfloat16* __restrict__ wb, __nv_bfloat16* s) {
    for (int i = threadIdx.x; i < kNrcParams; i += blockDim.x) {
        int off;
        if (i < kNrcW1) off = kFwW0 + (i / 128) * kS0 + (i % 128);
        else if (i < kNrcW5) { int j = i - kNrcW1, l = j / 4096, k = j % 4096; off = kFwW1 + l * 64 * kS1 + (k / 64) * kS1 + (k % 64); }
        else { int j = i - kNrcW5; off = kFwW5 + (j / 64) * kS5 + (j % 64); }
        s[off] = wb[i];
    }
}
__device__ void load_weights_bwd(const __nv_bfloat16* __restrict__ wb, __nv_bfloat16* s) {
    for (int i = threadIdx.x; i < kNrcParams; i += blockDim.x) {
        int off;
        if (i < kNrcW1) { int o = i / 128, in = i % 128; off = kBwW0 + in * kT0 + o; }
        else if (i < kNrcW5) { int j = i - kNrcW1, l = j / 4096, k = j % 4096, o = k / 64, in = k % 64; off = kBwW1 + l * 64 * kT1 + in * kT1 + o; }
        else { int j = i - kNrcW5, o = j / 64, in = j % 64; off = kBwW5 + in * kT5 + o; }
        s[off] = wb[i];
    }
}

// acc[NT] += A[KT] x B, with B[k][n] = W[n][k] (row stride `stride`)
template <int KT, int NT>
__device__ __forceinline__ void mlp_layer(const uint32_t (&a)[KT][4], const __nv_bfloat16* W, int stride, float (&acc)[NT][4]) {
    const int lane = threadIdx.x & 31, r = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const __nv_bfloat16* wp = W + (nt * 8 + r) * stride + kt * 16 + c;
            uint32_t b0 = *reinterpret_cast<const uint32_t*>(wp);
            uint32_t b1 = *reinterpret_cast<const uint32_t*>(wp + 8);
            mma16816(acc[nt], a[kt], b0, b1);
        }
    }
}

// accumulator fragments of 2*KT n-tiles -> A fragments of KT k-tiles
template <int KT>
__device__ __forceinline__ void to_afrag(const float (&acc)[2 * KT][4], uint32_t (&a)[KT][4], bool relu) {
#pragma unroll
    for (int j = 0; j < KT; ++j) {
        float v[8] = {acc[2 * j][0], acc[2 * j][1], acc[2 * j][2], acc[2 * j][3],
                      acc[2 * j + 1][0], acc[2 * j + 1][1], acc[2 * j + 1][2], acc[2 * j + 1][3]};
        if (relu) {
#pragma unroll
            for (int e = 0; e < 8; ++e) v[e] = fmaxf(v[e], 0.f);
        }
        a[j][0] = pack2(v[0], v[1]);
        a[j][1] = pack2(v[2], v[3]);
        a[j][2] = pack2(v[4], v[5]);
        a[j][3] = pack2(v[6], v[7]);
    }
}

// zero the gradient entries whose forward activation (A fragments h) was <= 0
template <int KT>
__device__ __forceinline__ void relu_mask(float (&g)[2 * KT][4], const uint32_t (&h)[KT][4]) {
#pragma unroll
    for (int nt = 0; nt < 2 * KT; ++nt) {
        const int j = nt >> 1, q = (nt & 1) ? 2 : 0;
        if (!(lo_f(h[j][q]) > 0.f)) g[nt][0] = 0.f;
        if (!(hi_f(h[j][q]) > 0.f)) g[nt][1] = 0.f;
        if (!(lo_f(h[j][q + 1]) > 0.f)) g[nt][2] = 0.f;
        if (!(hi_f(h[j][q + 1]) > 0.f)) g[nt][3] = 0.f;
    }
}

// store A fragments (16 rows x 16*KT cols) as bf16 rows [row][ld]
template <int KT>
__device__ __forceinline__ void store_afrag(const uint32_t (&a)[KT][4], __nv_bfloat16* base, int row0, int nrows, int ld) {
    const int lane = threadIdx.x & 31, r = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = row0 + r + ((q & 1) ? 8 : 0);
            const int col = 16 * j + c + ((q & 2) ? 8 : 0);
            if (row < nrows) *reinterpret_cast<uint32_t*>(base + size_t(row) * ld + col) = a[j][q];
        }
    }
}

__device__ __forceinline__ void load_input(const __nv_bfloat16* X, int row0, int nrows, uint32_t (&a)[8][4]) {
    const int lane = threadIdx.x & 31, r = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
    for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = row0 + r + ((q & 1) ? 8 : 0);
            const int col = 16 * kt + c + ((q & 2) ? 8 : 0);
            a[kt][q] = row < nrows ? *reinterpret_cast<const uint32_t*>(X + size_t(row) * kNrcIn + col) : 0u;
        }
    }
}

// forward through all layers; h[l] (l = 0..4) = post-ReLU hidden activations
__device__ __forceinline__ void mlp_forward(const __nv_bfloat16* sw, const uint32_t (&ain)[8][4], uint32_t (&h)[5][4][4],
                                            float (&out)[2][4]) {
    float acc[8][4];
    mlp_layer<8, 8>(ain, sw + kFwW0, kS0, acc);
    to_afrag<4>(acc, h[0], true);
#pragma unroll
    for (int l = 1; l < 5; ++l) {
        mlp_layer<4, 8>(h[l - 1], sw + kFwW1 + (l - 1) * 64 * kS1, kS1, acc);
        to_afrag<4>(acc, h[l], true);
    }
    mlp_layer<4, 2>(h[4], sw + kFwW5, kS5, out);
}

// raw query records [n][16] -> encoded bf16 rows [n][128] (the training path;
// inference encodes inside k_nrc_infer_tc).  The row is built in 64 registers
// and stored as 16-byte chunks.
__global__ void __launch_bounds__(128) k_nrc_encode(NrcDev C, const float* __restrict__ feat, const int* n_dev, int64_t n_static,
                                                    int offset, int limit, __nv_bfloat16* __restrict__ X) {
    int64_t n = n_dev ? int64_t(*n_dev) : n_static;
    n = n - offset;
    if (limit > 0 && n > limit) n = limit;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint32_t w[kNrcIn / 2];
        encode_row(C, feat + (size_t(offset) + size_t(i)) * kNrcFeatFloats, w);
        uint4* dst = reinterpret_cast<uint4*>(X + size_t(i) * kNrcIn);
#pragma unroll
        for (int k = 0; k < kNrcIn / 8; ++k) dst[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    }
}

// ------------------------------------------------------------- inference
// out[i] = (r, g, b, 0) for the n encoded rows
__global__ void __launch_bounds__(128) k_nrc_infer(NrcDev C, const __nv_bfloat16* __restrict__ X, const int* n_dev,
                                                   int64_t n_static, float4* __restrict__ out) {
    extern __shared__ __align__(16) __nv_bfloat16 sw[];
    load_weights_fwd(C.wb, sw);
    __syncthreads();
    const int64_t n = n_dev ? int64_t(*n_dev) : n_static;
    const int lane = threadIdx.x & 31, r = lane >> 2, q = lane & 3;
    const int warps = blockDim.x / 32;
    for (int64_t tile = int64_t(blockIdx.x) * warps + (threadIdx.x >> 5); tile * 16 < n; tile += int64_t(gridDim.x) * warps) {
        const int row0 = int(tile * 16);
        uint32_t ain[8][4];
        load_input(X, row0, int(n), ain);
        uint32_t h[5][4][4];
        float o[2][4];
        mlp_forward(sw, ain, h, o);
        // columns 0,1 live in lanes with q == 0, column 2 in lanes with q == 1
        if (q <= 1) {
            for (int half = 0; half < 2; ++half) {
                const int row = row0 + r + 8 * half;
                if (row >= n) continue;
                float* dst = reinterpret_cast<float*>(out + row);
                if (q == 0) { dst[0] = o[0][2 * half]; dst[1] = o[0][2 * half + 1]; }
                else { dst[2] = o[0][2 * half]; dst[3] = 0.f; }
            }
        }
    }
}

// ------------------------------------------------------------- training
struct TrainBufs {
    const __nv_bfloat16* X;     // encoded inputs [B][128]
    const float4* target;       // [B]
    __nv_bfloat16* H;           // hidden activations h1..h5, [5][B][64]
    __nv_bfloat16* DZ;          // gradients of layer outputs: dZ0..dZ4 [5][B][64], dZ5 at DZ5
    __nv_bfloat16* DZ5;         // [B][16]
    float* dX;                  // [B][32] gradient of the hash-grid features
    float* loss;                // accumulated sum of the relative L2 terms
    int B;                      // rows in this step
};

__global__ void __launch_bounds__(128) k_nrc_train(NrcDev C, TrainBufs T, const int* n_dev, int offset, int limit) {
    extern __shared__ __align__(16) __nv_bfloat16 smem[];
    __nv_bfloat16* sw = smem;
    __nv_bfloat16* st = smem + kFwTotal;
    load_weights_fwd(C.wb, sw);
    load_weights_bwd(C.wb, st);
    __syncthreads();
    int n = n_dev ? *n_dev - offset : T.B;
    if (limit > 0 && n > limit) n = limit;
    const float invn = n > 0 ? 1.f / (3.f * float(n)) : 0.f;
    const int lane = threadIdx.x & 31, r = lane >> 2, q = lane & 3, c = q * 2;
    const int warps = blockDim.x / 32;
    float lsum = 0.f;
    for (int tile = blockIdx.x * warps + (threadIdx.x >> 5); tile * 16 < n; tile += gridDim.x * warps) {
        const int row0 = tile * 16;
        uint32_t ain[8][4];
        load_input(T.X, row0, n, ain);
        uint32_t h[5][4][4];
        float o[2][4];
        mlp_forward(sw, ain, h, o);
#pragma unroll
        for (int l = 0; l < 5; ++l) store_afrag<4>(h[l], T.H + size_t(l) * T.B * 64, row0, n, 64);
        // relative L2 loss gradient on the 3 used outputs (columns 0..2 of n-tile 0)
        float g[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = row0 + r + ((e & 2) ? 8 : 0);
            const int col = c + (e & 1);
            if (row < n && col < 3) {
                const float y = reinterpret_cast<const float*>(T.target + row)[col];
                const float p = o[0][e];
                const float den = p * p + 0.01f;
                const float d = p - y;
                lsum += d * d / den;
                g[0][e] = 2.f * d / den * invn;
            }
        }
        uint32_t adz[4][4];
        uint32_t adz5[1][4];
        to_afrag<1>(g, adz5, false);
        store_afrag<1>(adz5, T.DZ5, row0, n, 16);
        float acc[8][4];
        mlp_layer<1, 8>(adz5, st + kBwW5, kT5, acc);       // dH5 = dZ5 W5
        relu_mask<4>(acc, h[4]);
        to_afrag<4>(acc, adz, false);
        store_afrag<4>(adz, T.DZ + size_t(4) * T.B * 64, row0, n, 64);
#pragma unroll
        for (int l = 4; l >= 1; --l) {                      // dH_l = dZ_l W_l, masked by h_{l-1}
            mlp_layer<4, 8>(adz, st + kBwW1 + (l - 1) * 64 * kT1, kT1, acc);
            relu_mask<4>(acc, h[l - 1]);
            to_afrag<4>(acc, adz, false);
            store_afrag<4>(adz, T.DZ + size_t(l - 1) * T.B * 64, row0, n, 64);
        }
        float dx[4][4];                                     // dX (hash-grid columns 0..31) = dZ0 W0
        mlp_layer<4, 4>(adz, st + kBwW0, kT0, dx);
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = row0 + r + ((e & 2) ? 8 : 0);
                const int col = nt * 8 + c + (e & 1);
                if (row < n) T.dX[size_t(row) * 32 + col] = dx[nt][e];
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
    if (lane == 0) atomicAdd(T.loss, lsum);
}

// dW[o][i] += sum_s dZ[s][o] X[s][i] over this block's sample chunks (split K).
template <int OUT, int IN>
__global__ void __launch_bounds__(256) k_nrc_wgrad(const __nv_bfloat16* __restrict__ DZ, const __nv_bfloat16* __restrict__ X,
                                                   const int* n_dev, int offset, int limit, int Bstatic, float* __restrict__ dW) {
    constexpr int KC = 64, LD = KC + 8;   // samples per staged chunk (static shared memory <= 48 KB)
    constexpr int MT = OUT / 16, NTT = IN / 8, PAIRS = MT * NTT, PW = PAIRS / 8;
    __shared__ __align__(16) __nv_bfloat16 dzT[OUT * LD];
    __shared__ __align__(16) __nv_bfloat16 xT[IN * LD];
    int n = n_dev ? *n_dev - offset : Bstatic;
    if (limit > 0 && n > limit) n = limit;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, r = lane >> 2, c = (lane & 3) * 2;
    float acc[PW][4];
#pragma unroll
    for (int p = 0; p < PW; ++p) acc[p][0] = acc[p][1] = acc[p][2] = acc[p][3] = 0.f;
    for (int s0 = blockIdx.x * KC; s0 < n; s0 += gridDim.x * KC) {
        __syncthreads();
        for (int v = threadIdx.x; v < KC * (OUT / 8); v += blockDim.x) {
            const int sl = v / (OUT / 8), o0 = (v % (OUT / 8)) * 8;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) w = *reinterpret_cast<const uint4*>(DZ + size_t(s0 + sl) * OUT + o0);
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&w);
#pragma unroll
            for (int j = 0; j < 8; ++j) dzT[(o0 + j) * LD + sl] = e[j];
        }
        for (int v = threadIdx.x; v < KC * (IN / 8); v += blockDim.x) {
            const int sl = v / (IN / 8), i0 = (v % (IN / 8)) * 8;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (s0 + sl < n) w = *reinterpret_cast<const uint4*>(X + size_t(s0 + sl) * IN + i0);
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&w);
#pragma unroll
            for (int j = 0; j < 8; ++j) xT[(i0 + j) * LD + sl] = e[j];
        }
        __syncthreads();
#pragma unroll
        for (int p = 0; p < PW; ++p) {
            const int pair = warp + 8 * p;
            const int m0 = (pair % MT) * 16, n0 = (pair / MT) * 8;
#pragma unroll
            for (int k0 = 0; k0 < KC; k0 += 16) {
                uint32_t a[4];
                a[0] = *reinterpret_cast<const uint32_t*>(dzT + (m0 + r) * LD + k0 + c);
                a[1] = *reinterpret_cast<const uint32_t*>(dzT + (m0 + r + 8) * LD + k0 + c);
                a[2] = *reinterpret_cast<const uint32_t*>(dzT + (m0 + r) * LD + k0 + c + 8);
                a[3] = *reinterpret_cast<const uint32_t*>(dzT + (m0 + r + 8) * LD + k0 + c + 8);
                uint32_t b0 = *reinterpret_cast<const uint32_t*>(xT + (n0 + r) * LD + k0 + c);
                uint32_t b1 = *reinterpret_cast<const uint32_t*>(xT + (n0 + r) * LD + k0 + c + 8);
                mma16816(acc[p], a, b0, b1);
            }
        }
    }
#pragma unroll
    for (int p = 0; p < PW; ++p) {
        const int pair = warp + 8 * p;
        const int m0 = (pair % MT) * 16, n0 = (pair / MT) * 8;
        atomicAdd(dW + (m0 + r) * IN + n0 + c, acc[p][0]);
        atomicAdd(dW + (m0 + r) * IN + n0 + c + 1, acc[p][1]);
        atomicAdd(dW + (m0 + r + 8) * IN + n0 + c, acc[p][2]);
        atomicAdd(dW + (m0 + r + 8) * IN + n0 + c + 1, acc[p][3]);
    }
}

// hash-grid backward: scatter dX through the trilinear weights
__global__ void __launch_bounds__(128) k_nrc_grid_bwd(NrcDev C, const float* __restrict__ feat, const float* __restrict__ dX,
                                                      const int* n_dev, int offset, int limit, int Bstatic) {
    int n = n_dev ? *n_dev - offset : Bstatic;
    if (limit > 0 && n > limit) n = limit;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* f = feat + (size_t(offset) + size_t(i)) * kNrcFeatFloats;
        float fr[3] = {f[0], f[1], f[2]};
        float u[3];
        norm_pos(C, fr, u);
        for (int l = 0; l < kNrcLevels; ++l) {
            const float g0 = dX[size_t(i) * 32 + 2 * l], g1 = dX[size_t(i) * 32 + 2 * l + 1];
            if (g0 == 0.f && g1 == 0.f) continue;
            GridCorner g = grid_cell(C, l, u);
#pragma unroll
            for (int cidx = 0; cidx < 8; ++cidx) {
                const int dx = cidx & 1, dy = (cidx >> 1) & 1, dz = (cidx >> 2) & 1;
                const float w = (dx ? g.fx : 1.f - g.fx) * (dy ? g.fy : 1.f - g.fy) * (dz ? g.fz : 1.f - g.fz);
                const uint32_t idx = grid_index(C, l, g.x0 + dx, g.y0 + dy, g.z0 + dz);
                float* dst = C.grid_grad + (size_t(l) << C.log2_T) * 2 + size_t(idx) * 2;
                atomicAdd(reinterpret_cast<float2*>(dst), make_float2(w * g0, w * g1));   // both features, one vector atomic
            }
        }
    }
}

__global__ void k_nrc_step(int* step) { *step += 1; }

// Adam on fp32 masters; optionally writes a bf16 copy; clears the gradient.
__global__ void __launch_bounds__(256) k_nrc_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                                                  float* __restrict__ v, int64_t n, const int* step, float lr, float b1,
                                                  float b2, float eps, __nv_bfloat16* __restrict__ out) {
    const int t = *step;
    const float c1 = 1.f / (1.f - powf(b1, float(t))), c2 = 1.f / (1.f - powf(b2, float(t)));
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        g[i] = 0.f;
        if (out) out[i] = __float2bfloat16_rn(pi);
    }
}

// Adam over the hash grid, four parameters per thread.  A quad whose gradient
// and both moments are zero (table entries no sample has reached yet, among
// them the unused tails of the densely indexed coarse levels) is left as it
// is: the update would change none of its values.
__global__ void __launch_bounds__(256) k_nrc_adam4(float4* __restrict__ p, float4* __restrict__ g,
                                                   float4* __restrict__ m, float4* __restrict__ v, int64_t n4,
                                                   const int* step, float lr, float b1, float b2, float eps) {
    const int t = *step;
    const float c1 = 1.f / (1.f - powf(b1, float(t))), c2 = 1.f / (1.f - powf(b2, float(t)));
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n4; i += int64_t(gridDim.x) * blockDim.x) {
        const float4 gi = g[i], mi = m[i], vi = v[i];
        if (gi.x == 0.f && gi.y == 0.f && gi.z == 0.f && gi.w == 0.f && mi.x == 0.f && mi.y == 0.f && mi.z == 0.f &&
            mi.w == 0.f && vi.x == 0.f && vi.y == 0.f && vi.z == 0.f && vi.w == 0.f)
            continue;
        float4 pi = p[i], mo, vo;
        const float ga[4] = {gi.x, gi.y, gi.z, gi.w}, ma[4] = {mi.x, mi.y, mi.z, mi.w}, va[4] = {vi.x, vi.y, vi.z, vi.w};
        float pa[4] = {pi.x, pi.y, pi.z, pi.w}, mn[4], vn[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            mn[k] = b1 * ma[k] + (1.f - b1) * ga[k];
            vn[k] = b2 * va[k] + (1.f - b2) * ga[k] * ga[k];
            pa[k] = pa[k] - lr * (mn[k] * c1) / (sqrtf(vn[k] * c2) + eps);
        }
        mo = make_float4(mn[0], mn[1], mn[2], mn[3]);
        vo = make_float4(vn[0], vn[1], vn[2], vn[3]);
        m[i] = mo;
        v[i] = vo;
        p[i] = make_float4(pa[0], pa[1], pa[2], pa[3]);
        g[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

__global__ void k_nrc_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = __float2bfloat16_rn(p[i]);
}

}  // namespace bg

// ============================================================= host side
struct bg_cache {
    bg_scene* scene = nullptr;
    bg_cache_desc desc{};
    bg::NrcDev dev{};
    bg::DevBuf grid, grid_grad, grid_m, grid_v, w, w_grad, w_m, w_v, wb, step;
    bg::DevBuf X, H, DZ, DZ5, dX, loss;   // training scratch; X also holds encoded mma.sync queries
    int64_t train_cap = 0;                // training rows H, DZ, DZ5 and dX hold
    int64_t x_cap = 0;                    // encoded rows X holds
    int sms = 0;
    int64_t frame = 0;
    uint64_t id = 0;          // unique over the process (captured passes key on it)
    uint64_t buf_epoch = 0;   // a fresh process-unique value whenever the scratch moves
};

namespace bg {

void render_forget_cache(bg_scene* s, const bg_cache* c);   // render.cu

static int64_t grid_params(const bg_cache* c) { return int64_t(kNrcLevels) * (int64_t(1) << c->dev.log2_T) * kNrcFeat; }

static std::atomic<uint64_t> g_cache_ids{1};

// Scratch for up to `train_rows` rows of one Adam step (encoded rows, hidden
// activations and layer gradients of the fused training kernels) and for
// `query_rows` queries at a time.  The tcgen05 inference kernel encodes its
// queries in shared memory and needs none; the mma.sync path encodes them
// into X first.  (Sizing everything by the pass, 2^24 paths, took 28.6 GB.)
static int cache_scratch(bg_cache* c, int64_t train_rows, int64_t query_rows) {
    const int64_t xr = std::max(train_rows, c->desc.mlp_kernel == 0 ? int64_t(0) : query_rows);
    if (train_rows <= c->train_cap && xr <= c->x_cap) return BG_OK;
    c->buf_epoch = g_cache_ids.fetch_add(1);   // captured passes bake X in (mma.sync queries)
    int rc;
    if (xr > c->x_cap) {
        if ((rc = c->X.ensure(size_t(xr) * kNrcIn * 2))) return rc;
        c->x_cap = xr;
    }
    if (train_rows > c->train_cap) {
        const size_t R = size_t(train_rows);
        if ((rc = c->H.ensure(5 * R * 64 * 2)) || (rc = c->DZ.ensure(5 * R * 64 * 2)) || (rc = c->DZ5.ensure(R * 16 * 2)) ||
            (rc = c->dX.ensure(R * 32 * 4)))
            return rc;
        c->train_cap = train_rows;
    }
    return BG_OK;
}

static uint64_t mix64(uint64_t z) { return splitmix64(z); }

static int cache_init_params(bg_cache* c) {
    const int64_t gp = grid_params(c);
    std::vector<float> g(static_cast<size_t>(gp)), w(kNrcParams);
    uint64_t s = c->desc.seed * 0x9E3779B97F4A7C15ull + 12345u;
    for (int64_t i = 0; i < gp; ++i) {
        double u = double(mix64(s + uint64_t(i)) >> 11) * (1.0 / 9007199254740992.0);
        g[size_t(i)] = float((u * 2.0 - 1.0) * 1e-4);
    }
    auto fill = [&](int off, int out, int in, uint64_t salt) {
        const double lim = std::sqrt(6.0 / double(in + out));
        for (int i = 0; i < out * in; ++i) {
            double u = double(mix64(s ^ (salt * 0xD1B54A32D192ED03ull) ^ uint64_t(i)) >> 11) * (1.0 / 9007199254740992.0);
            w[size_t(off + i)] = float((u * 2.0 - 1.0) * lim);
        }
    };
    fill(kNrcW0, 64, 128, 1);
    for (int l = 0; l < 4; ++l) fill(kNrcW1 + l * 4096, 64, 64, 2 + l);
    fill(kNrcW5, 16, 64, 7);
    BG_CUDA(cudaMemcpy(c->grid.ptr, g.data(), g.size() * 4, cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemcpy(c->w.ptr, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemset(c->grid_grad.ptr, 0, size_t(gp) * 4));
    BG_CUDA(cudaMemset(c->grid_m.ptr, 0, size_t(gp) * 4));
    BG_CUDA(cudaMemset(c->grid_v.ptr, 0, size_t(gp) * 4));
    BG_CUDA(cudaMemset(c->w_grad.ptr, 0, kNrcParams * 4));
    BG_CUDA(cudaMemset(c->w_m.ptr, 0, kNrcParams * 4));
    BG_CUDA(cudaMemset(c->w_v.ptr, 0, kNrcParams * 4));
    BG_CUDA(cudaMemset(c->step.ptr, 0, 16));
    k_nrc_to_bf16<<<64, 256>>>(c->w.as<float>(), c->wb.as<__nv_bfloat16>(), kNrcParams);
    BG_CUDA(cudaGetLastError());
    BG_CUDA(cudaDeviceSynchronize());
    return BG_OK;
}

static constexpr int kInferSmem = kFwTotal * 2;
static constexpr int kTrainSmem = (kFwTotal + kBwTotal) * 2;

int nrc_encode(bg_cache* c, const float* feat, const int* n_dev, int64_t n_static, int offset, int limit, cudaStream_t st) {
    k_nrc_encode<<<c->sms * 8, 128, 0, st>>>(c->dev, feat, n_dev, n_static, offset, limit, c->X.as<__nv_bfloat16>());
    BG_CUDA(cudaGetLastError());
    return BG_OK;
}

int nrc_infer(bg_cache* c, const int* n_dev, int64_t n_static, float4* out, cudaStream_t st) {
    if (c->desc.mlp_kernel == 0)
        k_nrc_infer_tc<<<c->sms * kTiCtasPerSm, kTiThreads, kTiSmem, st>>>(c->dev, c->X.as<__nv_bfloat16>(), n_dev, n_static, out,
                                                          c->scene->dev.errflags, nullptr);
    else
        k_nrc_infer<<<c->sms * 4, 128, kInferSmem, st>>>(c->dev, c->X.as<__nv_bfloat16>(), n_dev, n_static, out);
    BG_CUDA(cudaGetLastError());
    return BG_OK;
}

// Cache prediction for raw query records: on tcgen05 the encoding is fused
// into the inference kernel; the mma.sync path encodes into X first.
int nrc_query(bg_cache* c, const float* feat, const int* n_dev, int64_t n_static, float4* out, cudaStream_t st) {
    if (c->desc.mlp_kernel == 0) {
        k_nrc_infer_tc<<<c->sms * kTiCtasPerSm, kTiThreads, kTiSmem, st>>>(c->dev, nullptr, n_dev, n_static, out, c->scene->dev.errflags,
                                                          feat);
        BG_CUDA(cudaGetLastError());
        return BG_OK;
    }
    int rc;
    if ((rc = nrc_encode(c, feat, n_dev, n_static, 0, 0, st))) return rc;
    return nrc_infer(c, n_dev, n_static, out, st);
}

// One Adam step on rows [offset, offset + B) of (feat, target); n from n_dev or B.
int nrc_train_step(bg_cache* c, const float* feat, const float4* target, const int* n_dev, int offset, int B, bool apply,
                   cudaStream_t st) {
    int rc;
    if ((rc = nrc_encode(c, feat, n_dev, B, offset, B, st))) return rc;
    TrainBufs T;
    T.X = c->X.as<__nv_bfloat16>();
    T.target = target + offset;
    T.H = c->H.as<__nv_bfloat16>();
    T.DZ = c->DZ.as<__nv_bfloat16>();
    T.DZ5 = c->DZ5.as<__nv_bfloat16>();
    T.dX = c->dX.as<float>();
    T.loss = c->loss.as<float>();
    T.B = B;
    if (c->desc.mlp_kernel == 0) {
        TcTrainArgs A{T.X, T.target, T.H, T.DZ, T.DZ5, T.dX, T.loss, T.B};
        k_nrc_train_tc<<<c->sms * 2, 128, kTtSmem, st>>>(c->dev, A, n_dev, offset, B, c->scene->dev.errflags);
    } else {
        k_nrc_train<<<c->sms * 2, 128, kTrainSmem, st>>>(c->dev, T, n_dev, offset, B);
    }
    const int wg = c->sms;
    const __nv_bfloat16* H = c->H.as<__nv_bfloat16>();
    const __nv_bfloat16* DZ = c->DZ.as<__nv_bfloat16>();
    float* dW = c->w_grad.as<float>();
    const size_t L = size_t(B) * 64;
    if (c->desc.mlp_kernel == 0) {
        // all six weight gradients in one tcgen05 kernel
        TcWgradArgs W{T.X, H, DZ, T.DZ5, dW, B};
        k_nrc_wgrad_tc<<<wg, kWgThreads, kWgSmem, st>>>(c->dev, W, n_dev, offset, B, c->scene->dev.errflags);
    } else {
        k_nrc_wgrad<64, 128><<<wg, 256, 0, st>>>(DZ, T.X, n_dev, offset, B, B, dW + kNrcW0);
        for (int l = 1; l < 5; ++l)
            k_nrc_wgrad<64, 64><<<wg, 256, 0, st>>>(DZ + l * L, H + (l - 1) * L, n_dev, offset, B, B,
                                                    dW + kNrcW1 + (l - 1) * 4096);
        k_nrc_wgrad<16, 64><<<wg, 256, 0, st>>>(T.DZ5, H + 4 * L, n_dev, offset, B, B, dW + kNrcW5);
    }
    k_nrc_grid_bwd<<<c->sms * 8, 128, 0, st>>>(c->dev, feat, T.dX, n_dev, offset, B, B);
    BG_CUDA(cudaGetLastError());
    if (apply) {
        k_nrc_step<<<1, 1, 0, st>>>(c->step.as<int>());
        k_nrc_adam<<<c->sms * 4, 256, 0, st>>>(c->w.as<float>(), dW, c->w_m.as<float>(), c->w_v.as<float>(), kNrcParams,
                                               c->step.as<int>(), c->dev.lr, c->dev.beta1, c->dev.beta2, c->dev.eps,
                                               c->wb.as<__nv_bfloat16>());
        const int64_t gp = grid_params(c);
        if (gp % 4 == 0)
            k_nrc_adam4<<<c->sms * 8, 256, 0, st>>>(c->grid.as<float4>(), c->grid_grad.as<float4>(),
                                                    c->grid_m.as<float4>(), c->grid_v.as<float4>(), gp / 4,
                                                    c->step.as<int>(), c->dev.lr, c->dev.beta1, c->dev.beta2,
                                                    c->dev.eps);
        else
            k_nrc_adam<<<c->sms * 8, 256, 0, st>>>(c->grid.as<float>(), c->grid_grad.as<float>(), c->grid_m.as<float>(),
                                                   c->grid_v.as<float>(), gp, c->step.as<int>(), c->dev.lr,
                                                   c->dev.beta1, c->dev.beta2, c->dev.eps, nullptr);
        BG_CUDA(cudaGetLastError());
    }
    return BG_OK;
}

int nrc_prepare(bg_cache* c, int64_t train_rows, int64_t query_rows) { return cache_scratch(c, train_rows, query_rows); }

// Captured passes do not depend on which cache they were captured with: the
// only arguments of a pass's kernels that belong to a cache are the NrcDev
// (parameters, grid, weights) and the encoded-row buffer X of the query
// kernels.  nrc_graph_node() says whether a captured kernel node is one of
// them and, with `exec`, points its copy in the executable graph at cache `c`
// (every other argument is kept as captured).
int nrc_graph_node(bg_cache* c, cudaGraphExec_t exec, cudaGraphNode_t node, bool* is_cache) {
    cudaKernelNodeParams kp;
    BG_CUDA(cudaGraphKernelNodeGetParams(node, &kp));
    *is_cache = false;
    void** a = kp.kernelParams;
    NrcDev C = c->dev;
    const __nv_bfloat16* Xc = c->X.as<__nv_bfloat16>();
    if (kp.func == reinterpret_cast<void*>(k_nrc_infer_tc)) {
        // (NrcDev, X, n_dev, n_static, out, errflags, feat); X is null when the kernel encodes
        *is_cache = true;
        if (!exec) return BG_OK;
        const __nv_bfloat16* X = *static_cast<const __nv_bfloat16* const*>(a[1]) ? Xc : nullptr;
        void* args[] = {&C, &X, a[2], a[3], a[4], a[5], a[6]};
        kp.kernelParams = args;
        kp.extra = nullptr;
        BG_CUDA(cudaGraphExecKernelNodeSetParams(exec, node, &kp));
    } else if (kp.func == reinterpret_cast<void*>(k_nrc_encode)) {
        // (NrcDev, feat, n_dev, n_static, offset, limit, X)
        *is_cache = true;
        if (!exec) return BG_OK;
        __nv_bfloat16* X = c->X.as<__nv_bfloat16>();
        void* args[] = {&C, a[1], a[2], a[3], a[4], a[5], &X};
        kp.kernelParams = args;
        kp.extra = nullptr;
        BG_CUDA(cudaGraphExecKernelNodeSetParams(exec, node, &kp));
    } else if (kp.func == reinterpret_cast<void*>(k_nrc_infer)) {
        // (NrcDev, X, n_dev, n_static, out)
        *is_cache = true;
        if (!exec) return BG_OK;
        void* args[] = {&C, &Xc, a[2], a[3], a[4]};
        kp.kernelParams = args;
        kp.extra = nullptr;
        BG_CUDA(cudaGraphExecKernelNodeSetParams(exec, node, &kp));
    }
    return BG_OK;
}
const bg_cache_desc* nrc_desc(const bg_cache* c) { return &c->desc; }
int64_t nrc_next_frame(bg_cache* c) { return c->frame++; }
int64_t nrc_frame(const bg_cache* c) { return c->frame; }
uint64_t nrc_id(const bg_cache* c) { return c->id; }
uint64_t nrc_buf_epoch(const bg_cache* c) { return c->buf_epoch; }
bg_scene* nrc_scene(const bg_cache* c) { return c->scene; }

}  // namespace bg

using namespace bg;

extern "C" {

int bg_cache_create(bg_scene* s, const bg_cache_desc* d, bg_cache** out) {
    if (!s || !d || !out) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (!s->committed) return set_error(BG_ERR_STATE, "scene not committed");
    if (d->levels != 0 && d->levels != kNrcLevels) return set_error(BG_ERR_UNSUPPORTED, "levels must be %d", kNrcLevels);
    if (d->log2_table_size < 4 || d->log2_table_size > 24) return set_error(BG_ERR_INVALID_ARG, "log2_table_size out of range 4..24");
    if (d->base_resolution < 2 || d->max_resolution < d->base_resolution || d->max_resolution > (1 << 20))
        return set_error(BG_ERR_INVALID_ARG, "bad grid resolutions");
    *out = nullptr;
    bg_cache* c = new bg_cache();
    c->scene = s;
    c->id = g_cache_ids.fetch_add(1);
    c->desc = *d;
    if (c->desc.train_paths <= 0) c->desc.train_paths = 65536;
    if (c->desc.train_batch <= 0) c->desc.train_batch = 16384;
    if (c->desc.train_steps < 0) c->desc.train_steps = 0;
    if (c->desc.cache_depth < 0) c->desc.cache_depth = 2;
    c->sms = s->ctx->num_sms;
    NrcDev& D = c->dev;
    D.log2_T = d->log2_table_size;
    const double b = std::exp((std::log(double(d->max_resolution)) - std::log(double(d->base_resolution))) / (kNrcLevels - 1));
    for (int l = 0; l < kNrcLevels; ++l) D.res[l] = int(std::floor(double(d->base_resolution) * std::pow(b, l)));
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = d->bbox_max[k] > d->bbox_min[k] ? d->bbox_min[k] : s->bbox_lo[k];
        hi[k] = d->bbox_max[k] > d->bbox_min[k] ? d->bbox_max[k] : s->bbox_hi[k];
        const float ext = std::max(hi[k] - lo[k], 1e-6f);
        D.bmin[k] = lo[k] - 1e-3f * ext;
        D.bscale[k] = 1.f / (ext * 1.002f);
    }
    D.lr = d->learning_rate > 0.f ? d->learning_rate : 1e-2f;
    if (d->wait_polls < 0) {
        delete c;
        return set_error(BG_ERR_INVALID_ARG, "wait_polls %d < 0", d->wait_polls);
    }
    D.wait_polls = uint32_t(d->wait_polls);
    D.beta1 = 0.9f;
    D.beta2 = 0.99f;
    D.eps = 1e-15f;
    const int64_t gp = grid_params(c);
    int rc;
    if ((rc = c->grid.ensure(size_t(gp) * 4)) || (rc = c->grid_grad.ensure(size_t(gp) * 4)) ||
        (rc = c->grid_m.ensure(size_t(gp) * 4)) || (rc = c->grid_v.ensure(size_t(gp) * 4)) ||
        (rc = c->w.ensure(kNrcParams * 4)) || (rc = c->w_grad.ensure(kNrcParams * 4)) ||
        (rc = c->w_m.ensure(kNrcParams * 4)) || (rc = c->w_v.ensure(kNrcParams * 4)) ||
        (rc = c->wb.ensure(kNrcParams * 2)) || (rc = c->step.ensure(16)) || (rc = c->loss.ensure(16))) {
        bg_cache_destroy(c);
        return rc;
    }
    D.grid = c->grid.as<float>(); D.grid_grad = c->grid_grad.as<float>();
    D.grid_m = c->grid_m.as<float>(); D.grid_v = c->grid_v.as<float>();
    D.w = c->w.as<float>(); D.w_grad = c->w_grad.as<float>(); D.w_m = c->w_m.as<float>(); D.w_v = c->w_v.as<float>();
    D.wb = c->wb.as<__nv_bfloat16>();
    D.step = c->step.as<int>();
    if (c->desc.mlp_kernel != 0 && c->desc.mlp_kernel != 1) {
        bg_cache_destroy(c);
        return set_error(BG_ERR_INVALID_ARG, "mlp_kernel %d: 0 (tcgen05) or 1 (mma.sync)", d->mlp_kernel);
    }
    if (c->desc.train_suffix < 0) {
        bg_cache_destroy(c);
        return set_error(BG_ERR_INVALID_ARG, "train_suffix %d < 0", d->train_suffix);
    }
    cudaFuncSetAttribute(k_nrc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
    cudaFuncSetAttribute(k_nrc_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTiSmem);
    cudaFuncSetAttribute(k_nrc_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTtSmem);
    cudaFuncSetAttribute(k_nrc_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem);
    cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
    if ((rc = cache_init_params(c))) { bg_cache_destroy(c); return rc; }
    // the scratch of one Adam step over train_batch rows, here rather than in
    // the first render that trains
    if ((rc = cache_scratch(c, c->desc.train_batch, 0))) { bg_cache_destroy(c); return rc; }
    *out = c;
    return BG_OK;
}

int bg_cache_destroy(bg_cache* c) {
    if (!c) return BG_OK;
    cudaDeviceSynchronize();
    render_forget_cache(c->scene, c);   // its pending training rows, if any, are dropped
    for (DevBuf* b : {&c->grid, &c->grid_grad, &c->grid_m, &c->grid_v, &c->w, &c->w_grad, &c->w_m, &c->w_v, &c->wb,
                      &c->step, &c->X, &c->H, &c->DZ, &c->DZ5, &c->dX, &c->loss})
        b->release();
    delete c;
    return BG_OK;
}

int bg_cache_query(bg_cache* c, const float* feat, float* out_rgba, int64_t n, void* stream) {
    if (!c || (n > 0 && (!feat || !out_rgba))) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (n < 0 || n > (int64_t(1) << 30)) return set_error(BG_ERR_INVALID_ARG, "bad query count");
    if (n == 0) return BG_OK;
    int rc;
    if ((rc = cache_scratch(c, 0, n))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return nrc_query(c, feat, nullptr, n, reinterpret_cast<float4*>(out_rgba), st);
}

int bg_cache_train(bg_cache* c, const float* feat, const float* target_rgba, int64_t n, int32_t apply, float* loss,
                   void* stream) {
    if (!c || (n > 0 && (!feat || !target_rgba))) return set_error(BG_ERR_INVALID_ARG, "NULL argument");
    if (n <= 0 || n > (int64_t(1) << 26)) return set_error(BG_ERR_INVALID_ARG, "bad training batch size");
    int rc;
    if ((rc = cache_scratch(c, n, 0))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BG_CUDA(cudaMemsetAsync(c->loss.ptr, 0, 4, st));
    if ((rc = nrc_train_step(c, feat, reinterpret_cast<const float4*>(target_rgba), nullptr, 0, int(n), apply != 0, st)))
        return rc;
    if (loss) {
        float l = 0.f;
        BG_CUDA(cudaMemcpyAsync(&l, c->loss.ptr, 4, cudaMemcpyDeviceToHost, st));
        BG_CUDA(cudaStreamSynchronize(st));
        *loss = l / float(3 * n);
    }
    return BG_OK;
}

int bg_cache_params(bg_cache* c, float* mlp, float* grid, float* mlp_grad, float* grid_grad) {
    if (!c) return set_error(BG_ERR_INVALID_ARG, "cache is NULL");
    BG_CUDA(cudaDeviceSynchronize());
    const size_t gp = size_t(grid_params(c));
    if (mlp) BG_CUDA(cudaMemcpy(mlp, c->w.ptr, kNrcParams * 4, cudaMemcpyDeviceToHost));
    if (grid) BG_CUDA(cudaMemcpy(grid, c->grid.ptr, gp * 4, cudaMemcpyDeviceToHost));
    if (mlp_grad) BG_CUDA(cudaMemcpy(mlp_grad, c->w_grad.ptr, kNrcParams * 4, cudaMemcpyDeviceToHost));
    if (grid_grad) BG_CUDA(cudaMemcpy(grid_grad, c->grid_grad.ptr, gp * 4, cudaMemcpyDeviceToHost));
    return BG_OK;
}

int bg_cache_set_params(bg_cache* c, const float* mlp, const float* grid) {
    if (!c) return set_error(BG_ERR_INVALID_ARG, "cache is NULL");
    BG_CUDA(cudaDeviceSynchronize());
    if (mlp) {
        BG_CUDA(cudaMemcpy(c->w.ptr, mlp, kNrcParams * 4, cudaMemcpyHostToDevice));
        k_nrc_to_bf16<<<64, 256>>>(c->w.as<float>(), c->wb.as<__nv_bfloat16>(), kNrcParams);
        BG_CUDA(cudaGetLastError());
    }
    if (grid) BG_CUDA(cudaMemcpy(c->grid.ptr, grid, size_t(grid_params(c)) * 4, cudaMemcpyHostToDevice));
    BG_CUDA(cudaMemset(c->w_grad.ptr, 0, kNrcParams * 4));
    BG_CUDA(cudaMemset(c->grid_grad.ptr, 0, size_t(grid_params(c)) * 4));
    BG_CUDA(cudaDeviceSynchronize());
    return BG_OK;
}

int bg_cache_info(bg_cache* c, int32_t* nparams_mlp, int64_t* nparams_grid, int32_t* resolutions, float* norm6) {
    if (!c) return set_error(BG_ERR_INVALID_ARG, "cache is NULL");
    if (nparams_mlp) *nparams_mlp = kNrcParams;
    if (nparams_grid) *nparams_grid = grid_params(c);
    if (resolutions) memcpy(resolutions, c->dev.res, sizeof(c->dev.res));
    if (norm6) {
        memcpy(norm6, c->dev.bmin, 3 * sizeof(float));
        memcpy(norm6 + 3, c->dev.bscale, 3 * sizeof(float));
    }
    return BG_OK;
}

}  // extern "C"
