// Commit-time scene preparation on the device: the meshes' arrays go up once
// (vertices, normals, uvs and per-face indices, 40 bytes per face plus the
// vertex data), and the world-space triangle boxes, the traversal records
// (TriRec, leaf order) and the shading records (ShadeRec, primitive order)
// are built from them in HBM.  The arithmetic is the host's: the same
// transform_point (math/mathutils.h:129-137) for the world boxes of
// Mesh::GetShapeWorldBounds (primitive/mesh.cpp:263-283), and the same float
// subtraction for the Moller-Trumbore edges (primitive/mesh.cpp:13-14), so the
// records are bit-identical to host-built ones.
#include <algorithm>
#include <cfloat>
#include <cstring>

#include "internal.h"
#include "qnode.h"

namespace bg {
namespace {

constexpr int kRT = 256;
constexpr int kRGrid = 148 * 8;

struct MeshOff {              // first vertex, normal, uv and face of a mesh in the concatenated arrays
    int64_t v, n, t, f;
};

__device__ __forceinline__ v3 load3(const float* a, int64_t i) { return mk(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }

__device__ __forceinline__ unsigned int ford(float f) {     // order-preserving float -> uint
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ordf(unsigned int u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
#else
    const unsigned int b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

// bundle of each face: the last mesh whose first face is <= t
__global__ void k_face_bundle(const MeshOff* __restrict__ offs, int nm, int64_t ntris, int32_t* __restrict__ bundle) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntris; t += int64_t(gridDim.x) * blockDim.x) {
        int lo = 0, hi = nm - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (offs[mid].f <= t) lo = mid; else hi = mid - 1;
        }
        bundle[t] = lo;
    }
}

__global__ void k_world_boxes(int64_t ntris, const int32_t* __restrict__ bundle, const MeshOff* __restrict__ offs,
                              const float* __restrict__ verts, const int32_t* __restrict__ vi,
                              const BundleRec* __restrict__ bundles, float* __restrict__ lo, float* __restrict__ hi,
                              unsigned int* __restrict__ bbox) {
    unsigned int mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntris; t += int64_t(gridDim.x) * blockDim.x) {
        const int b = bundle[t];
        const BundleRec& br = bundles[b];
        const int64_t v0 = offs[b].v;
        v3 p[3];
        for (int k = 0; k < 3; ++k) p[k] = xf_point(br.m, load3(verts, v0 + vi[3 * t + k]));
        const float l[3] = {qmin(p[0].x, qmin(p[1].x, p[2].x)), qmin(p[0].y, qmin(p[1].y, p[2].y)),
                            qmin(p[0].z, qmin(p[1].z, p[2].z))};
        const float h[3] = {qmax(p[0].x, qmax(p[1].x, p[2].x)), qmax(p[0].y, qmax(p[1].y, p[2].y)),
                            qmax(p[0].z, qmax(p[1].z, p[2].z))};
        for (int k = 0; k < 3; ++k) {
            lo[3 * t + k] = l[k];
            hi[3 * t + k] = h[k];
            if (isfinite(l[k])) mn[k] = min(mn[k], ford(l[k] + 0.f));   // + 0: -0 counts as +0
            if (isfinite(h[k])) mx[k] = max(mx[k], ford(h[k] + 0.f));
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[k] = min(mn[k], __shfl_down_sync(0xffffffffu, mn[k], off));
            mx[k] = max(mx[k], __shfl_down_sync(0xffffffffu, mx[k], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(bbox + k, mn[k]);
            atomicMax(bbox + 3 + k, mx[k]);
        }
    }
}

// TriRec k (leaf order): object-space v0 = p1, e1 = p2 - p1, e2 = p3 - p1;
// v0.w = bundle (-1 when its transform is the identity), e1.w = primitive id
__global__ void k_tri_records(int64_t ntris, const int32_t* __restrict__ order, const int32_t* __restrict__ bundle,
                              const MeshOff* __restrict__ offs, const float* __restrict__ verts,
                              const int32_t* __restrict__ vi, const BundleRec* __restrict__ bundles,
                              TriRec* __restrict__ tris, int vertices, const int32_t* __restrict__ mat,
                              const int32_t* __restrict__ mat_class, int nmat) {
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < ntris; k += int64_t(gridDim.x) * blockDim.x) {
        const int64_t t = order[k];
        const int b = bundle[t];
        const int64_t v0 = offs[b].v;
        const v3 p1 = load3(verts, v0 + vi[3 * t]), p2 = load3(verts, v0 + vi[3 * t + 1]),
                 p3 = load3(verts, v0 + vi[3 * t + 2]);
        const v3 e1 = vertices ? p2 : sub(p2, p1), e2 = vertices ? p3 : sub(p3, p1);
        const int bcode = bundles[b].identity ? -1 : b;
        TriRec r;
        r.v0 = make_float4(p1.x, p1.y, p1.z, __int_as_float(bcode));
        r.e1 = make_float4(e1.x, e1.y, e1.z, __int_as_float(int32_t(t)));
        const int m = mat[t];
        r.e2 = make_float4(e2.x, e2.y, e2.z, __int_as_float(m >= 0 && m < nmat ? mat_class[m] : 0));
        tris[k] = r;
    }
}

// ShadeRec t: vertices, normals and uvs of face t as Mesh::FillHit reads them
// (primitive/mesh.cpp:47-97), with the bundle and the face material
__global__ void k_shade_records(int64_t ntris, const int32_t* __restrict__ bundle, const MeshOff* __restrict__ offs,
                                const float* __restrict__ verts, const float* __restrict__ normals,
                                const float* __restrict__ uvs, const int32_t* __restrict__ vi,
                                const int32_t* __restrict__ ni, const int32_t* __restrict__ ti,
                                const int32_t* __restrict__ mat, ShadeRec* __restrict__ shade) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < ntris; t += int64_t(gridDim.x) * blockDim.x) {
        const int b = bundle[t];
        const MeshOff o = offs[b];
        const v3 p1 = load3(verts, o.v + vi[3 * t]), p2 = load3(verts, o.v + vi[3 * t + 1]),
                 p3 = load3(verts, o.v + vi[3 * t + 2]);
        const v3 n1 = load3(normals, o.n + ni[3 * t]), n2 = load3(normals, o.n + ni[3 * t + 1]),
                 n3 = load3(normals, o.n + ni[3 * t + 2]);
        const float* t1 = uvs + 2 * (o.t + ti[3 * t]);
        const float* t2 = uvs + 2 * (o.t + ti[3 * t + 1]);
        const float* t3 = uvs + 2 * (o.t + ti[3 * t + 2]);
        ShadeRec r;
        r.a = make_float4(p1.x, p1.y, p1.z, __int_as_float(b));
        r.b = make_float4(p2.x, p2.y, p2.z, __int_as_float(mat[t]));
        r.c = make_float4(p3.x, p3.y, p3.z, t1[0]);
        r.d = make_float4(n1.x, n1.y, n1.z, t1[1]);
        r.e = make_float4(n2.x, n2.y, n2.z, t2[0]);
        r.f = make_float4(n3.x, n3.y, n3.z, t2[1]);
        r.g = make_float4(t3[0], t3[1], 0.f, 0.f);
        shade[t] = r;
    }
}

int grid_for(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>(kRGrid, (n + kRT - 1) / kRT))); }

}  // namespace

int upload_mesh_arrays(const std::vector<MeshHost>& meshes, int64_t ntris, MeshArrays& A) {
    const int nm = int(meshes.size());
    std::vector<MeshOff> offs(static_cast<size_t>(nm));
    int64_t nv = 0, nn = 0, nt = 0, nf = 0;
    for (int i = 0; i < nm; ++i) {
        const MeshHost& mh = meshes[size_t(i)];
        offs[size_t(i)] = MeshOff{nv, nn, nt, nf};
        nv += int64_t(mh.verts.size());
        nn += int64_t(mh.normals.size());
        nt += int64_t(mh.uvs.size() / 2);
        nf += mh.nfaces;
    }
    if (nf != ntris) return set_error(BG_ERR_STATE, "mesh face count changed during commit");
    const size_t F = size_t(ntris);
    int rc;
    if ((rc = A.verts.ensure(std::max<int64_t>(1, nv) * 12)) || (rc = A.normals.ensure(std::max<int64_t>(1, nn) * 12)) ||
        (rc = A.uvs.ensure(std::max<int64_t>(1, nt) * 8)) || (rc = A.vi.ensure(F * 12)) || (rc = A.ni.ensure(F * 12)) ||
        (rc = A.ti.ensure(F * 12)) || (rc = A.mat.ensure(F * 4)) || (rc = A.offs.ensure(size_t(nm) * sizeof(MeshOff))) ||
        (rc = A.bundle.ensure(F * 4)) || (rc = A.lo.ensure(F * 12)) || (rc = A.hi.ensure(F * 12)) ||
        (rc = A.bbox.ensure(6 * sizeof(unsigned int))))
        return rc;
    auto put = [](ScratchBuf& dst, int64_t at, const void* src, size_t bytes) -> int {
        if (bytes == 0) return BG_OK;
        BG_CUDA(cudaMemcpy(static_cast<char*>(dst.ptr) + at, src, bytes, cudaMemcpyHostToDevice));
        return BG_OK;
    };
    for (int i = 0; i < nm; ++i) {
        const MeshHost& mh = meshes[size_t(i)];
        const MeshOff& o = offs[size_t(i)];
        const size_t f3 = 3 * size_t(mh.nfaces) * 4;
        if ((rc = put(A.verts, o.v * 12, mh.verts.data(), mh.verts.size() * 12)) ||
            (rc = put(A.normals, o.n * 12, mh.normals.data(), mh.normals.size() * 12)) ||
            (rc = put(A.uvs, o.t * 8, mh.uvs.data(), (mh.uvs.size() / 2) * 8)) ||
            (rc = put(A.vi, o.f * 12, mh.vi.data(), f3)) || (rc = put(A.ni, o.f * 12, mh.ni.data(), f3)) ||
            (rc = put(A.ti, o.f * 12, mh.ti.data(), f3)) || (rc = put(A.mat, o.f * 4, mh.m.data(), size_t(mh.nfaces) * 4)))
            return rc;
    }
    BG_CUDA(cudaMemcpy(A.offs.ptr, offs.data(), size_t(nm) * sizeof(MeshOff), cudaMemcpyHostToDevice));
    k_face_bundle<<<grid_for(ntris), kRT>>>(A.offs.as<MeshOff>(), nm, ntris, A.bundle.as<int32_t>());
    BG_CUDA(cudaGetLastError());
    return BG_OK;
}

int device_world_boxes(MeshArrays& A, const BundleRec* bundles, int64_t ntris, float bbox_lo[3], float bbox_hi[3]) {
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BG_CUDA(cudaMemcpy(A.bbox.ptr, init, sizeof(init), cudaMemcpyHostToDevice));
    k_world_boxes<<<grid_for(ntris), kRT>>>(ntris, A.bundle.as<int32_t>(), A.offs.as<MeshOff>(), A.verts.as<float>(),
                                            A.vi.as<int32_t>(), bundles, A.lo.as<float>(), A.hi.as<float>(),
                                            A.bbox.as<unsigned int>());
    BG_CUDA(cudaGetLastError());
    unsigned int h[6];
    BG_CUDA(cudaMemcpy(h, A.bbox.ptr, sizeof(h), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; ++k) {                 // no finite value: the empty box
        bbox_lo[k] = h[k] == 0xffffffffu ? FLT_MAX : ordf(h[k]);
        bbox_hi[k] = h[3 + k] == 0u ? -FLT_MAX : ordf(h[3 + k]);
    }
    return BG_OK;
}

int device_records(const MeshArrays& A, const BundleRec* bundles, const int32_t* order, int64_t ntris, TriRec* tris,
                   ShadeRec* shade, bool vertices, const int32_t* mat_class, int nmat) {
    k_tri_records<<<grid_for(ntris), kRT>>>(ntris, order, A.bundle.as<int32_t>(), A.offs.as<MeshOff>(),
                                            A.verts.as<float>(), A.vi.as<int32_t>(), bundles, tris, vertices ? 1 : 0,
                                            A.mat.as<int32_t>(), mat_class, nmat);
    k_shade_records<<<grid_for(ntris), kRT>>>(ntris, A.bundle.as<int32_t>(), A.offs.as<MeshOff>(), A.verts.as<float>(),
                                              A.normals.as<float>(), A.uvs.as<float>(), A.vi.as<int32_t>(),
                                              A.ni.as<int32_t>(), A.ti.as<int32_t>(), A.mat.as<int32_t>(), shade);
    BG_CUDA(cudaGetLastError());
    BG_CUDA(cudaStreamSynchronize(0));
    return BG_OK;
}

}  // namespace bg
