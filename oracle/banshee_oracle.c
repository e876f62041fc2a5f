/*
 * banshee_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see banshee_oracle.h).
 *
 * Plain-C restatement of Banshee's hot path.  Arithmetic follows the
 * reference operation by operation (same operand order, float throughout,
 * -ffp-contract=off, the same libm float functions) so that, on the same
 * machine, it reproduces the reference bit for bit.  Citations are
 * file:line under FireRays/Banshee/.
 *
 * Toolchain-dependent detail reproduced here: RandomSampler::Sample2D
 * (sampler/random_sampler.h:58-61) returns float2(NextFloat(), NextFloat());
 * g++ evaluates those two arguments right to left, so x is the SECOND draw
 * and y the FIRST.  Probed with g++ 13.3 -O2 on the reference sources.
 */
#include "banshee_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define PI 3.14159265358979323846f  /* math/mathutils.h:48 */
#define MINPDF 0.05f                /* tracer/gitracer.cpp:10, ditracer.cpp:17 */
#define MAXRADIANCE 4.f             /* tracer/gitracer.cpp:11 */

/* ------------------------------------------------------------------ math */
typedef struct { float x, y, z; } v3;
typedef struct { float x, y; } v2;
typedef struct { float m[4][4]; } mat4;

static inline v3 V3(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v2 V2(float x, float y) { v2 r; r.x = x; r.y = y; return r; }
/* float3 operators, math/float3.h:49-96 */
static inline v3 add(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mulv(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float c) { return V3(a.x * c, a.y * c, a.z * c); }
static inline v3 neg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float sqnorm(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
/* float3::normalize / operator/= (float3.h:50,57): v * (1 / sqrt(|v|^2)) */
static inline v3 normalize(v3 v) {
    if (sqnorm(v) > 0.f) {
        float cinv = 1.f / sqrtf(sqnorm(v));
        v.x *= cinv; v.y *= cinv; v.z *= cinv;
    }
    return v;
}
/* float3.h:103-109 */
static inline v3 cross(v3 a, v3 b) {
    return V3(a.y * b.z - b.y * a.z, b.x * a.z - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* std::min / std::max semantics: min(a,b) = b < a ? b : a; max(a,b) = a < b ? b : a */
static inline float fmin_std(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_std(float a, float b) { return (a < b) ? b : a; }
static inline v3 vmin(v3 a, v3 b) { return V3(fmin_std(a.x, b.x), fmin_std(a.y, b.y), fmin_std(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return V3(fmax_std(a.x, b.x), fmax_std(a.y, b.y), fmax_std(a.z, b.z)); }
static inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
/* clamp(float), math/mathutils.h:90-93 */
static inline float clampf_ref(float x, float a, float b) { return x < a ? a : (x > b ? b : x); }

/* matrix * float3, math/matrix.h:208-220: res[i] = ((0 + m[i][0]v0) + m[i][1]v1) + m[i][2]v2 */
static inline v3 mat_mul(const mat4* m, v3 v) {
    float r[3], a[3] = {v.x, v.y, v.z};
    for (int i = 0; i < 3; ++i) {
        r[i] = 0.f;
        for (int j = 0; j < 3; ++j) r[i] += m->m[i][j] * a[j];
    }
    return V3(r[0], r[1], r[2]);
}
/* transform_point, math/mathutils.h:129-137 */
static inline v3 transform_point(v3 p, const mat4* m) {
    v3 r = mat_mul(m, p);
    r.x += m->m[0][3]; r.y += m->m[1][3]; r.z += m->m[2][3];
    return r;
}
/* transform_normal = minv^T * n, math/mathutils.h:148-151 */
static inline v3 transform_normal(v3 n, const mat4* minv) {
    mat4 t;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) t.m[j][i] = minv->m[i][j];
    return mat_mul(&t, n);
}

/* orthovector, math/mathutils.h:214-227 */
static inline v3 orthovector(v3 n) {
    v3 p;
    if (fabsf(n.z) > 0.707106781186547524401f) {
        float k = sqrtf(n.y * n.y + n.z * n.z);
        p.x = 0; p.y = -n.z / k; p.z = n.y / k;
    } else {
        float k = sqrtf(n.x * n.x + n.y * n.y);
        p.x = -n.y / k; p.y = n.x / k; p.z = 0;
    }
    return p;
}

/* map_to_hemisphere(n, s, e), math/mathutils.h:230-244 */
static inline v3 map_to_hemisphere(v3 n, v2 s, float e) {
    v3 u = orthovector(n);
    v3 v = cross(u, n);
    u = cross(n, v);
    float sinpsi = sinf(2 * PI * s.x);
    float cospsi = cosf(2 * PI * s.x);
    float costheta = powf(1.f - s.y, 1.f / (e + 1.f));
    float sintheta = sqrtf(1.f - costheta * costheta);
    return normalize(add(add(muls(muls(u, sintheta), cospsi), muls(muls(v, sintheta), sinpsi)),
                         muls(n, costheta)));
}

/* PowerHeuristic, math/mathutils.h:291-296 */
static inline float power_heuristic(int nf, float fpdf, int ng, float gpdf) {
    float f = nf * fpdf;
    float g = ng * gpdf;
    return (f * f) / (f * f + g * g);
}

/* ------------------------------------------------------------------ bbox */
typedef struct { v3 pmin, pmax; } bbox_t;

static inline bbox_t bbox_empty(void) {  /* math/bbox.h:45-54 */
    bbox_t b;
    b.pmin = V3(FLT_MAX, FLT_MAX, FLT_MAX);
    b.pmax = V3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    return b;
}
static inline bbox_t bbox_pts(v3 p1, v3 p2) { bbox_t b; b.pmin = vmin(p1, p2); b.pmax = vmax(p1, p2); return b; }
static inline void grow_pt(bbox_t* b, v3 p) { b->pmin = vmin(b->pmin, p); b->pmax = vmax(b->pmax, p); }
static inline void grow_box(bbox_t* b, bbox_t o) { b->pmin = vmin(b->pmin, o.pmin); b->pmax = vmax(b->pmax, o.pmax); }
static inline v3 center(bbox_t b) { return muls(add(b.pmax, b.pmin), 0.5f); }  /* bbox.h:68 */
static inline v3 extents(bbox_t b) { return sub(b.pmax, b.pmin); }             /* bbox.h:69 */
static inline int maxdim(bbox_t b) {                                             /* bbox.h:219-231 */
    v3 e = extents(b);
    if (e.x >= e.y && e.x >= e.z) return 0;
    if (e.y >= e.x && e.y >= e.z) return 1;
    if (e.z >= e.x && e.z >= e.y) return 2;
    return 0;
}
static inline float surface_area(bbox_t b) {                                     /* bbox.h:233-237 */
    v3 e = extents(b);
    return 2.f * (e.x * e.y + e.x * e.z + e.y * e.z);
}

/* Fast slab test, math/bbox.h:166-188 */
static inline int slab_test(v3 o, float tminray, v3 invrd, const bbox_t* box, const int dirneg[3], float maxt) {
    const v3* b = &box->pmin;  /* box[0] = pmin, box[1] = pmax */
    float tmin = (b[dirneg[0]].x - o.x) * invrd.x;
    float tmax = (b[1 - dirneg[0]].x - o.x) * invrd.x;
    float tymin = (b[dirneg[1]].y - o.y) * invrd.y;
    float tymax = (b[1 - dirneg[1]].y - o.y) * invrd.y;
    if ((tmin > tymax) || (tymin > tmax)) return 0;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    float tzmin = (b[dirneg[2]].z - o.z) * invrd.z;
    float tzmax = (b[1 - dirneg[2]].z - o.z) * invrd.z;
    if ((tmin > tzmax) || (tzmin > tmax)) return 0;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    return (tmin < maxt) && (tmax > tminray);
}

/* ------------------------------------------------------------------ world */
typedef struct { int vi0, vi1, vi2, ni0, ni1, ni2, ti0, ti1, ti2, m; } face_t;  /* mesh.h:57-63 */

typedef struct {
    v3* verts; int nverts;
    v3* normals; int nnormals;
    v2* uvs; int nuvs;
    face_t* faces; int nfaces;
    mat4 m, minv;
    int arealight;     /* ShapeBundle::arealight_: the LAST AreaLight made on it, arealight.cpp:22 */
    int64_t start;     /* Bvh::bundlestartidx_, bvh.cpp:23-39 */
} mesh_t;

typedef struct { bg_material_desc d; } material_t;
typedef struct { bg_light_desc d; v3 dir; int matidx; } light_t;

typedef struct {        /* Bvh::Node, bvh.h:153-176 (indices instead of pointers) */
    bbox_t bounds;
    int type;           /* 0 internal, 1 leaf */
    int lc, rc;
    int startidx, numprims;
} node_t;

struct or_world {
    mesh_t* meshes; int nmeshes;
    material_t* mats; int nmats;
    light_t* lights; int nlights;
    v3 bgcolor;
    int64_t ntris;
    node_t* nodes; int64_t nnodes;
    int* primids;
    int64_t* starts;    /* bundle start indices for upper_bound */
};

/* Hit, primitive/shapebundle.h:156-176 (+ the global primitive id) */
typedef struct {
    float t;
    v3 p, n, ng, dpdu, dpdv;
    v2 uv;
    int m;
    int mesh;
    int64_t prim;
    float a, b;
} hit_t;

/* Mesh::IntersectFace, primitive/mesh.cpp:7-45 */
static int intersect_face(const mesh_t* me, const face_t* f, v3 o, v3 d, float tmin, float tmax,
                          float* t, float* a, float* b) {
    v3 p1 = me->verts[f->vi0], p2 = me->verts[f->vi1], p3 = me->verts[f->vi2];
    v3 e1 = sub(p2, p1);
    v3 e2 = sub(p3, p1);
    v3 s1 = cross(d, e2);
    float invd = 1.f / dot(s1, e1);
    v3 dd = sub(o, p1);
    float b1 = dot(dd, s1) * invd;
    if (b1 < 0.f || b1 > 1.0) return 0;
    v3 s2 = cross(dd, e1);
    float b2 = dot(d, s2) * invd;
    if (b2 < 0.f || b1 + b2 > 1.f) return 0;
    float tmp = dot(e2, s2) * invd;
    if (tmp > tmin && tmp <= tmax) {
        *t = tmp; *a = b1; *b = b2;
        return 1;
    }
    return 0;
}

/* Mesh::FillHit, primitive/mesh.cpp:47-97 */
static void fill_hit(const mesh_t* me, int meshidx, const face_t* f, float t, float a, float b, hit_t* hit) {
    v3 p1 = me->verts[f->vi0], p2 = me->verts[f->vi1], p3 = me->verts[f->vi2];
    v3 n1 = me->normals[f->ni0], n2 = me->normals[f->ni1], n3 = me->normals[f->ni2];
    v2 t1 = me->uvs[f->ti0], t2 = me->uvs[f->ti1], t3 = me->uvs[f->ti2];
    float w0 = 1.f - a - b;
    hit->t = t;
    hit->p = transform_point(add(add(muls(p1, w0), muls(p2, a)), muls(p3, b)), &me->m);
    hit->n = normalize(transform_normal(add(add(muls(n1, w0), muls(n2, a)), muls(n3, b)), &me->minv));
    hit->ng = normalize(transform_normal(cross(sub(p3, p1), sub(p2, p1)), &me->minv));
    if (dot(hit->n, hit->ng) < 0) hit->ng = neg(hit->ng);
    float du1 = t1.x - t3.x, du2 = t2.x - t3.x, dv1 = t1.y - t3.y, dv2 = t2.y - t3.y;
    v3 dp1 = sub(p1, p3), dp2 = sub(p2, p3);
    float det = du1 * dv2 - dv1 * du2;
    if (det != 0.f) {
        float invdet = 1.f / det;
        hit->dpdu = normalize(transform_normal(muls(sub(muls(dp1, dv2), muls(dp2, dv1)), invdet), &me->minv));
        hit->dpdv = normalize(transform_normal(muls(add(muls(dp1, -du2), muls(dp2, du1)), invdet), &me->minv));
    } else {
        hit->dpdu = orthovector(hit->n);
        hit->dpdv = cross(hit->n, hit->dpdu);
    }
    hit->uv = V2(t1.x * w0 + t2.x * a + t3.x * b, t1.y * w0 + t2.y * a + t3.y * b);
    hit->m = f->m;
    hit->mesh = meshidx;
    hit->a = a; hit->b = b;
}

/* transform_ray through minv, math/mathutils.h:154-157 */
static inline void transform_ray(const mesh_t* me, v3 o, v3 d, v3* oo, v3* od) {
    *oo = transform_point(o, &me->minv);
    *od = mat_mul(&me->minv, d);
}

/* Mesh::IntersectShape(idx, r, hit), primitive/mesh.cpp:216-238 */
static int intersect_shape(const or_world* w, int meshidx, int idx, v3 o, v3 d, float tmin, hit_t* hit) {
    const mesh_t* me = &w->meshes[meshidx];
    const face_t* f = &me->faces[idx];
    v3 ro, rd;
    transform_ray(me, o, d, &ro, &rd);
    float t, a, b;
    if (intersect_face(me, f, ro, rd, tmin, hit->t, &t, &a, &b)) {
        fill_hit(me, meshidx, f, t, a, b, hit);
        hit->prim = me->start + idx;
        return 1;
    }
    return 0;
}

/* Mesh::IntersectShape(idx, r), primitive/mesh.cpp:240-261 */
static int intersect_shape_any(const or_world* w, int meshidx, int idx, v3 o, v3 d, float tmin, float tmax) {
    const mesh_t* me = &w->meshes[meshidx];
    v3 ro, rd;
    transform_ray(me, o, d, &ro, &rd);
    float t, a, b;
    return intersect_face(me, &me->faces[idx], ro, rd, tmin, tmax, &t, &a, &b);
}

/* Bvh::GetShapeBundleIdx: upper_bound over bundle starts minus one, bvh.cpp:649-661 */
static inline int bundle_of(const or_world* w, int64_t prim) {
    int lo = 0, hi = w->nmeshes;  /* first index with start > prim */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (w->starts[mid] > prim) hi = mid; else lo = mid + 1;
    }
    return lo - 1;
}

/* ------------------------------------------------------------- BVH build */
typedef struct {
    int64_t startidx, numprims;
    int* ptr;            /* parent's child slot */
    bbox_t bounds, centroid_bounds;
    int level;
} split_req_t;

typedef struct {
    or_world* w;
    const bbox_t* bounds;
    const v3* centroids;
    int* primindices;
    int64_t nodecnt;
} build_ctx_t;

/* Bvh::FindSahSplit, accelerator/bvh.cpp:247-355 */
static void find_sah_split(const split_req_t* req, const bbox_t* bounds, const v3* centroids,
                           const int* primindices, int* out_dim, float* out_split) {
    enum { kNumBins = 64 };
    int splitidx = -1;
    float sah = FLT_MAX;
    int dim = 0;
    float split = NAN;
    v3 cext = extents(req->centroid_bounds);
    if (sqnorm(cext) == 0.f) { *out_dim = dim; *out_split = split; return; }
    static __thread struct { bbox_t bounds; int count; } bins[3][kNumBins];
    float invarea = 1.f / surface_area(req->bounds);
    v3 rootmin = req->centroid_bounds.pmin;
    for (int axis = 0; axis < 3; ++axis) {
        float rootminc = comp(rootmin, axis);
        float centroid_rng = comp(cext, axis);
        float invcentroid_rng = 1.f / centroid_rng;
        if (centroid_rng == 0.f) continue;
        for (int i = 0; i < kNumBins; ++i) { bins[axis][i].count = 0; bins[axis][i].bounds = bbox_empty(); }
        for (int64_t i = req->startidx; i < req->startidx + req->numprims; ++i) {
            int idx = primindices[i];
            float fb = kNumBins * ((comp(centroids[idx], axis) - rootminc) * invcentroid_rng);
            int binidx = (int)fmin_std(fb, (float)(kNumBins - 1));
            ++bins[axis][binidx].count;
            grow_box(&bins[axis][binidx].bounds, bounds[idx]);
        }
        bbox_t rightbounds[kNumBins - 1];
        bbox_t rightbox = bbox_empty();
        for (int i = kNumBins - 1; i > 0; --i) {
            grow_box(&rightbox, bins[axis][i].bounds);
            rightbounds[i - 1] = rightbox;
        }
        bbox_t leftbox = bbox_empty();
        int leftcount = 0;
        int rightcount = (int)req->numprims;
        for (int i = 0; i < kNumBins - 1; ++i) {
            grow_box(&leftbox, bins[axis][i].bounds);
            leftcount += bins[axis][i].count;
            rightcount -= bins[axis][i].count;
            float sahtmp = 10.f + (leftcount * surface_area(leftbox) + rightcount * surface_area(rightbounds[i])) * invarea;
            if (sahtmp < sah) { dim = axis; splitidx = i; sah = sahtmp; }
        }
    }
    if (splitidx != -1) split = comp(rootmin, dim) + (splitidx + 1) * (comp(cext, dim) / kNumBins);
    *out_dim = dim; *out_split = split;
}

/* Bvh::BuildNode, accelerator/bvh.cpp:68-245 (usesah = true as World::Commit sets, world.cpp:9) */
static void build_node(build_ctx_t* c, const split_req_t* req) {
    int64_t nodeidx = c->nodecnt++;
    node_t* node = &c->w->nodes[nodeidx];
    node->bounds = req->bounds;
    const bbox_t* bounds = c->bounds;
    const v3* centroids = c->centroids;
    int* pi = c->primindices;
    if (req->numprims < 2) {
        node->type = 1;
        node->startidx = (int)req->startidx;
        node->numprims = (int)req->numprims;
    } else {
        node->type = 0;
        int axis = maxdim(req->centroid_bounds);
        float border = comp(center(req->centroid_bounds), axis);
        if (req->level < 10) {
            int sdim; float ssplit;
            find_sah_split(req, bounds, centroids, pi, &sdim, &ssplit);
            if (!(ssplit != ssplit)) { axis = sdim; border = ssplit; }
        }
        bbox_t lb = bbox_empty(), rb = bbox_empty(), lcb = bbox_empty(), rcb = bbox_empty();
        int64_t splitidx = req->startidx;
        int near2far = (int)((req->numprims + req->startidx) & 0x1);
        if (comp(extents(req->centroid_bounds), axis) > 0.f) {
            int64_t first = req->startidx;
            int64_t last = req->startidx + req->numprims;
            if (near2far) {
                for (;;) {
                    while ((first != last) && comp(centroids[pi[first]], axis) < border) {
                        grow_box(&lb, bounds[pi[first]]); grow_pt(&lcb, centroids[pi[first]]); ++first;
                    }
                    if (first == last--) break;
                    grow_box(&rb, bounds[pi[first]]); grow_pt(&rcb, centroids[pi[first]]);
                    while ((first != last) && comp(centroids[pi[last]], axis) >= border) {
                        grow_box(&rb, bounds[pi[last]]); grow_pt(&rcb, centroids[pi[last]]); --last;
                    }
                    if (first == last) break;
                    grow_box(&lb, bounds[pi[last]]); grow_pt(&lcb, centroids[pi[last]]);
                    int tmp = pi[first]; pi[first] = pi[last]; pi[last] = tmp; ++first;
                }
            } else {
                for (;;) {
                    while ((first != last) && comp(centroids[pi[first]], axis) >= border) {
                        grow_box(&lb, bounds[pi[first]]); grow_pt(&lcb, centroids[pi[first]]); ++first;
                    }
                    if (first == last--) break;
                    grow_box(&rb, bounds[pi[first]]); grow_pt(&rcb, centroids[pi[first]]);
                    while ((first != last) && comp(centroids[pi[last]], axis) < border) {
                        grow_box(&rb, bounds[pi[last]]); grow_pt(&rcb, centroids[pi[last]]); --last;
                    }
                    if (first == last) break;
                    grow_box(&lb, bounds[pi[last]]); grow_pt(&lcb, centroids[pi[last]]);
                    int tmp = pi[first]; pi[first] = pi[last]; pi[last] = tmp; ++first;
                }
            }
            splitidx = first;
        }
        if (splitidx == req->startidx || splitidx == req->startidx + req->numprims) {
            splitidx = req->startidx + (req->numprims >> 1);
            for (int64_t i = req->startidx; i < splitidx; ++i) { grow_box(&lb, bounds[pi[i]]); grow_pt(&lcb, centroids[pi[i]]); }
            for (int64_t i = splitidx; i < req->startidx + req->numprims; ++i) { grow_box(&rb, bounds[pi[i]]); grow_pt(&rcb, centroids[pi[i]]); }
        }
        split_req_t left = { req->startidx, splitidx - req->startidx, &node->lc, lb, lcb, req->level + 1 };
        split_req_t right = { splitidx, req->numprims - (splitidx - req->startidx), &node->rc, rb, rcb, req->level + 1 };
        build_node(c, &left);
        node = &c->w->nodes[nodeidx];
        build_node(c, &right);
        node = &c->w->nodes[nodeidx];
    }
    if (req->ptr) *req->ptr = (int)nodeidx;
}

/* Bvh::Build + BuildImpl, accelerator/bvh.cpp:16-54, 357-496 */
static void bvh_build(or_world* w) {
    int64_t n = w->ntris;
    bbox_t* bounds = (bbox_t*)malloc(sizeof(bbox_t) * (size_t)n);
    v3* centroids = (v3*)malloc(sizeof(v3) * (size_t)n);
    for (int i = 0; i < w->nmeshes; ++i) {      /* Mesh::GetShapeWorldBounds, mesh.cpp:263-283 */
        const mesh_t* me = &w->meshes[i];
        for (int j = 0; j < me->nfaces; ++j) {
            const face_t* f = &me->faces[j];
            v3 p1 = transform_point(me->verts[f->vi0], &me->m);
            v3 p2 = transform_point(me->verts[f->vi1], &me->m);
            v3 p3 = transform_point(me->verts[f->vi2], &me->m);
            bbox_t b = bbox_pts(p1, p2);
            grow_pt(&b, p3);
            bounds[me->start + j] = b;
        }
    }
    w->nnodes = 2 * n - 1;
    w->nodes = (node_t*)calloc((size_t)w->nnodes, sizeof(node_t));
    w->primids = (int*)malloc(sizeof(int) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) w->primids[i] = (int)i;
    bbox_t cb = bbox_empty(), tb = bbox_empty();
    for (int64_t i = 0; i < n; ++i) {
        v3 c = center(bounds[i]);
        grow_pt(&cb, c);
        centroids[i] = c;
        grow_box(&tb, bounds[i]);
    }
    build_ctx_t ctx = { w, bounds, centroids, w->primids, 0 };
    split_req_t init = { 0, n, NULL, tb, cb, 0 };
    build_node(&ctx, &init);
    free(bounds);
    free(centroids);
}

/* ---------------------------------------------------------- traversal */
typedef struct { int* data; int size, cap; } stack_t_;
static inline void spush(stack_t_* s, int v) {
    if (s->size == s->cap) { s->cap = s->cap ? 2 * s->cap : 128; s->data = (int*)realloc(s->data, sizeof(int) * (size_t)s->cap); }
    s->data[s->size++] = v;
}

/* Bvh::Intersect(ray, Hit&), accelerator/bvh.cpp:499-573, with World::Intersect
 * setting hit.t = r.t.y first (world/world.cpp:19-23). */
static int world_intersect(const or_world* w, v3 o, v3 d, float tmin, float tmax, hit_t* hit,
                           uint64_t* cnodes, uint64_t* ctris) {
    hit->t = tmax;
    hit->prim = -1;
    stack_t_ st = { NULL, 0, 0 };
    v3 invrd = V3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    int dirneg[3] = { d.x < 0.f ? 1 : 0, d.y < 0.f ? 1 : 0, d.z < 0.f ? 1 : 0 };
    int node = 0;
    int bhit = 0;
    for (;;) {
        const node_t* nd = &w->nodes[node];
        if (cnodes) ++*cnodes;
        if (nd->type == 1) {
            for (int i = nd->startidx; i < nd->startidx + nd->numprims; ++i) {
                int bi = bundle_of(w, w->primids[i]);
                int si = (int)(w->primids[i] - w->starts[bi]);
                if (ctris) ++*ctris;
                if (intersect_shape(w, bi, si, o, d, tmin, hit)) bhit = 1;
            }
        } else {
            int addleft = slab_test(o, tmin, invrd, &w->nodes[nd->lc].bounds, dirneg, hit->t);
            int addright = slab_test(o, tmin, invrd, &w->nodes[nd->rc].bounds, dirneg, hit->t);
            if (addleft) {
                if (addright) spush(&st, nd->rc);
                node = nd->lc;
                continue;
            } else if (addright) {
                node = nd->rc;
                continue;
            }
        }
        if (st.size == 0) break;
        node = st.data[--st.size];
    }
    free(st.data);
    return bhit;
}

/* Bvh::Intersect(ray), accelerator/bvh.cpp:575-647 */
static int world_occluded(const or_world* w, v3 o, v3 d, float tmin, float tmax,
                          uint64_t* cnodes, uint64_t* ctris) {
    stack_t_ st = { NULL, 0, 0 };
    v3 invrd = V3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    int dirneg[3] = { d.x < 0.f ? 1 : 0, d.y < 0.f ? 1 : 0, d.z < 0.f ? 1 : 0 };
    int node = 0;
    int res = 0;
    for (;;) {
        const node_t* nd = &w->nodes[node];
        if (cnodes) ++*cnodes;
        if (nd->type == 1) {
            for (int i = nd->startidx; i < nd->startidx + nd->numprims; ++i) {
                int bi = bundle_of(w, w->primids[i]);
                int si = (int)(w->primids[i] - w->starts[bi]);
                if (ctris) ++*ctris;
                if (intersect_shape_any(w, bi, si, o, d, tmin, tmax)) { res = 1; goto done; }
            }
        } else {
            int addleft = slab_test(o, tmin, invrd, &w->nodes[nd->lc].bounds, dirneg, tmax);
            int addright = slab_test(o, tmin, invrd, &w->nodes[nd->rc].bounds, dirneg, tmax);
            if (addleft) {
                if (addright) spush(&st, nd->rc);
                node = nd->lc;
                continue;
            } else if (addright) {
                node = nd->rc;
                continue;
            }
        }
        if (st.size == 0) break;
        node = st.data[--st.size];
    }
done:
    free(st.data);
    return res;
}

/* ------------------------------------------------------- world create */
static mat4 mat_from(const float* a) {
    mat4 m;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) m.m[i][j] = a[4 * i + j];
    return m;
}

/* Mesh::Mesh, primitive/mesh.cpp:126-214 */
static int mesh_init(mesh_t* me, const bg_mesh_desc* d) {
    int vstride = d->vstride == 0 ? (int)(3 * sizeof(float)) : d->vstride;
    int nstride = d->nstride == 0 ? (int)(3 * sizeof(float)) : d->nstride;
    int vis = d->vistride == 0 ? (int)sizeof(int) : d->vistride;
    int nis = d->nistride == 0 ? (int)sizeof(int) : d->nistride;
    int uis = d->uistride == 0 ? (int)sizeof(int) : d->uistride;
    if (d->nfaces < 0 || d->nvertices < 0 || (d->nfaces > 0 && (!d->vertices || !d->vidx || !d->nidx || !d->normals || !d->materials)))
        return -1;
    me->nverts = d->nvertices;
    me->verts = (v3*)malloc(sizeof(v3) * (size_t)(d->nvertices > 0 ? d->nvertices : 1));
    for (int i = 0; i < d->nvertices; ++i) {
        const float* c = (const float*)((const char*)d->vertices + (size_t)i * vstride);
        me->verts[i] = V3(c[0], c[1], c[2]);
    }
    me->nnormals = d->nnormals;
    me->normals = (v3*)malloc(sizeof(v3) * (size_t)(d->nnormals > 0 ? d->nnormals : 1));
    for (int i = 0; i < d->nnormals; ++i) {
        const float* c = (const float*)((const char*)d->normals + (size_t)i * nstride);
        me->normals[i] = V3(c[0], c[1], c[2]);
    }
    int hasuv = d->uvs && d->nuvs > 0;
    if (hasuv) {
        int us = d->ustride == 0 ? (int)(2 * sizeof(float)) : d->ustride;
        me->nuvs = d->nuvs;
        me->uvs = (v2*)malloc(sizeof(v2) * (size_t)d->nuvs);
        for (int i = 0; i < d->nuvs; ++i) {
            const float* c = (const float*)((const char*)d->uvs + (size_t)i * us);
            me->uvs[i] = V2(c[0], c[1]);
        }
    } else {
        me->nuvs = 1;
        me->uvs = (v2*)malloc(sizeof(v2));
        me->uvs[0] = V2(0, 0);
    }
    me->nfaces = d->nfaces;
    me->faces = (face_t*)malloc(sizeof(face_t) * (size_t)(d->nfaces > 0 ? d->nfaces : 1));
#define IDX(p, k, s) (*(const int*)((const char*)(p) + (size_t)(k) * (s)))
    for (int i = 0; i < d->nfaces; ++i) {
        face_t* f = &me->faces[i];
        f->vi0 = IDX(d->vidx, 3 * i, vis); f->vi1 = IDX(d->vidx, 3 * i + 1, vis); f->vi2 = IDX(d->vidx, 3 * i + 2, vis);
        f->ni0 = IDX(d->nidx, 3 * i, nis); f->ni1 = IDX(d->nidx, 3 * i + 1, nis); f->ni2 = IDX(d->nidx, 3 * i + 2, nis);
        if (hasuv) {
            f->ti0 = IDX(d->uidx, 3 * i, uis); f->ti1 = IDX(d->uidx, 3 * i + 1, uis); f->ti2 = IDX(d->uidx, 3 * i + 2, uis);
        } else {
            f->ti0 = f->ti1 = f->ti2 = 0;
        }
        f->m = IDX(d->materials, i, d->mstride);
        if (f->vi0 < 0 || f->vi0 >= me->nverts || f->vi1 < 0 || f->vi1 >= me->nverts || f->vi2 < 0 || f->vi2 >= me->nverts ||
            f->ni0 < 0 || f->ni0 >= me->nnormals || f->ni1 < 0 || f->ni1 >= me->nnormals || f->ni2 < 0 || f->ni2 >= me->nnormals ||
            f->ti0 < 0 || f->ti0 >= me->nuvs || f->ti1 < 0 || f->ti1 >= me->nuvs || f->ti2 < 0 || f->ti2 >= me->nuvs)
            return -1;
    }
#undef IDX
    me->m = mat_from(d->m);
    me->minv = mat_from(d->minv);
    me->arealight = -1;
    return 0;
}

or_world* or_world_create(const bg_mesh_desc* meshes, int32_t nmeshes,
                          const bg_material_desc* mats, int32_t nmats,
                          const bg_light_desc* lights, int32_t nlights,
                          const float* bgcolor) {
    if (nmeshes <= 0 || !meshes) return NULL;
    or_world* w = (or_world*)calloc(1, sizeof(or_world));
    w->nmeshes = nmeshes;
    w->meshes = (mesh_t*)calloc((size_t)nmeshes, sizeof(mesh_t));
    w->starts = (int64_t*)calloc((size_t)nmeshes, sizeof(int64_t));
    int64_t sum = 0;
    for (int i = 0; i < nmeshes; ++i) {
        if (mesh_init(&w->meshes[i], &meshes[i]) != 0) { or_world_destroy(w); return NULL; }
        w->meshes[i].start = sum;
        w->starts[i] = sum;
        sum += w->meshes[i].nfaces;
    }
    w->ntris = sum;
    if (sum == 0) { or_world_destroy(w); return NULL; }
    w->nmats = nmats;
    w->mats = (material_t*)calloc((size_t)(nmats > 0 ? nmats : 1), sizeof(material_t));
    for (int i = 0; i < nmats; ++i) w->mats[i].d = mats[i];
    w->nlights = nlights;
    w->lights = (light_t*)calloc((size_t)(nlights > 0 ? nlights : 1), sizeof(light_t));
    for (int i = 0; i < nlights; ++i) {
        light_t* L = &w->lights[i];
        L->d = lights[i];
        if (L->d.type == BG_LIGHT_AREA) {
            /* AreaLight ctor, light/arealight.cpp:11-23: material must be emissive */
            if (L->d.mesh < 0 || L->d.mesh >= nmeshes) { or_world_destroy(w); return NULL; }
            mesh_t* me = &w->meshes[L->d.mesh];
            if (L->d.face < 0 || L->d.face >= me->nfaces) { or_world_destroy(w); return NULL; }
            int mi = me->faces[L->d.face].m;
            if (mi < 0 || mi >= nmats || w->mats[mi].d.type != BG_MAT_EMISSIVE) { or_world_destroy(w); return NULL; }
            L->matidx = mi;
            me->arealight = i;
        } else if (L->d.type == BG_LIGHT_DIRECTIONAL) {
            L->dir = normalize(V3(L->d.d[0], L->d.d[1], L->d.d[2]));  /* directional_light.h:44 */
        }
    }
    w->bgcolor = bgcolor ? V3(bgcolor[0], bgcolor[1], bgcolor[2]) : V3(0, 0, 0);
    bvh_build(w);
    return w;
}

void or_world_destroy(or_world* w) {
    if (!w) return;
    for (int i = 0; i < w->nmeshes; ++i) {
        free(w->meshes[i].verts); free(w->meshes[i].normals); free(w->meshes[i].uvs); free(w->meshes[i].faces);
    }
    free(w->meshes); free(w->starts); free(w->mats); free(w->lights);
    free(w->nodes); free(w->primids);
    free(w);
}

int64_t or_world_ntriangles(const or_world* w) { return w->ntris; }
int64_t or_world_nnodes(const or_world* w) { return w->nnodes; }

/* --------------------------------------------------------- threading */
typedef struct {
    void (*fn)(void* arg, int64_t begin, int64_t end);
    void* arg;
    int64_t n, chunk;
    int64_t next;
    pthread_mutex_t mu;
} pool_t;

static void* pool_worker(void* p) {
    pool_t* pl = (pool_t*)p;
    for (;;) {
        pthread_mutex_lock(&pl->mu);
        int64_t b = pl->next;
        pl->next += pl->chunk;
        pthread_mutex_unlock(&pl->mu);
        if (b >= pl->n) break;
        int64_t e = b + pl->chunk < pl->n ? b + pl->chunk : pl->n;
        pl->fn(pl->arg, b, e);
    }
    return NULL;
}

static void parallel_for(int64_t n, int64_t chunk, int nthreads, void (*fn)(void*, int64_t, int64_t), void* arg) {
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pool_t pl;
    pl.fn = fn; pl.arg = arg; pl.n = n; pl.chunk = chunk < 1 ? 1 : chunk; pl.next = 0;
    pthread_mutex_init(&pl.mu, NULL);
    if (nthreads == 1) { pool_worker(&pl); pthread_mutex_destroy(&pl.mu); return; }
    pthread_t th[256];
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, pool_worker, &pl);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&pl.mu);
}

/* ------------------------------------------------------------- ray casts */
typedef struct { const or_world* w; const bg_ray* rays; bg_hit* hits; uint8_t* occ; } cast_arg_t;

static void cast_closest_range(void* a, int64_t b, int64_t e) {
    cast_arg_t* c = (cast_arg_t*)a;
    for (int64_t i = b; i < e; ++i) {
        const bg_ray* r = &c->rays[i];
        hit_t h;
        int hit = world_intersect(c->w, V3(r->o[0], r->o[1], r->o[2]), V3(r->d[0], r->d[1], r->d[2]),
                                  r->tmin, r->tmax, &h, NULL, NULL);
        c->hits[i].t = hit ? h.t : r->tmax;
        c->hits[i].primid = hit ? (int32_t)h.prim : -1;
        c->hits[i].u = hit ? h.a : 0.f;
        c->hits[i].v = hit ? h.b : 0.f;
    }
}

static void cast_any_range(void* a, int64_t b, int64_t e) {
    cast_arg_t* c = (cast_arg_t*)a;
    for (int64_t i = b; i < e; ++i) {
        const bg_ray* r = &c->rays[i];
        c->occ[i] = (uint8_t)world_occluded(c->w, V3(r->o[0], r->o[1], r->o[2]), V3(r->d[0], r->d[1], r->d[2]),
                                            r->tmin, r->tmax, NULL, NULL);
    }
}

void or_intersect_closest(const or_world* w, const bg_ray* rays, bg_hit* hits, int64_t n, int32_t nthreads) {
    cast_arg_t c = { w, rays, hits, NULL };
    parallel_for(n, 4096, nthreads, cast_closest_range, &c);
}

void or_intersect_any(const or_world* w, const bg_ray* rays, uint8_t* occ, int64_t n, int32_t nthreads) {
    cast_arg_t c = { w, rays, NULL, occ };
    parallel_for(n, 4096, nthreads, cast_any_range, &c);
}

void or_traversal_counts(const or_world* w, const bg_ray* rays, int64_t n, int32_t any_hit,
                         uint64_t* nodes, uint64_t* tris) {
    uint64_t cn = 0, ct = 0;
    for (int64_t i = 0; i < n; ++i) {
        const bg_ray* r = &rays[i];
        v3 o = V3(r->o[0], r->o[1], r->o[2]), d = V3(r->d[0], r->d[1], r->d[2]);
        if (any_hit) world_occluded(w, o, d, r->tmin, r->tmax, &cn, &ct);
        else { hit_t h; world_intersect(w, o, d, r->tmin, r->tmax, &h, &cn, &ct); }
    }
    *nodes = cn; *tris = ct;
}

int32_t or_triangle_test(const or_world* w, int64_t primid, const bg_ray* r, float* t, float* u, float* v) {
    if (primid < 0 || primid >= w->ntris) return 0;
    int bi = bundle_of(w, primid);
    int si = (int)(primid - w->starts[bi]);
    hit_t h;
    h.t = r->tmax;
    if (!intersect_shape(w, bi, si, V3(r->o[0], r->o[1], r->o[2]), V3(r->d[0], r->d[1], r->d[2]), r->tmin, &h)) return 0;
    *t = h.t; *u = h.a; *v = h.b;
    return 1;
}

/* ------------------------------------------------------ sampler / RNG */
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct { uint64_t key; uint32_t counter; } keyed_t;

static inline void keyed_init(keyed_t* k, uint64_t seed, uint32_t pixel, uint32_t sample) {
    k->key = splitmix64(seed ^ splitmix64(((uint64_t)pixel << 32) | sample));
    k->counter = 0;
}
/* the global rand() of the sampler contract, 31-bit like glibc's RAND_MAX */
static inline uint32_t keyed_rand(keyed_t* k) {
    uint64_t c = (uint64_t)(k->counter++);
    return (uint32_t)(splitmix64(k->key ^ (c * 0xD1B54A32D192ED03ull)) >> 33);
}
uint32_t or_keyed_rand(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t counter) {
    keyed_t k; keyed_init(&k, seed, pixel, sample); k.counter = counter;
    return keyed_rand(&k);
}
/* rand_float / rand_uint, math/mathutils.h:62-65: (float)rand() / RAND_MAX */
static inline float rand_float(keyed_t* k) { return (float)(int)keyed_rand(k) / (float)2147483647; }
static inline uint32_t rand_uint(keyed_t* k) { return keyed_rand(k); }

/* McRng, rng/mcrng.h:45-76 */
typedef struct { uint32_t z, w; } mcrng_t;
static inline void mcrng_init(mcrng_t* r, keyed_t* k) { r->z = rand_uint(k); r->w = rand_uint(k); }
static inline uint32_t mc_next_uint(mcrng_t* r) {
    r->z = 36969u * (r->z & 65535u) + (r->z >> 16);
    r->w = 18000u * (r->w & 65535u) + (r->w >> 16);
    return (r->z << 16) + r->w;
}
static inline float mc_next_float(mcrng_t* r) { return (float)mc_next_uint(r) * 2.328306e-10f; }
/* RandomSampler::Sample2D: x = second draw, y = first (see file header) */
static inline v2 sample2d(mcrng_t* r) {
    float first = mc_next_float(r);
    float second = mc_next_float(r);
    return V2(second, first);
}

/* --------------------------------------------------------- materials */
#define BSDF_REFLECTION (1 << 0)
#define BSDF_DIFFUSE    (1 << 2)
#define BSDF_SPECULAR   (1 << 3)
#define BSDF_GLOSSY     (1 << 4)

/* GgxDistribution::D, bsdf/microfacet_distribution.h:206-220 */
static float ggx_D(float a_, v3 m, v3 n) {
    float ndotm = dot(m, n);
    if (ndotm <= 0.f) return 0.f;
    float ndotm2 = ndotm * ndotm;
    float sinmn = sqrtf(1.f - clampf_ref(ndotm * ndotm, 0.f, 1.f));
    float tanmn = sinmn / ndotm;
    float a2 = a_ * a_;
    return (a2 / (PI * ndotm2 * ndotm2 * (a2 + tanmn * tanmn) * (a2 + tanmn * tanmn)));
}
/* GgxDistribution::GetPdf, microfacet_distribution.h:246-255 */
static float ggx_pdf(float a_, const hit_t* hit, v3 wi, v3 wo) {
    v3 m = normalize(add(wi, wo));
    float mpdf = ggx_D(a_, m, hit->n) * fabsf(dot(hit->n, m));
    return mpdf / (4.f * dot(wo, m));
}
/* GgxDistribution::G1 / G, microfacet_distribution.h:257-280 */
static float ggx_G1(float a_, v3 v, v3 m, v3 n) {
    float ndotv = dot(n, v);
    float mdotv = dot(m, v);
    if (ndotv * mdotv <= 0.f) return 0.f;
    float sinnv = sqrtf(1.f - clampf_ref(ndotv * ndotv, 0.f, 1.f));
    float tannv = sinnv / ndotv;
    float a2 = a_ * a_;
    return 2.f / (1.f + sqrtf(1.f + a2 * tannv * tannv));
}
static float ggx_G(float a_, v3 wi, v3 wo, v3 wh, v3 n) { return ggx_G1(a_, wi, wh, n) * ggx_G1(a_, wo, wh, n); }
/* GgxDistribution::Sample, microfacet_distribution.h:223-243 */
static void ggx_sample(float a_, const hit_t* hit, v2 s, v3 wi, v3* wo, float* pdf) {
    float temp = atanf(a_ * sqrtf(s.x) / sqrtf(1.f - s.x));
    float theta = (float)((temp >= 0) ? temp : (temp + 2 * PI));
    float costheta = cosf(theta);
    float sintheta = sqrtf(1.f - clampf_ref(costheta * costheta, 0.f, 1.f));
    float cosphi = cosf(2.f * PI * s.y);
    float sinphi = sinf(2.f * PI * s.y);
    v3 wh = normalize(add(add(muls(muls(hit->dpdu, sintheta), cosphi), muls(muls(hit->dpdv, sintheta), sinphi)),
                          muls(hit->n, costheta)));
    *wo = add(neg(wi), muls(wh, 2.f * dot(wi, wh)));
    *pdf = ggx_pdf(a_, hit, wi, *wo);
}
/* FresnelDielectric::Evaluate, bsdf/fresnel.h:59-90 */
static float fresnel_dielectric(float etai, float etat, float ndotwi) {
    float ei = etai, et = etat;
    if (ndotwi < 0) { ei = etat; et = etai; ndotwi = -ndotwi; }
    float sint = (ei / et) * sqrtf(fmax_std(0.f, 1.f - ndotwi * ndotwi));
    if (sint > 1.f) return 1.f;
    float ndotwt = sqrtf(fmax_std(0.f, 1.f - sint * sint));
    float rparl = ((et * ndotwi) - (ei * ndotwt)) / ((et * ndotwi) + (ei * ndotwt));
    float rperp = ((ei * ndotwi) - (et * ndotwt)) / ((ei * ndotwi) + (et * ndotwt));
    return (rparl * rparl + rperp * rperp) * 0.5f;
}
/* Microfacet::Evaluate, bsdf/microfacet.h:98-129 */
static v3 microfacet_eval(const bg_material_desc* md, const hit_t* hit, v3 wi, v3 wo) {
    float sameside = dot(wi, hit->n) * dot(wo, hit->n);
    if (sameside < 0.f) return V3(0, 0, 0);
    v3 n = dot(hit->n, wi) < 0.f ? neg(hit->n) : hit->n;
    float cos_theta_o = dot(n, wo);
    float cos_theta_i = dot(n, wi);
    if (cos_theta_i == 0.f || cos_theta_o == 0.f) return V3(0, 0, 0);
    v3 wh = normalize(add(wi, wo));
    float fresnel = fresnel_dielectric(1.f, md->eta, dot(wi, wh));
    v3 ks = V3(md->ks[0], md->ks[1], md->ks[2]);
    return muls(ks, (ggx_D(md->roughness, wh, n) * ggx_G(md->roughness, wi, wo, wh, n) * fresnel /
                     (4.f * cos_theta_i * cos_theta_o)));
}
/* Microfacet::Sample, bsdf/microfacet.h:80-95 */
static v3 microfacet_sample(const bg_material_desc* md, const hit_t* hit, v2 s, v3 wi, v3* wo, float* pdf) {
    hit_t hl = *hit;
    if (dot(hit->n, wi) < 0.f) { hl.n = neg(hl.n); hl.dpdu = neg(hl.dpdu); hl.dpdv = neg(hl.dpdv); }
    ggx_sample(md->roughness, &hl, s, wi, wo, pdf);
    return microfacet_eval(md, hit, wi, *wo);
}
/* Microfacet::GetPdf, bsdf/microfacet.h:132-148 */
static float microfacet_pdf(const bg_material_desc* md, const hit_t* hit, v3 wi, v3 wo) {
    float sameside = dot(wi, hit->n) * dot(wo, hit->n);
    if (sameside < 0.f) return 0.f;
    hit_t hl = *hit;
    if (dot(hl.n, wi) < 0) { hl.n = neg(hl.n); hl.dpdu = neg(hl.dpdu); hl.dpdv = neg(hl.dpdv); }
    return ggx_pdf(md->roughness, &hl, wi, wo);
}
/* Lambert, bsdf/lambert.h:66-127 */
static v3 lambert_sample(const bg_material_desc* md, const hit_t* hit, v2 s, v3 wi, v3* wo, float* pdf) {
    v3 n = dot(wi, hit->ng) >= 0.f ? hit->n : neg(hit->n);
    *wo = map_to_hemisphere(n, s, 1.f);
    float invpi = 1.f / PI;
    *pdf = dot(n, *wo) * invpi;
    return muls(V3(md->kd[0], md->kd[1], md->kd[2]), invpi);
}
static v3 lambert_eval(const bg_material_desc* md, const hit_t* hit, v3 wi, v3 wo) {
    float sameside = dot(wi, hit->ng) * dot(wo, hit->ng);
    if (sameside > 0.f) return muls(V3(md->kd[0], md->kd[1], md->kd[2]), 1.f / PI);
    return V3(0.f, 0.f, 0.f);
}
static float lambert_pdf(const hit_t* hit, v3 wi, v3 wo) {
    float sameside = dot(wi, hit->ng) * dot(wo, hit->ng);
    if (sameside > 0.f) {
        v3 n = dot(wi, hit->ng) >= 0.f ? hit->n : neg(hit->n);
        return dot(n, wo) * (1.f / PI);
    }
    return 0.f;
}
/* Emissive::GetLe, material/emissive.h:84-93 */
static v3 emissive_le(const bg_material_desc* md, v3 n, v3 wo) {
    float ndotwo = dot(n, wo);
    if (ndotwo > 0.f) return muls(V3(md->e[0], md->e[1], md->e[2]), ndotwo);
    return V3(0, 0, 0);
}

/* Material dispatch: SimpleMaterial (material/simplematerial.h:54-70) and
 * Emissive (material/emissive.h:55-81). */
static v3 mat_sample(const bg_material_desc* md, const hit_t* hit, v2 s, v3 wi, v3* wo, float* pdf, int* type) {
    switch (md->type) {
    case BG_MAT_LAMBERT: *type = BSDF_REFLECTION | BSDF_DIFFUSE; return lambert_sample(md, hit, s, wi, wo, pdf);
    case BG_MAT_MICROFACET_GGX: *type = BSDF_REFLECTION | BSDF_GLOSSY; return microfacet_sample(md, hit, s, wi, wo, pdf);
    default: *pdf = 0.f; return emissive_le(md, hit->n, wi);   /* type left unchanged, as the reference */
    }
}
static v3 mat_eval(const bg_material_desc* md, const hit_t* hit, v3 wi, v3 wo) {
    switch (md->type) {
    case BG_MAT_LAMBERT: return lambert_eval(md, hit, wi, wo);
    case BG_MAT_MICROFACET_GGX: return microfacet_eval(md, hit, wi, wo);
    default: return emissive_le(md, hit->n, wi);
    }
}
static float mat_pdf(const bg_material_desc* md, const hit_t* hit, v3 wi, v3 wo) {
    switch (md->type) {
    case BG_MAT_LAMBERT: return lambert_pdf(hit, wi, wo);
    case BG_MAT_MICROFACET_GGX: return microfacet_pdf(md, hit, wi, wo);
    default: return 0.f;
    }
}

/* ------------------------------------------------------------- lights */
/* Mesh::GetShapeSurfaceArea, primitive/mesh.cpp:304-321 */
static float shape_area(const mesh_t* me, int idx) {
    const face_t* f = &me->faces[idx];
    v3 p1 = transform_point(me->verts[f->vi0], &me->m);
    v3 p2 = transform_point(me->verts[f->vi1], &me->m);
    v3 p3 = transform_point(me->verts[f->vi2], &me->m);
    return sqrtf(fabsf(sqnorm(cross(sub(p3, p1), sub(p3, p2))))) * 0.5f;
}

/* AreaLight::GetSample -> Mesh::GetSampleOnShape + FillSample,
 * light/arealight.cpp:25-51, primitive/mesh.cpp:99-123,323-336 */
static v3 area_getsample(const or_world* w, const light_t* L, const hit_t* hit, v2 u, v3* d, float* pdf) {
    const mesh_t* me = &w->meshes[L->d.mesh];
    const face_t* f = &me->faces[L->d.face];
    float a = sqrtf(u.x) * (1.f - u.y);
    float b = sqrtf(u.x) * u.y;
    v3 p1 = me->verts[f->vi0], p2 = me->verts[f->vi1], p3 = me->verts[f->vi2];
    v3 n1 = me->normals[f->ni0], n2 = me->normals[f->ni1], n3 = me->normals[f->ni2];
    float w0 = 1.f - a - b;
    v3 sp = transform_point(add(add(muls(p1, w0), muls(p2, a)), muls(p3, b)), &me->m);
    v3 sn = normalize(transform_normal(add(add(muls(n1, w0), muls(n2, a)), muls(n3, b)), &me->minv));
    float spdf = 1.f / (sqrtf(fabsf(sqnorm(cross(sub(p3, p1), sub(p3, p2))))) * 0.5f);
    *d = sub(sp, hit->p);
    if (spdf > 0.f && dot(sn, neg(normalize(*d))) > 0.f) {
        *pdf = spdf;
        float d2inv = 1.f / sqnorm(*d);
        return muls(emissive_le(&w->mats[L->matidx].d, sn, neg(normalize(*d))), d2inv);
    }
    *pdf = 0.f;
    return V3(0, 0, 0);
}

/* AreaLight::GetPdf -> Mesh::GetPdfOnShape, light/arealight.cpp:54-58, primitive/mesh.cpp:354-378 */
static float area_getpdf(const or_world* w, const light_t* L, const hit_t* hit, v3 wv) {
    hit_t h;
    h.t = 100000.f;
    if (intersect_shape(w, L->d.mesh, L->d.face, hit->p, wv, 0.001f, &h) && dot(neg(wv), h.n) > 0.f) {
        v3 d = sub(hit->p, h.p);
        return sqnorm(d) / (dot(normalize(d), h.n) * shape_area(&w->meshes[L->d.mesh], L->d.face));
    }
    return 0.f;
}

/* EnvironmentLight over a constant texel: scale * pow(texel, 1/gamma)
 * (light/environment_light.cpp:36-65; pow is the double ::pow there). */
static v3 env_value(const light_t* L) {
    float invgamma = 1.f / L->d.gamma;
    v3 val = V3((float)pow((double)L->d.e[0], (double)invgamma), (float)pow((double)L->d.e[1], (double)invgamma),
                (float)pow((double)L->d.e[2], (double)invgamma));
    return muls(val, L->d.scale);
}

static v3 light_getsample(const or_world* w, const light_t* L, const hit_t* hit, v2 s, v3* d, float* pdf) {
    switch (L->d.type) {
    case BG_LIGHT_AREA: return area_getsample(w, L, hit, s, d, pdf);
    case BG_LIGHT_DIRECTIONAL:     /* light/directional_light.cpp:5-14 */
        *d = muls(neg(L->dir), 100000000.f);
        *pdf = 1.f;
        return V3(L->d.e[0], L->d.e[1], L->d.e[2]);
    default: {                     /* light/environment_light.cpp:8-33 */
        float invpi = 1.f / PI;
        *d = map_to_hemisphere(hit->n, s, 1.f);
        *pdf = dot(hit->n, *d) * invpi;
        *d = muls(*d, 10000000.f);
        return env_value(L);
    }
    }
}
static v3 light_getle(const light_t* L) {
    return L->d.type == BG_LIGHT_ENVIRONMENT ? env_value(L) : V3(0, 0, 0);
}
static float light_getpdf(const or_world* w, const light_t* L, const hit_t* hit, v3 wv) {
    switch (L->d.type) {
    case BG_LIGHT_AREA: return area_getpdf(w, L, hit, wv);
    case BG_LIGHT_DIRECTIONAL: return 0.f;
    default: return dot(hit->n, normalize(wv)) * (1.f / PI);   /* environment_light.cpp:62-68 */
    }
}
static int light_singular(const light_t* L) { return L->d.type == BG_LIGHT_DIRECTIONAL; }

/* ------------------------------------------------------------- tracers */
typedef struct { mcrng_t light, brdf; keyed_t* key; } samplers_t;

/* ------------------------------------------------------ image samplers */
/* SobolSampler::Sample2D, sampler/sobol_sampler.cpp:3-37: x from the
 * scrambled radical inverse in base 2, y from the scrambled Sobol (0,2)
 * generator matrix; both keep the top 24 bits. */
static float sobol_vdc(uint32_t n, uint32_t scramble) {
    uint32_t r = 0;
    for (int b = 0; b < 32; ++b) r |= ((n >> b) & 1u) << (31 - b);      /* bit reversal */
    r ^= scramble;
    return (float)((r >> 8) & 0xffffffu) / (float)(1 << 24);
}
static float sobol_02(uint32_t n, uint32_t scramble) {
    uint32_t col = 0x80000000u;
    while (n) {
        if (n & 1u) scramble ^= col;
        n >>= 1;
        col ^= col >> 1;
    }
    return (float)((scramble >> 8) & 0xffffffu) / (float)(1 << 24);
}

/* CmjSampler, sampler/cmj_sampler.cpp:3-73 (Kensler, "Correlated
 * Multi-Jittered Sampling", 2013): hashed permutation within [0, l) by
 * cycle walking, hashed jitter in [0, 1). */
static uint32_t cmj_permute(uint32_t i, uint32_t l, uint32_t p) {
    uint32_t w = l - 1;
    w |= w >> 1; w |= w >> 2; w |= w >> 4; w |= w >> 8; w |= w >> 16;
    do {
        i ^= p;             i *= 0xe170893du;
        i ^= p >> 16;       i ^= (i & w) >> 4;
        i ^= p >> 8;        i *= 0x0929eb3fu;
        i ^= p >> 23;       i ^= (i & w) >> 1;
        i *= 1u | p >> 27;  i *= 0x6935fa69u;
        i ^= (i & w) >> 11; i *= 0x74dcb303u;
        i ^= (i & w) >> 2;  i *= 0x9e501cc3u;
        i ^= (i & w) >> 2;  i *= 0xc860a3dfu;
        i &= w;
        i ^= i >> 5;
    } while (i >= l);
    return (i + p) % l;
}
static float cmj_jitter(uint32_t i, uint32_t p) {
    i ^= p;
    i ^= i >> 17; i ^= i >> 10; i *= 0xb36534e5u;
    i ^= i >> 12; i ^= i >> 21; i *= 0x93fc4795u;
    i ^= 0xdf6e307fu; i ^= i >> 17; i *= 1u | p >> 18;
    return (float)i * (1.0f / 4294967808.0f);
}
static v2 cmj_sample(int s, int m, int n, int p) {
    const uint32_t up = (uint32_t)p;
    int sx = (int)cmj_permute((uint32_t)(s % m), (uint32_t)m, up * 0xa511e9b3u);
    int sy = (int)cmj_permute((uint32_t)(s / m), (uint32_t)n, up * 0x63d83595u);
    float jx = cmj_jitter((uint32_t)s, up * 0xa399d265u);
    float jy = cmj_jitter((uint32_t)s, up * 0x711ad6a5u);
    return V2(((float)(s % m) + ((float)sy + jx) / (float)n) / (float)m,
              ((float)(s / m) + ((float)sx + jy) / (float)m) / (float)n);
}

/* Image sample of camera sample (pixel, s); img is the sample's keyed McRng. */
static v2 image_sample(int kind, int grid, uint64_t seed, uint32_t pixel, uint32_t s, mcrng_t* img) {
    if (kind == BG_SAMPLER_SOBOL) {
        keyed_t k; keyed_init(&k, seed, pixel, 0xFFFFFFFFu);
        mcrng_t m; mcrng_init(&m, &k);
        uint32_t sc0 = mc_next_uint(&m);
        uint32_t sc1 = mc_next_uint(&m);
        return V2(sobol_vdc(s, sc0), sobol_02(s, sc1));
    }
    if (kind == BG_SAMPLER_CMJ) {
        uint32_t g2 = (uint32_t)(grid * grid);
        keyed_t k; keyed_init(&k, seed, pixel, 0x80000000u + s / g2);
        mcrng_t m; mcrng_init(&m, &k);
        int pattern = (int)mc_next_uint(&m);
        return cmj_sample((int)(s % g2), grid, grid, pattern);
    }
    return sample2d(img);
}

/* DiTracer::GetDi, tracer/ditracer.cpp:57-239 (num_samples = 1) */
static v3 get_di(const or_world* w, int li, samplers_t* S, v3 wo, const hit_t* hit) {
    const light_t* L = &w->lights[li];
    v3 radiance = V3(0, 0, 0);
    v2 lightsample = sample2d(&S->light);
    v2 bsdfsample = sample2d(&S->brdf);
    int singular = light_singular(L);
    const bg_material_desc* mat = &w->mats[hit->m].d;
    float lightpdf = 0.f, bsdfpdf = 0.f;
    hit_t hl = *hit;
    v3 lightdir;
    v3 le = light_getsample(w, L, &hl, lightsample, &lightdir, &lightpdf);
    if (lightpdf > MINPDF && sqnorm(le) > 0.f) {
        v3 wi = normalize(lightdir);
        float dist = sqrtf(sqnorm(lightdir));
        int occluded = world_occluded(w, hl.p, wi, 0.01f, dist - 0.01f, NULL, NULL);
        float shadow = occluded ? 0.f : 1.f;
        if (shadow > 0.f) {
            v3 bsdf = mat_eval(mat, &hl, wi, wo);
            if (singular) {
                radiance = add(radiance, muls(muls(mulv(le, bsdf), fabsf(dot(hl.n, wi))), (1.f / lightpdf)));
            } else {
                bsdfpdf = mat_pdf(mat, &hl, wi, wo);
                float weight = power_heuristic(1, lightpdf, 1, bsdfpdf);
                radiance = add(radiance, muls(muls(muls(mulv(le, bsdf), fabsf(dot(hl.n, wi))), weight), (1.f / lightpdf)));
            }
        }
    }
    if (!singular) {
        int bsdftype = 0;
        v3 wi;
        v3 bsdf = mat_sample(mat, &hl, bsdfsample, wo, &wi, &bsdfpdf, &bsdftype);
        wi = normalize(wi);
        if (sqnorm(bsdf) > 0.f && bsdfpdf > MINPDF) {
            float weight = 1.f;
            int skip = 0;
            if (!(bsdftype & BSDF_SPECULAR)) {
                lightpdf = light_getpdf(w, L, &hl, wi);
                if (lightpdf < MINPDF) skip = 1;
                else weight = power_heuristic(1, bsdfpdf, 1, lightpdf);
            }
            if (!skip) {
                hit_t sh;
                v3 lev = V3(0.f, 0.f, 0.f);
                if (world_intersect(w, hl.p, wi, 0.01f, 10000000.f, &sh, NULL, NULL)) {
                    if (w->meshes[sh.mesh].arealight == li) {
                        const bg_material_desc* lightmat = &w->mats[sh.m].d;
                        v3 d = sub(sh.p, hl.p);
                        if (dot(sh.n, neg(wi)) > 0.f) {
                            float d2inv = 1.f / sqnorm(d);
                            lev = muls(emissive_le(lightmat, sh.n, neg(wi)), d2inv);
                        }
                    }
                } else {
                    lev = light_getle(L);
                }
                if (sqnorm(lev) > 0.f)
                    radiance = add(radiance, muls(muls(muls(mulv(lev, bsdf), fabsf(dot(hl.n, wi))), weight), (1.f / bsdfpdf)));
            }
        }
    }
    return muls(radiance, 1.f / 1);
}

/* GiTracer::GetLi, tracer/gitracer.cpp:13-140 */
static v3 gi_getli(const or_world* w, int maxdepth, v3 ro, v3 rd, float rtmin, float rtmax, samplers_t* S) {
    v3 radiance = V3(0, 0, 0);
    hit_t hp;
    if (!world_intersect(w, ro, rd, rtmin, rtmax, &hp, NULL, NULL)) {
        radiance = add(radiance, w->bgcolor);
        for (int i = 0; i < w->nlights; ++i) radiance = add(radiance, light_getle(&w->lights[i]));
        return radiance;
    }
    v2 sample0 = sample2d(&S->brdf);
    {
        v3 o = ro, d = rd;
        hit_t hit = hp;
        v3 thr = V3(1.f, 1.f, 1.f);
        for (int bounce = 0; bounce < maxdepth; ++bounce) {
            const bg_material_desc* mat = &w->mats[hit.m].d;
            if (bounce == 0 && mat->type == BG_MAT_EMISSIVE) {
                radiance = add(radiance, emissive_le(mat, hit.n, neg(d)));
                break;
            }
            if (bounce != 0) {
                int numlights = w->nlights;
                int idx = (int)(rand_uint(S->key) % (uint32_t)numlights);
                radiance = add(radiance, muls(mulv(thr, get_di(w, idx, S, neg(d), &hit)), (float)numlights));
            } else {
                for (int i = 0; i < w->nlights; ++i)
                    radiance = add(radiance, mulv(thr, get_di(w, i, S, neg(d), &hit)));
            }
            int bsdftype = 0;
            float bsdfpdf = 0.f;
            v3 wi;
            v3 bsdf = mat_sample(mat, &hit, sample0, neg(d), &wi, &bsdfpdf, &bsdftype);
            if (sqnorm(bsdf) == 0.f || bsdfpdf < MINPDF) break;
            o = hit.p;
            d = normalize(wi);
            thr = mulv(thr, muls(bsdf, (fabsf(dot(hit.n, wi)) / bsdfpdf)));
            if (bounce > 3) {
                float rnd = rand_float(S->key);
                float luminance = 0.2126f * thr.x + 0.7152f * thr.y + 0.0722f * thr.z;
                float q = fmin_std(0.5f, luminance);
                if (rnd > q) break;
                thr = muls(thr, (1.f / q));
            }
            if (!world_intersect(w, o, d, 0.01f, 1000000.f, &hit, NULL, NULL)) break;
        }
    }
    v3 r = muls(radiance, (1.f / 1));
    return V3(clampf_ref(r.x, 0.f, MAXRADIANCE), clampf_ref(r.y, 0.f, MAXRADIANCE), clampf_ref(r.z, 0.f, MAXRADIANCE));
}

/* DiTracer::GetLi, tracer/ditracer.cpp:19-55 */
static v3 di_getli(const or_world* w, v3 ro, v3 rd, float rtmin, float rtmax, samplers_t* S) {
    hit_t hit;
    v3 radiance = V3(0, 0, 0);
    if (world_intersect(w, ro, rd, rtmin, rtmax, &hit, NULL, NULL)) {
        const bg_material_desc* mat = &w->mats[hit.m].d;
        if (mat->type == BG_MAT_EMISSIVE) return V3(0, 0, 0);
        for (int i = 0; i < w->nlights; ++i) radiance = add(radiance, get_di(w, i, S, neg(rd), &hit));
    } else {
        radiance = w->bgcolor;
        for (int i = 0; i < w->nlights; ++i) radiance = add(radiance, light_getle(&w->lights[i]));
    }
    return radiance;
}

/* --------------------------------------------------------------- camera */
typedef struct { v3 forward, right, up, p; v2 zcap, dim; } camera_t;

/* PerscpectiveCamera ctor, camera/perspective_camera.cpp:5-23 */
static camera_t camera_make(const bg_camera_desc* c) {
    camera_t k;
    v3 eye = V3(c->eye[0], c->eye[1], c->eye[2]), at = V3(c->at[0], c->at[1], c->at[2]), up = V3(c->up[0], c->up[1], c->up[2]);
    k.p = eye;
    k.zcap = V2(c->znear, c->zfar);
    k.forward = normalize(sub(at, eye));
    k.right = cross(k.forward, normalize(up));
    k.up = cross(k.right, k.forward);
    k.dim.x = 2 * tanf(c->fovy * 0.5f) * k.zcap.x;
    k.dim.y = k.dim.x / c->aspect;
    return k;
}
/* PerscpectiveCamera::GenerateRay, camera/perspective_camera.cpp:25-38 */
static void camera_ray(const camera_t* k, v2 s, v3* o, v3* d, float* tmin, float* tmax) {
    v2 hs = V2(s.x - 0.5f, s.y - 0.5f);
    v2 cs = V2(hs.x * k->dim.x, hs.y * k->dim.y);
    *o = k->p;
    *d = normalize(add(add(muls(k->forward, k->zcap.x), muls(k->right, cs.x)), muls(k->up, cs.y)));
    *tmin = k->zcap.x;
    *tmax = k->zcap.y;
}

void or_camera_rays(const bg_camera_desc* cam, const float* samples, bg_ray* rays, int64_t n) {
    camera_t k = camera_make(cam);
    for (int64_t i = 0; i < n; ++i) {
        v3 o, d; float t0, t1;
        camera_ray(&k, V2(samples[2 * i], samples[2 * i + 1]), &o, &d, &t0, &t1);
        rays[i].o[0] = o.x; rays[i].o[1] = o.y; rays[i].o[2] = o.z; rays[i].tmin = t0;
        rays[i].d[0] = d.x; rays[i].d[1] = d.y; rays[i].d[2] = d.z; rays[i].tmax = t1;
    }
}

/* AoTracer::GetLi, tracer/aotracer.cpp:9-49 (lightsampler.num_samples() = 1):
 * one cosine-distributed ray about the shading normal, t in (0.00002, radius). */
static v3 ao_getli(const or_world* w, float radius, v3 ro, v3 rd, float rtmin, float rtmax, samplers_t* S) {
    hit_t hit;
    if (!world_intersect(w, ro, rd, rtmin, rtmax, &hit, NULL, NULL)) return V3(0.f, 0.f, 0.f);
    v2 sample = sample2d(&S->light);
    v3 d = map_to_hemisphere(hit.n, sample, 1.f);
    float occlusion = world_occluded(w, hit.p, d, 0.00002f, radius, NULL, NULL) ? 1.f : 0.f;
    occlusion *= 1.f / 1.f;
    return V3(1.f - occlusion, 1.f - occlusion, 1.f - occlusion);
}

/* ------------------------------------------------------------- renderer */
typedef struct {
    const or_world* w;
    camera_t cam;
    int kind, maxdepth, W, H, spp, soff, skind, sgrid;
    float ao_radius;
    uint64_t seed;
    float* accum;
    int x0, x1, y0;
} render_arg_t;

/* ImageRenderer::Render body, renderer/imagerenderer.cpp:25-43, one row per task */
static void render_rows(void* a, int64_t b, int64_t e) {
    render_arg_t* r = (render_arg_t*)a;
    for (int64_t row = b; row < e; ++row) {
        int y = r->y0 + (int)row;
        for (int x = r->x0; x < r->x1; ++x) {
            for (int s = 0; s < r->spp; ++s) {
                keyed_t key;
                keyed_init(&key, r->seed, (uint32_t)(y * r->W + x), (uint32_t)(r->soff + s));
                mcrng_t img;
                samplers_t S;
                mcrng_init(&img, &key);
                mcrng_init(&S.light, &key);
                mcrng_init(&S.brdf, &key);
                S.key = &key;
                v2 smp = image_sample(r->skind, r->sgrid, r->seed, (uint32_t)(y * r->W + x),
                                      (uint32_t)(r->soff + s), &img);
                v2 is = V2((float)x / r->W + (1.f / r->W) * smp.x, (float)y / r->H + (1.f / r->H) * smp.y);
                v3 o, d; float t0, t1;
                camera_ray(&r->cam, is, &o, &d, &t0, &t1);
                v3 L = r->kind == BG_TRACER_DI   ? di_getli(r->w, o, d, t0, t1, &S)
                       : r->kind == BG_TRACER_AO ? ao_getli(r->w, r->ao_radius, o, d, t0, t1, &S)
                                                 : gi_getli(r->w, r->maxdepth, o, d, t0, t1, &S);
                /* FileImagePlane::WriteSample, imageplane/fileimageplane.cpp:29-34 */
                float* px = &r->accum[4 * ((size_t)r->W * (size_t)(r->H - 1 - y) + (size_t)x)];
                px[0] += L.x; px[1] += L.y; px[2] += L.z; px[3] += 1.f;
            }
        }
    }
}

void or_render(const or_world* w, const bg_camera_desc* cam, int32_t tracer_kind, int32_t maxdepth,
               int32_t width, int32_t height, int32_t spp, int32_t sample_offset, uint64_t seed,
               float* accum, int32_t x0, int32_t y0, int32_t x1, int32_t y1, int32_t nthreads,
               int32_t sampler_kind, int32_t sampler_grid, float ao_radius) {
    render_arg_t r;
    r.w = w; r.cam = camera_make(cam); r.kind = tracer_kind; r.maxdepth = maxdepth;
    r.skind = sampler_kind; r.sgrid = sampler_grid; r.ao_radius = ao_radius;
    r.W = width; r.H = height; r.spp = spp; r.soff = sample_offset; r.seed = seed; r.accum = accum;
    r.x0 = x0; r.x1 = x1; r.y0 = y0;
    parallel_for(y1 - y0, 1, nthreads, render_rows, &r);
}
