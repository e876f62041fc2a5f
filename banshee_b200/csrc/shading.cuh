// Surface interaction, BSDFs and lights for the wavefront tracer.
//
// Restates, in the reference's operation order:
//   Mesh::FillHit / FillSample           primitive/mesh.cpp:47-123
//   Lambert                              bsdf/lambert.h:66-127
//   Microfacet + GgxDistribution         bsdf/microfacet.h:80-148,
//                                        bsdf/microfacet_distribution.h:196-286
//   FresnelDielectric                    bsdf/fresnel.h:59-90
//   Emissive::GetLe                      material/emissive.h:84-93
//   AreaLight / DirectionalLight / EnvironmentLight
//                                        light/arealight.cpp, directional_light.cpp,
//                                        environment_light.cpp
//   map_to_hemisphere / orthovector / PowerHeuristic   math/mathutils.h:214-296
//
// The BSDF and light-sampling functions are __noinline__: k_shade calls them
// from several places, and one shared copy keeps the shading kernel inside the
// instruction cache (measured: the fully inlined kernel stalled on instruction
// fetch).  fill_hit, called once, is inlined so that its hit record stays in
// registers instead of the call frame (measured: +6.7 % frame throughput
// together with inlining emit_di).
#pragma once

#include "device_common.cuh"
#include "scene_types.h"
#include "traverse.cuh"

namespace bg {

constexpr int kBsdfReflection = 1 << 0;
constexpr int kBsdfDiffuse = 1 << 2;
constexpr int kBsdfSpecular = 1 << 3;
constexpr int kBsdfGlossy = 1 << 4;

struct SHit {            // ShapeBundle::Hit (primitive/shapebundle.h:156-176)
    v3 p, n, ng, dpdu, dpdv;
    float u, v;
    int m;
    int bundle;
};

__device__ __forceinline__ v3 f4xyz(float4 a) { return mk(a.x, a.y, a.z); }

__device__ __forceinline__ void load_xf(const BundleRec* b, float* m, float* minv) {
#pragma unroll
    for (int k = 0; k < 12; ++k) { m[k] = __ldg(b->m + k); minv[k] = __ldg(b->minv + k); }
}

// orthovector, math/mathutils.h:214-227
__device__ __forceinline__ v3 orthovector(v3 n) {
    v3 p;
    if (fabsf(n.z) > 0.707106781186547524401f) {
        float k = sqrtf(n.y * n.y + n.z * n.z);
        p.x = 0.f; p.y = -n.z / k; p.z = n.y / k;
    } else {
        float k = sqrtf(n.x * n.x + n.y * n.y);
        p.x = -n.y / k; p.y = n.x / k; p.z = 0.f;
    }
    return p;
}

// Mesh::FillHit, primitive/mesh.cpp:47-97
__device__ __forceinline__ void fill_hit(const DevScene& S, int prim, float a, float b, SHit& h) {
    const float4* sr = reinterpret_cast<const float4*>(S.shade + prim);
    float4 ra = __ldg(sr), rb = __ldg(sr + 1), rc = __ldg(sr + 2), rd = __ldg(sr + 3);
    float4 re = __ldg(sr + 4), rf = __ldg(sr + 5), rg = __ldg(sr + 6);
    v3 p1 = f4xyz(ra), p2 = f4xyz(rb), p3 = f4xyz(rc);
    v3 n1 = f4xyz(rd), n2 = f4xyz(re), n3 = f4xyz(rf);
    float t1x = rc.w, t1y = rd.w, t2x = re.w, t2y = rf.w, t3x = rg.x, t3y = rg.y;
    h.bundle = __float_as_int(ra.w);
    h.m = __float_as_int(rb.w);
    const BundleRec* B = S.bundles + h.bundle;
    const bool ident = __ldg(&B->identity) != 0;
    float m[12], mi[12];
    if (!ident) load_xf(B, m, mi);
    float w0 = 1.f - a - b;
    v3 p = add(add(muls(p1, w0), muls(p2, a)), muls(p3, b));
    h.p = ident ? p : xf_point(m, p);
    v3 n = add(add(muls(n1, w0), muls(n2, a)), muls(n3, b));
    h.n = normalize(ident ? n : xf_normal(mi, n));
    v3 g = cross(sub(p3, p1), sub(p2, p1));
    h.ng = normalize(ident ? g : xf_normal(mi, g));
    if (dot(h.n, h.ng) < 0) h.ng = neg(h.ng);
    float du1 = t1x - t3x, du2 = t2x - t3x, dv1 = t1y - t3y, dv2 = t2y - t3y;
    v3 dp1 = sub(p1, p3), dp2 = sub(p2, p3);
    float det = du1 * dv2 - dv1 * du2;
    if (det != 0.f) {
        float invdet = 1.f / det;
        v3 tu = muls(sub(muls(dp1, dv2), muls(dp2, dv1)), invdet);
        v3 tv = muls(add(muls(dp1, -du2), muls(dp2, du1)), invdet);
        h.dpdu = normalize(ident ? tu : xf_normal(mi, tu));
        h.dpdv = normalize(ident ? tv : xf_normal(mi, tv));
    } else {
        h.dpdu = orthovector(h.n);
        h.dpdv = cross(h.n, h.dpdu);
    }
    h.u = t1x * w0 + t2x * a + t3x * b;
    h.v = t1y * w0 + t2y * a + t3y * b;
}

// map_to_hemisphere(n, s, e), math/mathutils.h:230-244
__device__ __forceinline__ v3 map_to_hemisphere_body(v3 n, float sx, float sy, float e) {
    v3 u = orthovector(n);
    v3 v = cross(u, n);
    u = cross(n, v);
    float sinpsi = sinf(2 * BG_PI * sx);
    float cospsi = cosf(2 * BG_PI * sx);
    float costheta = powf(1.f - sy, 1.f / (e + 1.f));
    float sintheta = sqrtf(1.f - costheta * costheta);
    return normalize(add(add(muls(muls(u, sintheta), cospsi), muls(muls(v, sintheta), sinpsi)), muls(n, costheta)));
}
__device__ __noinline__ v3 map_to_hemisphere(v3 n, float sx, float sy, float e) { return map_to_hemisphere_body(n, sx, sy, e); }
// INL: inline copy (the material-class shading kernels) or the shared out-of-line one
template <bool INL>
__device__ __forceinline__ v3 hemisphere(v3 n, float sx, float sy, float e) {
    return INL ? map_to_hemisphere_body(n, sx, sy, e) : map_to_hemisphere(n, sx, sy, e);
}

__device__ __forceinline__ float power_heuristic(float fpdf, float gpdf) {
    float f = 1 * fpdf;
    float g = 1 * gpdf;
    return (f * f) / (f * f + g * g);
}

// --------------------------------------------------------------- BSDFs
__device__ __forceinline__ float ggx_D(float a_, v3 m, v3 n) {
    float ndotm = dot(m, n);
    if (ndotm <= 0.f) return 0.f;
    float ndotm2 = ndotm * ndotm;
    float sinmn = sqrtf(1.f - clamp_ref(ndotm * ndotm, 0.f, 1.f));
    float tanmn = sinmn / ndotm;
    float a2 = a_ * a_;
    return (a2 / (BG_PI * ndotm2 * ndotm2 * (a2 + tanmn * tanmn) * (a2 + tanmn * tanmn)));
}
__device__ __forceinline__ float ggx_pdf(float a_, v3 hn, v3 wi, v3 wo) {
    v3 m = normalize(add(wi, wo));
    float mpdf = ggx_D(a_, m, hn) * fabsf(dot(hn, m));
    return mpdf / (4.f * dot(wo, m));
}
__device__ __forceinline__ float ggx_G1(float a_, v3 v, v3 m, v3 n) {
    float ndotv = dot(n, v);
    float mdotv = dot(m, v);
    if (ndotv * mdotv <= 0.f) return 0.f;
    float sinnv = sqrtf(1.f - clamp_ref(ndotv * ndotv, 0.f, 1.f));
    float tannv = sinnv / ndotv;
    float a2 = a_ * a_;
    return 2.f / (1.f + sqrtf(1.f + a2 * tannv * tannv));
}
__device__ __forceinline__ float fresnel_dielectric(float etai, float etat, float ndotwi) {
    float ei = etai, et = etat;
    if (ndotwi < 0) { ei = etat; et = etai; ndotwi = -ndotwi; }
    float sint = (ei / et) * sqrtf(fmax_std(0.f, 1.f - ndotwi * ndotwi));
    if (sint > 1.f) return 1.f;
    float ndotwt = sqrtf(fmax_std(0.f, 1.f - sint * sint));
    float rparl = ((et * ndotwi) - (ei * ndotwt)) / ((et * ndotwi) + (ei * ndotwt));
    float rperp = ((ei * ndotwi) - (et * ndotwt)) / ((ei * ndotwi) + (et * ndotwt));
    return (rparl * rparl + rperp * rperp) * 0.5f;
}
// The out-of-line BSDF functions take and return values only (no reference to
// the caller's hit record or material), so the caller's registers stay
// registers across the call instead of being written to a local-memory frame.
struct BsdfSample {
    v3 f, wo;
    float pdf;
};

// Microfacet::Evaluate (bsdf/microfacet.h:110-148) for the shading normal hn
__device__ __forceinline__ v3 microfacet_eval_body(v3 ks, float eta, float a, v3 hn, v3 wi, v3 wo) {
    float sameside = dot(wi, hn) * dot(wo, hn);
    if (sameside < 0.f) return mk(0.f, 0.f, 0.f);
    v3 n = dot(hn, wi) < 0.f ? neg(hn) : hn;
    float cos_o = dot(n, wo);
    float cos_i = dot(n, wi);
    if (cos_i == 0.f || cos_o == 0.f) return mk(0.f, 0.f, 0.f);
    v3 wh = normalize(add(wi, wo));
    float F = fresnel_dielectric(1.f, eta, dot(wi, wh));
    float G = ggx_G1(a, wi, wh, n) * ggx_G1(a, wo, wh, n);
    return muls(ks, (ggx_D(a, wh, n) * G * F / (4.f * cos_i * cos_o)));
}
__device__ __noinline__ v3 microfacet_eval(v3 ks, float eta, float a, v3 hn, v3 wi, v3 wo) {
    return microfacet_eval_body(ks, eta, a, hn, wi, wo);
}
// Microfacet::Sample + GgxDistribution::Sample (bsdf/microfacet.h:80-108,
// bsdf/microfacet_distribution.h:236-262); the value is Evaluate on the
// unflipped hit
__device__ __forceinline__ BsdfSample microfacet_sample_body(v3 ks, float eta, float a, v3 hn, v3 hdu, v3 hdv, float sx, float sy,
                                                     v3 wi) {
    v3 n = hn, du = hdu, dv = hdv;
    if (dot(hn, wi) < 0.f) { n = neg(n); du = neg(du); dv = neg(dv); }
    float temp = atanf(a * sqrtf(sx) / sqrtf(1.f - sx));
    float theta = (float)((temp >= 0) ? temp : (temp + 2 * BG_PI));
    float costheta = cosf(theta);
    float sintheta = sqrtf(1.f - clamp_ref(costheta * costheta, 0.f, 1.f));
    float cosphi = cosf(2.f * BG_PI * sy);
    float sinphi = sinf(2.f * BG_PI * sy);
    v3 wh = normalize(add(add(muls(muls(du, sintheta), cosphi), muls(muls(dv, sintheta), sinphi)), muls(n, costheta)));
    BsdfSample r;
    r.wo = add(neg(wi), muls(wh, 2.f * dot(wi, wh)));
    r.pdf = ggx_pdf(a, n, wi, r.wo);
    r.f = microfacet_eval_body(ks, eta, a, hn, wi, r.wo);
    return r;
}
__device__ __noinline__ BsdfSample microfacet_sample(v3 ks, float eta, float a, v3 hn, v3 hdu, v3 hdv, float sx, float sy,
                                                     v3 wi) {
    return microfacet_sample_body(ks, eta, a, hn, hdu, hdv, sx, sy, wi);
}
// Microfacet::GetPdf (bsdf/microfacet.h:150-165)
__device__ __forceinline__ float microfacet_pdf_body(float a, v3 hn, v3 wi, v3 wo) {
    float sameside = dot(wi, hn) * dot(wo, hn);
    if (sameside < 0.f) return 0.f;
    v3 n = dot(hn, wi) < 0 ? neg(hn) : hn;
    return ggx_pdf(a, n, wi, wo);
}
__device__ __noinline__ float microfacet_pdf(float a, v3 hn, v3 wi, v3 wo) {
    return microfacet_pdf_body(a, hn, wi, wo);
}
// Lambert::Sample (bsdf/lambert.h:66-86)
__device__ __forceinline__ BsdfSample lambert_sample_body(v3 kd, v3 hn, v3 ng, float sx, float sy, v3 wi) {
    v3 n = dot(wi, ng) >= 0.f ? hn : neg(hn);
    BsdfSample r;
    r.wo = map_to_hemisphere_body(n, sx, sy, 1.f);
    float invpi = 1.f / BG_PI;
    r.pdf = dot(n, r.wo) * invpi;
    r.f = muls(kd, invpi);
    return r;
}
__device__ __noinline__ BsdfSample lambert_sample(v3 kd, v3 hn, v3 ng, float sx, float sy, v3 wi) {
    return lambert_sample_body(kd, hn, ng, sx, sy, wi);
}
__device__ __forceinline__ v3 lambert_eval(const MatRec& M, const SHit& h, v3 wi, v3 wo) {
    float sameside = dot(wi, h.ng) * dot(wo, h.ng);
    if (sameside > 0.f) return muls(mk(M.kd[0], M.kd[1], M.kd[2]), 1.f / BG_PI);
    return mk(0.f, 0.f, 0.f);
}
__device__ __forceinline__ float lambert_pdf(const SHit& h, v3 wi, v3 wo) {
    float sameside = dot(wi, h.ng) * dot(wo, h.ng);
    if (sameside > 0.f) {
        v3 n = dot(wi, h.ng) >= 0.f ? h.n : neg(h.n);
        return dot(n, wo) * (1.f / BG_PI);
    }
    return 0.f;
}
__device__ __forceinline__ v3 emissive_le(const MatRec& M, v3 n, v3 wo) {
    float ndotwo = dot(n, wo);
    if (ndotwo > 0.f) return muls(mk(M.e[0], M.e[1], M.e[2]), ndotwo);
    return mk(0.f, 0.f, 0.f);
}

__device__ __forceinline__ MatRec load_mat(const DevScene& S, int m) {
    MatRec r;
    const MatRec* p = S.mats + m;
    r.type = __ldg(&p->type);
#pragma unroll
    for (int k = 0; k < 3; ++k) { r.kd[k] = __ldg(p->kd + k); r.ks[k] = __ldg(p->ks + k); r.e[k] = __ldg(p->e + k); }
    r.eta = __ldg(&p->eta);
    r.a = __ldg(&p->a);
    return r;
}

// SimpleMaterial / Emissive dispatch (material/simplematerial.h:54-70, emissive.h:55-81)
template <bool INL = false>
__device__ __forceinline__ v3 mat_sample(const MatRec& M, const SHit& h, float sx, float sy, v3 wi, v3& wo, float& pdf, int& type) {
    if (M.type == BG_MAT_LAMBERT) {
        type = kBsdfReflection | kBsdfDiffuse;
        const v3 kd = mk(M.kd[0], M.kd[1], M.kd[2]);
        const BsdfSample r = INL ? lambert_sample_body(kd, h.n, h.ng, sx, sy, wi) : lambert_sample(kd, h.n, h.ng, sx, sy, wi);
        wo = r.wo;
        pdf = r.pdf;
        return r.f;
    }
    if (M.type == BG_MAT_MICROFACET_GGX) {
        type = kBsdfReflection | kBsdfGlossy;
        const v3 ks = mk(M.ks[0], M.ks[1], M.ks[2]);
        const BsdfSample r = INL ? microfacet_sample_body(ks, M.eta, M.a, h.n, h.dpdu, h.dpdv, sx, sy, wi)
                                 : microfacet_sample(ks, M.eta, M.a, h.n, h.dpdu, h.dpdv, sx, sy, wi);
        wo = r.wo;
        pdf = r.pdf;
        return r.f;
    }
    pdf = 0.f;
    wo = mk(0.f, 0.f, 0.f);
    return emissive_le(M, h.n, wi);
}
template <bool INL = false>
__device__ __forceinline__ v3 mat_eval(const MatRec& M, const SHit& h, v3 wi, v3 wo) {
    if (M.type == BG_MAT_LAMBERT) return lambert_eval(M, h, wi, wo);
    if (M.type == BG_MAT_MICROFACET_GGX) {
        const v3 ks = mk(M.ks[0], M.ks[1], M.ks[2]);
        return INL ? microfacet_eval_body(ks, M.eta, M.a, h.n, wi, wo) : microfacet_eval(ks, M.eta, M.a, h.n, wi, wo);
    }
    return emissive_le(M, h.n, wi);
}
template <bool INL = false>
__device__ __forceinline__ float mat_pdf(const MatRec& M, const SHit& h, v3 wi, v3 wo) {
    if (M.type == BG_MAT_LAMBERT) return lambert_pdf(h, wi, wo);
    if (M.type == BG_MAT_MICROFACET_GGX) return INL ? microfacet_pdf_body(M.a, h.n, wi, wo) : microfacet_pdf(M.a, h.n, wi, wo);
    return 0.f;
}

// --------------------------------------------------------------- lights
__device__ __forceinline__ LightRec load_light(const DevScene& S, int i) {
    LightRec L;
    const LightRec* p = S.lights + i;
    L.type = __ldg(&p->type);
    L.mesh = __ldg(&p->mesh);
    L.face = __ldg(&p->face);
    L.matidx = __ldg(&p->matidx);
#pragma unroll
    for (int k = 0; k < 3; ++k) { L.dir[k] = __ldg(p->dir + k); L.e[k] = __ldg(p->e + k); L.env[k] = __ldg(p->env + k); }
    L.area_world = __ldg(&p->area_world);
    L.pdf_obj = __ldg(&p->pdf_obj);
    return L;
}

// AreaLight::GetSample (light/arealight.cpp:25-51) with Mesh::GetSampleOnShape /
// FillSample (primitive/mesh.cpp:99-123,323-336); the area pdf 1/area in object
// space is precomputed on the host (same float ops).
__device__ __noinline__ v3 area_getsample(const DevScene& S, const LightRec& L, v3 hp, float ux, float uy, v3& d, float& pdf) {
    const int prim = int(__ldg(&S.bundles[L.mesh].start)) + L.face;
    const float4* sr = reinterpret_cast<const float4*>(S.shade + prim);
    float4 ra = __ldg(sr), rb = __ldg(sr + 1), rc = __ldg(sr + 2), rd = __ldg(sr + 3), re = __ldg(sr + 4), rf = __ldg(sr + 5);
    float a = sqrtf(ux) * (1.f - uy);
    float b = sqrtf(ux) * uy;
    float w0 = 1.f - a - b;
    const BundleRec* B = S.bundles + L.mesh;
    const bool ident = __ldg(&B->identity) != 0;
    float m[12], mi[12];
    if (!ident) load_xf(B, m, mi);
    v3 sp = add(add(muls(f4xyz(ra), w0), muls(f4xyz(rb), a)), muls(f4xyz(rc), b));
    if (!ident) sp = xf_point(m, sp);
    v3 sn = add(add(muls(f4xyz(rd), w0), muls(f4xyz(re), a)), muls(f4xyz(rf), b));
    sn = normalize(ident ? sn : xf_normal(mi, sn));
    d = sub(sp, hp);
    if (L.pdf_obj > 0.f && dot(sn, neg(normalize(d))) > 0.f) {
        pdf = L.pdf_obj;
        float d2inv = 1.f / sqnorm(d);
        MatRec M = load_mat(S, L.matidx);
        return muls(emissive_le(M, sn, neg(normalize(d))), d2inv);
    }
    pdf = 0.f;
    return mk(0.f, 0.f, 0.f);
}

// AreaLight::GetPdf -> Mesh::GetPdfOnShape (primitive/mesh.cpp:354-378): intersect the
// light's own triangle from p along w with t in (0.001, 1e5].
__device__ __noinline__ float area_getpdf(const DevScene& S, const LightRec& L, v3 hp, v3 w) {
    const int prim = int(__ldg(&S.bundles[L.mesh].start)) + L.face;
    const float4* sr = reinterpret_cast<const float4*>(S.shade + prim);
    float4 ra = __ldg(sr), rb = __ldg(sr + 1), rc = __ldg(sr + 2);
    v3 p1 = f4xyz(ra), p2 = f4xyz(rb), p3 = f4xyz(rc);
    const BundleRec* B = S.bundles + L.mesh;
    v3 o = hp, d = w;
    if (!__ldg(&B->identity)) {
        float mi[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) mi[k] = __ldg(B->minv + k);
        o = xf_point(mi, hp);
        d = xf_vector(mi, w);
    }
    float t, a, b;
    if (!mt_test(o, d, p1, sub(p2, p1), sub(p3, p1), 0.001f, 100000.f, t, a, b)) return 0.f;
    SHit h;
    fill_hit(S, prim, a, b, h);
    if (dot(neg(w), h.n) > 0.f) {
        v3 dd = sub(hp, h.p);
        return sqnorm(dd) / (dot(normalize(dd), h.n) * L.area_world);
    }
    return 0.f;
}

__device__ __forceinline__ bool light_singular(const LightRec& L) { return L.type == BG_LIGHT_DIRECTIONAL; }

// AREA = false: the scene has no area light (the shading variant without the
// area-light code; its lights are directional or environment lights).
template <bool AREA, bool INL = false>
__device__ __forceinline__ v3 light_getsample(const DevScene& S, const LightRec& L, const SHit& h, float sx, float sy, v3& d, float& pdf) {
    if (AREA && L.type == BG_LIGHT_AREA) return area_getsample(S, L, h.p, sx, sy, d, pdf);
    if (L.type == BG_LIGHT_DIRECTIONAL) {                       // directional_light.cpp:5-14
        d = muls(neg(mk(L.dir[0], L.dir[1], L.dir[2])), 100000000.f);
        pdf = 1.f;
        return mk(L.e[0], L.e[1], L.e[2]);
    }
    float invpi = 1.f / BG_PI;                                    // environment_light.cpp:8-33
    d = hemisphere<INL>(h.n, sx, sy, 1.f);
    pdf = dot(h.n, d) * invpi;
    d = muls(d, 10000000.f);
    return mk(L.env[0], L.env[1], L.env[2]);
}
template <bool AREA>
__device__ __forceinline__ float light_getpdf(const DevScene& S, const LightRec& L, const SHit& h, v3 w) {
    if (AREA && L.type == BG_LIGHT_AREA) return area_getpdf(S, L, h.p, w);
    if (L.type == BG_LIGHT_DIRECTIONAL) return 0.f;
    return dot(h.n, normalize(w)) * (1.f / BG_PI);
}

}  // namespace bg
