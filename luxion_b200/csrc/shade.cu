// shade.cu -- camera generation, shading, light sampling, accumulation and tonemapping.
//
// Compiled with --fmad=false: every float multiply and add is rounded on its own, in the
// order the reference writes it, so these kernels agree with the reference's host build
// except where CUDA's transcendental functions differ from the host's by an ulp.
//
//   k_camera      generateRayFromCamera (src/kernels/generate_ray_from_camera.cu:8-39) and the
//                 bounce-0 sampleDirectLight (src/kernels/sample_direct_light.cu:9-101)
//   k_shade       shadePath (src/kernels/shade_path.cu:94-364) with the uber-shader
//                 (src/shaders/cook_torrance.cu), material queries (src/material_queries.cu),
//                 throughput/RR (src/update_throughput_materials.cu:23-67), the warp-aggregated
//                 survivor append (:355-363) and, fused behind it, the next bounce's
//                 sampleDirectLight: that kernel seeds its RNG with the pre-increment depth,
//                 which equals the post-increment depth this shade just used
//                 (src/pathtrace.cu:193,264,299), so the stream is the same.
//   k_accumulate  finalGather (src/kernels/image_kernels.cu:49-60), samples added in order
//   k_tonemap     sendImageToPBO (src/kernels/image_kernels.cu:6-46, src/tonemapping.cu)

#include "device_scene.h"
#include "device_math.cuh"
#include "launch.h"

#include <algorithm>
#include <map>
#include <mutex>

namespace lux {
namespace {

// A closest hit as the shading reads it. The tangent frame is only read under a normal map,
// so it is rebuilt there from the hit (hit_tangent) instead of for every hit.
struct Isect {
    float t;
    f3 normal;
    int inst, prim;
    int material;
    float u, v;
};

LUX_DI float4 tex(unsigned long long t, float u, float v) { return tex2D<float4>(cudaTextureObject_t(t), u, v); }

LUX_DI void tt_apply(const DevTexTransform& tt, float& u, float& v) {  // src/material_queries.cu:3-17
    u *= tt.scale[0];
    v *= tt.scale[1];
    if (tt.rotation != 0.0f) {
        float c = cosf(tt.rotation), s = sinf(tt.rotation);
        float nu = c * u - s * v, nv = s * u + c * v;
        u = nu;
        v = nv;
    }
    u = u + tt.offset[0];
    v = v + tt.offset[1];
}

LUX_DI void mesh_tri(const DevScene& S, const DevInstance& I, int prim, uint32_t& i0, uint32_t& i1, uint32_t& i2) {
    const uint32_t* id = S.idx + (size_t(I.idx_base) + prim) * 3;
    i0 = I.vert_base + __ldg(id);
    i1 = I.vert_base + __ldg(id + 1);
    i2 = I.vert_base + __ldg(id + 2);
}

// closest-hit program (src/optixshaders/optix_triangle.cu:156-243); its tangent is hit_tangent
LUX_DI Isect ch_radiance(const DevScene& S, float t, int inst, int prim, float bu, float bv) {
    Isect r;
    const DevInstance& I = S.insts[inst];
    uint32_t i0, i1, i2;
    mesh_tri(S, I, prim, i0, i1, i2);
    f3 n;
    float bA = 1.0f - bu - bv;
    if (I.flags & kInstHasNormals) {
        f3 nA = ld3(S.nrm + i0 * 3), nB = ld3(S.nrm + i1 * 3), nC = ld3(S.nrm + i2 * 3);
        n = normalize(bA * nA + bu * nB + bv * nC);
    } else {
        f3 A = ld3(S.pos + i0 * 3), B = ld3(S.pos + i1 * 3), C = ld3(S.pos + i2 * 3);
        n = normalize(cross(B - A, C - A));
    }
    float uu = 0.0f, vv = 0.0f;
    if (I.flags & kInstHasUVs) {
        float ax = S.uv[i0 * 2], ay = S.uv[i0 * 2 + 1], bx = S.uv[i1 * 2], by = S.uv[i1 * 2 + 1];
        float cx = S.uv[i2 * 2], cy = S.uv[i2 * 2 + 1];
        uu = bA * ax + bu * bx + bv * cx;
        vv = bA * ay + bu * by + bv * cy;
    }
    r.t = t;
    r.normal = normalize(xform(I.MinvT, n, 0.0f));
    r.inst = inst;
    r.prim = prim;
    r.material = I.material;
    r.u = uu;
    r.v = vv;
    return r;
}

// The closest-hit program's world tangent (optix_triangle.cu:194-223): the object-space
// tangent from the uv deltas, transformed by the instance, then made orthogonal to the world
// normal n (the hit's is.normal).
LUX_DI f3 hit_tangent(const DevScene& S, int inst, int prim, f3 n) {
    const DevInstance& I = S.insts[inst];
    uint32_t i0, i1, i2;
    mesh_tri(S, I, prim, i0, i1, i2);
    f3 tg = mk(1.0f, 0.0f, 0.0f);
    if (I.flags & kInstHasUVs) {
        f3 A = ld3(S.pos + i0 * 3), B = ld3(S.pos + i1 * 3), C = ld3(S.pos + i2 * 3);
        f3 e1 = B - A, e2 = C - A;
        float ax = S.uv[i0 * 2], ay = S.uv[i0 * 2 + 1], bx = S.uv[i1 * 2], by = S.uv[i1 * 2 + 1];
        float cx = S.uv[i2 * 2], cy = S.uv[i2 * 2 + 1];
        float d1x = bx - ax, d1y = by - ay, d2x = cx - ax, d2y = cy - ay;
        float det = d1x * d2y - d2x * d1y;
        float f = (fabsf(det) < 1e-10f) ? 0.0f : 1.0f / det;
        if (f != 0.0f) {
            tg.x = f * (d2y * e1.x - d1y * e2.x);
            tg.y = f * (d2y * e1.y - d1y * e2.y);
            tg.z = f * (d2y * e1.z - d1y * e2.z);
        }
    }
    tg = normalize(xform(I.M, tg, 0.0f));
    f3 T = tg - dot(tg, n) * n;
    float l2 = dot(T, T);
    if (l2 > 1e-10f) {
        tg = T * (1.0f / sqrtf(l2));
    } else {
        tg = (fabsf(n.x) > 0.9f) ? mk(0.0f, 1.0f, 0.0f) : mk(1.0f, 0.0f, 0.0f);
        tg = normalize(cross(tg, n));
    }
    return tg;
}

// direct-light closest-hit program (src/optixshaders/optix_triangle.cu:259-305)
LUX_DI Isect ch_direct_light(const DevScene& S, float t, int inst, int prim, float bu, float bv) {
    Isect r;
    const DevInstance& I = S.insts[inst];
    uint32_t i0, i1, i2;
    mesh_tri(S, I, prim, i0, i1, i2);
    float bA = 1.0f - bu - bv;
    f3 n;
    if (I.flags & kInstHasNormals) {
        n = normalize(bA * ld3(S.nrm + i0 * 3) + bu * ld3(S.nrm + i1 * 3) + bv * ld3(S.nrm + i2 * 3));
    } else {
        f3 A = ld3(S.pos + i0 * 3), B = ld3(S.pos + i1 * 3), C = ld3(S.pos + i2 * 3);
        n = normalize(cross(B - A, C - A));
    }
    float uu = 0.0f, vv = 0.0f;
    if (I.flags & kInstHasUVs) {
        uu = bA * S.uv[i0 * 2] + bu * S.uv[i1 * 2] + bv * S.uv[i2 * 2];
        vv = bA * S.uv[i0 * 2 + 1] + bu * S.uv[i1 * 2 + 1] + bv * S.uv[i2 * 2 + 1];
    }
    r.t = t;
    r.normal = normalize(xform(I.MinvT, n, 0.0f));
    r.inst = inst;
    r.prim = prim;
    r.material = I.material;
    r.u = uu;
    r.v = vv;
    return r;
}

// ---- material queries (src/material_queries.cu:19-117)
LUX_DI f3 get_albedo(const DevMaterial& m, float u, float v) {
    if (m.flags & kMatAlbedoTex) {
        tt_apply(m.albedo_tt, u, v);
        float4 t = tex(m.albedo_tex, u, v);
        return vpow(mk(t.x, t.y, t.z), 2.2f);
    }
    return mk(m.color[0], m.color[1], m.color[2]);
}
LUX_DI f3 get_normal(const DevScene& S, const DevMaterial& m, const Isect& is) {
    if (m.flags & kMatNormalTex) {
        float u = is.u, v = is.v;
        tt_apply(m.normal_tt, u, v);
        float4 t = tex(m.normal_tex, u, v);
        f3 ln = mk(t.x * 2.0f - 1.0f, t.y * 2.0f - 1.0f, t.z * 2.0f - 1.0f);
        const f3 N = is.normal;
        if (!(dot(ln, ln) > 1e-12f)) return N;
        const f3 tangent = hit_tangent(S, is.inst, is.prim, N);
        f3 T = tangent - dot(tangent, N) * N;
        float t2 = dot(T, T);
        if (!(t2 > 1e-12f)) return N;
        T = T * (1.0f / sqrtf(t2));
        f3 Bt = cross(N, T);
        f3 mp = mk(T.x * ln.x + Bt.x * ln.y + N.x * ln.z, T.y * ln.x + Bt.y * ln.y + N.y * ln.z,
                   T.z * ln.x + Bt.z * ln.y + N.z * ln.z);
        float m2 = dot(mp, mp);
        if (!(m2 > 1e-12f)) return N;
        mp = mp * (1.0f / sqrtf(m2));
        if (!(dot(mp, N) > 1e-4f)) return N;
        return mp;
    }
    return is.normal;
}
LUX_DI void get_mr(const DevMaterial& m, float u, float v, float& rough, float& metal) {
    rough = m.roughness;
    metal = m.metallic;
    if (m.flags & kMatMRTex) {
        tt_apply(m.mr_tt, u, v);
        float4 t = tex(m.mr_tex, u, v);
        rough *= t.y;
        metal *= t.z;
    }
}
LUX_DI f3 get_emission(const DevMaterial& m, float u, float v) {
    f3 e = mk(m.emission[0], m.emission[1], m.emission[2]);
    if (m.flags & kMatEmissiveTex) {
        tt_apply(m.emissive_tt, u, v);
        float4 t = tex(m.emissive_tex, u, v);
        e = e * vpow(mk(t.x, t.y, t.z), 2.2f);
    }
    return e;
}

// The normal-map texel get_normal reads (src/material_queries.cu:32-40), or (0.5, 0.5, 1)
// without a normal texture.
LUX_DI f3 normal_map_texel(const DevMaterial& m, float u, float v) {
    if (!(m.flags & kMatNormalTex)) return mk(0.5f, 0.5f, 1.0f);
    tt_apply(m.normal_tt, u, v);
    float4 t = tex(m.normal_tex, u, v);
    return mk(t.x, t.y, t.z);
}
// get_alpha (src/material_queries.cu:119-137)
LUX_DI float get_alpha(const DevMaterial& m, float u, float v) {
    if (m.alpha_mode == 0) return 1.0f;
    float alpha = m.alpha;
    if (m.flags & kMatAlbedoTex) {
        tt_apply(m.albedo_tt, u, v);
        alpha *= tex(m.albedo_tex, u, v).w;
    }
    if (m.alpha_mode == 1) return alpha >= m.alpha_cutoff ? 1.0f : 0.0f;
    return alpha;
}
// render_material_debug_mode (src/material_debug_render.cu:3-26)
LUX_DI f3 material_debug_color(int mode, f3 mc, f3 normal, f3 nmap, float rough, float metal, float alpha) {
    switch (mode) {
        case 1: return mc;
        case 2: return normal * 0.5f + mk(0.5f, 0.5f, 0.5f);
        case 3: return nmap;
        case 4: return mk(rough, rough, rough);
        case 5: return mk(metal, metal, metal);
        case 6: return mk(alpha, alpha, alpha);
    }
    return mk(0.0f, 0.0f, 0.0f);
}

// ---- Cook-Torrance (src/shaders/cook_torrance.cu:8-331)
LUX_DI float D_GGX(f3 h, f3 n, float alpha) {
    float ndh = dot(n, h);
    if (ndh <= 0.0f) return 0.0f;
    float a2 = alpha * alpha;
    float ndh2 = ndh * ndh;
    float dc = (ndh2 * a2) + (1.0f - ndh2);
    float den = dc * dc * kPI;
    return a2 / gmax(den, kEPS_CT);
}
LUX_DI f3 F_schlick(float vdh, f3 f0) {
    float m = 1.0f - vdh;
    float m2 = m * m;
    return f0 + ((mk(1.0f, 1.0f, 1.0f) - f0) * (m2 * m2 * m));
}
LUX_DI float F_dielectric(float ci, float etaI, float etaT) {
    ci = gclamp(ci, 0.0f, 1.0f);
    float si = sqrtf(gmax(0.0f, 1.0f - ci * ci));
    float st = (etaI / etaT) * si;
    if (st >= 1.0f) return 1.0f;
    float ct = sqrtf(gmax(0.0f, 1.0f - st * st));
    float rpa = ((etaT * ci) - (etaI * ct)) / ((etaT * ci) + (etaI * ct));
    float rpe = ((etaI * ci) - (etaT * ct)) / ((etaI * ci) + (etaT * ct));
    return (rpa * rpa + rpe * rpe) / 2.0f;
}
LUX_DI f3 half_t(f3 wo, f3 wi, float etaI, float etaT) { return normalize(-(etaI * wo + etaT * wi)); }
LUX_DI float smith(f3 w, f3 n, float alpha) {
    float a2 = alpha * alpha;
    float nw = gmax(dot(n, w), 0.0f);
    float num = 2.0f * nw;
    float us = a2 + (1.0f - a2) * (nw * nw);
    float den = nw + sqrtf(us);
    return num / gmax(den, kEPS_CT);
}
LUX_DI f3 fresnel(float c, f3 albedo, float metal, float etaI, float etaT) {
    float d = F_dielectric(c, etaI, etaT);
    return vmix(mk(d, d, d), F_schlick(c, albedo), metal);
}
LUX_DI f3 BRDF(f3 v, f3 n, f3 l, f3 albedo, float rough, float metal, float ior, float trans) {
    ior = gmax(ior, 1.0001f);
    bool enter = dot(v, n) > 0.0f;
    f3 nf = enter ? n : -n;
    float etaI = enter ? 1.0f : ior, etaT = enter ? ior : 1.0f;
    f3 h = normalize(v + l);
    rough = gclamp(rough, 0.0001f, 1.0f);
    float alpha = rough * rough;
    float D = D_GGX(h, nf, alpha);
    f3 F = fresnel(gmax(dot(v, h), 0.0f), albedo, metal, etaI, etaT);
    float G = smith(v, nf, alpha) * smith(l, nf, alpha);
    f3 num = D * F * G;
    float den = 4.0f * gmax(dot(nf, v), 0.0f) * gmax(dot(nf, l), 0.0f);
    f3 spec = num / gmax(den, kEPS_CT);
    f3 kD = (1.0f - metal) * (mk(1.0f, 1.0f, 1.0f) - F) * (1.0f - trans);
    f3 diffuse = kD * albedo * kINV_PI;
    return diffuse + spec;
}
LUX_DI f3 BTDF(f3 wo, f3 n, f3 wi, f3 albedo, float rough, float metal, float ior, float trans) {
    bool enter = dot(wo, n) > 0.0f;
    float etaI = enter ? 1.0f : ior, etaT = enter ? ior : 1.0f;
    f3 ht = half_t(wo, wi, etaI, etaT);
    float jd = (etaT * dot(wi, ht) + etaI * dot(wo, ht));
    float jac = (etaI * etaI) / gmax(jd * jd, kEPS_CT);
    float cnum = fabsf(dot(wi, ht)) * fabsf(dot(wo, ht));
    float cden = fabsf(dot(wi, n)) * fabsf(dot(wo, n));
    rough = gclamp(rough, 0.0001f, 1.0f);
    float alpha = rough * rough;
    float D = D_GGX(ht, n, alpha);
    float F = F_dielectric(fabsf(dot(wo, ht)), etaI, etaT);
    bool gv = dot(wi, ht) * dot(wi, n) > 0.0f && dot(wo, ht) * dot(wo, n) > 0.0f;
    float G = gv ? smith(dot(wi, n) > 0.0f ? wi : -wi, n, alpha) * smith(dot(wo, n) > 0.0f ? wo : -wo, n, alpha) : 0.0f;
    float DFG = D * G * (1.0f - F);
    return albedo * (trans * (1.0f - metal) * (cnum / cden) * jac * DFG);
}
// calculateRandomDirectionInHemisphere (src/interactions.cu:7-45)
LUX_DI f3 hemisphere(f3 n, Rng& rng) {
    float up = sqrtf(rng.u01());
    float over = sqrtf(1.0f - up * up);
    float around = rng.u01() * kTWO_PI;
    f3 dnn;
    if (fabsf(n.x) < kSQRT13) dnn = mk(1.0f, 0.0f, 0.0f);
    else if (fabsf(n.y) < kSQRT13) dnn = mk(0.0f, 1.0f, 0.0f);
    else dnn = mk(0.0f, 0.0f, 1.0f);
    f3 p1 = normalize(cross(n, dnn));
    f3 p2 = normalize(cross(n, p1));
    return up * n + cosf(around) * over * p1 + sinf(around) * over * p2;
}
LUX_DI void lobe_probs(f3 wo, f3 n, float metal, f3 color, float ior, float trans, float& pR, float& pD, float& pS) {
    bool enter = dot(wo, n) > 0.0f;
    float etaI = enter ? 1.0f : ior, etaT = enter ? ior : 1.0f;
    float cm = fabsf(dot(wo, n));
    f3 Fa = fresnel(cm, color, metal, etaI, etaT);
    float sr = gclamp((Fa.x + Fa.y + Fa.z) / 3.0f, 0.01f, 0.99f);
    float Fm = F_dielectric(cm, etaI, etaT);
    pR = trans * (1.0f - metal) * (1.0f - Fm);
    pD = (1.0f - pR) * (1.0f - sr) * (1.0f - metal);
    pS = 1.0f - pR - pD;
}
// The lobe probabilities depend on the outgoing direction and the material only, so one
// evaluation serves the direction sampling and every pdf of a shading point (the reference
// evaluates them in each call, with the same operands).
struct Lobes {
    float pR, pD, pS;
};
LUX_DI Lobes lobes_of(f3 wo, f3 n, float metal, f3 color, float ior, float trans) {
    Lobes L;
    lobe_probs(wo, n, metal, color, gmax(ior, 1.0001f), trans, L.pR, L.pD, L.pS);
    return L;
}
// sampleCookTorrance (src/shaders/cook_torrance.cu:156-224); L = lobes_of(wo, n, metal, color, ior, trans)
LUX_DI f3 sample_ct(f3 wo, f3 n, float rough, Rng& rng, float ior, const Lobes& L) {
    float r = rng.u01();
    ior = gmax(ior, 1.0001f);
    rough = gclamp(rough, 0.0001f, 1.0f);
    float alpha = rough * rough;
    bool enter = dot(wo, n) > 0.0f;
    f3 nf = enter ? n : -n;
    float etaI = enter ? 1.0f : ior, etaT = enter ? ior : 1.0f;
    const float pD = L.pD, pS = L.pS;
    if (r > pS && r <= pS + pD) return hemisphere(nf, rng);
    float x1 = rng.u01(), x2 = rng.u01();
    float th = atanf((alpha * sqrtf(x1)) / sqrtf(1.0f - x1));
    float ph = 2.0f * kPI * x2;
    f3 h = normalize(mk(1.0f * sinf(th) * cosf(ph), 1.0f * sinf(th) * sinf(ph), 1.0f * cosf(th)));
    f3 t = normalize(fabsf(nf.z) < 0.999f ? cross(mk(0.0f, 0.0f, 1.0f), nf) : cross(mk(1.0f, 0.0f, 0.0f), nf));
    f3 b = cross(nf, t);
    f3 hw = h.x * t + h.y * b + h.z * nf;
    if (r <= pS) {
        f3 wi = reflect(-wo, hw);
        if (dot(wi, nf) <= 0.0f) return mk(0.0f, 0.0f, 0.0f);
        return normalize(wi);
    }
    f3 wi = refract(-wo, hw, etaI / etaT);
    if (dot(wi, wi) < kEPS_CT || isnan(wi.x) || isnan(wi.y) || isnan(wi.z) || dot(wi, nf) >= 0.0f)
        return mk(0.0f, 0.0f, 0.0f);
    return normalize(wi);
}
LUX_DI float pdf_ggx(f3 wo, f3 wi, f3 n, float rough) {
    f3 h = normalize(wo + wi);
    rough = gclamp(rough, 0.0001f, 1.0f);
    float alpha = rough * rough;
    float ph = D_GGX(h, n, alpha) * dot(n, h);
    return ph / gmax((4.0f * fabsf(dot(wo, h))), kEPS_CT);
}
LUX_DI float pdf_ggx_t(f3 wo, f3 wi, f3 n, float rough, float ior) {
    bool enter = dot(wo, n) > 0.0f;
    float etaI = enter ? 1.0f : ior, etaT = enter ? ior : 1.0f;
    f3 ht = half_t(wo, wi, etaI, etaT);
    rough = gclamp(rough, 0.0001f, 1.0f);
    float alpha = rough * rough;
    float den = etaT * dot(wi, ht) + etaI * dot(wo, ht);
    float ph = D_GGX(ht, n, alpha) * fabsf(dot(n, ht));
    return ph * (etaT * etaT * fabsf(dot(wi, ht))) / gmax(den * den, kEPS_CT);
}
// L = lobes_of(wo, n, metal, color, ior, trans)
LUX_DI float PDF(f3 wo, f3 wi, f3 n, float rough, float ior, const Lobes& L) {
    ior = gmax(ior, 1.0001f);
    f3 nf = dot(wo, n) < 0.0f ? -n : n;
    float pdfD = fmaxf(0.0f, dot(wi, nf)) * kINV_PI;
    float pdfS = pdf_ggx(wo, wi, nf, rough);
    float pdfR = pdf_ggx_t(wo, wi, n, rough, ior);
    bool refr = (dot(wi, n) * dot(wo, n)) < 0.0f;
    float pdf = refr ? L.pR * pdfR : L.pD * pdfD + L.pS * pdfS;
    return gmax(pdf, kPDF_CLAMP);
}
LUX_DI f3 shade_ct(f3 wo, f3 albedo, f3 n, f3 wi, float rough, float metal, float ior, float trans) {
    ior = gmax(ior, 1.0001f);
    bool refr = (dot(wi, n) * dot(wo, n)) < 0.0f;
    f3 f = refr ? BTDF(wo, n, wi, albedo, rough, metal, ior, trans) : BRDF(wo, n, wi, albedo, rough, metal, ior, trans);
    return f * fabsf(dot(wi, n));
}

// ---- environment (src/kernels/shade_path.cu:27-42, :207-215)
LUX_DI float envmap_pdf(const DevScene& S, f3 d) {
    const int W = S.env_w, H = S.env_h;
    float phi = atan2f(d.z, d.x);
    float theta = acosf(gclamp(d.y, -1.0f, 1.0f));
    float u = (phi + kPI) / (2.0f * kPI);
    float v = theta / kPI;
    int col = gclampi(int(u * float(W)), 0, W - 1);
    int row = gclampi(int(v * float(H)), 0, H - 1);
    float pm = (__ldg(S.marginal + row) - (row == 0 ? 0.0f : __ldg(S.marginal + row - 1))) * float(H);
    const float* cr = S.conditional + size_t(row) * W;
    float pc = (__ldg(cr + col) - (col == 0 ? 0.0f : __ldg(cr + col - 1))) * float(W);
    float st = sinf(theta);
    return (st > 1e-6f) ? (pm * pc) / (2.0f * kPI * kPI * st) : 0.0f;
}
LUX_DI f3 env_lookup(const DevScene& S, f3 d, float intensity) {
    float phi = atan2f(d.z, d.x);
    float theta = acosf(gclamp(d.y, -1.0f, 1.0f));
    float u = float((double(phi) + kM_PI_SHADE) * (double(1.0f) / (double(2.0f) * kM_PI_SHADE)));
    float v = float(double(theta) * (double(1.0f) / kM_PI_SHADE));
    float4 e = tex(S.env_tex, u, v);
    return mk(e.x, e.y, e.z) * intensity;
}

// NEE mode of a kernel instantiation: -1 = read from the options at run time, 0 = none,
// 1 = emitter sampling only (-dmis), 2 = environment sampling (-emis, with or without -dmis;
// the reference's shading then takes the environment branch, src/kernels/shade_path.cu:166-249).
template <int NEE> LUX_DI bool nee_env(const DevOptions& O) { return NEE < 0 ? O.env != 0 : NEE == 2; }
template <int NEE> LUX_DI bool nee_dl(const DevOptions& O) {
    return NEE < 0 ? O.dl != 0 : (NEE == 1 || (NEE == 2 && O.dl != 0));
}
inline int nee_mode_of(const DevOptions& O) { return O.env ? 2 : (O.dl ? 1 : 0); }

// sampleDirectLight for one path (src/kernels/sample_direct_light.cu:31-100). With both -dmis
// and -emis the reference draws the emitter point and then keeps only the environment
// direction (the shading reads one of the two); want_dl = false skips the emitter point's CDF
// searches and vertex loads and only advances the random stream past its three draws.
template <int NEE = -1>
LUX_DI f3 light_sample(const DevScene& S, const DevOptions& O, int iter, int pixel, int depth, f3& env_dir,
                       bool want_dl = true) {
    Rng rng = Rng::seeded(iter, pixel, depth);
    f3 dl = mk(0.0f, 0.0f, 0.0f);
    env_dir = mk(0.0f, 0.0f, 0.0f);
    const bool dl_on = nee_dl<NEE>(O);
    if (dl_on && !want_dl) {
        rng.skip3();
    } else if (dl_on) {
        float rnd = rng.u01();
        int sel = select_from_cdf(S.emissive_prefix, S.num_emissive, rnd);
        int ii = __ldg(S.emissive_inst + sel);
        const DevInstance& I = S.insts[ii];
        float lower = (sel == 0) ? 0.0f : __ldg(S.emissive_prefix + sel - 1);
        float upper = __ldg(S.emissive_prefix + sel);
        float den = upper - lower;
        float off = (den > 1e-10f) ? (rnd - lower) / den : 0.0f;
        off = gclamp(off, 0.0f, 1.0f);
        int ts = select_from_cdf(S.tri_prefix + __ldg(S.tri_prefix_off + sel), I.num_tris, off);
        uint32_t i0, i1, i2;
        mesh_tri(S, I, ts, i0, i1, i2);
        f3 v0 = ld3(S.pos + i0 * 3), v1 = ld3(S.pos + i1 * 3), v2 = ld3(S.pos + i2 * 3);
        float r1 = sqrtf(rng.u01());
        float r2 = rng.u01();
        float u = 1.0f - r1, v = r2 * r1;
        f3 lp = u * v0 + v * v1 + (1.0f - u - v) * v2;
        dl = xform(I.M, lp, 1.0f);
    }
    if (nee_env<NEE>(O)) {
        float rnd = rng.u01();
        const int H = S.env_h, W = S.env_w;
        int mg = select_from_cdf_guided(S.marginal, S.marginal_guide, S.guide_marg, rnd);
        float lower = (mg == 0) ? 0.0f : __ldg(S.marginal + mg - 1);
        float upper = __ldg(S.marginal + mg);
        float den = upper - lower;
        float off = (den > 1e-10f) ? (rnd - lower) / den : 0.0f;
        off = gclamp(off, 0.0f, 1.0f);
        int cn = select_from_cdf_guided(S.conditional + size_t(mg) * W,
                                        S.conditional_guide + size_t(mg) * (S.guide_cond + 1), S.guide_cond, off);
        float u = (float(cn) + 0.5f) / float(W);
        float v = (float(mg) + 0.5f) / float(H);
        float phi = float(double(u) * 2.0 * double(kPI) - double(kPI));
        float theta = v * kPI;
        float st = sinf(theta);
        env_dir = mk(st * cosf(phi), cosf(theta), st * sinf(phi));
    }
    return dl;
}

// A path as shade_one sees it. d, thr, spec, pixel and iter are read on entry; the other
// fields are outputs: the new origin, radiance and pdf of a surviving path (color always).
struct PathState {
    f3 o, d, thr, color;
    float last_pdf;
    bool spec;
    int pixel, iter;
};

// The path fields shade_one reads late, loaded where they are used instead of being held in
// registers across the shading (origin, radiance so far, pdf of the last bounce, NEE sample).
struct WavePathIn {
    const DevWave& W;
    int pid;
    LUX_DI f3 origin() const { float4 a = ld_stream(&W.s0[pid]); return mk(a.x, a.y, a.z); }
    LUX_DI float last_pdf() const { return ld_stream(&W.s0[pid]).w; }
    LUX_DI f3 color0() const { float4 a = ld_stream(&W.s3[pid]); return mk(a.x, a.y, a.z); }
    LUX_DI f3 nee() const { float4 a = ld_stream(&W.s4[pid]); return mk(a.x, a.y, a.z); }
};

// shadePath for one path; returns true if the path survives (is not killed).
// sh_t: DL shadow hit t (or env occlusion); sh_* the DL shadow hit record.
// MATDBG: the instantiation that also renders the material debug views (O.material_debug).
// NEE: as for light_sample. At most one radiance term is added per call (emission, the NEE
// contribution or the environment on a miss), so p.color = color0 + that term.
// SPAWN_KILLED: also sample the next direction and spawn the ray of a path that an emitter
// hit kills, as the reference does (its result is then unused; the parity entry reports it).
// The NEE terms draw no random numbers, so sampling the direction after them leaves the
// random stream as the reference's (sample first, then Russian roulette).
template <bool MATDBG, int NEE, bool SPAWN_KILLED, class In>
LUX_DI bool shade_one(const DevScene& S, const DevOptions& O, int depth, PathState& p, const In& in, float t, int inst,
                      int prim, float bu, float bv, float sh_t, int sh_inst, int sh_prim, float sh_u, float sh_v) {
    Rng rng = Rng::seeded(p.iter, p.pixel, depth);
    f3 add = mk(0.0f, 0.0f, 0.0f);
    bool added = false;
    const bool has_exr = S.has_env != 0;
    bool kill = false;
    if (inst >= 0 && t > 0.0f) {
        Isect is = ch_radiance(S, t, inst, prim, bu, bv);
        const DevMaterial& m = S.mats[is.material];
        f3 mc = get_albedo(m, is.u, is.v);
        f3 normal = get_normal(S, m, is);
        float rough, metal;
        get_mr(m, is.u, is.v, rough, metal);
        if (MATDBG && O.material_debug) {
            // the debug view replaces the colour and ends the path (shade_path.cu:154-164)
            p.color = material_debug_color(O.material_debug, mc, normal, normal_map_texel(m, is.u, is.v), rough, metal,
                                           get_alpha(m, is.u, is.v));
            return false;
        }
        f3 emission = get_emission(m, is.u, is.v);
        bool is_spec = rough < kSPEC_ROUGH;
        f3 nf = dot(-p.d, normal) < 0.0f ? -normal : normal;
        const float ior = m.ior, trans = m.transmission;
        bool emissive = length(emission) > kEPS_UTIL;
        const Lobes L = lobes_of(-p.d, normal, metal, mc, ior, trans);
        if (nee_env<NEE>(O)) {
            if (emissive) {
                float w = 1.0f;
                if (depth > 1 && !p.spec) {
                    float pb = in.last_pdf();
                    float pe = envmap_pdf(S, p.d);
                    w = (pb * pb) / (pb * pb + pe * pe);
                }
                add = p.thr * (w * emission);
                added = true;
                kill = true;
            } else if (sh_t < 0.0f && !is_spec && has_exr) {
                f3 ed = in.nee();
                float pee = envmap_pdf(S, ed);
                float pbe = PDF(-p.d, ed, normal, rough, ior, L);
                float w = (pee * pee) / (pee * pee + pbe * pbe);
                f3 brdf = BRDF(-p.d, normal, ed, mc, rough, metal, ior, trans);
                f3 el = env_lookup(S, normalize(ed), O.env_intensity);
                float cs = dot(nf, ed);
                if (cs > 0.0f && pee > 1e-8f) {
                    f3 contrib = (el * brdf * cs) / pee;
                    add = p.thr * contrib * w;
                    added = true;
                }
            }
        } else if (nee_dl<NEE>(O)) {
            if (emissive) {
                float w = 1.0f;
                if (depth > 1 && !p.spec) {
                    float pb = in.last_pdf();
                    float dsq = is.t * is.t;
                    float cl = dot(is.normal, -p.d);
                    if (cl > 0.0001f) {
                        float pa = 1.0f / S.total_area;
                        float ps = pa * (dsq / cl);
                        w = (pb * pb) / (pb * pb + ps * ps);
                    } else {
                        w = 0.0f;
                    }
                }
                add = p.thr * (w * emission);
                added = true;
                kill = true;
            } else if (sh_inst >= 0 && sh_t > 0.0f && !is_spec) {
                Isect dli = ch_direct_light(S, sh_t, sh_inst, sh_prim, sh_u, sh_v);
                f3 sp = is.t * p.d + in.origin();
                f3 lv = in.nee() - sp;
                float dsq = dot(lv, lv);
                float dist = sqrtf(dsq);
                f3 ld = lv / dist;
                float cs = dot(nf, ld);
                float cl = dot(dli.normal, -ld);
                if (cs > 0.0f && cl > 0.0f) {
                    float pa = 1.0f / S.total_area;
                    float ps = pa * (dsq / cl);
                    float pb = PDF(-p.d, ld, normal, rough, ior, L);
                    float w = (ps * ps) / (ps * ps + pb * pb);
                    f3 brdf = BRDF(-p.d, normal, ld, mc, rough, metal, ior, trans);
                    const DevMaterial& lm = S.mats[dli.material];
                    f3 lr = get_emission(lm, dli.u, dli.v);
                    f3 contrib = (lr * brdf * cs) / ps;
                    add = p.thr * contrib * w;
                    added = true;
                }
            }
        } else if (emissive) {
            add = p.thr * emission;
            added = true;
            kill = true;
        }
        if (kill && !SPAWN_KILLED) {
            p.color = in.color0() + add;
            return false;
        }
        f3 sd = sample_ct(-p.d, normal, rough, rng, ior, L);
        if (!kill) {
            bool transmitted = dot(-p.d, normal) * dot(sd, normal) < 0.0f;
            bool spec = is_spec || transmitted;
            f3 f = shade_ct(-p.d, mc, normal, sd, rough, metal, ior, trans);
            float pdf = PDF(-p.d, sd, normal, rough, ior, L);
            p.thr = p.thr * (f / pdf);
            p.last_pdf = pdf;
            p.spec = spec;
            if (depth >= kRR_MIN_DEPTH) {
                float mx = gmax(p.thr.x, gmax(p.thr.y, p.thr.z));
                float surv = gclamp(mx, 0.0f, 1.0f);
                if (rng.u01() >= surv) kill = true;
                else p.thr = p.thr / surv;
            }
        }
        p.color = added ? in.color0() + add : in.color0();
        // ray spawn (shade_path.cu:333-353), run for paths killed above as well
        f3 hp = in.origin() + (is.t - .0001f) * normalize(p.d);
        float sl2 = dot(sd, sd);
        if (!(sl2 > 1e-12f) || !isfinite(sl2)) return false;
        p.d = sd;
        if (dot(p.d, is.normal) > 0.0f) p.o = hp + (is.normal * kGLASS_EPS);
        else p.o = hp - (is.normal * kGLASS_EPS);
        return !kill;
    }
    if (has_exr) {
        f3 d = normalize(p.d);
        f3 er = env_lookup(S, d, O.env_intensity);
        float w = 1.0f;
        if (nee_env<NEE>(O) && depth > 1 && !p.spec) {
            float pb = in.last_pdf();
            float pe = envmap_pdf(S, d);
            w = (pb * pb) / (pb * pb + pe * pe);
        }
        add = p.thr * er * w;
        added = true;
    }
    p.color = added ? in.color0() + add : in.color0();
    return false;
}

// The fields shade_one reads on entry.
LUX_DI PathState load_path(const DevWave& W, int pid) {
    float4 b = ld_stream(&W.s1[pid]), c = ld_stream(&W.s2[pid]);
    PathState p;
    p.d = mk(b.x, b.y, b.z);
    p.spec = (__float_as_int(b.w) & 1) != 0;
    p.thr = mk(c.x, c.y, c.z);
    p.pixel = __float_as_int(c.w);
    p.iter = __float_as_int(ld_stream(&W.s3[pid]).w);
    return p;
}

// Pixel of the t-th path of a sample: 8x4 pixel tiles in row-major tile order, so that a warp's
// 32 camera rays (and, through the order-preserving survivor queue, their later bounces) start
// from one compact patch of the image rather than a 32x1 strip. Pixels outside the whole tiles
// (a right margin of W % 8 columns and a bottom margin of H % 4 rows) follow in row order.
LUX_HDI int tiled_pixel(int t, int W, int H) {
    const int W8 = W - W % 8, H4 = H - H % 4;
    const int a = W8 * H4;
    if (t < a) {
        const int tile = t >> 5, k = t & 31, tpr = W8 >> 3;
        return ((tile / tpr) * 4 + (k >> 3)) * W + (tile % tpr) * 8 + (k & 7);
    }
    t -= a;
    const int rw = W - W8;
    if (t < rw * H4) return (t / rw) * W + W8 + t % rw;
    t -= rw * H4;
    return (H4 + t / W) * W + t % W;
}

// Paths [0, n) of a wave in lane `lane`: path ids and queue slots from lane * lane_stride on.
__global__ void __launch_bounds__(kShadeBlock, 16) k_camera(DevScene S, DevWave W, DevOptions O, DevCamera C, int n,
                                                            int lane, const int* wave_iter) {
    const int first_iter = wave_iter[0];
    const bool nee = O.dl || O.env;
    const int base = lane * W.lane_stride;
    for (int local = blockIdx.x * blockDim.x + threadIdx.x; local < n; local += gridDim.x * blockDim.x) {
        const int pid = base + local;
        int s = local / W.npix, index = tiled_pixel(local - s * W.npix, C.width, C.height);
        int iter = first_iter + s;
        int x = index % C.width, y = index / C.width;
        Rng rng = Rng::seeded(iter, index, O.trace_depth);
        float x1 = rng.u01() - 0.5f;
        float x2 = rng.u01() - 0.5f;
        float pX = (float(x) + x1 + 0.5f) - float(C.width) * 0.5f;
        float pY = (float(y) + x2 + 0.5f) - float(C.height) * 0.5f;
        f3 view = ld3(C.view), right = ld3(C.right), up = ld3(C.up);
        f3 d = normalize(view - (right * C.pixel_length[0] * pX) - (up * C.pixel_length[1] * pY));
        st_stream(&W.s0[pid], make_float4(C.pos[0], C.pos[1], C.pos[2], -1.0f));
        st_stream(&W.s1[pid], make_float4(d.x, d.y, d.z, __int_as_float(0)));
        st_stream(&W.s2[pid], make_float4(1.0f, 1.0f, 1.0f, __int_as_float(index)));
        st_stream(&W.s3[pid], make_float4(0.0f, 0.0f, 0.0f, __int_as_float(iter)));
        if (nee) {
            f3 ed;
            f3 dl = light_sample(S, O, iter, index, 0, ed, !O.env);
            f3 v = O.env ? ed : dl;
            st_stream(&W.s4[pid], make_float4(v.x, v.y, v.z, 0.0f));
        }
        st_stream(&W.queue[0][pid], pid);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) (W.ctr + lane)->count[0] = n;
}

// JOBS: the shared wavefront of the job engine; each path shades against its job's scene
// (lights, environment) and stops compacting at its job's trace depth.
// Full occupancy (16 blocks of 128 threads per SM, 32 registers): the kernel waits mostly on
// texture fetches and gathers, and hiding that latency with more warps pays more than the
// register spills cost (shade per 16-spp step of the 1M-triangle 1080p workload: 28.3 ms at
// 5 blocks per SM, 22.6 at 8, 20.4 at 12, 18.8 at 16).
// G: the (lane, bounce) segments of waves in flight this launch shades; the paths of segment k
// are its lane's queue at its bounce, and its survivors go to the lane's next queue.
template <bool JOBS, bool MATDBG, int NEE>
__global__ void __launch_bounds__(kShadeBlock, 16) k_shade(const __grid_constant__ DevScene S0, DevWave W, DevOptions O,
                                                       const __grid_constant__ Segs G) {
    __shared__ int seg_first[kMaxSegs + 1];
    if (threadIdx.x == 0) {
        int t = 0;
        seg_first[0] = 0;
        for (int k = 0; k < kMaxSegs; ++k) {
            if (k < G.n) t += *(volatile const int*)&(W.ctr + G.lane[k])->count[G.bounce[k]];
            seg_first[k + 1] = t;
        }
    }
    __syncthreads();
    const int n = seg_first[kMaxSegs];
    const bool nee = nee_dl<NEE>(O) || nee_env<NEE>(O);
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    // uniform trip count across the warp so the append below runs converged
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int item = base + threadIdx.x;
        bool alive = false;
        int pid = 0, k = 0;
        if (item < n) {
            while (k + 1 < G.n && item >= seg_first[k + 1]) ++k;
            const int slot = G.lane[k] * W.lane_stride + (item - seg_first[k]);
            const int depth = G.bounce[k] + 1;
            pid = ld_stream(&W.queue[G.bounce[k] & 1][slot]);
            int job_compact = G.compact[k];
            const DevScene* sp = &S0;
            if (JOBS) {
                const DevJob& J = W.jobs[W.path_job[pid]];
                sp = &W.scenes[J.scene];
                job_compact = depth < J.trace_depth;
            }
            const DevScene& S = *sp;
            PathState p = load_path(W, pid);
            float4 h = ld_stream(&W.hit[slot]);
            int inst = __float_as_int(h.w);
            int prim = ld_stream(&W.hit_prim[slot]);
            float sh_t = -1.0f, su = 0.0f, sv = 0.0f;
            int si = -1, spr = -1;
            if (nee && inst >= 0) {
                float4 sh = ld_stream(&W.sh_hit[slot]);
                sh_t = sh.x;
                if (!nee_env<NEE>(O)) {
                    su = sh.y;
                    sv = sh.z;
                    si = __float_as_int(sh.w);
                    spr = ld_stream(&W.sh_prim[slot]);
                }
            }
            alive = shade_one<MATDBG, NEE, false>(S, O, depth, p, WavePathIn{W, pid}, h.x, inst, prim, h.y, h.z, sh_t, si, spr,
                                           su, sv) &&
                    job_compact;
            st_stream(&W.s3[pid], make_float4(p.color.x, p.color.y, p.color.z, __int_as_float(p.iter)));
            if (alive) {
                st_stream(&W.s0[pid], make_float4(p.o.x, p.o.y, p.o.z, p.last_pdf));
                st_stream(&W.s1[pid], make_float4(p.d.x, p.d.y, p.d.z, __int_as_float(p.spec ? 1 : 0)));
                st_stream(&W.s2[pid], make_float4(p.thr.x, p.thr.y, p.thr.z, __int_as_float(p.pixel)));
                if (nee) {
                    f3 ed;
                    f3 dl = light_sample<NEE>(S, O, p.iter, p.pixel, depth, ed, !nee_env<NEE>(O));
                    f3 v = nee_env<NEE>(O) ? ed : dl;
                    st_stream(&W.s4[pid], make_float4(v.x, v.y, v.z, 0.0f));
                }
            }
        }
        // warp-aggregated survivor append (src/kernels/shade_path.cu:355-363), one atomic per
        // segment present in the warp
        const unsigned am = __ballot_sync(0xffffffffu, alive);
        if (am) {
            const unsigned grp = __match_any_sync(0xffffffffu, alive ? k : -1);
            if (alive) {
                const int lk = G.lane[k], nb = G.bounce[k] + 1;
                const int leader = __ffs(grp) - 1;
                int b = 0;
                if (lane == leader) b = atomicAdd(&(W.ctr + lk)->count[nb], __popc(grp));
                b = __shfl_sync(grp, b, leader);
                st_stream(&W.queue[nb & 1][lk * W.lane_stride + b + __popc(grp & ((1u << lane) - 1u))], pid);
            }
        }
    }
}

// Path t of every sample of the wave is pixel tiled_pixel(t) (k_camera).
__global__ void k_accumulate(const float4* __restrict__ s3, float* __restrict__ image, float* __restrict__ comp,
                             int width, int height, int nsamples, int compensated) {
    const int npix = width * height;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npix; t += gridDim.x * blockDim.x) {
        const int p = tiled_pixel(t, width, height);
        float r = image[p * 3], g = image[p * 3 + 1], b = image[p * 3 + 2];
        if (compensated) {
            // Kahan-compensated running sum (precision form)
            float cr = comp[p * 3], cg = comp[p * 3 + 1], cb = comp[p * 3 + 2];
            for (int s = 0; s < nsamples; ++s) {
                float4 c = ld_stream(&s3[size_t(s) * npix + t]);
                float yr = c.x - cr, tr = r + yr;
                cr = (tr - r) - yr;
                r = tr;
                float yg = c.y - cg, tg = g + yg;
                cg = (tg - g) - yg;
                g = tg;
                float yb = c.z - cb, tb = b + yb;
                cb = (tb - b) - yb;
                b = tb;
            }
            comp[p * 3] = cr;
            comp[p * 3 + 1] = cg;
            comp[p * 3 + 2] = cb;
        } else {
            for (int s = 0; s < nsamples; ++s) {
                float4 c = ld_stream(&s3[size_t(s) * npix + t]);
                r += c.x;
                g += c.y;
                b += c.z;
            }
        }
        image[p * 3] = r;
        image[p * 3 + 1] = g;
        image[p * 3 + 2] = b;
    }
}

// Segment of the wave holding index v of a prefix array (path0 or pix0), by binary search
// over the segment table staged in shared memory.
template <int FIELD>
LUX_DI int find_segment(const DevSegment* segs, int nsegs, int v) {
    int lo = 0, hi = nsegs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        int start = FIELD == 0 ? segs[mid].path0 : segs[mid].pix0;
        if (start <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Camera rays of a job-engine wave (generateRayFromCamera, src/kernels/generate_ray_from_camera.cu:8-39,
// per job): path pid belongs to the segment covering it; its sample s and pixel index give the
// job-local iteration and pixel that seed the RNG, exactly as a single-job render would.
// W.segs and W.wave_hdr are the wave's own tables; its paths go to lane `lane`.
__global__ void __launch_bounds__(kShadeBlock) k_camera_jobs(DevWave W, DevOptions O, int lane) {
    __shared__ DevSegment segs[kMaxSegments];
    const int nsegs = W.wave_hdr[0], n = min(W.wave_hdr[1], W.lane_stride);
    for (int k = threadIdx.x; k < nsegs; k += blockDim.x) segs[k] = W.segs[k];
    __syncthreads();
    const bool nee = O.dl || O.env;
    const int base = lane * W.lane_stride;
    for (int local = blockIdx.x * blockDim.x + threadIdx.x; local < n; local += gridDim.x * blockDim.x) {
        const int pid = base + local;
        const DevSegment& g = segs[find_segment<0>(segs, nsegs, local)];
        const DevJob& J = W.jobs[g.job];
        int off = local - g.path0;
        int s = off / J.npix, index = off - s * J.npix;
        int iter = J.first_iter + g.sample0 + s;
        int x = index % J.width, y = index / J.width;
        Rng rng = Rng::seeded(iter, index, J.trace_depth);
        float x1 = rng.u01() - 0.5f;
        float x2 = rng.u01() - 0.5f;
        float pX = (float(x) + x1 + 0.5f) - float(J.width) * 0.5f;
        float pY = (float(y) + x2 + 0.5f) - float(J.height) * 0.5f;
        f3 view = ld3(J.view), right = ld3(J.right), up = ld3(J.up);
        f3 d = normalize(view - (right * J.pixel_length[0] * pX) - (up * J.pixel_length[1] * pY));
        W.s0[pid] = make_float4(J.pos[0], J.pos[1], J.pos[2], -1.0f);
        W.s1[pid] = make_float4(d.x, d.y, d.z, __int_as_float(0));
        W.s2[pid] = make_float4(1.0f, 1.0f, 1.0f, __int_as_float(index));
        W.s3[pid] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(iter));
        if (nee) {
            f3 ed;
            f3 dl = light_sample(W.scenes[J.scene], O, iter, index, 0, ed, !O.env);
            f3 v = O.env ? ed : dl;
            W.s4[pid] = make_float4(v.x, v.y, v.z, 0.0f);
        }
        W.path_job[pid] = g.job;
        W.queue[0][pid] = pid;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) (W.ctr + lane)->count[0] = n;
}

// image[job pixel] (+comp) += radiance of the segment's samples, in sample order, so that a
// job's image is the same bit for bit however its samples were split into waves.
__global__ void k_accumulate_jobs(DevWave W, int compensated, int lane) {
    __shared__ DevSegment segs[kMaxSegments];
    const int nsegs = W.wave_hdr[0], total = W.wave_hdr[2];
    const float4* __restrict__ s3 = W.s3 + size_t(lane) * W.lane_stride;
    for (int k = threadIdx.x; k < nsegs; k += blockDim.x) segs[k] = W.segs[k];
    __syncthreads();
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const DevSegment& g = segs[find_segment<1>(segs, nsegs, q)];
        const DevJob& J = W.jobs[g.job];
        const int p = q - g.pix0;
        const size_t o = size_t(p) * 3;
        float* __restrict__ image = J.image;
        float* __restrict__ comp = J.comp;
        float r = image[o], gr = image[o + 1], b = image[o + 2];
        if (compensated) {
            float cr = comp[o], cg = comp[o + 1], cb = comp[o + 2];
            for (int s = 0; s < g.nsamples; ++s) {
                float4 c = ld_stream(&s3[size_t(g.path0) + size_t(s) * J.npix + p]);
                float yr = c.x - cr, tr = r + yr;
                cr = (tr - r) - yr;
                r = tr;
                float yg = c.y - cg, tg = gr + yg;
                cg = (tg - gr) - yg;
                gr = tg;
                float yb = c.z - cb, tb = b + yb;
                cb = (tb - b) - yb;
                b = tb;
            }
            comp[o] = cr;
            comp[o + 1] = cg;
            comp[o + 2] = cb;
        } else {
            for (int s = 0; s < g.nsamples; ++s) {
                float4 c = ld_stream(&s3[size_t(g.path0) + size_t(s) * J.npix + p]);
                r += c.x;
                gr += c.y;
                b += c.z;
            }
        }
        image[o] = r;
        image[o + 1] = gr;
        image[o + 2] = b;
    }
}

LUX_DI f3 aces(f3 x) {  // src/tonemapping.cu:3-11
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    f3 num = x * (a * x + mk(b, b, b));
    f3 den = x * (c * x + mk(d, d, d)) + mk(e, e, e);
    return mk(gclamp(num.x / den.x, 0.0f, 1.0f), gclamp(num.y / den.y, 0.0f, 1.0f), gclamp(num.z / den.z, 0.0f, 1.0f));
}
LUX_DI f3 agx(f3 v) {  // src/tonemapping.cu:13-30
    float c[3] = {v.x, v.y, v.z};
    for (int i = 0; i < 3; ++i) {
        c[i] = gmax(c[i], 1e-6f);
        c[i] = (log2f(c[i]) + 10.0f) / 16.0f;
        c[i] = gclamp(c[i], 0.0f, 1.0f);
        float x2 = c[i] * c[i], x4 = x2 * x2;
        c[i] = 15.5f * x4 * c[i] - 40.14f * x4 + 31.96f * x2 * c[i] - 6.86f * x2 + 0.429f * c[i] + 0.0322f;
    }
    float r = c[0] * 1.1968790f - c[1] * 0.0980208f - c[2] * 0.0990297f;
    float g = -c[0] * 0.0528968f + c[1] * 1.1519031f - c[2] * 0.0989611f;
    float b = -c[0] * 0.0529716f - c[1] * 0.0980434f + c[2] * 1.1510736f;
    return mk(gclamp(r, 0.0f, 1.0f), gclamp(g, 0.0f, 1.0f), gclamp(b, 0.0f, 1.0f));
}

__global__ void k_tonemap(const float* __restrict__ image, uchar4* __restrict__ out, int npix, float iter, int mode) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        float inv = __frcp_rn(iter);
        f3 p = mk(image[i * 3], image[i * 3 + 1], image[i * 3 + 2]) * inv;
        if (mode >= 0) {  // mode < 0: material debug view, shown without tone map or gamma
            if (mode == 0) p = mk(p.x / (p.x + 1.0f), p.y / (p.y + 1.0f), p.z / (p.z + 1.0f));
            else if (mode == 1) p = agx(p);
            else p = aces(p);
            p = vpow(p, 0.45f);
        }
        out[i] = make_uchar4((unsigned char)gclampi(int(double(p.x) * 255.0), 0, 255),
                             (unsigned char)gclampi(int(double(p.y) * 255.0), 0, 255),
                             (unsigned char)gclampi(int(double(p.z) * 255.0), 0, 255), 0);
    }
}

// ---- kernel-level parity entry points ------------------------------------------------
// Path rows of 24 floats: origin 0-2, direction 3-5, radiance 6-8, throughput 9-11, DL point
// 12-14, env direction 15-17, pixel 18, killed 19, specular 20, pdf 21.
struct RowPathIn {
    const float* f;
    bool env;
    LUX_DI f3 origin() const { return mk(f[0], f[1], f[2]); }
    LUX_DI float last_pdf() const { return f[21]; }
    LUX_DI f3 color0() const { return mk(f[6], f[7], f[8]); }
    LUX_DI f3 nee() const { return env ? mk(f[15], f[16], f[17]) : mk(f[12], f[13], f[14]); }
};

__global__ void k_shade_ext(DevScene S, DevOptions O, float* paths, const uint32_t* hits, int n, int iter, int depth,
                            int compact, int* survivors, int* n_out) {
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        int i = base + threadIdx.x;
        bool alive = false;
        if (i < n) {
            float* f = paths + size_t(i) * 24;
            PathState p;
            p.o = mk(f[0], f[1], f[2]);
            p.d = mk(f[3], f[4], f[5]);
            p.thr = mk(f[9], f[10], f[11]);
            p.pixel = __float_as_int(f[18]);
            p.spec = f[20] != 0.0f;
            p.last_pdf = f[21];
            p.iter = iter;
            const uint32_t* h = hits + size_t(i) * 10;
            float t = __uint_as_float(h[0]);
            int inst = int(h[1]), prim = int(h[2]);
            float su = __uint_as_float(h[8]), sv = __uint_as_float(h[9]);
            int si = int(h[6]), spr = int(h[7]);
            if (O.env) si = -1;
            bool survived = shade_one<true, -1, true>(S, O, depth, p, RowPathIn{f, O.env != 0}, t, inst, prim,
                                                __uint_as_float(h[3]), __uint_as_float(h[4]), __uint_as_float(h[5]), si,
                                                spr, su, sv);
            alive = survived && compact;
            f[0] = p.o.x; f[1] = p.o.y; f[2] = p.o.z;
            f[3] = p.d.x; f[4] = p.d.y; f[5] = p.d.z;
            f[6] = p.color.x; f[7] = p.color.y; f[8] = p.color.z;
            f[9] = p.thr.x; f[10] = p.thr.y; f[11] = p.thr.z;
            f[19] = survived ? 0.0f : 1.0f;
            f[20] = p.spec ? 1.0f : 0.0f;
            f[21] = p.last_pdf;
        }
        unsigned am = __ballot_sync(0xffffffffu, alive);
        if (am) {
            int b = 0, leader = __ffs(am) - 1;
            if (lane == leader) b = atomicAdd(n_out, __popc(am));
            b = __shfl_sync(0xffffffffu, b, leader);
            if (alive) survivors[b + __popc(am & ((1u << lane) - 1u))] = i;
        }
    }
}

__global__ void k_light_ext(DevScene S, DevOptions O, int iter, int depth, const int* pixels, int n, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        f3 ed;
        f3 dl = light_sample(S, O, iter, pixels[i], depth, ed);
        float* o = out + size_t(i) * 6;
        o[0] = dl.x; o[1] = dl.y; o[2] = dl.z;
        o[3] = ed.x; o[4] = ed.y; o[5] = ed.z;
    }
}

__global__ void k_rng_ext(int iter, int index, int depth, int n, float* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Rng r = Rng::seeded(iter, index, depth);
        for (int i = 0; i < n; ++i) out[i] = r.u01();
    }
}

__global__ void k_tex_ext(unsigned long long t, const float* uv, int n, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 v = tex(t, uv[i * 2], uv[i * 2 + 1]);
        out[i * 4] = v.x; out[i * 4 + 1] = v.y; out[i * 4 + 2] = v.z; out[i * 4 + 3] = v.w;
    }
}

}  // namespace

// Grid of the shading kernels: SMs x resident blocks per SM, cached per device ordinal under a
// lock, as trace_grid_blocks is.
int shade_grid_blocks() {
    static std::mutex mu;
    static std::map<int, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    int& cached = cache[dev];
    if (cached == 0) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int per_jobs = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_shade<false, false, 2>, kShadeBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_jobs, k_shade<true, false, 2>, kShadeBlock, 0);
        per = std::min(per, per_jobs);
        cached = sms * (per > 0 ? per : 1);
    }
    return cached;
}

cudaError_t launch_camera(const DevScene& S, const DevWave& W, const DevOptions& O, const DevCamera& C, int n,
                          int lane, const int* wave_iter, cudaStream_t st) {
    if (n > W.lane_stride || lane < 0) return cudaErrorInvalidValue;
    int grid = std::min((n + kShadeBlock - 1) / kShadeBlock, shade_grid_blocks() * 2);
    if (grid < 1) grid = 1;
    k_camera<<<grid, kShadeBlock, 0, st>>>(S, W, O, C, n, lane, wave_iter);
    return cudaGetLastError();
}

cudaError_t launch_shade(const DevScene& S, const DevWave& W, const DevOptions& O, int bounce, int compact,
                         cudaStream_t st) {
    return launch_shade_segs(S, W, O, one_seg(bounce, compact), st);
}

cudaError_t launch_shade_segs(const DevScene& S, const DevWave& W, const DevOptions& O, const Segs& G,
                              cudaStream_t st) {
    if (G.n < 1 || G.n > kMaxSegs) return cudaErrorInvalidValue;
    const int g = shade_grid_blocks(), mode = nee_mode_of(O);
    if (O.material_debug && !W.path_job) {
        k_shade<false, true, -1><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
    } else if (W.path_job) {
        if (mode == 2) k_shade<true, false, 2><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
        else if (mode == 1) k_shade<true, false, 1><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
        else k_shade<true, false, 0><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
    } else {
        if (mode == 2) k_shade<false, false, 2><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
        else if (mode == 1) k_shade<false, false, 1><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
        else k_shade<false, false, 0><<<g, kShadeBlock, 0, st>>>(S, W, O, G);
    }
    return cudaGetLastError();
}

cudaError_t launch_camera_jobs(const DevWave& W, const DevOptions& O, int max_paths, int lane, cudaStream_t st) {
    if (lane < 0) return cudaErrorInvalidValue;
    int grid = std::min((max_paths + kShadeBlock - 1) / kShadeBlock, shade_grid_blocks() * 2);
    if (grid < 1) grid = 1;
    k_camera_jobs<<<grid, kShadeBlock, 0, st>>>(W, O, lane);
    return cudaGetLastError();
}

cudaError_t launch_accumulate_jobs(const DevWave& W, int compensated, int lane, cudaStream_t st) {
    if (lane < 0) return cudaErrorInvalidValue;
    k_accumulate_jobs<<<148 * 8, 256, 0, st>>>(W, compensated, lane);
    return cudaGetLastError();
}

cudaError_t launch_accumulate(const DevWave& W, int lane, float* image, float* comp, int nsamples, int compensated,
                              cudaStream_t st) {
    if (lane < 0 || size_t(nsamples) * size_t(W.npix) > size_t(W.lane_stride)) return cudaErrorInvalidValue;
    int grid = std::min((W.npix + 255) / 256, 148 * 8);
    if (grid < 1) grid = 1;
    if (W.width * W.height != W.npix) return cudaErrorInvalidValue;
    k_accumulate<<<grid, 256, 0, st>>>(W.s3 + size_t(lane) * W.lane_stride, image, comp, W.width, W.height, nsamples,
                                       compensated);
    return cudaGetLastError();
}

cudaError_t launch_tonemap(const float* image, uint8_t* rgba, int npix, float iter, int color_mode, cudaStream_t st) {
    int grid = std::min((npix + 255) / 256, 148 * 8);
    if (grid < 1) grid = 1;
    k_tonemap<<<grid, 256, 0, st>>>(image, reinterpret_cast<uchar4*>(rgba), npix, iter, color_mode);
    return cudaGetLastError();
}

cudaError_t launch_shade_ext(const DevScene& S, const DevOptions& O, float* paths, const uint32_t* hits, int n,
                             int iter, int depth, int compact, int* survivors, int* n_out, cudaStream_t st) {
    int grid = std::max(1, std::min((n + kShadeBlock - 1) / kShadeBlock, 1024));
    k_shade_ext<<<grid, kShadeBlock, 0, st>>>(S, O, paths, hits, n, iter, depth, compact, survivors, n_out);
    return cudaGetLastError();
}

cudaError_t launch_light_ext(const DevScene& S, const DevOptions& O, int iter, int depth, const int* pixels, int n,
                             float* out, cudaStream_t st) {
    int grid = std::max(1, std::min((n + 127) / 128, 1024));
    k_light_ext<<<grid, 128, 0, st>>>(S, O, iter, depth, pixels, n, out);
    return cudaGetLastError();
}

cudaError_t launch_rng_ext(int iter, int index, int depth, int n, float* out, cudaStream_t st) {
    k_rng_ext<<<1, 32, 0, st>>>(iter, index, depth, n, out);
    return cudaGetLastError();
}

cudaError_t launch_tex_ext(unsigned long long t, const float* uv, int n, float* out, cudaStream_t st) {
    int grid = std::max(1, std::min((n + 127) / 128, 1024));
    k_tex_ext<<<grid, 128, 0, st>>>(t, uv, n, out);
    return cudaGetLastError();
}

}  // namespace lux
