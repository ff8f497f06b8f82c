// ref_driver.cpp -- host harness around the reference's own render-path sources.
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile together with the reference files it
// names, compiled unmodified from the reference tree, into oracle/_ref/libluxref.so. The
// library pins the oracle restatement (golden vectors under tests/golden/) and serves as the
// "reference" CPU baseline of the benchmark.
//
// What runs is the reference's code: generateRayFromCamera, sampleDirectLight and shadePath
// (called once per path with a one-thread launch shape), the Cook-Torrance shader, material
// queries, hemisphere sampling, select_from_cdf, Scene::precompute_emissive_mesh_area /
// precompute_hdri_emission, fill_bvh, BoundingBox::RayBoxInterection, meshIntersectionTest
// and rayMortonCode. What the reference only has as OptiX device programs is restated here:
// the closest-hit traversal of its software BVH with the primitive recorded (structure of
// src/intersections/mesh_isect.cu:48-139, ties toward the lowest primitive), the closest-hit
// attribute programs (src/optixshaders/optix_triangle.cu:156-305), the raygen shadow rays
// (:82-136) and the alpha any-hit (:317-366, hash keyed on the pixel). The texture fetch
// stands in for the CUDA hardware filter.

#include "sceneStructs.h"
#include "common.h"
#include "scene.h"
#include "texture.h"
#include "pathtrace/dev_options.h"
#include "kernels/shade_path.h"
#include "kernels/sample_direct_light.h"
#include "kernels/generate_ray_from_camera.h"
#include "shaders/cook_torrance.h"
#include "interactions.h"
#include "mesh/bvh_build.h"
#include "mesh/bounding_box.h"
#include "morton_codes.h"
#include "intersections/mesh_isect.h"

#include "../../include/luxion.h"

#include <cstring>
#include <cfloat>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;

// The reference's Scene constructor lives in scene.cpp (the glTF loader), which is not part
// of the host build; the harness fills a Scene's members directly.
Scene::Scene(std::string, const char*) {}

namespace {

struct HostTex {
    int w = 0, h = 0;
    std::vector<float> t;
};
std::vector<HostTex>* g_texs = nullptr;  // handle k -> (*g_texs)[k-1]

float half_to_float(uint16_t h) {
    uint32_t sign = uint32_t(h >> 15) << 31, exp = (h >> 10) & 0x1f, man = h & 0x3ff, bits;
    if (exp == 0) {
        if (man == 0) bits = sign;
        else {
            int e = -1;
            do { ++e; man <<= 1; } while ((man & 0x400) == 0);
            bits = sign | uint32_t(127 - 15 - e) << 23 | (man & 0x3ff) << 13;
        }
    } else if (exp == 31) bits = sign | 0x7f800000u | (man << 13);
    else bits = sign | (exp + 112) << 23 | (man << 13);
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

void load(HostTex& t, int w, int h, int fmt, const void* data) {
    t.w = w;
    t.h = h;
    size_t n = size_t(w) * h * 4;
    t.t.resize(n);
    for (size_t i = 0; i < n; ++i) {
        if (fmt == LUX_TEX_RGBA8) t.t[i] = float(static_cast<const uint8_t*>(data)[i]) / 255.0f;
        else if (fmt == LUX_TEX_RGBA16) t.t[i] = float(static_cast<const uint16_t*>(data)[i]) / 65535.0f;
        else if (fmt == LUX_TEX_RGBA16F) t.t[i] = half_to_float(static_cast<const uint16_t*>(data)[i]);
        else t.t[i] = static_cast<const float*>(data)[i];
    }
}

// The CUDA hardware linear filter on float4 texels, as measured on B200 (the same rule the
// oracle restates): the normalized coordinate wraps into a 21-bit fixed-point fraction by
// truncation, the texel position u * n - 0.5 is formed exactly from it, 8-bit 1-D weights
// round half up and the 2-D weights sum to 256.
void axis(float u, int n, int& i0, int& a) {
    double s = std::floor(double(u) * 2097152.0);
    s -= std::floor(s / 2097152.0) * 2097152.0;
    int64_t X = int64_t(s) * n - (int64_t(1) << 20);
    int64_t fi = X >> 21;
    a = int(((X - (fi << 21)) + (1 << 12)) >> 13);
    i0 = int(fi);
}

float4 fetch(const HostTex& t, float u, float v) {
    int fi, fj, a, b;
    axis(u, t.w, fi, a);
    axis(v, t.h, fj, b);
    int w00 = ((256 - a) * (256 - b) + 128) >> 8, w11 = (a * b + 128) >> 8;
    int w10 = (256 - b) - w00, w01 = b - w11;
    auto wrap = [](int i, int n) { int r = i % n; return r < 0 ? r + n : r; };
    int i0 = wrap(fi, t.w), i1 = wrap(fi + 1, t.w), j0 = wrap(fj, t.h), j1 = wrap(fj + 1, t.h);
    const float* t00 = &t.t[(size_t(j0) * t.w + i0) * 4];
    const float* t10 = &t.t[(size_t(j0) * t.w + i1) * 4];
    const float* t01 = &t.t[(size_t(j1) * t.w + i0) * 4];
    const float* t11 = &t.t[(size_t(j1) * t.w + i1) * 4];
    float r[4];
    for (int c = 0; c < 4; ++c)
        r[c] = ((float(w00) * t00[c] + float(w10) * t10[c]) + (float(w01) * t01[c] + float(w11) * t11[c])) * (1.0f / 256.0f);
    return make_float4(r[0], r[1], r[2], r[3]);
}

}  // namespace

template <> float4 tex2D<float4>(cudaTextureObject_t tex, float u, float v) {
    return fetch((*g_texs)[size_t(tex) - 1], u, v);
}

struct ref_scene {
    Scene* sc = nullptr;
    std::vector<HostTex> texs;           // scene textures then (last) the env map
    std::vector<TextureData> texdata;
    cudaTextureObject_t env_tex = 0;
    std::vector<std::vector<BVHNode>> bvh;
    std::vector<std::vector<glm::vec3>> normals;
    std::vector<std::vector<glm::vec2>> uvs;
    std::vector<int> uses_normals, uses_uvs;
    int trace_depth = 8;
    lux_camera_desc cam{};
};

namespace {

inline uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

struct RHit {
    float t = -1.0f;
    int geom = -1, prim = -1;
    float u = 0, v = 0;
};

bool alpha_accept(const ref_scene& R, int gi, int prim, float bu, float bv, glm::vec3 wdir, int pixel, int iter) {
    const Geom& g = R.sc->geoms[gi];
    const Material& m = R.sc->materials[g.materialid];
    if (m.alpha_mode == ALPHA_MODE_OPAQUE) return true;
    float alpha = m.alpha;
    if (m.albedo_tex >= 0) {
        glm::vec2 uv(0.0f);
        if (g.mesh.has_uvs) {
            const Triangle& tri = g.mesh.h_triangles[prim];
            float bA = 1.0f - bu - bv;
            glm::vec2 A = g.mesh.h_uvs[tri.uv_indices[0]], B = g.mesh.h_uvs[tri.uv_indices[1]], C = g.mesh.h_uvs[tri.uv_indices[2]];
            uv = glm::vec2(bA * A.x + bu * B.x + bv * C.x, bA * A.y + bu * B.y + bv * C.y);
        }
        uv = uv * m.albedo_tex_transform.scale;
        if (m.albedo_tex_transform.rotation != 0.0f) {
            float c = cosf(m.albedo_tex_transform.rotation), s = sinf(m.albedo_tex_transform.rotation);
            uv = glm::vec2(c * uv.x - s * uv.y, s * uv.x + c * uv.y);
        }
        uv = uv + m.albedo_tex_transform.offset;
        float4 tx = tex2D<float4>(R.texdata[m.albedo_tex].tex, uv.x, uv.y);
        alpha *= tx.w;
    }
    if (m.alpha_mode == ALPHA_MODE_MASK) return !(alpha < m.alpha_cutoff);
    uint32_t bx, by, bz;
    std::memcpy(&bx, &wdir.x, 4);
    std::memcpy(&by, &wdir.y, 4);
    std::memcpy(&bz, &wdir.z, 4);
    uint32_t h = hash_u32(uint32_t(pixel) ^ hash_u32(uint32_t(iter)));
    h = hash_u32(h ^ bx);
    h = hash_u32(h ^ by);
    h = hash_u32(h ^ bz);
    h = hash_u32(h ^ uint32_t(gi));
    h = hash_u32(h ^ uint32_t(prim));
    float rnd = (h >> 8) * (1.0f / 16777216.0f);
    return !(rnd >= alpha);
}

// Closest (or any, mode 2) accepted hit over every geom, each traversed in object space
// through its fill_bvh tree as meshIntersectionTest does.
bool trace(const ref_scene& R, glm::vec3 o, glm::vec3 d, float tmax, int mode, int pixel, int iter, RHit& best) {
    best = RHit();
    const float eps = 1.1920929E-7F;
    for (int gi = 0; gi < int(R.sc->geoms.size()); ++gi) {
        const Geom& g = R.sc->geoms[gi];
        Ray r;
        r.origin = glm::vec3(g.inverseTransform * glm::vec4(o, 1.0f));
        r.direction = glm::vec3(g.inverseTransform * glm::vec4(d, 0.0f));
        r.inv_direction.x = __frcp_rn(r.direction.x);
        r.inv_direction.y = __frcp_rn(r.direction.y);
        r.inv_direction.z = __frcp_rn(r.direction.z);
        r.sign.x = (r.inv_direction.x < 0.0f) ? 1 : 0;
        r.sign.y = (r.inv_direction.y < 0.0f) ? 1 : 0;
        r.sign.z = (r.inv_direction.z < 0.0f) ? 1 : 0;
        const std::vector<BVHNode>& bvh = R.bvh[gi];
        const std::vector<glm::vec3>& verts = g.mesh.h_verts;
        const std::vector<Triangle>& tris = g.mesh.h_triangles;
        float min_t = -1.0f;
        int min_tri = -1;
        float min_u = 0, min_v = 0;
        int stack[64];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            int bi = stack[--sp];
            const BVHNode& nd = bvh[bi];
            if (!nd.isLeaf) {
                int left = nd.left_child, right = nd.left_child + 1;
                float tl = -FLT_MAX, tr = -FLT_MAX;
                bool hl = bvh[left].isLeaf || const_cast<BoundingBox&>(bvh[left].box).RayBoxInterection(r, tl);
                bool hr = bvh[right].isLeaf || const_cast<BoundingBox&>(bvh[right].box).RayBoxInterection(r, tr);
                float lim = (mode == 2) ? -1.0f : min_t;
                if (hl && tl > lim && lim >= 0.0f) hl = false;
                if (hr && tr > lim && lim >= 0.0f) hr = false;
                if (hl && hr) {
                    stack[sp++] = tl <= tr ? right : left;
                    stack[sp++] = tl <= tr ? left : right;
                } else if (hl) stack[sp++] = left;
                else if (hr) stack[sp++] = right;
            } else {
                int tri = nd.tri_index;
                glm::vec3 a = verts[tris[tri].v_indices[0]];
                glm::vec3 edge1 = verts[tris[tri].v_indices[1]] - a;
                glm::vec3 edge2 = verts[tris[tri].v_indices[2]] - a;
                glm::vec3 cr = glm::cross(r.direction, edge2);
                float det = glm::dot(edge1, cr);
                if (det > -eps && det < eps) continue;
                float inv_det = __frcp_rn(det);
                a = r.origin - a;
                float u = inv_det * glm::dot(a, cr);
                if (u < -eps || u > 1.0f + eps) continue;
                cr = glm::cross(a, edge1);
                float v = inv_det * glm::dot(r.direction, cr);
                if ((v < 0 && glm::abs(v) > eps) || (u + v > 1 && glm::abs(u + v - 1) > eps)) continue;
                float t = inv_det * glm::dot(edge2, cr);
                if (!(t > eps)) continue;
                if (!(t <= tmax)) continue;
                bool take = mode == 2 || min_t < 0 || t < min_t || (t == min_t && tri < min_tri);
                if (!take) continue;
                // a candidate that cannot win across geoms does not run the any-hit either
                if (mode != 2 && best.geom >= 0 && !(t < best.t)) continue;
                if (!alpha_accept(R, gi, tri, u, v, d, pixel, iter)) continue;
                min_t = t;
                min_tri = tri;
                min_u = u;
                min_v = v;
                if (mode == 2) {
                    best.t = t;
                    best.geom = gi;
                    best.prim = tri;
                    return true;
                }
            }
        }
        if (min_t > 0.0f && (best.geom < 0 || best.t > min_t)) {
            best.t = min_t;
            best.geom = gi;
            best.prim = min_tri;
            best.u = min_u;
            best.v = min_v;
        }
    }
    return best.geom >= 0;
}

ShadeableIntersection ch_radiance(const ref_scene& R, const RHit& h) {
    ShadeableIntersection s{};
    const Geom& g = R.sc->geoms[h.geom];
    const Triangle& tri = g.mesh.h_triangles[h.prim];
    glm::vec3 A = g.mesh.h_verts[tri.v_indices[0]], B = g.mesh.h_verts[tri.v_indices[1]], C = g.mesh.h_verts[tri.v_indices[2]];
    glm::vec3 edge1 = B - A, edge2 = C - A;
    glm::vec3 normal = glm::normalize(glm::cross(edge1, edge2));
    float bA = 1.0f - h.u - h.v;
    if (g.mesh.has_normal_buffers) {
        glm::vec3 nA = g.mesh.h_normals[tri.n_indices[0]], nB = g.mesh.h_normals[tri.n_indices[1]], nC = g.mesh.h_normals[tri.n_indices[2]];
        normal = glm::normalize(bA * nA + h.u * nB + h.v * nC);
    }
    glm::vec3 tangent(1.0f, 0.0f, 0.0f);
    glm::vec2 uv(0.0f);
    if (g.mesh.has_uvs) {
        glm::vec2 a = g.mesh.h_uvs[tri.uv_indices[0]], b = g.mesh.h_uvs[tri.uv_indices[1]], c = g.mesh.h_uvs[tri.uv_indices[2]];
        uv = glm::vec2(bA * a.x + h.u * b.x + h.v * c.x, bA * a.y + h.u * b.y + h.v * c.y);
        glm::vec2 duv1 = b - a, duv2 = c - a;
        float det = (duv1.x * duv2.y - duv2.x * duv1.y);
        float f = (fabsf(det) < 1e-10f) ? 0.0f : 1.0f / det;
        if (f == 0.0f) tangent = glm::vec3(1.0f, 0.0f, 0.0f);
        else {
            tangent.x = f * (duv2.y * edge1.x - duv1.y * edge2.x);
            tangent.y = f * (duv2.y * edge1.y - duv1.y * edge2.y);
            tangent.z = f * (duv2.y * edge1.z - duv1.y * edge2.z);
        }
    }
    normal = glm::normalize(glm::vec3(g.invTranspose * glm::vec4(normal, 0.0f)));
    tangent = glm::normalize(glm::vec3(g.transform * glm::vec4(tangent, 0.0f)));
    glm::vec3 T = tangent - glm::dot(tangent, normal) * normal;
    float len2 = glm::dot(T, T);
    if (len2 > 1e-10f) tangent = T * (1.0f / sqrtf(len2));
    else {
        tangent = (fabsf(normal.x) > 0.9f) ? glm::vec3(0, 1, 0) : glm::vec3(1, 0, 0);
        tangent = glm::normalize(glm::cross(tangent, normal));
    }
    s.t = h.t;
    s.surfaceNormal = normal;
    s.surfaceTangent = tangent;
    s.materialId = g.materialid;
    s.uvs = uv;
    return s;
}

ShadeableIntersection ch_direct_light(const ref_scene& R, const RHit& h) {
    ShadeableIntersection s{};
    const Geom& g = R.sc->geoms[h.geom];
    const Triangle& tri = g.mesh.h_triangles[h.prim];
    float bA = 1.0f - h.u - h.v;
    glm::vec3 normal;
    if (g.mesh.has_normal_buffers) {
        normal = glm::normalize(bA * g.mesh.h_normals[tri.n_indices[0]] + h.u * g.mesh.h_normals[tri.n_indices[1]] +
                                h.v * g.mesh.h_normals[tri.n_indices[2]]);
    } else {
        glm::vec3 A = g.mesh.h_verts[tri.v_indices[0]], B = g.mesh.h_verts[tri.v_indices[1]], C = g.mesh.h_verts[tri.v_indices[2]];
        normal = glm::normalize(glm::cross(B - A, C - A));
    }
    glm::vec2 uv(0.0f);
    if (g.mesh.has_uvs) {
        glm::vec2 a = g.mesh.h_uvs[tri.uv_indices[0]], b = g.mesh.h_uvs[tri.uv_indices[1]], c = g.mesh.h_uvs[tri.uv_indices[2]];
        uv = glm::vec2(bA * a.x + h.u * b.x + h.v * c.x, bA * a.y + h.u * b.y + h.v * c.y);
    }
    s.t = h.t;
    s.surfaceNormal = glm::normalize(glm::vec3(g.invTranspose * glm::vec4(normal, 0.0f)));
    s.materialId = g.materialid;
    s.uvs = uv;
    return s;
}

void set_options(const lux_options* o) {
    DEV_OPTIONS.debug_bvh = false;
    DEV_OPTIONS.material_debug_mode = o ? o->material_debug_mode : 0;
    DEV_OPTIONS.color_mode = o ? o->color_mode : 2;
    DEV_OPTIONS.envmap_intensity = o ? o->envmap_intensity : 1.0f;
    DEV_OPTIONS.direct_light_sampling = o ? o->direct_light_sampling != 0 : false;
    DEV_OPTIONS.environment_map_importance_sampling = o ? o->env_importance_sampling != 0 : false;
}

void one_thread() {
    blockIdx = make_uint3(0, 0, 0);
    threadIdx = make_uint3(0, 0, 0);
    blockDim = dim3(1, 1, 1);
}

void do_light_sample(const ref_scene& R, int iter, int depth, PathSegment& seg) {
    one_thread();
    int zero = 0;
    Scene& S = *R.sc;
    sampleDirectLight(iter, 1, &seg, &zero, depth, int(S.emissive_geoms.size()), S.emissive_geoms.data(),
                      S.emissive_geom_area_prefix.data(), S.geoms.data(), S.total_emissive_mesh_area,
                      S.hdri_marginal_cdf.data(), S.hdri_conditional_cdfs.data(), S.exr_width, S.exr_height);
}

bool do_shade(const ref_scene& R, int iter, int depth, bool compact, PathSegment& seg, ShadeableIntersection& is,
              ShadeableIntersection& dl, ShadeableIntersection& env) {
    one_thread();
    int zero = 0, next = -1, count = 0;
    Scene& S = *R.sc;
    bool has_exr = !S.exr_data.empty();
    shadePath(iter, 1, &seg, &zero, compact ? &next : nullptr, &count, S.materials.data(), &is, &dl, &env, depth,
              has_exr, R.env_tex, const_cast<TextureData*>(R.texdata.data()), int(S.emissive_geoms.size()),
              S.emissive_geoms.data(), S.emissive_geom_area_prefix.data(), S.geoms.data(), S.total_emissive_mesh_area,
              S.hdri_marginal_cdf.data(), S.hdri_conditional_cdfs.data(), S.exr_width, S.exr_height);
    return count > 0;
}

// raygen of src/optixshaders/optix_triangle.cu:52-143 for one path
void do_trace(const ref_scene& R, int iter, const PathSegment& p, ShadeableIntersection& is,
              ShadeableIntersection& dl, ShadeableIntersection& env, double& nsh) {
    is = ShadeableIntersection{};
    dl = ShadeableIntersection{};
    env = ShadeableIntersection{};
    RHit h;
    if (!trace(R, p.ray.origin, p.ray.direction, 1e16f, 0, p.pixelIndex, iter, h)) {
        is.t = -1.0f;
        dl.t = -1.0f;
        env.t = -0.5f;
        return;
    }
    is = ch_radiance(R, h);
    glm::vec3 hp = p.ray.origin + is.t * p.ray.direction;
    glm::vec3 so = hp + (is.surfaceNormal * 1e-4f);
    bool emis = DEV_OPTIONS.environment_map_importance_sampling;
    dl.t = -1.0f;
    env.t = 1.0f;
    if (DEV_OPTIONS.direct_light_sampling && !emis) {
        glm::vec3 ld = p.direct_light_sample - so;
        float dist = sqrtf(glm::dot(ld, ld));
        ld = ld * (1.0f / dist);
        RHit s;
        if (trace(R, so, ld, dist * 1.0001f + 1e-4f, 1, p.pixelIndex, iter, s)) dl = ch_direct_light(R, s);
        nsh += 1;
    }
    if (emis) {
        RHit s;
        bool occ = trace(R, so, p.environment_map_sample, 1e16f, 2, p.pixelIndex, iter, s);
        env.t = occ ? 1.0f : -1.0f;
        nsh += 1;
    }
}

void ps_store(const PathSegment& p, float* f) {
    float v[18] = {p.ray.origin.x, p.ray.origin.y, p.ray.origin.z, p.ray.direction.x, p.ray.direction.y,
                   p.ray.direction.z, p.color.x, p.color.y, p.color.z, p.throughput.x, p.throughput.y,
                   p.throughput.z, p.direct_light_sample.x, p.direct_light_sample.y, p.direct_light_sample.z,
                   p.environment_map_sample.x, p.environment_map_sample.y, p.environment_map_sample.z};
    std::memcpy(f, v, sizeof(v));
    int32_t px = p.pixelIndex;
    std::memcpy(&f[18], &px, 4);
    f[19] = p.kill ? 1.0f : 0.0f;
    f[20] = p.last_bounce_was_specular ? 1.0f : 0.0f;
    f[21] = p.last_pdf;
    f[22] = f[23] = 0.0f;
}
void ps_load(PathSegment& p, const float* f) {
    p.ray.origin = glm::vec3(f[0], f[1], f[2]);
    p.ray.direction = glm::vec3(f[3], f[4], f[5]);
    p.color = glm::vec3(f[6], f[7], f[8]);
    p.throughput = glm::vec3(f[9], f[10], f[11]);
    p.direct_light_sample = glm::vec3(f[12], f[13], f[14]);
    p.environment_map_sample = glm::vec3(f[15], f[16], f[17]);
    int32_t px;
    std::memcpy(&px, &f[18], 4);
    p.pixelIndex = px;
    p.kill = f[19] != 0.0f;
    p.last_bounce_was_specular = f[20] != 0.0f;
    p.last_pdf = f[21];
}

RHit read_hit(const uint32_t* w) {
    RHit h;
    std::memcpy(&h.t, &w[0], 4);
    h.geom = int32_t(w[1]);
    h.prim = int32_t(w[2]);
    std::memcpy(&h.u, &w[3], 4);
    std::memcpy(&h.v, &w[4], 4);
    return h;
}

}  // namespace

extern "C" {

void ref_rng_stream(int iter, int index, int depth, int n, float* out) {
    thrust::default_random_engine rng = makeSeededRandomEngine(iter, index, depth);
    thrust::uniform_real_distribution<float> u01(0, 1);
    for (int i = 0; i < n; ++i) out[i] = u01(rng);
}

uint32_t ref_utilhash(uint32_t a) { return utilhash(a); }

int ref_select_from_cdf(const float* cdf, int size, float xi) {
    return cudaUtils::select_from_cdf(const_cast<float*>(cdf), size, xi);
}

// same record layout as orc_eval_bsdf
void ref_eval_bsdf(const float* in, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        const float* r = in + i * 16;
        glm::vec3 wo(r[0], r[1], r[2]), nn(r[3], r[4], r[5]), wi(r[6], r[7], r[8]), al(r[9], r[10], r[11]);
        float ro = r[12], me = r[13], ior = r[14], tr = r[15];
        glm::vec3 b = CookTorrance::BRDF(wo, nn, wi, al, ro, me, ior, tr);
        glm::vec3 t = CookTorrance::BTDF(wo, nn, wi, al, ro, me, glm::max(ior, 1.0001f), tr);
        PathSegment p{};
        p.ray.direction = -wo;
        glm::vec3 sh = CookTorrance::shadePathCookTorrance(p, al, nn, wi, ro, me, ior, tr);
        float pdf = CookTorrance::PDF(wo, wi, nn, ro, me, al, ior, tr);
        float rc = glm::clamp(ro, 0.0001f, 1.0f);
        glm::vec3 h = glm::normalize(wo + wi);
        float D = CookTorrance::D_TrowbridgeReitz(h, nn, rc * rc);
        float G = CookTorrance::Smith_G(wo, wi, nn, rc * rc);
        float Fd = CookTorrance::FresnelDielectric(glm::dot(nn, wo), 1.0f, glm::max(ior, 1.0001f));
        glm::vec3 Fs = CookTorrance::F_SchlickApprox(glm::max(glm::dot(wo, h), 0.0f), al);
        glm::vec3 Fm = CookTorrance::Fresnel(glm::max(glm::dot(wo, h), 0.0f), al, me, 1.0f, glm::max(ior, 1.0001f));
        float v[16] = {b.x, b.y, b.z, t.x, t.y, t.z, sh.x, sh.y, sh.z, pdf, D, G, Fd, Fs.x, Fm.x, 0.0f};
        std::memcpy(out + i * 16, v, sizeof(v));
    }
}

void ref_sample_bsdf(const float* in, const int* seeds, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        const float* r = in + i * 16;
        glm::vec3 wo(r[0], r[1], r[2]), nn(r[3], r[4], r[5]), al(r[9], r[10], r[11]);
        thrust::default_random_engine rng = makeSeededRandomEngine(seeds[i * 3], seeds[i * 3 + 1], seeds[i * 3 + 2]);
        thrust::default_random_engine ref = rng;
        PathSegment p{};
        CookTorrance::sampleCookTorrance(p, 0, 0, 0, wo, nn, r[12], r[13], rng, al, r[14], r[15]);
        int used = 0;
        while (!(ref == rng) && used < 16) { ref(); ++used; }
        out[i * 4] = p.sample_dir.x;
        out[i * 4 + 1] = p.sample_dir.y;
        out[i * 4 + 2] = p.sample_dir.z;
        out[i * 4 + 3] = float(used);
    }
}

void ref_hemisphere(const float* normals, const int* seeds, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        thrust::default_random_engine rng = makeSeededRandomEngine(seeds[i * 3], seeds[i * 3 + 1], seeds[i * 3 + 2]);
        glm::vec3 d = calculateRandomDirectionInHemisphere(glm::vec3(normals[i * 3], normals[i * 3 + 1], normals[i * 3 + 2]), rng);
        out[i * 3] = d.x;
        out[i * 3 + 1] = d.y;
        out[i * 3 + 2] = d.z;
    }
}

ref_scene* ref_scene_create(const lux_scene_desc* d) {
    ref_scene* R = new ref_scene();
    R->sc = new Scene(std::string(), nullptr);
    Scene& S = *R->sc;
    R->trace_depth = d->trace_depth;
    R->cam = d->camera;
    for (int i = 0; i < d->num_textures; ++i) {
        R->texs.emplace_back();
        load(R->texs.back(), d->textures[i].width, d->textures[i].height, d->textures[i].format, d->textures[i].data);
    }
    if (d->env_data) {
        R->texs.emplace_back();
        load(R->texs.back(), d->env_width, d->env_height, d->env_format, d->env_data);
        R->env_tex = cudaTextureObject_t(R->texs.size());
        const HostTex& e = R->texs.back();
        S.exr_width = e.w;
        S.exr_height = e.h;
        S.exr_data.resize(size_t(e.w) * e.h);
        for (size_t k = 0; k < S.exr_data.size(); ++k)
            S.exr_data[k] = glm::vec4(e.t[k * 4], e.t[k * 4 + 1], e.t[k * 4 + 2], e.t[k * 4 + 3]);
    } else {
        S.exr_width = S.exr_height = 0;
    }
    for (int i = 0; i < d->num_textures; ++i) {
        TextureData td;
        td.width = d->textures[i].width;
        td.height = d->textures[i].height;
        td.tex = cudaTextureObject_t(i + 1);
        R->texdata.push_back(td);
    }
    for (int i = 0; i < d->num_materials; ++i) {
        const lux_material_desc& md = d->materials[i];
        Material m{};
        m.material_type = MaterialType::Microfacet;
        m.color = glm::vec3(md.color[0], md.color[1], md.color[2]);
        m.albedo_tex = md.albedo_tex;
        m.alpha = md.alpha;
        m.alpha_mode = AlphaMode(md.alpha_mode);
        m.alpha_cutoff = md.alpha_cutoff;
        m.emission.emission_strength = md.emission_strength;
        m.emission.emission_color = glm::vec3(md.emission_color[0], md.emission_color[1], md.emission_color[2]);
        m.emission.emissive_tex = md.emissive_tex;
        auto tt = [](const lux_tex_transform& s, TextureTransform& o) {
            o.offset = glm::vec2(s.offset[0], s.offset[1]);
            o.scale = glm::vec2(s.scale[0], s.scale[1]);
            o.rotation = s.rotation;
        };
        tt(md.emissive_tt, m.emission.emissive_tex_transform);
        m.roughness = md.roughness;
        m.metallic = md.metallic;
        m.normal_tex = md.normal_tex;
        m.metallic_roughness_tex = md.metallic_roughness_tex;
        m.transmission = md.transmission;
        m.indexOfRefraction = md.ior;
        tt(md.albedo_tt, m.albedo_tex_transform);
        tt(md.normal_tt, m.normal_tex_transform);
        tt(md.metallic_roughness_tt, m.metallic_roughness_tex_transform);
        S.materials.push_back(m);
    }
    S.geoms.resize(d->num_instances);
    R->bvh.resize(d->num_instances);
    for (int i = 0; i < d->num_instances; ++i) {
        const lux_instance_desc& id = d->instances[i];
        const lux_mesh_desc& md = d->meshes[id.mesh];
        Geom& g = S.geoms[i];
        g.type = GeomType::MESH;
        g.materialid = id.material;
        std::memcpy(&g.transform[0][0], id.transform, 64);
        std::memcpy(&g.inverseTransform[0][0], id.inverse, 64);
        std::memcpy(&g.invTranspose[0][0], id.inv_transpose, 64);
        std::vector<glm::vec3> v(md.num_verts), n;
        std::vector<glm::vec2> uv;
        for (int k = 0; k < md.num_verts; ++k) v[k] = glm::vec3(md.positions[k * 3], md.positions[k * 3 + 1], md.positions[k * 3 + 2]);
        if (md.normals) {
            n.resize(md.num_verts);
            for (int k = 0; k < md.num_verts; ++k) n[k] = glm::vec3(md.normals[k * 3], md.normals[k * 3 + 1], md.normals[k * 3 + 2]);
        }
        if (md.uvs) {
            uv.resize(md.num_verts);
            for (int k = 0; k < md.num_verts; ++k) uv[k] = glm::vec2(md.uvs[k * 2], md.uvs[k * 2 + 1]);
        }
        std::vector<int> idx(md.indices, md.indices + size_t(md.num_tris) * 3);
        // Mesh::make_mesh_host (src/mesh/mesh_host.cu:10-70) with one shared index stream,
        // as the glTF loader passes it (src/scene/scene_load_gltf.cpp:430)
        g.mesh.make_mesh_host(v, idx, n, idx, uv, idx);
        g.mesh.d_verts = g.mesh.h_verts.data();
        g.mesh.d_triangles = g.mesh.h_triangles.data();
        g.mesh.d_normals = g.mesh.h_normals.data();
        g.mesh.d_uvs = g.mesh.h_uvs.data();
        // the reference BVH, built by its own fill_bvh (src/mesh/bvh.cu:18-38 without the upload)
        int nl = int(g.mesh.h_triangles.size());
        R->bvh[i].resize(size_t(2 * nl - 1));
        std::vector<int> ti(nl);
        for (int k = 0; k < nl; ++k) ti[k] = k;
        int alloc = 1;
        fill_bvh(0, 0, nl - 1, R->bvh[i], g.mesh.h_verts, g.mesh.h_triangles, ti, alloc);
        g.mesh.bvh.num_nodes = 2 * nl - 1;
        g.mesh.bvh.dev_bvh = R->bvh[i].data();
        g.mesh.bvh.initizalized = true;
    }
    S.precompute_emissive_mesh_area();
    for (auto& g : S.geoms) g.mesh.d_triangle_area_percentage_prefix = g.mesh.h_triangle_area_percentage_prefix.data();
    if (!S.exr_data.empty()) S.precompute_hdri_emission();
    return R;
}

void ref_scene_destroy(ref_scene* R) {
    if (!R) return;
    delete R->sc;
    delete R;
}

int ref_get_cdfs(ref_scene* R, float* ep, float* tp, float* mg, float* cd, float* ta) {
    Scene& S = *R->sc;
    if (ep) std::copy(S.emissive_geom_area_prefix.begin(), S.emissive_geom_area_prefix.end(), ep);
    if (tp) {
        size_t o = 0;
        for (int e : S.emissive_geoms) {
            auto& v = S.geoms[e].mesh.h_triangle_area_percentage_prefix;
            std::copy(v.begin(), v.end(), tp + o);
            o += v.size();
        }
    }
    if (mg) std::copy(S.hdri_marginal_cdf.begin(), S.hdri_marginal_cdf.end(), mg);
    if (cd) std::copy(S.hdri_conditional_cdfs.begin(), S.hdri_conditional_cdfs.end(), cd);
    if (ta) *ta = S.total_emissive_mesh_area;
    return 0;
}

void ref_cdf_sizes(ref_scene* R, int* sizes) {
    Scene& S = *R->sc;
    sizes[0] = int(S.emissive_geoms.size());
    size_t tl = 0;
    for (int e : S.emissive_geoms) tl += S.geoms[e].mesh.h_triangle_area_percentage_prefix.size();
    sizes[1] = int(tl);
    sizes[2] = S.exr_height;
    sizes[3] = S.exr_width;
}

void ref_trace(ref_scene* R, const float* rays, int n, int mode, int iter, uint32_t* hits) {
    g_texs = &R->texs;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const float* r = rays + size_t(i) * 8;
        int32_t px;
        std::memcpy(&px, &r[7], 4);
        RHit h;
        bool any = trace(*R, glm::vec3(r[0], r[1], r[2]), glm::vec3(r[4], r[5], r[6]), mode == 1 ? r[3] : 1e16f, mode, px, iter, h);
        uint32_t* w = hits + size_t(i) * 5;
        float t = mode == 2 ? (any ? 1.0f : -1.0f) : (any ? h.t : -1.0f);
        std::memcpy(&w[0], &t, 4);
        w[1] = uint32_t(mode == 2 ? -1 : (any ? h.geom : -1));
        w[2] = uint32_t(mode == 2 ? -1 : (any ? h.prim : -1));
        float u = any && mode != 2 ? h.u : 0.0f, v = any && mode != 2 ? h.v : 0.0f;
        std::memcpy(&w[3], &u, 4);
        std::memcpy(&w[4], &v, 4);
    }
}

// The reference's own closest t per ray: meshIntersectionTest over every geom and the
// computeIntersections reduction (src/kernels/compute_intersections.cu:32-71).
void ref_mesh_isect_t(ref_scene* R, const float* rays, int n, float* t_out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const float* r = rays + size_t(i) * 8;
        Ray ray;
        ray.origin = glm::vec3(r[0], r[1], r[2]);
        ray.direction = glm::vec3(r[4], r[5], r[6]);
        float t_min = FLT_MAX;
        int hit = -1;
        for (int g = 0; g < int(R->sc->geoms.size()); ++g) {
            glm::vec3 ip, nn;
            bool outside;
            float t = meshIntersectionTest(R->sc->geoms[g], ray, ip, nn, outside);
            if (t > 0.0f && t_min > t) {
                t_min = t;
                hit = g;
            }
        }
        t_out[i] = hit < 0 ? -1.0f : t_min;
    }
}

void ref_morton(ref_scene* R, const float* rays, int n, const float* bmin, const float* bmax, uint32_t* keys) {
    const Geom& g = R->sc->geoms[0];
    BoundingBox bbox;
    bbox.box_min = glm::vec3(bmin[0], bmin[1], bmin[2]);
    bbox.box_max = glm::vec3(bmax[0], bmax[1], bmax[2]);
    for (int i = 0; i < n; ++i) {
        const float* rr = rays + size_t(i) * 8;
        // intersectionPrecompute (src/kernels/intersection_precompute.cu:6-33)
        Ray r;
        r.origin = glm::vec3(g.inverseTransform * glm::vec4(glm::vec3(rr[0], rr[1], rr[2]), 1.0f));
        r.direction = glm::vec3(g.inverseTransform * glm::vec4(glm::vec3(rr[4], rr[5], rr[6]), 0.0f));
        r.inv_direction.x = __frcp_rn(r.direction.x);
        r.inv_direction.y = __frcp_rn(r.direction.y);
        r.inv_direction.z = __frcp_rn(r.direction.z);
        r.sign.x = (r.inv_direction.x < 0.0f) ? 1 : 0;
        r.sign.y = (r.inv_direction.y < 0.0f) ? 1 : 0;
        r.sign.z = (r.inv_direction.z < 0.0f) ? 1 : 0;
        float ext = glm::length(bbox.box_max - bbox.box_min);
        float t;
        keys[i] = bbox.RayBoxInterection(r, t) ? rayMortonCode(r, ext) : MORTON_CODE_MISS;
    }
}

void ref_light_samples(ref_scene* R, const lux_options* opt, int iter, int depth, const int* pixels, int n, float* out) {
    set_options(opt);
    g_texs = &R->texs;
    for (int i = 0; i < n; ++i) {
        PathSegment seg{};
        seg.pixelIndex = pixels[i];
        seg.kill = false;
        do_light_sample(*R, iter, depth, seg);
        float v[6] = {seg.direct_light_sample.x, seg.direct_light_sample.y, seg.direct_light_sample.z,
                      seg.environment_map_sample.x, seg.environment_map_sample.y, seg.environment_map_sample.z};
        std::memcpy(out + i * 6, v, sizeof(v));
    }
}

void ref_camera_rays(ref_scene* R, int iter, const int* pixels, int n, float* paths) {
    const lux_camera_desc* cam = &R->cam;
    Camera c{};
    c.resolution = glm::ivec2(cam->width, cam->height);
    c.position = glm::vec3(cam->position[0], cam->position[1], cam->position[2]);
    c.lookAt = glm::vec3(cam->look_at[0], cam->look_at[1], cam->look_at[2]);
    c.view = glm::vec3(cam->view[0], cam->view[1], cam->view[2]);
    c.up = glm::vec3(cam->up[0], cam->up[1], cam->up[2]);
    c.right = glm::vec3(cam->right[0], cam->right[1], cam->right[2]);
    c.fov = glm::vec2(cam->fov[0], cam->fov[1]);
    c.pixelLength = glm::vec2(cam->pixel_length[0], cam->pixel_length[1]);
    for (int i = 0; i < n; ++i) {
        int index = pixels[i];
        PathSegment seg{};
        int qi = -1;
        blockIdx = make_uint3(0, 0, 0);
        blockDim = dim3(1, 1, 1);
        threadIdx = make_uint3(uint32_t(index % cam->width), uint32_t(index / cam->width), 0);
        // the kernel writes pathSegments[index]; hand it a base that lands on seg
        PathSegment* base = reinterpret_cast<PathSegment*>(reinterpret_cast<uintptr_t>(&seg) - uintptr_t(index) * sizeof(PathSegment));
        int* qbase = reinterpret_cast<int*>(reinterpret_cast<uintptr_t>(&qi) - uintptr_t(index) * sizeof(int));
        generateRayFromCamera(c, iter, R->trace_depth, base, qbase);
        ps_store(seg, paths + size_t(i) * LUX_PS_FLOATS);
    }
}

void ref_shade_step(ref_scene* R, const lux_options* opt, int iter, int depth, int compact, float* paths, int n,
                    const uint32_t* hits, int* survivors, int* n_out) {
    set_options(opt);
    g_texs = &R->texs;
    int k = 0;
    for (int i = 0; i < n; ++i) {
        PathSegment seg{};
        ps_load(seg, paths + size_t(i) * LUX_PS_FLOATS);
        RHit rh = read_hit(hits + size_t(i) * 10), sh = read_hit(hits + size_t(i) * 10 + 5);
        ShadeableIntersection is{}, dl{}, env{};
        if (rh.geom >= 0) is = ch_radiance(*R, rh);
        else is.t = -1.0f;
        dl.t = -1.0f;
        env.t = sh.t;
        if (!opt->env_importance_sampling && sh.geom >= 0 && sh.t > 0.0f) dl = ch_direct_light(*R, sh);
        bool alive = do_shade(*R, iter, depth, compact != 0, seg, is, dl, env);
        ps_store(seg, paths + size_t(i) * LUX_PS_FLOATS);
        if (alive) survivors[k++] = i;
    }
    *n_out = k;
}

int ref_render(ref_scene* R, const lux_options* opt, int first_iter, int n_iter, int x0, int y0, int w, int h,
               int threads, float* image, double* stats) {
    set_options(opt);
    g_texs = &R->texs;
    int tdepth = opt->trace_depth > 0 ? opt->trace_depth : R->trace_depth;
    if (opt->material_debug_mode) tdepth = 1;  // src/pathtrace.cu:107
    const lux_camera_desc& cd = R->cam;
    Camera c{};
    c.resolution = glm::ivec2(cd.width, cd.height);
    c.position = glm::vec3(cd.position[0], cd.position[1], cd.position[2]);
    c.lookAt = glm::vec3(cd.look_at[0], cd.look_at[1], cd.look_at[2]);
    c.view = glm::vec3(cd.view[0], cd.view[1], cd.view[2]);
    c.up = glm::vec3(cd.up[0], cd.up[1], cd.up[2]);
    c.right = glm::vec3(cd.right[0], cd.right[1], cd.right[2]);
    c.fov = glm::vec2(cd.fov[0], cd.fov[1]);
    c.pixelLength = glm::vec2(cd.pixel_length[0], cd.pixel_length[1]);
    double st[4] = {0, 0, 0, 0};
    int nt = 1;
#ifdef _OPENMP
    nt = threads > 0 ? threads : omp_get_max_threads();
#endif
    (void)threads;
    const bool nee = DEV_OPTIONS.direct_light_sampling || DEV_OPTIONS.environment_map_importance_sampling;
#pragma omp parallel num_threads(nt)
    {
        double lst[4] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
        for (int yy = 0; yy < h; ++yy) {
            for (int xx = 0; xx < w; ++xx) {
                const int index = (y0 + yy) * cd.width + (x0 + xx);
                float acc[3] = {0, 0, 0};
                for (int it = first_iter; it < first_iter + n_iter; ++it) {
                    // generateRayFromCamera for this pixel; the kernel writes
                    // pathSegments[index], so it is handed a base that lands on seg
                    PathSegment seg{};
                    int qi = -1;
                    blockIdx = make_uint3(0, 0, 0);
                    blockDim = dim3(1, 1, 1);
                    threadIdx = make_uint3(uint32_t(index % cd.width), uint32_t(index / cd.width), 0);
                    PathSegment* base = reinterpret_cast<PathSegment*>(reinterpret_cast<uintptr_t>(&seg) -
                                                                       uintptr_t(index) * sizeof(PathSegment));
                    int* qbase = reinterpret_cast<int*>(reinterpret_cast<uintptr_t>(&qi) - uintptr_t(index) * sizeof(int));
                    generateRayFromCamera(c, it, tdepth, base, qbase);
                    // the bounce loop of pathtrace() (src/pathtrace.cu:129-343) for one path
                    int depth = 0;
                    if (nee) do_light_sample(*R, it, depth, seg);
                    while (true) {
                        ShadeableIntersection is, dl, env;
                        do_trace(*R, it, seg, is, dl, env, lst[1]);
                        lst[0] += 1;
                        ++depth;
                        lst[2] += 1;
                        bool alive = do_shade(*R, it, depth, depth < tdepth, seg, is, dl, env);
                        if (!alive || depth >= tdepth) break;
                        if (nee) do_light_sample(*R, it, depth, seg);
                    }
                    // finalGather (src/kernels/image_kernels.cu:49-60), iteration order
                    acc[0] += seg.color.x;
                    acc[1] += seg.color.y;
                    acc[2] += seg.color.z;
                    lst[3] += 1;
                }
                float* o = image + (size_t(yy) * w + xx) * 3;
                o[0] = acc[0];
                o[1] = acc[1];
                o[2] = acc[2];
            }
        }
#pragma omp critical
        for (int k = 0; k < 4; ++k) st[k] += lst[k];
    }
    if (stats)
        for (int k = 0; k < 4; ++k) stats[k] = st[k];
    return 0;
}

}  // extern "C"
