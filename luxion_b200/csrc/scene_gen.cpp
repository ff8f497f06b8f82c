// scene_gen.cpp -- seeded procedural scenes in the host scene IR (include/luxion.h).
//
// The reference renders glTF files (src/scene/scene_load_gltf.cpp:61-529); the workloads the
// B200 build is measured on are synthetic, so they are generated here, deterministically
// from a seed, straight into lux_scene_desc views:
//   * Cornell-36: 5 wall quads, a short diffuse box, a tall GGX-metal box (roughness 0.3)
//     and a ceiling area light with Le = (17, 12, 4); albedos as in scenes/cornell.glb.
//   * random instanced scene: icospheres and displaced grids with random transforms,
//     random uber-shader materials, value-noise base-colour textures and an HDRI made of a
//     log-normal sky and a Gaussian sun lobe.
//   * white furnace: a sphere under a constant environment of 1, by default smooth white
//     metal; any material can be given (a Lambert-like albedo-1 dielectric, rough GGX metal).
// Camera conventions follow the glTF loader (scene_load_gltf.cpp:465-500): view = -z of the
// camera frame, pixelLength = 2*tan(fovy/2)*(aspect, 1)/resolution.

#include "../../include/luxion.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

struct lux_host_scene {
    std::vector<std::vector<float>> pos, nrm, uv;
    std::vector<std::vector<uint32_t>> idx;
    std::vector<lux_mesh_desc> meshes;
    std::vector<lux_instance_desc> insts;
    std::vector<lux_material_desc> mats;
    std::vector<std::vector<uint8_t>> tex_bytes;
    std::vector<lux_texture_desc> texs;
    std::vector<float> env32;
    std::vector<uint16_t> env16;
    lux_scene_desc desc;
    int64_t instanced_tris = 0;

    void finalize() {
        meshes.resize(pos.size());
        for (size_t i = 0; i < pos.size(); ++i) {
            lux_mesh_desc& m = meshes[i];
            m.num_verts = int32_t(pos[i].size() / 3);
            m.num_tris = int32_t(idx[i].size() / 3);
            m.positions = pos[i].data();
            m.normals = nrm[i].empty() ? nullptr : nrm[i].data();
            m.uvs = uv[i].empty() ? nullptr : uv[i].data();
            m.indices = idx[i].data();
        }
        for (size_t i = 0; i < texs.size(); ++i) texs[i].data = tex_bytes[i].data();
        desc.num_meshes = int32_t(meshes.size());
        desc.num_instances = int32_t(insts.size());
        desc.num_materials = int32_t(mats.size());
        desc.num_textures = int32_t(texs.size());
        desc.meshes = meshes.data();
        desc.instances = insts.data();
        desc.materials = mats.data();
        desc.textures = texs.empty() ? nullptr : texs.data();
        instanced_tris = 0;
        for (auto& in : insts) instanced_tris += meshes[in.mesh].num_tris;
        if (!env32.empty()) desc.env_data = env32.data();
        else if (!env16.empty()) desc.env_data = env16.data();
        else desc.env_data = nullptr;
    }
};

namespace {

// ---- small deterministic RNG (splitmix64) ----------------------------------------------
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x1234567ull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uni(double a, double b) { return a + (b - a) * uni(); }
    double normal() {
        double u1 = std::max(uni(), 1e-300), u2 = uni();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// ---- 4x4 column-major matrices (glm layout) ----------------------------------------------
struct M4 {
    double m[16];  // m[col*4 + row]
};
M4 identity() {
    M4 r{};
    for (int i = 0; i < 4; ++i) r.m[i * 4 + i] = 1.0;
    return r;
}
M4 mul(const M4& a, const M4& b) {
    M4 r{};
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a.m[k * 4 + rr] * b.m[c * 4 + k];
            r.m[c * 4 + rr] = s;
        }
    return r;
}
M4 translate(double x, double y, double z) {
    M4 r = identity();
    r.m[12] = x;
    r.m[13] = y;
    r.m[14] = z;
    return r;
}
M4 scale(double x, double y, double z) {
    M4 r = identity();
    r.m[0] = x;
    r.m[5] = y;
    r.m[10] = z;
    return r;
}
M4 quat(double w, double x, double y, double z) {
    double n = std::sqrt(w * w + x * x + y * y + z * z);
    w /= n; x /= n; y /= n; z /= n;
    M4 r = identity();
    r.m[0] = 1 - 2 * (y * y + z * z);
    r.m[1] = 2 * (x * y + w * z);
    r.m[2] = 2 * (x * z - w * y);
    r.m[4] = 2 * (x * y - w * z);
    r.m[5] = 1 - 2 * (x * x + z * z);
    r.m[6] = 2 * (y * z + w * x);
    r.m[8] = 2 * (x * z + w * y);
    r.m[9] = 2 * (y * z - w * x);
    r.m[10] = 1 - 2 * (x * x + y * y);
    return r;
}
M4 rot_y(double deg) {
    double a = deg * 3.141592653589793 / 180.0;
    return quat(std::cos(a / 2), 0, std::sin(a / 2), 0);
}
bool invert(const M4& a, M4& out) {
    // Gauss-Jordan with partial pivoting in double
    double t[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            t[r][c] = a.m[c * 4 + r];
            t[r][c + 4] = (r == c) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(t[r][c]) > std::fabs(t[p][c])) p = r;
        if (std::fabs(t[p][c]) < 1e-300) return false;
        for (int k = 0; k < 8; ++k) std::swap(t[c][k], t[p][k]);
        double d = t[c][c];
        for (int k = 0; k < 8; ++k) t[c][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = t[r][c];
                for (int k = 0; k < 8; ++k) t[r][k] -= f * t[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out.m[c * 4 + r] = t[r][c + 4];
    return true;
}

lux_instance_desc make_instance(int mesh, int material, const M4& M) {
    lux_instance_desc d{};
    d.mesh = mesh;
    d.material = material;
    d.has_inverse = 1;
    M4 inv;
    invert(M, inv);
    for (int i = 0; i < 16; ++i) {
        d.transform[i] = float(M.m[i]);
        d.inverse[i] = float(inv.m[i]);
    }
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) d.inv_transpose[c * 4 + r] = float(inv.m[r * 4 + c]);
    return d;
}

lux_material_desc default_material() {
    lux_material_desc m{};
    m.color[0] = m.color[1] = m.color[2] = 1.0f;
    m.albedo_tex = -1;
    m.alpha = 1.0f;
    m.alpha_mode = LUX_ALPHA_OPAQUE;
    m.alpha_cutoff = 0.5f;
    m.emission_strength = 1.0f;
    m.emissive_tex = -1;
    m.roughness = 1.0f;
    m.metallic = 0.0f;
    m.normal_tex = -1;
    m.metallic_roughness_tex = -1;
    m.transmission = 0.0f;
    m.ior = 1.55f;  // reference glTF default (src/scene/scene_load_gltf.cpp:177)
    lux_tex_transform id{{0.f, 0.f}, {1.f, 1.f}, 0.f};
    m.albedo_tt = m.emissive_tt = m.normal_tt = m.metallic_roughness_tt = id;
    return m;
}

void set_camera(lux_camera_desc& c, int w, int h, const double pos[3], const double look[3], double fovy_deg) {
    c.width = w;
    c.height = h;
    double v[3] = {look[0] - pos[0], look[1] - pos[1], look[2] - pos[2]};
    double vl = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (double& x : v) x /= vl;
    double upw[3] = {0, 1, 0};
    double r[3] = {v[1] * upw[2] - v[2] * upw[1], v[2] * upw[0] - v[0] * upw[2], v[0] * upw[1] - v[1] * upw[0]};
    double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (double& x : r) x /= rl;
    double u[3] = {r[1] * v[2] - r[2] * v[1], r[2] * v[0] - r[0] * v[2], r[0] * v[1] - r[1] * v[0]};
    for (int i = 0; i < 3; ++i) {
        c.position[i] = float(pos[i]);
        c.look_at[i] = float(pos[i] + v[i]);
        c.view[i] = float(v[i]);
        c.right[i] = float(r[i]);
        c.up[i] = float(u[i]);
    }
    const float kPI = 3.1415926535897932384626422832795028841971f;
    float fovy = float(fovy_deg);
    float yscaled = std::tan(0.5f * fovy * (kPI / 180));
    float xscaled = (yscaled * float(w)) / float(h);
    float fovx = (2.0f * std::atan(xscaled) * 180) / kPI;
    c.fov[0] = fovx;
    c.fov[1] = fovy;
    c.pixel_length[0] = 2 * xscaled / float(w);
    c.pixel_length[1] = 2 * yscaled / float(h);
}

// Quad with four corners (counter-clockwise when seen from the side the normal points to).
void add_quad(lux_host_scene& s, const float q[4][3], const float n[3]) {
    std::vector<float> P, N;
    for (int i = 0; i < 4; ++i)
        for (int a = 0; a < 3; ++a) {
            P.push_back(q[i][a]);
            N.push_back(n[a]);
        }
    // orient the winding so cross(B-A, C-A) points along n
    float e1[3], e2[3];
    for (int a = 0; a < 3; ++a) { e1[a] = q[1][a] - q[0][a]; e2[a] = q[2][a] - q[0][a]; }
    float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    bool ok = c[0] * n[0] + c[1] * n[1] + c[2] * n[2] > 0;
    std::vector<uint32_t> I = ok ? std::vector<uint32_t>{0, 1, 2, 0, 2, 3} : std::vector<uint32_t>{0, 2, 1, 0, 3, 2};
    std::vector<float> UV = {0, 0, 1, 0, 1, 1, 0, 1};
    s.pos.push_back(P);
    s.nrm.push_back(N);
    s.uv.push_back(UV);
    s.idx.push_back(I);
}

void add_unit_cube(lux_host_scene& s) {
    std::vector<float> P, N, UV;
    std::vector<uint32_t> I;
    for (int axis = 0; axis < 3; ++axis)
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            float n[3] = {0, 0, 0};
            n[axis] = float(sgn);
            int u = (axis + 1) % 3, v = (axis + 2) % 3;
            float q[4][3];
            float cu[4] = {-0.5f, 0.5f, 0.5f, -0.5f}, cv[4] = {-0.5f, -0.5f, 0.5f, 0.5f};
            for (int k = 0; k < 4; ++k) {
                q[k][axis] = 0.5f * float(sgn);
                q[k][u] = cu[k];
                q[k][v] = cv[k];
            }
            uint32_t base = uint32_t(P.size() / 3);
            for (int k = 0; k < 4; ++k)
                for (int a = 0; a < 3; ++a) {
                    P.push_back(q[k][a]);
                    N.push_back(n[a]);
                }
            UV.insert(UV.end(), {0, 0, 1, 0, 1, 1, 0, 1});
            float e1[3], e2[3];
            for (int a = 0; a < 3; ++a) { e1[a] = q[1][a] - q[0][a]; e2[a] = q[2][a] - q[0][a]; }
            float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            bool ok = c[0] * n[0] + c[1] * n[1] + c[2] * n[2] > 0;
            if (ok) I.insert(I.end(), {base, base + 1, base + 2, base, base + 2, base + 3});
            else I.insert(I.end(), {base, base + 2, base + 1, base, base + 3, base + 2});
        }
    s.pos.push_back(P);
    s.nrm.push_back(N);
    s.uv.push_back(UV);
    s.idx.push_back(I);
}

// ---- value noise -------------------------------------------------------------------------
inline uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t h = x * 0x8da6b343u ^ y * 0xd8163841u ^ z * 0xcb1ab31fu;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    return h;
}
inline double lattice(int x, int y, uint32_t seed, int period) {
    if (period > 0) {
        x = ((x % period) + period) % period;
        y = ((y % period) + period) % period;
    }
    return double(hash3(uint32_t(x), uint32_t(y), seed) & 0xffffff) / double(0xffffff);
}
double value_noise(double x, double y, uint32_t seed, int period) {
    int xi = int(std::floor(x)), yi = int(std::floor(y));
    double fx = x - xi, fy = y - yi;
    double sx = fx * fx * (3 - 2 * fx), sy = fy * fy * (3 - 2 * fy);
    double a = lattice(xi, yi, seed, period), b = lattice(xi + 1, yi, seed, period);
    double c = lattice(xi, yi + 1, seed, period), d = lattice(xi + 1, yi + 1, seed, period);
    return (a + (b - a) * sx) + ((c + (d - c) * sx) - (a + (b - a) * sx)) * sy;
}
double fbm(double x, double y, uint32_t seed, int period, int oct) {
    double s = 0, amp = 0.5, norm = 0;
    for (int o = 0; o < oct; ++o) {
        s += amp * value_noise(x, y, seed + uint32_t(o) * 101u, period);
        norm += amp;
        amp *= 0.5;
        x *= 2;
        y *= 2;
        if (period > 0) period *= 2;
    }
    return s / norm;
}

uint16_t float_to_half(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    int32_t e = int32_t((x >> 23) & 0xff) - 127 + 15;
    uint32_t man = x & 0x7fffffu;
    if (((x >> 23) & 0xff) == 0xff) return uint16_t(sign | 0x7c00u | (man ? 0x200u : 0u));
    if (e >= 31) return uint16_t(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return uint16_t(sign);
        man |= 0x800000u;
        uint32_t shift = uint32_t(14 - e);
        uint32_t half = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u), mid = 1u << (shift - 1);
        if (rem > mid || (rem == mid && (half & 1u))) ++half;
        return uint16_t(sign | half);
    }
    uint32_t half = sign | (uint32_t(e) << 10) | (man >> 13);
    uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) ++half;
    return uint16_t(half);
}

void make_noise_texture(lux_host_scene& s, int size, uint32_t seed, bool alpha_noise, bool half) {
    lux_texture_desc t{};
    t.width = size;
    t.height = size;
    t.format = half ? LUX_TEX_RGBA16F : LUX_TEX_RGBA8;
    std::vector<uint8_t> bytes(size_t(size) * size * 4 * (half ? 2 : 1));
    Rng r(seed);
    double c0[3] = {r.uni(0.2, 1.0), r.uni(0.2, 1.0), r.uni(0.2, 1.0)};
    double c1[3] = {r.uni(0.0, 0.6), r.uni(0.0, 0.6), r.uni(0.0, 0.6)};
    const int cells = 16;
    for (int y = 0; y < size; ++y)
        for (int x = 0; x < size; ++x) {
            double u = double(x) / size * cells, v = double(y) / size * cells;
            double n = fbm(u, v, seed, cells, 5);
            double a = alpha_noise ? fbm(u * 0.5 + 3.7, v * 0.5 + 1.3, seed ^ 0x55u, cells / 2, 3) : 1.0;
            double rgba[4];
            for (int c = 0; c < 3; ++c) rgba[c] = c1[c] + (c0[c] - c1[c]) * n;
            rgba[3] = a;
            size_t o = (size_t(y) * size + x) * 4;
            for (int c = 0; c < 4; ++c) {
                double val = std::min(1.0, std::max(0.0, rgba[c]));
                if (half) {
                    uint16_t hv = float_to_half(float(std::round(val * 255.0) / 255.0));
                    std::memcpy(&bytes[(o + c) * 2], &hv, 2);
                } else {
                    bytes[o + c] = uint8_t(std::lround(val * 255.0));
                }
            }
        }
    s.tex_bytes.push_back(std::move(bytes));
    s.texs.push_back(t);
}

void add_icosphere(lux_host_scene& s, int freq, uint32_t seed, double bump) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    double V[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                       {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    int F[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                    {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                    {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    std::vector<float> P, N, UV;
    std::vector<uint32_t> I;
    auto radius = [&](double x, double y, double z) {
        double u = std::atan2(z, x) / 6.283185307179586 + 0.5, v = std::acos(std::max(-1.0, std::min(1.0, y))) / 3.141592653589793;
        return 1.0 + bump * (fbm(u * 8, v * 4, seed, 8, 3) - 0.5);
    };
    for (int f = 0; f < 20; ++f) {
        const double* a = V[F[f][0]];
        const double* b = V[F[f][1]];
        const double* c = V[F[f][2]];
        uint32_t base = uint32_t(P.size() / 3);
        for (int i = 0; i <= freq; ++i)
            for (int j = 0; j <= freq - i; ++j) {
                double wa = double(freq - i - j) / freq, wb = double(i) / freq, wc = double(j) / freq;
                double p[3];
                for (int k = 0; k < 3; ++k) p[k] = wa * a[k] + wb * b[k] + wc * c[k];
                double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
                for (double& x : p) x /= l;
                double rr = radius(p[0], p[1], p[2]);
                for (int k = 0; k < 3; ++k) {
                    P.push_back(float(p[k] * rr));
                    N.push_back(float(p[k]));
                }
                UV.push_back(float(std::atan2(p[2], p[0]) / 6.283185307179586 + 0.5));
                UV.push_back(float(std::acos(std::max(-1.0, std::min(1.0, p[1]))) / 3.141592653589793));
            }
        auto id = [&](int i, int j) {
            // row i has freq-i+1 entries
            int off = 0;
            for (int r = 0; r < i; ++r) off += freq - r + 1;
            return base + uint32_t(off + j);
        };
        for (int i = 0; i < freq; ++i)
            for (int j = 0; j < freq - i; ++j) {
                I.insert(I.end(), {id(i, j), id(i + 1, j), id(i, j + 1)});
                if (j < freq - i - 1) I.insert(I.end(), {id(i + 1, j), id(i + 1, j + 1), id(i, j + 1)});
            }
    }
    // orient all triangles outward
    for (size_t k = 0; k < I.size(); k += 3) {
        const float* A = &P[I[k] * 3];
        const float* B = &P[I[k + 1] * 3];
        const float* C = &P[I[k + 2] * 3];
        float e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
        float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        if (cr[0] * A[0] + cr[1] * A[1] + cr[2] * A[2] < 0) std::swap(I[k + 1], I[k + 2]);
    }
    s.pos.push_back(P);
    s.nrm.push_back(N);
    s.uv.push_back(UV);
    s.idx.push_back(I);
}

void add_grid(lux_host_scene& s, int n, uint32_t seed, double amp) {
    std::vector<float> P, N, UV;
    std::vector<uint32_t> I;
    auto hgt = [&](double x, double z) { return amp * (fbm(x * 2 + 10, z * 2 + 10, seed, 0, 4) - 0.5); };
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
            double x = -1 + 2.0 * i / n, z = -1 + 2.0 * j / n;
            double y = hgt(x, z);
            double e = 1e-3;
            double dx = (hgt(x + e, z) - hgt(x - e, z)) / (2 * e), dz = (hgt(x, z + e) - hgt(x, z - e)) / (2 * e);
            double nn[3] = {-dx, 1, -dz};
            double l = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
            P.insert(P.end(), {float(x), float(y), float(z)});
            N.insert(N.end(), {float(nn[0] / l), float(nn[1] / l), float(nn[2] / l)});
            UV.insert(UV.end(), {float(i) / n, float(j) / n});
        }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            uint32_t a = uint32_t(j * (n + 1) + i), b = a + 1, c = a + uint32_t(n + 1), d = c + 1;
            // +y facing: cross(B-A, C-A) > 0 in y for (a, c, b)
            I.insert(I.end(), {a, c, b, b, c, d});
        }
    s.pos.push_back(P);
    s.nrm.push_back(N);
    s.uv.push_back(UV);
    s.idx.push_back(I);
}

void make_sky(lux_host_scene& s, int W, int H, uint64_t seed, bool half) {
    Rng r(seed ^ 0xabcdefull);
    double sun_theta = r.uni(0.35, 1.0), sun_phi = r.uni(-3.14159, 3.14159);
    double sd[3] = {std::sin(sun_theta) * std::cos(sun_phi), std::cos(sun_theta), std::sin(sun_theta) * std::sin(sun_phi)};
    const double sigma = 0.02;  // radians
    std::vector<float> px(size_t(W) * H * 4);
    for (int y = 0; y < H; ++y) {
        double v = (y + 0.5) / H, theta = v * 3.141592653589793;
        for (int x = 0; x < W; ++x) {
            double u = (x + 0.5) / W, phi = u * 6.283185307179586 - 3.141592653589793;
            double d[3] = {std::sin(theta) * std::cos(phi), std::cos(theta), std::sin(theta) * std::sin(phi)};
            double g = fbm(u * 16, v * 8, uint32_t(seed), 16, 5);
            double ln = 0.0 + 0.8 * (g - 0.5) * 2.0;  // log-normal sky brightness
            double sky = std::exp(ln);
            double base[3];
            if (d[1] >= 0) {
                double k = d[1];
                base[0] = 0.5 + 0.2 * (1 - k);
                base[1] = 0.6 + 0.2 * (1 - k);
                base[2] = 0.9;
            } else {
                base[0] = 0.25;
                base[1] = 0.22;
                base[2] = 0.2;
            }
            double cosang = d[0] * sd[0] + d[1] * sd[1] + d[2] * sd[2];
            double ang = std::acos(std::max(-1.0, std::min(1.0, cosang)));
            double sun = 1e4 * std::exp(-(ang * ang) / (2 * sigma * sigma));
            size_t o = (size_t(y) * W + x) * 4;
            px[o] = float(base[0] * sky + sun);
            px[o + 1] = float(base[1] * sky + sun * 0.95);
            px[o + 2] = float(base[2] * sky + sun * 0.85);
            px[o + 3] = 1.0f;
        }
    }
    s.desc.env_width = W;
    s.desc.env_height = H;
    if (half) {
        s.env16.resize(px.size());
        for (size_t i = 0; i < px.size(); ++i) s.env16[i] = float_to_half(px[i]);
        s.desc.env_format = LUX_TEX_RGBA16F;
    } else {
        s.env32 = std::move(px);
        s.desc.env_format = LUX_TEX_RGBA32F;
    }
}

}  // namespace

extern "C" {

void lux_make_camera(int width, int height, const float pos[3], const float look[3], float fovy_deg,
                     lux_camera_desc* out) {
    if (!out || !pos || !look) return;
    const double p[3] = {pos[0], pos[1], pos[2]}, l[3] = {look[0], look[1], look[2]};
    std::memset(out, 0, sizeof(*out));
    set_camera(*out, width, height, p, l, fovy_deg);
}

lux_host_scene* lux_scene_cornell36(int width, int height) {
    auto s = std::make_unique<lux_host_scene>();
    std::memset(&s->desc, 0, sizeof(s->desc));
    lux_material_desc white = default_material(), red = default_material(), green = default_material(),
                      metal = default_material(), light = default_material();
    white.color[0] = 0.725f; white.color[1] = 0.71f; white.color[2] = 0.68f;
    red.color[0] = 0.63f; red.color[1] = 0.065f; red.color[2] = 0.05f;
    green.color[0] = 0.14f; green.color[1] = 0.45f; green.color[2] = 0.091f;
    metal.color[0] = 0.725f; metal.color[1] = 0.71f; metal.color[2] = 0.68f;
    metal.metallic = 1.0f;
    metal.roughness = 0.3f;
    light.color[0] = light.color[1] = light.color[2] = 0.78f;
    light.emission_color[0] = 17.0f; light.emission_color[1] = 12.0f; light.emission_color[2] = 4.0f;
    light.emission_strength = 1.0f;
    s->mats = {white, red, green, metal, light};
    // walls: floor y=0, ceiling y=2, back z=-1, left x=-1 (red), right x=1 (green)
    const float fl[4][3] = {{-1, 0, -1}, {1, 0, -1}, {1, 0, 1}, {-1, 0, 1}};
    const float ce[4][3] = {{-1, 2, -1}, {1, 2, -1}, {1, 2, 1}, {-1, 2, 1}};
    const float bk[4][3] = {{-1, 0, -1}, {1, 0, -1}, {1, 2, -1}, {-1, 2, -1}};
    const float lf[4][3] = {{-1, 0, -1}, {-1, 0, 1}, {-1, 2, 1}, {-1, 2, -1}};
    const float rt[4][3] = {{1, 0, -1}, {1, 0, 1}, {1, 2, 1}, {1, 2, -1}};
    const float li[4][3] = {{-0.25f, 1.98f, -0.25f}, {0.25f, 1.98f, -0.25f}, {0.25f, 1.98f, 0.25f}, {-0.25f, 1.98f, 0.25f}};
    const float ny[3] = {0, 1, 0}, nny[3] = {0, -1, 0}, nz[3] = {0, 0, 1}, nx[3] = {1, 0, 0}, nnx[3] = {-1, 0, 0};
    add_quad(*s, fl, ny);   // mesh 0
    add_quad(*s, ce, nny);  // mesh 1
    add_quad(*s, bk, nz);   // mesh 2
    add_quad(*s, lf, nx);   // mesh 3
    add_quad(*s, rt, nnx);  // mesh 4
    add_quad(*s, li, nny);  // mesh 5
    add_unit_cube(*s);      // mesh 6
    M4 I = identity();
    s->insts.push_back(make_instance(0, 0, I));
    s->insts.push_back(make_instance(1, 0, I));
    s->insts.push_back(make_instance(2, 0, I));
    s->insts.push_back(make_instance(3, 1, I));
    s->insts.push_back(make_instance(4, 2, I));
    s->insts.push_back(make_instance(5, 4, I));
    s->insts.push_back(make_instance(6, 0, mul(translate(0.33, 0.3, 0.3), mul(rot_y(-18), scale(0.6, 0.6, 0.6)))));
    s->insts.push_back(make_instance(6, 3, mul(translate(-0.33, 0.6, -0.32), mul(rot_y(20), scale(0.6, 1.2, 0.6)))));
    double pos[3] = {0, 1, 3.4}, look[3] = {0, 1, 0};
    set_camera(s->desc.camera, width, height, pos, look, 40.0);
    s->desc.trace_depth = 8;
    s->finalize();
    return s.release();
}

void lux_default_random_scene_params(lux_random_scene_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->seed = 0;
    p->num_instances = 200;
    p->total_tris = 1000000;
    p->min_tris = 2000;
    p->max_tris = 50000;
    p->num_emissive = 12;
    p->num_textures = 16;
    p->texture_size = 1024;
    p->env_width = 2048;
    p->env_height = 1024;
    p->width = 1920;
    p->height = 1080;
    p->trace_depth = 12;
    p->env_half = 0;
    p->tex_half = 0;
}

lux_host_scene* lux_scene_random(const lux_random_scene_params* prm) {
    if (!prm || prm->num_instances < 1 || prm->total_tris < 1) return nullptr;
    auto s = std::make_unique<lux_host_scene>();
    std::memset(&s->desc, 0, sizeof(s->desc));
    Rng r(prm->seed);
    const int NI = prm->num_instances;
    // triangle budgets: log-uniform in [min,max], rescaled toward the total
    std::vector<double> want(NI);
    for (int i = 0; i < NI; ++i)
        want[i] = std::exp(r.uni(std::log(double(prm->min_tris)), std::log(double(prm->max_tris))));
    for (int pass = 0; pass < 8; ++pass) {
        double sum = 0;
        for (double w : want) sum += w;
        double f = double(prm->total_tris) / sum;
        for (double& w : want) w = std::min(double(prm->max_tris), std::max(double(prm->min_tris), w * f));
    }
    // textures
    const int NT = std::max(0, prm->num_textures);
    for (int t = 0; t < NT; ++t)
        make_noise_texture(*s, prm->texture_size, uint32_t(prm->seed * 977 + t * 31 + 7), (t % 4) == 3, prm->tex_half != 0);
    // meshes + materials + instances
    std::vector<int> emissive_ids;
    {
        std::vector<int> ids(NI - 1);
        for (int i = 0; i < NI - 1; ++i) ids[i] = i + 1;
        for (int i = NI - 2; i > 0; --i) std::swap(ids[i], ids[r.next() % uint64_t(i + 1)]);
        for (int k = 0; k < std::min(prm->num_emissive, NI - 1); ++k) emissive_ids.push_back(ids[k]);
    }
    for (int i = 0; i < NI; ++i) {
        bool ground = (i == 0);
        bool grid = ground || (r.uni() < 0.5);
        int tris = int(want[i]);
        if (grid) {
            int n = std::max(2, int(std::lround(std::sqrt(tris / 2.0))));
            add_grid(*s, n, uint32_t(prm->seed * 131 + i), ground ? 0.15 : 0.6);
        } else {
            int f = std::max(2, int(std::lround(std::sqrt(tris / 20.0))));
            add_icosphere(*s, f, uint32_t(prm->seed * 131 + i), 0.15);
        }
        lux_material_desc m = default_material();
        m.roughness = float(r.uni(0.05, 1.0));
        m.metallic = r.uni() < 0.3 ? 1.0f : 0.0f;
        bool transmissive = r.uni() < 0.10;
        bool masked = r.uni() < 0.05;
        if (transmissive) {
            m.transmission = 1.0f;
            m.ior = 1.5f;
            m.metallic = 0.0f;
        }
        if (NT > 0) {
            m.albedo_tex = int(r.next() % uint64_t(NT));
            if (masked) {
                m.alpha_mode = LUX_ALPHA_MASK;
                m.alpha_cutoff = 0.5f;
                // the mask reads the texture alpha: pick an alpha-noise texture if one exists
                int t4 = (m.albedo_tex / 4) * 4 + 3;
                if (t4 < NT) m.albedo_tex = t4;
            }
        }
        for (int c = 0; c < 3; ++c) m.color[c] = float(r.uni(0.2, 0.9));
        if (std::find(emissive_ids.begin(), emissive_ids.end(), i) != emissive_ids.end()) {
            double hue = r.uni();
            m.emission_color[0] = float(0.6 + 0.4 * std::cos(6.2831853 * hue));
            m.emission_color[1] = float(0.6 + 0.4 * std::cos(6.2831853 * (hue + 0.33)));
            m.emission_color[2] = float(0.6 + 0.4 * std::cos(6.2831853 * (hue + 0.67)));
            m.emission_strength = float(std::exp(r.uni(std::log(1.0), std::log(50.0))));
            m.alpha_mode = LUX_ALPHA_OPAQUE;
            m.transmission = 0.0f;
        }
        s->mats.push_back(m);
        M4 M;
        if (ground) {
            M = mul(translate(0, -0.6, 0), scale(16, 1, 16));
        } else {
            double w = r.normal(), x = r.normal(), y = r.normal(), z = r.normal();
            double sc = r.uni(0.5, 2.0);
            M = mul(translate(r.uni(-12, 12), r.uni(0.2, 5), r.uni(-12, 12)), mul(quat(w, x, y, z), scale(sc, sc, sc)));
        }
        s->insts.push_back(make_instance(i, i, M));
    }
    if (prm->env_width > 0 && prm->env_height > 0) make_sky(*s, prm->env_width, prm->env_height, prm->seed, prm->env_half != 0);
    double pos[3] = {0, 7, 25}, look[3] = {0, 1, 0};
    set_camera(s->desc.camera, prm->width, prm->height, pos, look, 45.0);
    s->desc.trace_depth = prm->trace_depth;
    s->finalize();
    return s.release();
}

lux_host_scene* lux_scene_furnace(int width, int height, int subdiv) {
    lux_material_desc m = default_material();
    m.metallic = 1.0f;
    m.roughness = 0.01f;
    return lux_scene_furnace_material(width, height, subdiv, &m, 1);
}

lux_host_scene* lux_scene_furnace_material(int width, int height, int subdiv, const lux_material_desc* mat,
                                           int vertex_normals) {
    if (!mat) return nullptr;
    auto s = std::make_unique<lux_host_scene>();
    std::memset(&s->desc, 0, sizeof(s->desc));
    add_icosphere(*s, std::max(2, subdiv), 1u, 0.0);
    if (!vertex_normals) s->nrm.back().clear();
    s->mats.push_back(*mat);
    s->insts.push_back(make_instance(0, 0, identity()));
    const int W = 64, H = 32;
    s->env32.assign(size_t(W) * H * 4, 1.0f);
    s->desc.env_width = W;
    s->desc.env_height = H;
    s->desc.env_format = LUX_TEX_RGBA32F;
    double pos[3] = {0, 0, 3.5}, look[3] = {0, 0, 0};
    set_camera(s->desc.camera, width, height, pos, look, 45.0);
    s->desc.trace_depth = 8;
    s->finalize();
    return s.release();
}

void lux_default_material(lux_material_desc* m) {
    if (m) *m = default_material();
}

const lux_scene_desc* lux_scene_get_desc(const lux_host_scene* s) { return s ? &s->desc : nullptr; }
int64_t lux_scene_instanced_tris(const lux_host_scene* s) { return s ? s->instanced_tris : 0; }
void lux_scene_destroy(lux_host_scene* s) { delete s; }

}  // extern "C"
