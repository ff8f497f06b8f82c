// lux_oracle.cpp -- CPU restatement of the seabiscuit-iv/luxion render path.
//
// TEST INFRASTRUCTURE ONLY: loaded by the test suite, the smoke check and the CPU-baseline leg
// of the benchmark, as the checker of the CUDA path. Nothing in the product links it.
//
// Every function restates one piece of the reference, cited as path:line within the
// reference project. The arithmetic follows the reference's evaluation order (glm 0.9.6 and
// sutil semantics) so that, compiled with -ffp-contract=off, the FP32 build agrees with the
// reference's own host-compiled sources (oracle/_ref) to the last bit wherever glibc is the
// math library on both sides. The same templates instantiated with double form the FP64
// integrator used as the converged-image error oracle.
//
// Deviations from the reference, each deliberate:
//  * trace: closest hit over every triangle the reference's Moller-Trumbore test accepts
//    (src/intersections/mesh_isect.cu:78-137), ties on equal t broken toward the lowest
//    (instance, primitive); the reference keeps the first one its traversal order finds.
//  * the alpha-blend any-hit hash is keyed on the pixel index instead of the OptiX launch
//    index (src/optixshaders/optix_triangle.cu:355), which is a queue slot and therefore
//    depends on the order of atomics.
//  * with -dmis and -emis both on, the reference traces a DL shadow ray its shader never
//    reads (src/kernels/shade_path.cu:182,226); it is not traced here.
//  * the Morton box is the first instance's mesh bounds padded once by 1e-5; the reference
//    pads once per level of its own BVH (src/mesh/bvh_build.cu:306-315).

#include "lux_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------------------
// glm 0.9.6 scalar semantics (external/include/glm/detail/func_common.inl:409-472)
template <class T> inline T gmin(T a, T b) { return a < b ? a : b; }
template <class T> inline T gmax(T a, T b) { return a > b ? a : b; }
template <class T> inline T gclamp(T x, T lo, T hi) { return gmin(gmax(x, lo), hi); }

template <class T> struct V2 { T x, y; };
template <class T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
// glm compute_dot<tvec3>: (x.x*y.x + x.y*y.y) + x.z*y.z (func_geometric.inl:65-72); sutil
// dot has the same order (sutil/vec_math.h:503-506).
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// glm cross (func_geometric.inl:134-142)
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
// glm normalize = x * inversesqrt(dot(x,x)), inversesqrt = 1/sqrt (func_exponential.inl:150-153)
template <class T> inline V3<T> normalize(V3<T> v) { return v * (T(1) / std::sqrt(dot(v, v))); }
template <class T> inline T length(V3<T> v) { return std::sqrt(dot(v, v)); }
template <class T> inline V3<T> vmix(V3<T> x, V3<T> y, T a) { return x + a * (y - x); }
template <class T> inline V3<T> reflect(V3<T> I, V3<T> N) { return I - N * dot(N, I) * T(2); }
// glm refract (func_geometric.inl:193-200); sqrt of a negative k gives NaN times 0 = NaN.
template <class T> inline V3<T> refract(V3<T> I, V3<T> N, T eta) {
    T d = dot(N, I);
    T k = T(1) - eta * eta * (T(1) - d * d);
    return (eta * I - (eta * d + std::sqrt(k)) * N) * T(k >= T(0));
}
template <class T> inline V3<T> vpow(V3<T> v, T e) { return {std::pow(v.x, e), std::pow(v.y, e), std::pow(v.z, e)}; }
template <class T, class U> inline V3<T> cvt(V3<U> v) { return {T(v.x), T(v.y), T(v.z)}; }

// glm mat4 * vec4 (detail/type_mat4x4.inl:592-629): (m0*v0 + m1*v1) + (m2*v2 + m3*v3)
template <class T> inline V3<T> mul_point(const float* m, V3<T> p, T w) {
    V3<T> r;
    for (int c = 0; c < 3; ++c) {
        T a0 = T(m[0 * 4 + c]) * p.x;
        T a1 = T(m[1 * 4 + c]) * p.y;
        T a2 = T(m[2 * 4 + c]) * p.z;
        T a3 = T(m[3 * 4 + c]) * w;
        r[c] = (a0 + a1) + (a2 + a3);
    }
    return r;
}

constexpr float kPI = 3.1415926535897932384626422832795028841971f;      // include/utilities.h:13
constexpr float kTWO_PI = 6.2831853071795864769252867665590057683943f;  // include/utilities.h:14
constexpr float kSQRT13 = 0.5773502691896257645091487805019574556476f;  // include/utilities.h:15
constexpr float kEPS_UTIL = 0.00001f;                                  // include/utilities.h:16
constexpr float kINV_PI = 0.3183098f;                      // include/shaders/cook_torrance.h:13
constexpr float kEPS_CT = 1e-30f;                                    // src/shaders/cook_torrance.cu:3
constexpr float kPDF_CLAMP = 1e-5f;                                  // src/shaders/cook_torrance.cu:4
constexpr double kM_PI_SHADE = 3.14159;                              // src/kernels/shade_path.cu:23
constexpr float kGLASS_EPS = 0.01f;                                  // src/kernels/shade_path.cu:24
constexpr float kSPEC_ROUGH = 0.05f;                                 // src/kernels/shade_path.cu:25
constexpr int kRR_MIN_DEPTH = 3;                                     // include/config.h:7

// ---------------------------------------------------------------------------------------
// RNG: utilhash (include/intersections.h:13-22), makeSeededRandomEngine
// (include/common.h:38-47), thrust::minstd_rand and uniform_real_distribution<float>(0,1)
// ((x - min) / (1 + (max - min)), thrust/random/detail/uniform_real_distribution.inl:61-75).
uint32_t utilhash(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}

struct MinStd {
    uint32_t x;
    explicit MinStd(uint32_t s) {
        uint32_t r = s % 2147483647u;
        x = (r == 0u) ? 1u : r;
    }
    uint32_t next() {
        x = uint32_t((uint64_t(x) * 48271ull) % 2147483647ull);
        return x;
    }
    template <class T> T u01() {
        uint32_t v = next();
        T r = static_cast<T>(v - 1u);
        r /= (T(1) + static_cast<T>(2147483646u - 1u));
        return (r * (T(1) - T(0))) + T(0);
    }
};

MinStd seeded(int iter, int index, int depth) {
    uint32_t k = (1u << 31) | (uint32_t(depth) << 22) | uint32_t(iter);
    int h = int(utilhash(k) ^ utilhash(uint32_t(index)));
    return MinStd(uint32_t(h));
}

// cudaUtils::select_from_cdf (src/common.cu:3-15)
template <class T> int select_from_cdf(const T* cdf, int size, T xi) {
    int low = 0, high = size - 1;
    while (low < high) {
        int mid = low + (high - low) / 2;
        if (cdf[mid] < xi) low = mid + 1;
        else high = mid;
    }
    return low;
}

// ---------------------------------------------------------------------------------------
// Textures. The reference uploads every texture as float4 (RGBA8 / 255, RGBA16 / 65535,
// scene_load_gltf.cpp:115-143) into a cudaArray with linear filtering, wrap addressing and
// normalised coordinates (src/texture.cu:51-56). The fetch below restates the CUDA hardware
// filter as measured on B200 (tests/golden/texture_filter_probe.npz holds the measurement):
// after wrap, x = u*W - 0.5, i = floor(x), the 1-D weight a = floor(frac(x)*256 + 0.5) in
// 1/256 units (round half up; the programming guide's "9-bit fixed point with 8 fractional
// bits"), likewise b; the 2-D weights are w00 = ((256-a)(256-b)+128)>>8, w11 = (ab+128)>>8,
// w10 = (256-b) - w00, w01 = b - w11, summing to 256. Float texels are combined as
// sum(w*T)/256; 8-bit unorm texels are expanded to 16 bits (c*257), combined in integers,
// rounded half up to 16 bits and divided by 65535.
struct Tex {
    int w = 0, h = 0;
    bool unorm8 = false;         // texels kept as 8-bit unorm (hardware unorm path)
    bool half = false;           // texels held as binary16 on the device (half filter path)
    std::vector<float> texels;   // w*h*4 (float path)
    std::vector<uint8_t> bytes;  // w*h*4 (unorm8 path)
};

inline float half_to_float(uint16_t h) {
    uint32_t sign = uint32_t(h >> 15) << 31;
    uint32_t exp = (h >> 10) & 0x1f, man = h & 0x3ff;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) bits = sign;
        else {
            int e = -1;
            do { ++e; man <<= 1; } while ((man & 0x400) == 0);
            bits = sign | uint32_t(127 - 15 - e) << 23 | (man & 0x3ff) << 13;
        }
    } else if (exp == 31) {
        bits = sign | 0x7f800000u | (man << 13);
    } else {
        bits = sign | (exp + 112) << 23 | (man << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

inline float round_to_half(float f) {  // IEEE binary16 round-to-nearest-even, back to float
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    int32_t e = int32_t((x >> 23) & 0xff) - 127 + 15;
    uint32_t man = x & 0x7fffffu;
    uint16_t hb;
    if (((x >> 23) & 0xff) == 0xff) hb = uint16_t(sign | 0x7c00u | (man ? 0x200u : 0u));
    else if (e >= 31) hb = uint16_t(sign | 0x7c00u);
    else if (e <= 0) {
        if (e < -10) hb = uint16_t(sign);
        else {
            man |= 0x800000u;
            uint32_t shift = uint32_t(14 - e);
            uint32_t half = man >> shift, rem = man & ((1u << shift) - 1u), mid = 1u << (shift - 1);
            if (rem > mid || (rem == mid && (half & 1u))) ++half;
            hb = uint16_t(sign | half);
        }
    } else {
        uint32_t half = sign | (uint32_t(e) << 10) | (man >> 13), rem = man & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) ++half;
        hb = uint16_t(half);
    }
    return half_to_float(hb);
}

// storage: LUX_TEXSTORE_FLOAT converts 8-bit texels to float as the reference does,
// LUX_TEXSTORE_UNORM8 keeps them on the hardware unorm path, LUX_TEXSTORE_HALF rounds every
// texel to binary16. Binary16 input stays binary16 on the device under every storage.
void load_tex(Tex& t, int w, int h, int fmt, const void* data, int storage = LUX_TEXSTORE_FLOAT) {
    t.w = w;
    t.h = h;
    size_t n = size_t(w) * size_t(h) * 4;
    t.unorm8 = storage == LUX_TEXSTORE_UNORM8 && fmt == LUX_TEX_RGBA8;
    t.half = !t.unorm8 && (storage == LUX_TEXSTORE_HALF || fmt == LUX_TEX_RGBA16F);
    if (t.unorm8) {
        t.bytes.assign(static_cast<const uint8_t*>(data), static_cast<const uint8_t*>(data) + n);
        return;
    }
    t.texels.resize(n);
    for (size_t i = 0; i < n; ++i) {
        switch (fmt) {
            case LUX_TEX_RGBA8: t.texels[i] = float(static_cast<const uint8_t*>(data)[i]) / 255.0f; break;
            case LUX_TEX_RGBA16: t.texels[i] = float(static_cast<const uint16_t*>(data)[i]) / 65535.0f; break;
            case LUX_TEX_RGBA16F: t.texels[i] = half_to_float(static_cast<const uint16_t*>(data)[i]); break;
            default: t.texels[i] = static_cast<const float*>(data)[i]; break;
        }
        if (storage == LUX_TEXSTORE_HALF) t.texels[i] = round_to_half(t.texels[i]);
    }
}

// Filter coordinate of one axis, as the B200 texture unit forms it (measured with
// tests/golden/probe_texture_filter.py): the normalized coordinate wraps into a 21-bit fixed
// point fraction by truncation, q = floor(u * 2^21) mod 2^21; the texel-space position
// X = q * n - 2^20 (units of 2^-21 texel, i.e. u * n - 0.5) is exact; the lower texel is
// X >> 21 and the 8-bit weight of the upper one rounds half up, a = (X mod 2^21 + 2^12) >> 13.
// Binary16 rounding of a double, ties away from zero (the rounding of the half filter below).
inline float round_half_away_to_half(double s) {
    if (s == 0.0) return 0.0f;
    double a = std::fabs(s);
    int ex;
    std::frexp(a, &ex);                         // a = m * 2^ex, m in [0.5, 1)
    double ulp = std::ldexp(1.0, std::max(ex - 1, -14) - 10);
    double q = std::floor(a / ulp + 0.5) * ulp;
    if (q > 65504.0) q = double(INFINITY);
    return float(s < 0 ? -q : q);
}

// The filter of a binary16 texture, as the B200 texture unit computes it (measured with
// tests/golden/probe_texture_filter.py on random texels over six decades): the texels with a
// non-zero weight are aligned to the leading bit of the largest of them and truncated to 15
// significant bits, the weighted sum of those integers is exact, and the result rounds to
// binary16 with ties away from zero. Measured on non-negative texels; negative ones take the
// same rule on magnitudes.
inline float half_filter(const int w[4], const float t[4]) {
    double mx = 0.0;
    for (int k = 0; k < 4; ++k)
        if (w[k] > 0) mx = std::max(mx, std::fabs(double(t[k])));
    if (mx == 0.0) return 0.0f;
    int ex;
    std::frexp(mx, &ex);
    double ulp = std::ldexp(1.0, ex - 15);      // 2^(leading bit - 14)
    int64_t X = 0;
    for (int k = 0; k < 4; ++k) {
        if (w[k] <= 0) continue;
        double q = std::trunc(std::fabs(double(t[k])) / ulp);
        X += int64_t(w[k]) * int64_t(t[k] < 0 ? -q : q);
    }
    return round_half_away_to_half(double(X) * ulp / 256.0);
}

inline void tex_axis(float u, int n, int& i0, int& a) {
    double s = std::floor(double(u) * 2097152.0);
    s -= std::floor(s / 2097152.0) * 2097152.0;
    int64_t X = int64_t(s) * n - (int64_t(1) << 20);
    int64_t fi = X >> 21;  // arithmetic shift: floor for negative X
    a = int(((X - (fi << 21)) + (1 << 12)) >> 13);
    i0 = int(fi);
}

template <class T> void tex_fetch(const Tex& t, T u, T v, T out[4]) {
    int i0, j0, a, b;
    tex_axis(float(u), t.w, i0, a);
    tex_axis(float(v), t.h, j0, b);
    int w00 = ((256 - a) * (256 - b) + 128) >> 8;
    int w11 = (a * b + 128) >> 8;
    int w10 = (256 - b) - w00;
    int w01 = b - w11;
    auto wrap = [](int i, int n) { int r = i % n; return r < 0 ? r + n : r; };
    int i1 = wrap(i0 + 1, t.w), j1 = wrap(j0 + 1, t.h);
    i0 = wrap(i0, t.w);
    j0 = wrap(j0, t.h);
    size_t o00 = (size_t(j0) * t.w + i0) * 4, o10 = (size_t(j0) * t.w + i1) * 4;
    size_t o01 = (size_t(j1) * t.w + i0) * 4, o11 = (size_t(j1) * t.w + i1) * 4;
    for (int c = 0; c < 4; ++c) {
        if (t.unorm8) {
            int64_t s = int64_t(w00) * 257 * t.bytes[o00 + c] + int64_t(w10) * 257 * t.bytes[o10 + c] +
                        int64_t(w01) * 257 * t.bytes[o01 + c] + int64_t(w11) * 257 * t.bytes[o11 + c];
            int64_t r = (s + 128) >> 8;
            out[c] = T(float(double(r) / 65535.0));
        } else if (t.half) {
            const int w[4] = {w00, w10, w01, w11};
            const float tx[4] = {t.texels[o00 + c], t.texels[o10 + c], t.texels[o01 + c], t.texels[o11 + c]};
            out[c] = T(half_filter(w, tx));
        } else {
            float r = (float(w00) * t.texels[o00 + c] + float(w10) * t.texels[o10 + c]) +
                      (float(w01) * t.texels[o01 + c] + float(w11) * t.texels[o11 + c]);
            out[c] = T(r * (1.0f / 256.0f));
        }
    }
}

// ---------------------------------------------------------------------------------------
// Scene
struct Mesh {
    int nv = 0, nt = 0;
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx;
    bool has_n = false, has_uv = false;
    float bmin[3], bmax[3];
};
struct Inst {
    int mesh, material;
    float M[16], Minv[16], MinvT[16];
};

struct BNode {
    float bmin[3], bmax[3];
    int left = -1, right = -1, first = 0, count = 0;
};
struct BVH {
    std::vector<BNode> nodes;
    std::vector<int> prims;
};

void build_bvh(BVH& bvh, const std::vector<float>& boxes /*n*6*/, int n) {
    bvh.nodes.clear();
    bvh.prims.resize(n);
    for (int i = 0; i < n; ++i) bvh.prims[i] = i;
    if (n == 0) return;
    std::vector<float> cen(size_t(n) * 3);
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) cen[i * 3 + a] = 0.5f * (boxes[i * 6 + a] + boxes[i * 6 + 3 + a]);
    struct Task { int node, first, count; };
    std::vector<Task> stack;
    bvh.nodes.push_back(BNode());
    stack.push_back({0, 0, n});
    while (!stack.empty()) {
        Task tk = stack.back();
        stack.pop_back();
        BNode nd;
        for (int a = 0; a < 3; ++a) { nd.bmin[a] = FLT_MAX; nd.bmax[a] = -FLT_MAX; }
        float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = tk.first; i < tk.first + tk.count; ++i) {
            int p = bvh.prims[i];
            for (int a = 0; a < 3; ++a) {
                nd.bmin[a] = std::min(nd.bmin[a], boxes[p * 6 + a]);
                nd.bmax[a] = std::max(nd.bmax[a], boxes[p * 6 + 3 + a]);
                cmin[a] = std::min(cmin[a], cen[p * 3 + a]);
                cmax[a] = std::max(cmax[a], cen[p * 3 + a]);
            }
        }
        if (tk.count <= 4) {
            nd.first = tk.first;
            nd.count = tk.count;
            bvh.nodes[tk.node] = nd;
            continue;
        }
        int axis = 0;
        float ext = cmax[0] - cmin[0];
        for (int a = 1; a < 3; ++a)
            if (cmax[a] - cmin[a] > ext) { ext = cmax[a] - cmin[a]; axis = a; }
        int mid = tk.first + tk.count / 2;
        std::nth_element(bvh.prims.begin() + tk.first, bvh.prims.begin() + mid,
                         bvh.prims.begin() + tk.first + tk.count, [&](int x, int y) {
                             float cx = cen[x * 3 + axis], cy = cen[y * 3 + axis];
                             return cx < cy || (cx == cy && x < y);
                         });
        nd.left = int(bvh.nodes.size());
        nd.right = nd.left + 1;
        bvh.nodes.push_back(BNode());
        bvh.nodes.push_back(BNode());
        bvh.nodes[tk.node] = nd;
        stack.push_back({nd.left, tk.first, mid - tk.first});
        stack.push_back({nd.right, mid, tk.first + tk.count - mid});
    }
}

// Conservative slab test in double; NaN from 0*inf is ignored (fmin/fmax), so a ray lying in
// a slab plane is never rejected.
inline bool box_hit(const float* bmin, const float* bmax, const double o[3], const double inv[3],
                    double tmax, double& tnear) {
    double t0 = 0.0, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        double ta = (double(bmin[a]) - o[a]) * inv[a];
        double tb = (double(bmax[a]) - o[a]) * inv[a];
        double lo = std::fmin(ta, tb), hi = std::fmax(ta, tb);
        if (!std::isnan(lo)) t0 = std::fmax(t0, lo);
        if (!std::isnan(hi)) t1 = std::fmin(t1, hi);
    }
    tnear = t0;
    return t0 <= t1 * (1.0 + 1e-9) + 1e-30;
}

}  // namespace

struct orc_scene {
    lux_camera_desc cam;
    int trace_depth = 8;
    std::vector<Mesh> meshes;
    std::vector<Inst> insts;
    std::vector<lux_material_desc> mats;
    std::vector<Tex> texs;
    Tex env;
    bool has_env = false;
    // light CDFs (src/scene/scene_precompute.cpp:22-124); double copies for the FP64 form
    std::vector<int> emissive;             // instance ids
    std::vector<float> emissive_prefix;
    std::vector<std::vector<float>> tri_prefix;  // per instance
    float total_area = 0.0f;
    std::vector<float> marginal, conditional;
    std::vector<double> emissive_prefix_d, marginal_d, conditional_d;
    std::vector<std::vector<double>> tri_prefix_d;
    double total_area_d = 0.0;
    // acceleration
    std::vector<BVH> blas;
    BVH tlas;
    std::vector<float> inst_boxes;  // world boxes n*6
    float morton_bmin[3], morton_bmax[3];
};

namespace {

template <class T> V3<T> mesh_pos(const Mesh& m, uint32_t i) {
    return {T(m.pos[i * 3]), T(m.pos[i * 3 + 1]), T(m.pos[i * 3 + 2])};
}
template <class T> V3<T> mesh_nrm(const Mesh& m, uint32_t i) {
    return {T(m.nrm[i * 3]), T(m.nrm[i * 3 + 1]), T(m.nrm[i * 3 + 2])};
}
template <class T> V2<T> mesh_uv(const Mesh& m, uint32_t i) { return {T(m.uv[i * 2]), T(m.uv[i * 2 + 1])}; }

// Emissive-area CDF, Scene::precompute_emissive_mesh_area (src/scene/scene_precompute.cpp:22-73)
template <class T>
void precompute_emissive(orc_scene& s, std::vector<T>& prefix, std::vector<std::vector<T>>& tri,
                         T& total) {
    T emissive_area = T(0);
    s.emissive.clear();
    prefix.clear();
    tri.assign(s.insts.size(), {});
    for (size_t i = 0; i < s.insts.size(); ++i) {
        const Inst& g = s.insts[i];
        const Mesh& m = s.meshes[g.mesh];
        T cum = T(0);
        for (int k = 0; k < m.nt; ++k) {
            V3<T> A = mul_point<T>(g.M, mesh_pos<T>(m, m.idx[k * 3]), T(1));
            V3<T> B = mul_point<T>(g.M, mesh_pos<T>(m, m.idx[k * 3 + 1]), T(1));
            V3<T> C = mul_point<T>(g.M, mesh_pos<T>(m, m.idx[k * 3 + 2]), T(1));
            V3<T> u = B - A, v = C - A;
            cum += T(0.5) * length(cross(u, v));
            tri[i].push_back(cum);
        }
        for (auto& x : tri[i]) x /= cum;
        const lux_material_desc& mat = s.mats[g.material];
        V3<float> ec{mat.emission_color[0], mat.emission_color[1], mat.emission_color[2]};
        if (length(ec) * mat.emission_strength > kEPS_UTIL) {
            emissive_area += cum;
            s.emissive.push_back(int(i));
            prefix.push_back(emissive_area);
        }
    }
    for (auto& x : prefix) x /= emissive_area;
    total = emissive_area;
}

// HDRI marginal/conditional CDFs, Scene::precompute_hdri_emission
// (src/scene/scene_precompute.cpp:76-124). The weight is |rgba| (vec4 length, alpha
// included, :88) times sin(theta) of the row centre.
template <class T> bool precompute_hdri(const Tex& env, std::vector<T>& marg, std::vector<T>& cond) {
    int W = env.w, H = env.h;
    cond.assign(size_t(W) * H, T(0));
    marg.assign(H, T(0));
    T total = T(0);
    for (int y = 0; y < H; ++y) {
        T row_total = T(0);
        T theta = T(kPI) * (T(y) + T(0.5)) / T(H);
        T st = std::sin(theta);
        for (int x = 0; x < W; ++x) {
            const float* p = &env.texels[(size_t(y) * W + x) * 4];
            T e;
            {
                T a = T(p[0]) * T(p[0]), b = T(p[1]) * T(p[1]), c = T(p[2]) * T(p[2]),
                  d = T(p[3]) * T(p[3]);
                e = std::sqrt((a + b) + (c + d));  // glm compute_dot<tvec4>, func_geometric.inl:77-81
            }
            T w = e * st;
            row_total += w;
            cond[size_t(y) * W + x] = row_total;
        }
        if (row_total > T(0)) {
            for (int x = 0; x < W; ++x) cond[size_t(y) * W + x] /= row_total;
        } else {
            for (int x = 0; x < W; ++x) cond[size_t(y) * W + x] = T(x + 1) / T(W);
        }
        cond[size_t(y) * W + (W - 1)] = T(1);
        total += row_total;
        marg[y] = total;
    }
    if (total == T(0)) return false;
    for (int y = 0; y < H; ++y) marg[y] /= total;
    marg[H - 1] = T(1);
    return true;
}

// ---------------------------------------------------------------------------------------
// Trace. Ray into the instance's object space with inverseTransform
// (src/intersections/mesh_isect.cu:15-16), then Moller-Trumbore with eps = FLT_EPSILON
// (mesh_isect.cu:34,78-115), keep t > eps.
struct Hit {
    float t = -1.0f;
    int inst = -1, prim = -1;
    float u = 0.0f, v = 0.0f;
};
template <class T> struct HitT {
    T t = T(-1);
    int inst = -1, prim = -1;
    T u = T(0), v = T(0);
};

template <class T>
inline bool moller_trumbore(const Mesh& m, int tri, V3<T> o, V3<T> d, T& t_out, T& u_out, T& v_out) {
    const T eps = T(1.1920929E-7F);
    V3<T> a = mesh_pos<T>(m, m.idx[tri * 3]);
    V3<T> edge1 = mesh_pos<T>(m, m.idx[tri * 3 + 1]) - a;
    V3<T> edge2 = mesh_pos<T>(m, m.idx[tri * 3 + 2]) - a;
    V3<T> c = cross(d, edge2);
    T det = dot(edge1, c);
    if (det > -eps && det < eps) return false;
    T inv_det = T(1) / det;
    a = o - a;
    T u = inv_det * dot(a, c);
    if (u < -eps || u > T(1) + eps) return false;
    c = cross(a, edge1);
    T v = inv_det * dot(d, c);
    if ((v < T(0) && std::fabs(v) > eps) || (u + v > T(1) && std::fabs(u + v - T(1)) > eps)) return false;
    T t = inv_det * dot(edge2, c);
    if (!(t > eps)) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    return true;
}

inline uint32_t hash_u32(uint32_t x) {  // src/optixshaders/optix_triangle.cu:41-49
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

template <class T> V2<T> apply_tt(V2<T> uv, const lux_tex_transform& tt);

// Any-hit program (src/optixshaders/optix_triangle.cu:317-366): true = accept.
template <class T>
bool any_hit_accept(const orc_scene& s, int inst, int prim, T bu, T bv, V3<T> wdir, int pixel, int iter) {
    const Inst& g = s.insts[inst];
    const lux_material_desc& mat = s.mats[g.material];
    if (mat.alpha_mode == LUX_ALPHA_OPAQUE) return true;
    T alpha = T(mat.alpha);
    if (mat.albedo_tex >= 0) {
        const Mesh& m = s.meshes[g.mesh];
        V2<T> uv{T(0), T(0)};
        if (m.has_uv) {
            V2<T> A = mesh_uv<T>(m, m.idx[prim * 3]), B = mesh_uv<T>(m, m.idx[prim * 3 + 1]),
                  C = mesh_uv<T>(m, m.idx[prim * 3 + 2]);
            T bA = T(1) - bu - bv;
            uv.x = bA * A.x + bu * B.x + bv * C.x;
            uv.y = bA * A.y + bu * B.y + bv * C.y;
        }
        uv = apply_tt(uv, mat.albedo_tt);
        T texel[4];
        tex_fetch(s.texs[mat.albedo_tex], uv.x, uv.y, texel);
        alpha *= texel[3];
    }
    if (mat.alpha_mode == LUX_ALPHA_MASK) return !(alpha < T(mat.alpha_cutoff));
    float dx = float(wdir.x), dy = float(wdir.y), dz = float(wdir.z);
    uint32_t bx, by, bz;
    std::memcpy(&bx, &dx, 4);
    std::memcpy(&by, &dy, 4);
    std::memcpy(&bz, &dz, 4);
    uint32_t h = hash_u32(uint32_t(pixel) ^ hash_u32(uint32_t(iter)));
    h = hash_u32(h ^ bx);
    h = hash_u32(h ^ by);
    h = hash_u32(h ^ bz);
    h = hash_u32(h ^ uint32_t(inst));
    h = hash_u32(h ^ uint32_t(prim));
    float rnd = float(h >> 8) * (1.0f / 16777216.0f);
    return !(rnd >= float(alpha));
}

inline bool better(float t, int inst, int prim, const HitT<float>& b) {
    if (b.inst < 0) return true;
    if (t < b.t) return true;
    if (t == b.t) return inst < b.inst || (inst == b.inst && prim < b.prim);
    return false;
}
inline bool better(double t, int inst, int prim, const HitT<double>& b) {
    if (b.inst < 0) return true;
    if (t < b.t) return true;
    if (t == b.t) return inst < b.inst || (inst == b.inst && prim < b.prim);
    return false;
}

// mode 0/1: closest accepted hit with t <= tmax; mode 2: any accepted hit (occlusion).
template <class T>
bool trace_ray(const orc_scene& s, V3<T> o, V3<T> d, T tmax, int mode, int pixel, int iter, bool brute,
               HitT<T>& best) {
    best = HitT<T>();
    auto test_inst = [&](int ii) -> bool {
        const Inst& g = s.insts[ii];
        const Mesh& m = s.meshes[g.mesh];
        V3<T> oo = mul_point<T>(g.Minv, o, T(1));
        V3<T> od = mul_point<T>(g.Minv, d, T(0));
        auto test_tri = [&](int tri) -> bool {
            T t, u, v;
            if (!moller_trumbore(m, tri, oo, od, t, u, v)) return false;
            if (!(t <= tmax)) return false;
            if (mode != 2 && !better(t, ii, tri, best)) return false;
            if (!any_hit_accept(s, ii, tri, u, v, d, pixel, iter)) return false;
            best.t = t;
            best.inst = ii;
            best.prim = tri;
            best.u = u;
            best.v = v;
            return mode == 2;
        };
        if (brute) {
            for (int k = 0; k < m.nt; ++k)
                if (test_tri(k)) return true;
            return false;
        }
        const BVH& b = s.blas[g.mesh];
        double od3[3] = {double(oo.x), double(oo.y), double(oo.z)};
        double inv[3] = {1.0 / double(od.x), 1.0 / double(od.y), 1.0 / double(od.z)};
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const BNode& nd = b.nodes[stack[--sp]];
            double lim = (mode != 2 && best.inst >= 0) ? double(best.t) : double(tmax);
            double tn;
            if (!box_hit(nd.bmin, nd.bmax, od3, inv, lim, tn)) continue;
            if (nd.count) {
                for (int k = nd.first; k < nd.first + nd.count; ++k)
                    if (test_tri(b.prims[k])) return true;
            } else {
                stack[sp++] = nd.left;
                stack[sp++] = nd.right;
            }
        }
        return false;
    };
    if (brute) {
        for (int ii = 0; ii < int(s.insts.size()); ++ii)
            if (test_inst(ii)) return true;
        return best.inst >= 0;
    }
    double o3[3] = {double(o.x), double(o.y), double(o.z)};
    double inv[3] = {1.0 / double(d.x), 1.0 / double(d.y), 1.0 / double(d.z)};
    int stack[128];
    int sp = 0;
    if (!s.tlas.nodes.empty()) stack[sp++] = 0;
    while (sp) {
        const BNode& nd = s.tlas.nodes[stack[--sp]];
        double lim = (mode != 2 && best.inst >= 0) ? double(best.t) : double(tmax);
        double tn;
        if (!box_hit(nd.bmin, nd.bmax, o3, inv, lim, tn)) continue;
        if (nd.count) {
            for (int k = nd.first; k < nd.first + nd.count; ++k)
                if (test_inst(s.tlas.prims[k])) return true;
        } else {
            stack[sp++] = nd.left;
            stack[sp++] = nd.right;
        }
    }
    return best.inst >= 0;
}

// ---------------------------------------------------------------------------------------
// Hit attributes: closest-hit programs (src/optixshaders/optix_triangle.cu:156-243 radiance,
// :259-305 direct light).
template <class T> struct Isect {
    T t = T(-1);
    V3<T> normal, tangent;
    int material = 0;
    V2<T> uv{T(0), T(0)};
};

template <class T> V3<T> xform_normal(const Inst& g, V3<T> n) { return mul_point<T>(g.MinvT, n, T(0)); }
template <class T> V3<T> xform_vector(const Inst& g, V3<T> v) { return mul_point<T>(g.M, v, T(0)); }

template <class T> Isect<T> ch_radiance(const orc_scene& s, const HitT<T>& h) {
    Isect<T> r;
    const Inst& g = s.insts[h.inst];
    const Mesh& m = s.meshes[g.mesh];
    uint32_t i0 = m.idx[h.prim * 3], i1 = m.idx[h.prim * 3 + 1], i2 = m.idx[h.prim * 3 + 2];
    V3<T> A = mesh_pos<T>(m, i0), B = mesh_pos<T>(m, i1), C = mesh_pos<T>(m, i2);
    V3<T> edge1 = B - A, edge2 = C - A;
    V3<T> normal = normalize(cross(edge1, edge2));
    T bA = T(1) - h.u - h.v;
    if (m.has_n) {
        V3<T> nA = mesh_nrm<T>(m, i0), nB = mesh_nrm<T>(m, i1), nC = mesh_nrm<T>(m, i2);
        normal = normalize(bA * nA + h.u * nB + h.v * nC);
    }
    V3<T> tangent{T(1), T(0), T(0)};
    V2<T> uv{T(0), T(0)};
    if (m.has_uv) {
        V2<T> a = mesh_uv<T>(m, i0), b = mesh_uv<T>(m, i1), c = mesh_uv<T>(m, i2);
        uv.x = bA * a.x + h.u * b.x + h.v * c.x;
        uv.y = bA * a.y + h.u * b.y + h.v * c.y;
        V2<T> duv1{b.x - a.x, b.y - a.y}, duv2{c.x - a.x, c.y - a.y};
        T det = duv1.x * duv2.y - duv2.x * duv1.y;
        T f = (std::fabs(det) < T(1e-10f)) ? T(0) : T(1) / det;
        if (f == T(0)) {
            tangent = V3<T>(T(1), T(0), T(0));
        } else {
            tangent.x = f * (duv2.y * edge1.x - duv1.y * edge2.x);
            tangent.y = f * (duv2.y * edge1.y - duv1.y * edge2.y);
            tangent.z = f * (duv2.y * edge1.z - duv1.y * edge2.z);
        }
    }
    normal = normalize(xform_normal(g, normal));
    tangent = normalize(xform_vector(g, tangent));
    V3<T> Tg = tangent - dot(tangent, normal) * normal;
    T len2 = dot(Tg, Tg);
    if (len2 > T(1e-10f)) {
        tangent = Tg * (T(1) / std::sqrt(len2));
    } else {
        tangent = (std::fabs(normal.x) > T(0.9f)) ? V3<T>(T(0), T(1), T(0)) : V3<T>(T(1), T(0), T(0));
        tangent = normalize(cross(tangent, normal));
    }
    r.t = h.t;
    r.normal = normal;
    r.tangent = tangent;
    r.material = g.material;
    r.uv = uv;
    return r;
}

template <class T> Isect<T> ch_direct_light(const orc_scene& s, const HitT<T>& h) {
    Isect<T> r;
    const Inst& g = s.insts[h.inst];
    const Mesh& m = s.meshes[g.mesh];
    uint32_t i0 = m.idx[h.prim * 3], i1 = m.idx[h.prim * 3 + 1], i2 = m.idx[h.prim * 3 + 2];
    T bA = T(1) - h.u - h.v;
    V3<T> normal;
    if (m.has_n) {
        normal = normalize(bA * mesh_nrm<T>(m, i0) + h.u * mesh_nrm<T>(m, i1) + h.v * mesh_nrm<T>(m, i2));
    } else {
        V3<T> A = mesh_pos<T>(m, i0), B = mesh_pos<T>(m, i1), C = mesh_pos<T>(m, i2);
        normal = normalize(cross(B - A, C - A));
    }
    V2<T> uv{T(0), T(0)};
    if (m.has_uv) {
        V2<T> a = mesh_uv<T>(m, i0), b = mesh_uv<T>(m, i1), c = mesh_uv<T>(m, i2);
        uv.x = bA * a.x + h.u * b.x + h.v * c.x;
        uv.y = bA * a.y + h.u * b.y + h.v * c.y;
    }
    r.t = h.t;
    r.normal = normalize(xform_normal(g, normal));
    r.material = g.material;
    r.uv = uv;
    return r;
}

// ---------------------------------------------------------------------------------------
// Material queries (src/material_queries.cu:3-137)
template <class T> V2<T> apply_tt(V2<T> uv, const lux_tex_transform& tt) {
    uv.x *= T(tt.scale[0]);
    uv.y *= T(tt.scale[1]);
    if (tt.rotation != 0.0f) {
        T c = std::cos(T(tt.rotation)), s = std::sin(T(tt.rotation));
        V2<T> r{c * uv.x - s * uv.y, s * uv.x + c * uv.y};
        uv = r;
    }
    return {uv.x + T(tt.offset[0]), uv.y + T(tt.offset[1])};
}

template <class T> V3<T> get_albedo(const orc_scene& s, const lux_material_desc& m, V2<T> uv) {
    if (m.albedo_tex >= 0) {
        uv = apply_tt(uv, m.albedo_tt);
        T tx[4];
        tex_fetch(s.texs[m.albedo_tex], uv.x, uv.y, tx);
        return vpow(V3<T>(tx[0], tx[1], tx[2]), T(2.2f));
    }
    return {T(m.color[0]), T(m.color[1]), T(m.color[2])};
}

template <class T> V3<T> get_normal(const orc_scene& s, const lux_material_desc& m, const Isect<T>& is) {
    if (m.normal_tex >= 0) {
        V2<T> uv = apply_tt(is.uv, m.normal_tt);
        T tx[4];
        tex_fetch(s.texs[m.normal_tex], uv.x, uv.y, tx);
        V3<T> ln{tx[0] * T(2) - T(1), tx[1] * T(2) - T(1), tx[2] * T(2) - T(1)};
        const V3<T> N = is.normal;
        T l2 = dot(ln, ln);
        if (!(l2 > T(1e-12f))) return N;
        V3<T> Tg = is.tangent - dot(is.tangent, N) * N;
        T t2 = dot(Tg, Tg);
        if (!(t2 > T(1e-12f))) return N;
        Tg = Tg * (T(1) / std::sqrt(t2));
        V3<T> Bt = cross(N, Tg);
        // glm mat3(T, B, N) * v (detail/type_mat3x3.inl:487-493)
        V3<T> mapped{Tg.x * ln.x + Bt.x * ln.y + N.x * ln.z, Tg.y * ln.x + Bt.y * ln.y + N.y * ln.z,
                     Tg.z * ln.x + Bt.z * ln.y + N.z * ln.z};
        T m2 = dot(mapped, mapped);
        if (!(m2 > T(1e-12f))) return N;
        mapped = mapped * (T(1) / std::sqrt(m2));
        if (!(dot(mapped, N) > T(1e-4f))) return N;
        return mapped;
    }
    return is.normal;
}

// The normal-map texel get_normal hands out (src/material_queries.cu:32-40); (0.5, 0.5, 1)
// without a normal texture (:83-85).
template <class T> V3<T> normal_map_texel(const orc_scene& s, const lux_material_desc& m, V2<T> uv) {
    if (m.normal_tex < 0) return {T(0.5f), T(0.5f), T(1.0f)};
    uv = apply_tt(uv, m.normal_tt);
    T tx[4];
    tex_fetch(s.texs[m.normal_tex], uv.x, uv.y, tx);
    return {tx[0], tx[1], tx[2]};
}

// get_alpha (src/material_queries.cu:119-137)
template <class T> T get_alpha(const orc_scene& s, const lux_material_desc& m, V2<T> uv) {
    if (m.alpha_mode == LUX_ALPHA_OPAQUE) return T(1);
    T alpha = T(m.alpha);
    if (m.albedo_tex >= 0) {
        uv = apply_tt(uv, m.albedo_tt);
        T tx[4];
        tex_fetch(s.texs[m.albedo_tex], uv.x, uv.y, tx);
        alpha *= tx[3];
    }
    if (m.alpha_mode == LUX_ALPHA_MASK) return alpha >= T(m.alpha_cutoff) ? T(1) : T(0);
    return alpha;
}

template <class T> void get_metallic_roughness(const orc_scene& s, const lux_material_desc& m, V2<T> uv, T& r, T& mt) {
    r = T(m.roughness);
    mt = T(m.metallic);
    if (m.metallic_roughness_tex >= 0) {
        uv = apply_tt(uv, m.metallic_roughness_tt);
        T tx[4];
        tex_fetch(s.texs[m.metallic_roughness_tex], uv.x, uv.y, tx);
        r *= tx[1];
        mt *= tx[2];
    }
}

template <class T> V3<T> get_emission(const orc_scene& s, const lux_material_desc& m, V2<T> uv) {
    V3<T> e = V3<T>(T(m.emission_color[0]), T(m.emission_color[1]), T(m.emission_color[2])) * T(m.emission_strength);
    if (m.emissive_tex >= 0) {
        uv = apply_tt(uv, m.emissive_tt);
        T tx[4];
        tex_fetch(s.texs[m.emissive_tex], uv.x, uv.y, tx);
        e = e * vpow(V3<T>(tx[0], tx[1], tx[2]), T(2.2f));
    }
    return e;
}

// ---------------------------------------------------------------------------------------
// Cook-Torrance uber-shader (src/shaders/cook_torrance.cu:8-331)
template <class T> T D_GGX(V3<T> h, V3<T> n, T alpha) {
    T ndh = dot(n, h);
    if (ndh <= T(0)) return T(0);
    T a2 = alpha * alpha;
    T ndh2 = ndh * ndh;
    T dc = (ndh2 * a2) + (T(1) - ndh2);
    T den = dc * dc * T(kPI);
    return a2 / gmax(den, T(kEPS_CT));
}
template <class T> V3<T> F_schlick(T vdh, V3<T> f0) {
    T m = T(1) - vdh;
    T m2 = m * m;
    return f0 + ((V3<T>(T(1), T(1), T(1)) - f0) * (m2 * m2 * m));
}
template <class T> T F_dielectric(T cosI, T etaI, T etaT) {
    cosI = gclamp(cosI, T(0), T(1));
    T sinI = std::sqrt(gmax(T(0), T(1) - cosI * cosI));
    T sinT = (etaI / etaT) * sinI;
    if (sinT >= T(1)) return T(1);
    T cosT = std::sqrt(gmax(T(0), T(1) - sinT * sinT));
    T rpar = ((etaT * cosI) - (etaI * cosT)) / ((etaT * cosI) + (etaI * cosT));
    T rper = ((etaI * cosI) - (etaT * cosT)) / ((etaI * cosI) + (etaT * cosT));
    return (rpar * rpar + rper * rper) / T(2);
}
template <class T> V3<T> half_t(V3<T> wo, V3<T> wi, T etaI, T etaT) { return normalize(-(etaI * wo + etaT * wi)); }
template <class T> T smith_ggx(V3<T> w, V3<T> n, T alpha) {
    T a2 = alpha * alpha;
    T ndw = gmax(dot(n, w), T(0));
    T num = T(2) * ndw;
    T us = a2 + (T(1) - a2) * (ndw * ndw);
    T den = ndw + std::sqrt(us);
    return num / gmax(den, T(kEPS_CT));
}
template <class T> V3<T> fresnel(T c, V3<T> albedo, T metallic, T etaI, T etaT) {
    T d = F_dielectric(c, etaI, etaT);
    return vmix(V3<T>(d, d, d), F_schlick(c, albedo), metallic);
}
template <class T> V3<T> BRDF(V3<T> v, V3<T> n, V3<T> l, V3<T> albedo, T rough, T metal, T ior, T trans) {
    ior = gmax(ior, T(1.0001f));
    bool enter = dot(v, n) > T(0);
    V3<T> nf = enter ? n : -n;
    T etaI = enter ? T(1) : ior, etaT = enter ? ior : T(1);
    V3<T> h = normalize(v + l);
    rough = gclamp(rough, T(0.0001f), T(1));
    T alpha = rough * rough;
    T D = D_GGX(h, nf, alpha);
    V3<T> F = fresnel(gmax(dot(v, h), T(0)), albedo, metal, etaI, etaT);
    T G = smith_ggx(v, nf, alpha) * smith_ggx(l, nf, alpha);
    V3<T> num = D * F * G;
    T den = T(4) * gmax(dot(nf, v), T(0)) * gmax(dot(nf, l), T(0));
    V3<T> spec = num / gmax(den, T(kEPS_CT));
    V3<T> nonspec = V3<T>(T(1), T(1), T(1)) - F;
    V3<T> kD = (T(1) - metal) * nonspec * (T(1) - trans);
    V3<T> diffuse = kD * albedo * T(kINV_PI);
    return diffuse + spec;
}
template <class T> V3<T> BTDF(V3<T> wo, V3<T> n, V3<T> wi, V3<T> albedo, T rough, T metal, T ior, T trans) {
    T cI = dot(wo, n);
    bool enter = cI > T(0);
    T etaI = enter ? T(1) : ior, etaT = enter ? ior : T(1);
    V3<T> ht = half_t(wo, wi, etaI, etaT);
    T jd = (etaT * dot(wi, ht) + etaI * dot(wo, ht));
    T jac = (etaI * etaI) / gmax(jd * jd, T(kEPS_CT));
    T cnum = std::fabs(dot(wi, ht)) * std::fabs(dot(wo, ht));
    T cden = std::fabs(dot(wi, n)) * std::fabs(dot(wo, n));
    rough = gclamp(rough, T(0.0001f), T(1));
    T alpha = rough * rough;
    T D = D_GGX(ht, n, alpha);
    T F = F_dielectric(std::fabs(dot(wo, ht)), etaI, etaT);
    bool gvis = dot(wi, ht) * dot(wi, n) > T(0) && dot(wo, ht) * dot(wo, n) > T(0);
    T G = gvis ? smith_ggx(dot(wi, n) > T(0) ? wi : -wi, n, alpha) * smith_ggx(dot(wo, n) > T(0) ? wo : -wo, n, alpha)
               : T(0);
    T DFG = D * G * (T(1) - F);
    return albedo * (trans * (T(1) - metal) * (cnum / cden) * jac * DFG);
}
template <class T> V3<T> sph2cart(T r, T theta, T phi) {
    return {r * std::sin(theta) * std::cos(phi), r * std::sin(theta) * std::sin(phi), r * std::cos(theta)};
}

// calculateRandomDirectionInHemisphere (src/interactions.cu:7-45)
template <class T> V3<T> hemisphere(V3<T> normal, MinStd& rng) {
    T up = std::sqrt(rng.u01<T>());
    T over = std::sqrt(T(1) - up * up);
    T around = rng.u01<T>() * T(kTWO_PI);
    V3<T> dnn;
    if (std::fabs(normal.x) < T(kSQRT13)) dnn = V3<T>(T(1), T(0), T(0));
    else if (std::fabs(normal.y) < T(kSQRT13)) dnn = V3<T>(T(0), T(1), T(0));
    else dnn = V3<T>(T(0), T(0), T(1));
    V3<T> p1 = normalize(cross(normal, dnn));
    V3<T> p2 = normalize(cross(normal, p1));
    return up * normal + std::cos(around) * over * p1 + std::sin(around) * over * p2;
}

// CookTorrance::sampleCookTorrance (src/shaders/cook_torrance.cu:156-224)
template <class T>
V3<T> sample_ct(V3<T> wo, V3<T> n, T rough, T metal, MinStd& rng, V3<T> color, T ior, T trans) {
    T r = rng.u01<T>();
    ior = gmax(ior, T(1.0001f));
    rough = gclamp(rough, T(0.0001f), T(1));
    T alpha = rough * rough;
    bool enter = dot(wo, n) > T(0);
    V3<T> nf = enter ? n : -n;
    T etaI = enter ? T(1) : ior, etaT = enter ? ior : T(1);
    T cm = std::fabs(dot(wo, n));
    V3<T> Fa = fresnel(cm, color, metal, etaI, etaT);
    T sr = gclamp((Fa.x + Fa.y + Fa.z) / T(3), T(0.01f), T(0.99f));
    T Fm = F_dielectric(cm, etaI, etaT);
    T pR = trans * (T(1) - metal) * (T(1) - Fm);
    T pD = (T(1) - pR) * (T(1) - sr) * (T(1) - metal);
    T pS = T(1) - pR - pD;
    if (r > pS && r <= pS + pD) return hemisphere(nf, rng);
    T x1 = rng.u01<T>(), x2 = rng.u01<T>();
    T th = std::atan((alpha * std::sqrt(x1)) / std::sqrt(T(1) - x1));
    T ph = T(2) * T(kPI) * x2;
    V3<T> h = normalize(sph2cart(T(1), th, ph));
    V3<T> t = normalize(std::fabs(nf.z) < T(0.999f) ? cross(V3<T>(T(0), T(0), T(1)), nf)
                                                    : cross(V3<T>(T(1), T(0), T(0)), nf));
    V3<T> b = cross(nf, t);
    V3<T> hw = h.x * t + h.y * b + h.z * nf;
    if (r <= pS) {
        V3<T> wi = reflect(-wo, hw);
        if (dot(wi, nf) <= T(0)) return V3<T>();
        return normalize(wi);
    }
    V3<T> wi = refract(-wo, hw, etaI / etaT);
    if (dot(wi, wi) < T(kEPS_CT) || std::isnan(wi.x) || std::isnan(wi.y) || std::isnan(wi.z) || dot(wi, nf) >= T(0))
        return V3<T>();
    return normalize(wi);
}

template <class T> T pdf_ggx(V3<T> wo, V3<T> wi, V3<T> n, T rough) {
    V3<T> h = normalize(wo + wi);
    rough = gclamp(rough, T(0.0001f), T(1));
    T alpha = rough * rough;
    T ph = D_GGX(h, n, alpha) * dot(n, h);
    return ph / gmax((T(4) * std::fabs(dot(wo, h))), T(kEPS_CT));
}
template <class T> T pdf_ggx_t(V3<T> wo, V3<T> wi, V3<T> n, T rough, T ior) {
    T cI = dot(wo, n);
    bool enter = cI > T(0);
    T etaI = enter ? T(1) : ior, etaT = enter ? ior : T(1);
    V3<T> ht = half_t(wo, wi, etaI, etaT);
    rough = gclamp(rough, T(0.0001f), T(1));
    T alpha = rough * rough;
    T den = etaT * dot(wi, ht) + etaI * dot(wo, ht);
    T ph = D_GGX(ht, n, alpha) * std::fabs(dot(n, ht));
    return ph * (etaT * etaT * std::fabs(dot(wi, ht))) / gmax(den * den, T(kEPS_CT));
}
template <class T> T PDF(V3<T> wo, V3<T> wi, V3<T> n, T rough, T metal, V3<T> color, T ior, T trans) {
    ior = gmax(ior, T(1.0001f));
    V3<T> nf = dot(wo, n) < T(0) ? -n : n;
    T pdfD = std::max(T(0), dot(wi, nf)) * T(kINV_PI);
    T pdfS = pdf_ggx(wo, wi, nf, rough);
    T pdfR = pdf_ggx_t(wo, wi, n, rough, ior);
    bool refr = (dot(wi, n) * dot(wo, n)) < T(0);
    bool enter = dot(wo, n) > T(0);
    T etaI = enter ? T(1) : ior, etaT = enter ? ior : T(1);
    T cm = std::fabs(dot(wo, n));
    V3<T> Fa = fresnel(cm, color, metal, etaI, etaT);
    T sr = gclamp((Fa.x + Fa.y + Fa.z) / T(3), T(0.01f), T(0.99f));
    T Fm = F_dielectric(cm, etaI, etaT);
    T pR = trans * (T(1) - metal) * (T(1) - Fm);
    T pD = (T(1) - pR) * (T(1) - sr) * (T(1) - metal);
    T pS = T(1) - pR - pD;
    T pdf = refr ? pR * pdfR : pD * pdfD + pS * pdfS;
    return gmax(pdf, T(kPDF_CLAMP));
}
template <class T> V3<T> shade_ct(V3<T> wo, V3<T> albedo, V3<T> normal, V3<T> wi, T rough, T metal, T ior, T trans) {
    ior = gmax(ior, T(1.0001f));
    bool refr = (dot(wi, normal) * dot(wo, normal)) < T(0);
    V3<T> f = refr ? BTDF(wo, normal, wi, albedo, rough, metal, ior, trans)
                   : BRDF(wo, normal, wi, albedo, rough, metal, ior, trans);
    return f * std::fabs(dot(wi, normal));
}

// ---------------------------------------------------------------------------------------
// Path state (include/sceneStructs.h:154-166)
template <class T> struct Path {
    V3<T> o, d, color, thr, dl, env;
    int pixel = 0;
    bool kill = false, spec = false;
    T last_pdf = T(-1);
};

template <class T> void path_load(Path<T>& p, const float* f) {
    p.o = {T(f[0]), T(f[1]), T(f[2])};
    p.d = {T(f[3]), T(f[4]), T(f[5])};
    p.color = {T(f[6]), T(f[7]), T(f[8])};
    p.thr = {T(f[9]), T(f[10]), T(f[11])};
    p.dl = {T(f[12]), T(f[13]), T(f[14])};
    p.env = {T(f[15]), T(f[16]), T(f[17])};
    int32_t px;
    std::memcpy(&px, &f[18], 4);
    p.pixel = px;
    p.kill = f[19] != 0.0f;
    p.spec = f[20] != 0.0f;
    p.last_pdf = T(f[21]);
}
template <class T> void path_store(const Path<T>& p, float* f) {
    float v[18] = {float(p.o.x), float(p.o.y), float(p.o.z), float(p.d.x), float(p.d.y), float(p.d.z),
                   float(p.color.x), float(p.color.y), float(p.color.z), float(p.thr.x), float(p.thr.y),
                   float(p.thr.z), float(p.dl.x), float(p.dl.y), float(p.dl.z), float(p.env.x),
                   float(p.env.y), float(p.env.z)};
    std::memcpy(f, v, sizeof(v));
    int32_t px = p.pixel;
    std::memcpy(&f[18], &px, 4);
    f[19] = p.kill ? 1.0f : 0.0f;
    f[20] = p.spec ? 1.0f : 0.0f;
    f[21] = float(p.last_pdf);
    f[22] = 0.0f;
    f[23] = 0.0f;
}

template <class T> struct Cdfs {
    const std::vector<T>* em;
    const std::vector<std::vector<T>>* tri;
    T total;
    const std::vector<T>* marg;
    const std::vector<T>* cond;
};
template <class T> Cdfs<T> cdfs_of(const orc_scene& s);
template <> Cdfs<float> cdfs_of<float>(const orc_scene& s) {
    return {&s.emissive_prefix, &s.tri_prefix, s.total_area, &s.marginal, &s.conditional};
}
template <> Cdfs<double> cdfs_of<double>(const orc_scene& s) {
    return {&s.emissive_prefix_d, &s.tri_prefix_d, s.total_area_d, &s.marginal_d, &s.conditional_d};
}

// generateRayFromCamera (src/kernels/generate_ray_from_camera.cu:8-39)
template <class T> void camera_ray(const orc_scene& s, int iter, int index, int tdepth, Path<T>& p) {
    const lux_camera_desc& c = s.cam;
    int x = index % c.width, y = index / c.width;
    p.o = {T(c.position[0]), T(c.position[1]), T(c.position[2])};
    p.color = V3<T>();
    p.thr = V3<T>(T(1), T(1), T(1));
    p.kill = false;
    MinStd rng = seeded(iter, index, tdepth);
    T x1 = rng.u01<T>() - T(0.5f);
    T x2 = rng.u01<T>() - T(0.5f);
    T pX = (T(x) + x1 + T(0.5f)) - T(c.width) * T(0.5f);
    T pY = (T(y) + x2 + T(0.5f)) - T(c.height) * T(0.5f);
    V3<T> view{T(c.view[0]), T(c.view[1]), T(c.view[2])};
    V3<T> right{T(c.right[0]), T(c.right[1]), T(c.right[2])};
    V3<T> up{T(c.up[0]), T(c.up[1]), T(c.up[2])};
    p.d = normalize(view - (right * T(c.pixel_length[0]) * pX) - (up * T(c.pixel_length[1]) * pY));
    p.pixel = index;
}

// sampleDirectLight (src/kernels/sample_direct_light.cu:9-101). With both -dmis and -emis
// the DL draws still precede the env draw.
template <class T> void light_sample(const orc_scene& s, const lux_options& opt, int iter, int depth, Path<T>& p) {
    if (p.kill) return;
    MinStd rng = seeded(iter, p.pixel, depth);
    Cdfs<T> cd = cdfs_of<T>(s);
    if (opt.direct_light_sampling) {
        T rnd = rng.u01<T>();
        int ne = int(cd.em->size());
        int sel = select_from_cdf(cd.em->data(), ne, rnd);
        const Inst& g = s.insts[s.emissive[sel]];
        const Mesh& m = s.meshes[g.mesh];
        T lower = (sel == 0) ? T(0) : (*cd.em)[sel - 1];
        T upper = (*cd.em)[sel];
        T den = upper - lower;
        T off = (den > T(1e-10f)) ? (rnd - lower) / den : T(0);
        off = gclamp(off, T(0), T(1));
        const std::vector<T>& tp = (*cd.tri)[s.emissive[sel]];
        int ts = select_from_cdf(tp.data(), m.nt, off);
        V3<T> v0 = mesh_pos<T>(m, m.idx[ts * 3]), v1 = mesh_pos<T>(m, m.idx[ts * 3 + 1]),
              v2 = mesh_pos<T>(m, m.idx[ts * 3 + 2]);
        T r1 = std::sqrt(rng.u01<T>());
        T r2 = rng.u01<T>();
        T u = T(1) - r1, v = r2 * r1;
        V3<T> lp = u * v0 + v * v1 + (T(1) - u - v) * v2;
        p.dl = mul_point<T>(g.M, lp, T(1));
    }
    if (opt.env_importance_sampling) {
        T rnd = rng.u01<T>();
        int H = s.env.h, W = s.env.w;
        int mg = select_from_cdf(cd.marg->data(), H, rnd);
        T lower = (mg == 0) ? T(0) : (*cd.marg)[mg - 1];
        T upper = (*cd.marg)[mg];
        T den = upper - lower;
        T off = (den > T(1e-10f)) ? (rnd - lower) / den : T(0);
        off = gclamp(off, T(0), T(1));
        int cn = select_from_cdf(cd.cond->data() + size_t(mg) * W, W, off);
        T u = (T(cn) + T(0.5f)) / T(W);
        T v = (T(mg) + T(0.5f)) / T(H);
        T phi = T(double(u) * 2.0 * double(kPI) - double(kPI));
        T theta = v * T(kPI);
        T st = std::sin(theta);
        p.env = {st * std::cos(phi), std::cos(theta), st * std::sin(phi)};
    }
}

// envmap_pdf (src/kernels/shade_path.cu:27-42)
template <class T> T envmap_pdf(const orc_scene& s, V3<T> d) {
    Cdfs<T> cd = cdfs_of<T>(s);
    int W = s.env.w, H = s.env.h;
    T phi = std::atan2(d.z, d.x);
    T theta = std::acos(gclamp(d.y, T(-1), T(1)));
    T u = (phi + T(kPI)) / (T(2) * T(kPI));
    T v = theta / T(kPI);
    int col = gclamp(int(u * T(W)), 0, W - 1);
    int row = gclamp(int(v * T(H)), 0, H - 1);
    const std::vector<T>& mg = *cd.marg;
    const std::vector<T>& cn = *cd.cond;
    T pm = (mg[row] - (row == 0 ? T(0) : mg[row - 1])) * T(H);
    T pc = (cn[size_t(row) * W + col] - (col == 0 ? T(0) : cn[size_t(row) * W + col - 1])) * T(W);
    T st = std::sin(theta);
    return (st > T(1e-6f)) ? (pm * pc) / (T(2) * T(kPI) * T(kPI) * st) : T(0);
}

// env radiance lookup as in the shader (src/kernels/shade_path.cu:207-215,309-318): the
// uv mapping is evaluated in double with M_PI = 3.14159.
template <class T> V3<T> env_lookup(const orc_scene& s, V3<T> d, float intensity) {
    T phi = std::atan2(d.z, d.x);
    T theta = std::acos(gclamp(d.y, T(-1), T(1)));
    T u = T((double(phi) + kM_PI_SHADE) * (double(1.0f) / (double(2.0f) * kM_PI_SHADE)));
    T v = T(double(theta) * (double(1.0f) / kM_PI_SHADE));
    T tx[4];
    tex_fetch(s.env, u, v, tx);
    return V3<T>(tx[0], tx[1], tx[2]) * T(intensity);
}

struct ShadeIn {
    Hit rad, shadow;
};

// shadePath for one path (src/kernels/shade_path.cu:94-364). Returns true when the path
// survives into the next queue.
template <class T>
bool shade_path(const orc_scene& s, const lux_options& opt, int iter, int depth, bool compact, Path<T>& path,
                const HitT<T>& rh, const HitT<T>& sh, T env_occ) {
    MinStd rng = seeded(iter, path.pixel, depth);
    Cdfs<T> cd = cdfs_of<T>(s);
    bool has_exr = s.has_env;
    Isect<T> is;
    if (rh.inst >= 0) is = ch_radiance(s, rh);
    if (rh.inst >= 0 && is.t > T(0)) {
        const lux_material_desc& mat = s.mats[is.material];
        V3<T> mc = get_albedo(s, mat, is.uv);
        V3<T> normal = get_normal(s, mat, is);
        T rough, metal;
        get_metallic_roughness(s, mat, is.uv, rough, metal);
        if (opt.material_debug_mode) {
            // render_material_debug_mode (src/material_debug_render.cu:3-26) replaces the
            // colour and kills the path; shade_path.cu:154-164 skips the lighting
            const int md = opt.material_debug_mode;
            V3<T> c{T(0), T(0), T(0)};
            if (md == 1) c = mc;
            else if (md == 2) c = normal * T(0.5f) + V3<T>(T(0.5f), T(0.5f), T(0.5f));
            else if (md == 3) c = normal_map_texel(s, mat, is.uv);
            else if (md == 4) c = V3<T>(rough, rough, rough);
            else if (md == 5) c = V3<T>(metal, metal, metal);
            else if (md == 6) {
                T a = get_alpha(s, mat, is.uv);
                c = V3<T>(a, a, a);
            }
            path.color = c;
            path.kill = true;
            return false;
        }
        V3<T> emission = get_emission(s, mat, is.uv);
        bool is_spec = rough < T(kSPEC_ROUGH);
        V3<T> nf = dot(-path.d, normal) < T(0) ? -normal : normal;
        T ior = T(mat.ior), trans = T(mat.transmission);
        V3<T> sample_dir = sample_ct(-path.d, normal, rough, metal, rng, mc, ior, trans);
        bool emissive = length(emission) > T(kEPS_UTIL);
        if (opt.env_importance_sampling) {
            if (emissive) {
                T w = T(1);
                if (depth > 1 && !path.spec) {
                    T pb = path.last_pdf;
                    T pe = envmap_pdf(s, path.d);
                    w = (pb * pb) / (pb * pb + pe * pe);
                }
                path.color = path.color + path.thr * (w * emission);
                path.kill = true;
            } else if (env_occ < T(0) && !is_spec && !path.kill && has_exr) {
                V3<T> ed = path.env;
                T pee = envmap_pdf(s, ed);
                T pbe = PDF(-path.d, ed, normal, rough, metal, mc, ior, trans);
                T w = (pee * pee) / (pee * pee + pbe * pbe);
                V3<T> brdf = BRDF(-path.d, normal, ed, mc, rough, metal, ior, trans);
                V3<T> el = env_lookup(s, normalize(ed), opt.envmap_intensity);
                T cs = dot(nf, ed);
                if (cs > T(0) && pee > T(1e-8f)) {
                    V3<T> contrib = (el * brdf * cs) / pee;
                    path.color = path.color + path.thr * contrib * w;
                }
            }
        } else if (opt.direct_light_sampling) {
            if (emissive) {
                T w = T(1);
                if (depth > 1 && !path.spec) {
                    T pb = path.last_pdf;
                    T dsq = is.t * is.t;
                    T cl = dot(is.normal, -path.d);
                    if (cl > T(0.0001f)) {
                        T pa = T(1) / cd.total;
                        T ps = pa * (dsq / cl);
                        w = (pb * pb) / (pb * pb + ps * ps);
                    } else {
                        w = T(0);
                    }
                }
                path.color = path.color + path.thr * (w * emission);
                path.kill = true;
            } else if (sh.inst >= 0 && sh.t > T(0) && !is_spec && !path.kill) {
                Isect<T> dli = ch_direct_light(s, sh);
                V3<T> sp = is.t * path.d + path.o;
                V3<T> lv = path.dl - sp;
                T dsq = dot(lv, lv);
                T dist = std::sqrt(dsq);
                V3<T> ld = lv / dist;
                T cs = dot(nf, ld);
                T cl = dot(dli.normal, -ld);
                if (cs > T(0) && cl > T(0)) {
                    T pa = T(1) / cd.total;
                    T ps = pa * (dsq / cl);
                    T pb = PDF(-path.d, ld, normal, rough, metal, mc, ior, trans);
                    T w = (ps * ps) / (ps * ps + pb * pb);
                    V3<T> brdf = BRDF(-path.d, normal, ld, mc, rough, metal, ior, trans);
                    V3<T> lr = get_emission(s, s.mats[dli.material], dli.uv);
                    V3<T> contrib = (lr * brdf * cs) / ps;
                    path.color = path.color + path.thr * contrib * w;
                }
            }
        } else if (emissive) {
            path.color = path.color + path.thr * emission;
            path.kill = true;
        }
        if (!path.kill) {
            // update_throughput_materials (src/update_throughput_materials.cu:23-67)
            bool transmitted = dot(-path.d, normal) * dot(sample_dir, normal) < T(0);
            bool spec = is_spec || transmitted;
            V3<T> f = shade_ct(-path.d, mc, normal, sample_dir, rough, metal, ior, trans);
            T pdf = PDF(-path.d, sample_dir, normal, rough, metal, mc, ior, trans);
            path.thr = path.thr * (f / pdf);
            path.last_pdf = pdf;
            path.spec = spec;
            if (depth >= kRR_MIN_DEPTH) {
                T mx = gmax(path.thr.x, gmax(path.thr.y, path.thr.z));
                T surv = gclamp(mx, T(0), T(1));
                if (rng.u01<T>() >= surv) path.kill = true;
                else path.thr = path.thr / surv;
            }
        }
        // spawn the next ray (shade_path.cu:333-353, getPointOnRay include/intersections.h:29-32);
        // the reference runs it for paths killed above as well
        V3<T> hp = path.o + (is.t - T(.0001f)) * normalize(path.d);
        T sl2 = dot(sample_dir, sample_dir);
        if (!(sl2 > T(1e-12f)) || !std::isfinite(sl2)) {
            path.kill = true;
            return false;
        }
        path.d = sample_dir;
        if (dot(path.d, is.normal) > T(0)) path.o = hp + (is.normal * T(kGLASS_EPS));
        else path.o = hp - (is.normal * T(kGLASS_EPS));
        return compact && !path.kill;
    }
    if (!path.kill && has_exr) {
        V3<T> d = normalize(path.d);
        V3<T> er = env_lookup(s, d, opt.envmap_intensity);
        T w = T(1);
        if (opt.env_importance_sampling && depth > 1 && !path.spec) {
            T pb = path.last_pdf;
            T pe = envmap_pdf(s, d);
            w = (pb * pb) / (pb * pb + pe * pe);
        }
        path.color = path.color + path.thr * er * w;
    }
    path.kill = true;
    return false;
}

// Shadow rays of the raygen program (src/optixshaders/optix_triangle.cu:82-136): origin is
// hit + surfaceNormal*1e-4 with the raw world normal; the DL ray runs to dist*1.0001+1e-4.
template <class T>
void trace_shadow(const orc_scene& s, const lux_options& opt, int iter, const Path<T>& p, const HitT<T>& rh,
                  bool brute, HitT<T>& sh, T& env_occ, long long& nrays) {
    sh = HitT<T>();
    env_occ = T(-0.5f);
    if (rh.inst < 0) return;
    Isect<T> is = ch_radiance(s, rh);
    V3<T> hp = p.o + is.t * p.d;
    V3<T> so = hp + (is.normal * T(1e-4f));
    if (opt.env_importance_sampling) {
        HitT<T> tmp;
        bool occ = trace_ray(s, so, p.env, T(1e16f), 2, p.pixel, iter, brute, tmp);
        env_occ = occ ? T(1) : T(-1);
        ++nrays;
    } else if (opt.direct_light_sampling) {
        V3<T> ld = p.dl - so;
        T dist = length(ld);
        ld = ld * (T(1) / dist);
        trace_ray(s, so, ld, dist * T(1.0001f) + T(1e-4f), 1, p.pixel, iter, brute, sh);
        ++nrays;
    }
}

inline void write_hit(const Hit& h, uint32_t* w) {
    std::memcpy(&w[0], &h.t, 4);
    w[1] = uint32_t(h.inst);
    w[2] = uint32_t(h.prim);
    std::memcpy(&w[3], &h.u, 4);
    std::memcpy(&w[4], &h.v, 4);
}
inline Hit read_hit(const uint32_t* w) {
    Hit h;
    std::memcpy(&h.t, &w[0], 4);
    h.inst = int32_t(w[1]);
    h.prim = int32_t(w[2]);
    std::memcpy(&h.u, &w[3], 4);
    std::memcpy(&h.v, &w[4], 4);
    return h;
}
inline HitT<float> to_ht(const Hit& h) {
    HitT<float> r;
    r.t = h.t;
    r.inst = h.inst;
    r.prim = h.prim;
    r.u = h.u;
    r.v = h.v;
    if (h.inst < 0) r.t = -1.0f;
    return r;
}

// Morton key (src/kernels/intersection_precompute.cu:6-33, src/morton_codes.cu:13-24,
// include/morton_codes.h:12-38), including the reference slab test
// (src/mesh/bounding_box.cu:7-40).
inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
inline uint32_t morton3d(float x, float y, float z) {
    x = std::fmin(std::fmax(x * 1024.0f, 0.0f), 1023.0f);
    y = std::fmin(std::fmax(y * 1024.0f, 0.0f), 1023.0f);
    z = std::fmin(std::fmax(z * 1024.0f, 0.0f), 1023.0f);
    return (expand_bits(uint32_t(x)) << 2) | (expand_bits(uint32_t(y)) << 1) | expand_bits(uint32_t(z));
}
uint32_t morton_key(const orc_scene& s, V3<float> o, V3<float> d) {
    const Inst& g = s.insts[0];
    V3<float> ro = mul_point<float>(g.Minv, o, 1.0f);
    V3<float> rd = mul_point<float>(g.Minv, d, 0.0f);
    V3<float> inv{1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z};
    int sx = inv.x < 0.0f, sy = inv.y < 0.0f, sz = inv.z < 0.0f;
    V3<float> bmin{s.morton_bmin[0], s.morton_bmin[1], s.morton_bmin[2]};
    V3<float> bmax{s.morton_bmax[0], s.morton_bmax[1], s.morton_bmax[2]};
    V3<float> bounds[2] = {bmin, bmax};
    float tmin = (bounds[sx].x - ro.x) * inv.x;
    float tmax = (bounds[1 - sx].x - ro.x) * inv.x;
    float tymin = (bounds[sy].y - ro.y) * inv.y;
    float tymax = (bounds[1 - sy].y - ro.y) * inv.y;
    bool hit = true;
    if (tmin > tymax || tymin > tmax) hit = false;
    if (hit) {
        tmin = gmax(tmin, tymin);
        tmax = gmin(tmax, tymax);
        float tzmin = (bounds[sz].z - ro.z) * inv.z;
        float tzmax = (bounds[1 - sz].z - ro.z) * inv.z;
        if (tmin > tzmax || tzmin > tmax) hit = false;
        else {
            tmin = gmax(tmin, tzmin);
            if (tmax < 0.0f) hit = false;
            else hit = tmin < tmax;
        }
    }
    if (!hit) return 0xFFFFFFFFu;
    float ext = length(bmax - bmin);
    auto normp = [&](V3<float> p) {
        return V3<float>((p.x + ext) / (2.0f * ext), (p.y + ext) / (2.0f * ext), (p.z + ext) / (2.0f * ext));
    };
    V3<float> p0 = normp(ro);
    V3<float> far = ro + (rd * 1.0f);
    V3<float> p1 = normp(far);
    V3<float> mid = 0.5f * (p0 + p1);
    return morton3d(mid.x, mid.y, mid.z);
}

template <class T>
void render_path(const orc_scene& s, const lux_options& opt, int iter, int pixel, V3<T>& color, double* st) {
    Path<T> p;
    int tdepth = opt.trace_depth > 0 ? opt.trace_depth : s.trace_depth;
    if (opt.material_debug_mode) tdepth = 1;  // src/pathtrace.cu:107
    camera_ray(s, iter, pixel, tdepth, p);
    int depth = 0;
    bool nee = opt.direct_light_sampling || opt.env_importance_sampling;
    if (nee) light_sample(s, opt, iter, depth, p);
    long long nsh = 0;
    while (true) {
        HitT<T> rh;
        trace_ray(s, p.o, p.d, T(1e16f), 0, p.pixel, iter, false, rh);
        st[0] += 1;
        HitT<T> sh;
        T eo;
        trace_shadow(s, opt, iter, p, rh, false, sh, eo, nsh);
        ++depth;
        st[2] += 1;
        bool alive = shade_path(s, opt, iter, depth, depth < tdepth, p, rh, sh, eo);
        if (!alive || depth >= tdepth) break;
        if (nee) light_sample(s, opt, iter, depth, p);
    }
    st[1] += double(nsh);
    color = p.color;
}

inline void acesfilm(float* c) {  // src/tonemapping.cu:3-11
    for (int i = 0; i < 3; ++i) {
        float x = c[i];
        c[i] = gclamp((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.0f, 1.0f);
    }
}
inline void agx(float* v) {  // src/tonemapping.cu:13-30
    for (int i = 0; i < 3; ++i) {
        v[i] = gmax(v[i], 1e-6f);
        v[i] = (std::log2(v[i]) + 10.0f) / 16.0f;
        v[i] = gclamp(v[i], 0.0f, 1.0f);
        float x2 = v[i] * v[i], x4 = x2 * x2;
        v[i] = 15.5f * x4 * v[i] - 40.14f * x4 + 31.96f * x2 * v[i] - 6.86f * x2 + 0.429f * v[i] + 0.0322f;
    }
    float r = v[0] * 1.1968790f - v[1] * 0.0980208f - v[2] * 0.0990297f;
    float g = -v[0] * 0.0528968f + v[1] * 1.1519031f - v[2] * 0.0989611f;
    float b = -v[0] * 0.0529716f - v[1] * 0.0980434f + v[2] * 1.1510736f;
    v[0] = gclamp(r, 0.0f, 1.0f);
    v[1] = gclamp(g, 0.0f, 1.0f);
    v[2] = gclamp(b, 0.0f, 1.0f);
}

}  // namespace

// =======================================================================================
extern "C" {

uint32_t orc_utilhash(uint32_t a) { return utilhash(a); }

void orc_rng_stream(int iter, int index, int depth, int n, float* out) {
    MinStd r = seeded(iter, index, depth);
    for (int i = 0; i < n; ++i) out[i] = r.u01<float>();
}

int orc_select_from_cdf(const float* cdf, int size, float xi) { return select_from_cdf(cdf, size, xi); }

void orc_eval_bsdf(const float* in, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        const float* r = in + i * 16;
        V3<float> wo{r[0], r[1], r[2]}, nn{r[3], r[4], r[5]}, wi{r[6], r[7], r[8]}, al{r[9], r[10], r[11]};
        float ro = r[12], me = r[13], ior = r[14], tr = r[15];
        float* o = out + i * 16;
        V3<float> b = BRDF(wo, nn, wi, al, ro, me, ior, tr);
        V3<float> t = BTDF(wo, nn, wi, al, ro, me, gmax(ior, 1.0001f), tr);
        V3<float> sh = shade_ct(wo, al, nn, wi, ro, me, ior, tr);
        float pdf = PDF(wo, wi, nn, ro, me, al, ior, tr);
        float rc = gclamp(ro, 0.0001f, 1.0f);
        V3<float> h = normalize(wo + wi);
        float D = D_GGX(h, nn, rc * rc);
        float G = smith_ggx(wo, nn, rc * rc) * smith_ggx(wi, nn, rc * rc);
        float Fd = F_dielectric(dot(nn, wo), 1.0f, gmax(ior, 1.0001f));
        V3<float> Fs = F_schlick(gmax(dot(wo, h), 0.0f), al);
        V3<float> Fm = fresnel(gmax(dot(wo, h), 0.0f), al, me, 1.0f, gmax(ior, 1.0001f));
        float v[16] = {b.x, b.y, b.z, t.x, t.y, t.z, sh.x, sh.y, sh.z, pdf, D, G, Fd, Fs.x, Fm.x, 0.0f};
        std::memcpy(o, v, sizeof(v));
    }
}

void orc_sample_bsdf(const float* in, const int* seeds, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        const float* r = in + i * 16;
        V3<float> wo{r[0], r[1], r[2]}, nn{r[3], r[4], r[5]}, al{r[9], r[10], r[11]};
        MinStd rng = seeded(seeds[i * 3], seeds[i * 3 + 1], seeds[i * 3 + 2]);
        MinStd ref = rng;
        V3<float> d = sample_ct(wo, nn, r[12], r[13], rng, al, r[14], r[15]);
        int used = 0;
        while (ref.x != rng.x && used < 16) { ref.next(); ++used; }
        out[i * 4] = d.x;
        out[i * 4 + 1] = d.y;
        out[i * 4 + 2] = d.z;
        out[i * 4 + 3] = float(used);
    }
}

void orc_hemisphere(const float* normals, const int* seeds, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        MinStd rng = seeded(seeds[i * 3], seeds[i * 3 + 1], seeds[i * 3 + 2]);
        V3<float> d = hemisphere(V3<float>(normals[i * 3], normals[i * 3 + 1], normals[i * 3 + 2]), rng);
        out[i * 3] = d.x;
        out[i * 3 + 1] = d.y;
        out[i * 3 + 2] = d.z;
    }
}

orc_scene* orc_scene_create(const lux_scene_desc* d, int cdf_f64, int tex_storage) {
    if (!d) return nullptr;
    orc_scene* s = new orc_scene();
    s->cam = d->camera;
    s->trace_depth = d->trace_depth;
    s->meshes.resize(d->num_meshes);
    for (int i = 0; i < d->num_meshes; ++i) {
        const lux_mesh_desc& md = d->meshes[i];
        Mesh& m = s->meshes[i];
        m.nv = md.num_verts;
        m.nt = md.num_tris;
        m.pos.assign(md.positions, md.positions + size_t(m.nv) * 3);
        m.has_n = md.normals != nullptr;
        m.has_uv = md.uvs != nullptr;
        if (m.has_n) m.nrm.assign(md.normals, md.normals + size_t(m.nv) * 3);
        if (m.has_uv) m.uv.assign(md.uvs, md.uvs + size_t(m.nv) * 2);
        m.idx.assign(md.indices, md.indices + size_t(m.nt) * 3);
        for (int a = 0; a < 3; ++a) { m.bmin[a] = FLT_MAX; m.bmax[a] = -FLT_MAX; }
        for (int v = 0; v < m.nv; ++v)
            for (int a = 0; a < 3; ++a) {
                m.bmin[a] = std::min(m.bmin[a], m.pos[v * 3 + a]);
                m.bmax[a] = std::max(m.bmax[a], m.pos[v * 3 + a]);
            }
    }
    s->insts.resize(d->num_instances);
    for (int i = 0; i < d->num_instances; ++i) {
        const lux_instance_desc& id = d->instances[i];
        Inst& g = s->insts[i];
        g.mesh = id.mesh;
        g.material = id.material;
        std::memcpy(g.M, id.transform, sizeof(g.M));
        std::memcpy(g.Minv, id.inverse, sizeof(g.Minv));
        std::memcpy(g.MinvT, id.inv_transpose, sizeof(g.MinvT));
    }
    s->mats.assign(d->materials, d->materials + d->num_materials);
    s->texs.resize(d->num_textures);
    for (int i = 0; i < d->num_textures; ++i)
        load_tex(s->texs[i], d->textures[i].width, d->textures[i].height, d->textures[i].format, d->textures[i].data,
                 tex_storage);
    if (d->env_data) {
        s->has_env = true;
        load_tex(s->env, d->env_width, d->env_height, d->env_format, d->env_data,
                 tex_storage == LUX_TEXSTORE_HALF ? LUX_TEXSTORE_HALF : LUX_TEXSTORE_FLOAT);
    }
    precompute_emissive<float>(*s, s->emissive_prefix, s->tri_prefix, s->total_area);
    precompute_emissive<double>(*s, s->emissive_prefix_d, s->tri_prefix_d, s->total_area_d);
    if (cdf_f64) {
        for (size_t i = 0; i < s->emissive_prefix.size(); ++i) s->emissive_prefix[i] = float(s->emissive_prefix_d[i]);
        for (size_t i = 0; i < s->tri_prefix.size(); ++i)
            for (size_t k = 0; k < s->tri_prefix[i].size(); ++k) s->tri_prefix[i][k] = float(s->tri_prefix_d[i][k]);
        s->total_area = float(s->total_area_d);
    }
    if (s->has_env) {
        precompute_hdri<float>(s->env, s->marginal, s->conditional);
        precompute_hdri<double>(s->env, s->marginal_d, s->conditional_d);
        if (cdf_f64) {
            for (size_t i = 0; i < s->marginal.size(); ++i) s->marginal[i] = float(s->marginal_d[i]);
            for (size_t i = 0; i < s->conditional.size(); ++i) s->conditional[i] = float(s->conditional_d[i]);
        }
    }
    // acceleration: one BVH per mesh (object space), one over instance world boxes
    s->blas.resize(s->meshes.size());
    for (size_t mi = 0; mi < s->meshes.size(); ++mi) {
        const Mesh& m = s->meshes[mi];
        std::vector<float> boxes(size_t(m.nt) * 6);
        for (int k = 0; k < m.nt; ++k) {
            for (int a = 0; a < 3; ++a) { boxes[k * 6 + a] = FLT_MAX; boxes[k * 6 + 3 + a] = -FLT_MAX; }
            for (int c = 0; c < 3; ++c) {
                uint32_t vi = m.idx[k * 3 + c];
                for (int a = 0; a < 3; ++a) {
                    boxes[k * 6 + a] = std::min(boxes[k * 6 + a], m.pos[vi * 3 + a]);
                    boxes[k * 6 + 3 + a] = std::max(boxes[k * 6 + 3 + a], m.pos[vi * 3 + a]);
                }
            }
            for (int a = 0; a < 3; ++a) {
                float pad = 1e-5f + 1e-5f * std::max(std::fabs(boxes[k * 6 + a]), std::fabs(boxes[k * 6 + 3 + a]));
                boxes[k * 6 + a] -= pad;
                boxes[k * 6 + 3 + a] += pad;
            }
        }
        build_bvh(s->blas[mi], boxes, m.nt);
    }
    s->inst_boxes.assign(s->insts.size() * 6, 0.0f);
    for (size_t i = 0; i < s->insts.size(); ++i) {
        const Inst& g = s->insts[i];
        const Mesh& m = s->meshes[g.mesh];
        float* b = &s->inst_boxes[i * 6];
        for (int a = 0; a < 3; ++a) { b[a] = FLT_MAX; b[3 + a] = -FLT_MAX; }
        for (int c = 0; c < 8; ++c) {
            V3<double> p{double((c & 1) ? m.bmax[0] : m.bmin[0]), double((c & 2) ? m.bmax[1] : m.bmin[1]),
                         double((c & 4) ? m.bmax[2] : m.bmin[2])};
            V3<double> w = mul_point<double>(g.M, p, 1.0);
            for (int a = 0; a < 3; ++a) {
                b[a] = std::min(b[a], float(w[a]));
                b[3 + a] = std::max(b[3 + a], float(w[a]));
            }
        }
        for (int a = 0; a < 3; ++a) {
            float pad = 1e-4f + 1e-5f * std::max(std::fabs(b[a]), std::fabs(b[3 + a]));
            b[a] -= pad;
            b[3 + a] += pad;
        }
    }
    build_bvh(s->tlas, s->inst_boxes, int(s->insts.size()));
    if (!s->insts.empty()) {
        const Mesh& m0 = s->meshes[s->insts[0].mesh];
        for (int a = 0; a < 3; ++a) {
            s->morton_bmin[a] = m0.bmin[a] - kEPS_UTIL;
            s->morton_bmax[a] = m0.bmax[a] + kEPS_UTIL;
        }
    }
    return s;
}

void orc_scene_destroy(orc_scene* s) { delete s; }

void orc_cdf_sizes(orc_scene* s, int* sizes) {
    sizes[0] = int(s->emissive.size());
    size_t tl = 0;
    for (int e : s->emissive) tl += s->tri_prefix[e].size();
    sizes[1] = int(tl);
    sizes[2] = s->has_env ? s->env.h : 0;
    sizes[3] = s->has_env ? s->env.w : 0;
}

int orc_get_cdfs(orc_scene* s, float* ep, float* tp, float* mg, float* cd, float* ta) {
    if (ep) std::copy(s->emissive_prefix.begin(), s->emissive_prefix.end(), ep);
    if (tp) {
        size_t o = 0;
        for (int e : s->emissive) {
            std::copy(s->tri_prefix[e].begin(), s->tri_prefix[e].end(), tp + o);
            o += s->tri_prefix[e].size();
        }
    }
    if (mg) std::copy(s->marginal.begin(), s->marginal.end(), mg);
    if (cd) std::copy(s->conditional.begin(), s->conditional.end(), cd);
    if (ta) *ta = s->total_area;
    return 0;
}

void orc_trace(orc_scene* s, const float* rays, int n, int mode, int iter, uint32_t* hits, int brute) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const float* r = rays + size_t(i) * 8;
        int32_t px;
        std::memcpy(&px, &r[7], 4);
        HitT<float> h;
        float tmax = (mode == 1) ? r[3] : 1e16f;
        bool any = trace_ray(*s, V3<float>(r[0], r[1], r[2]), V3<float>(r[4], r[5], r[6]), tmax, mode, px, iter,
                             brute != 0, h);
        Hit o;
        if (mode == 2) {
            o.t = any ? 1.0f : -1.0f;
        } else if (h.inst >= 0) {
            o.t = h.t;
            o.inst = h.inst;
            o.prim = h.prim;
            o.u = h.u;
            o.v = h.v;
        }
        write_hit(o, hits + size_t(i) * 5);
    }
}

void orc_morton(orc_scene* s, const float* rays, int n, uint32_t* keys) {
    for (int i = 0; i < n; ++i) {
        const float* r = rays + size_t(i) * 8;
        keys[i] = morton_key(*s, V3<float>(r[0], r[1], r[2]), V3<float>(r[4], r[5], r[6]));
    }
}

void orc_light_samples(orc_scene* s, const lux_options* opt, int iter, int depth, const int* pixels, int n, float* out) {
    for (int i = 0; i < n; ++i) {
        Path<float> p;
        p.pixel = pixels[i];
        light_sample(*s, *opt, iter, depth, p);
        out[i * 6] = p.dl.x;
        out[i * 6 + 1] = p.dl.y;
        out[i * 6 + 2] = p.dl.z;
        out[i * 6 + 3] = p.env.x;
        out[i * 6 + 4] = p.env.y;
        out[i * 6 + 5] = p.env.z;
    }
}

void orc_camera_rays(orc_scene* s, int iter, const int* pixels, int n, float* paths) {
    for (int i = 0; i < n; ++i) {
        Path<float> p;
        camera_ray(*s, iter, pixels[i], s->trace_depth, p);
        path_store(p, paths + size_t(i) * LUX_PS_FLOATS);
    }
}

void orc_shade_step(orc_scene* s, const lux_options* opt, int iter, int depth, int compact, float* paths, int n,
                    const uint32_t* hits, int* survivors, int* n_out) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
        Path<float> p;
        path_load(p, paths + size_t(i) * LUX_PS_FLOATS);
        Hit rh = read_hit(hits + size_t(i) * 10);
        Hit sh = read_hit(hits + size_t(i) * 10 + 5);
        float eo = sh.t;
        HitT<float> shs = to_ht(sh);
        if (opt->env_importance_sampling) shs = HitT<float>();
        bool alive = shade_path(*s, *opt, iter, depth, compact != 0, p, to_ht(rh), shs, eo);
        path_store(p, paths + size_t(i) * LUX_PS_FLOATS);
        if (alive) survivors[k++] = i;
    }
    *n_out = k;
}

void orc_sample_texture(orc_scene* s, int tex, const float* uv, int n, float* out) {
    const Tex& t = tex < 0 ? s->env : s->texs[tex];
    for (int i = 0; i < n; ++i) tex_fetch(t, uv[i * 2], uv[i * 2 + 1], out + i * 4);
}

int orc_render(orc_scene* s, const lux_options* opt, int first_iter, int n_iter, int x0, int y0, int w, int h,
               int f64, int threads, float* image, double* stats) {
    double st[4] = {0, 0, 0, 0};
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
#endif
    const int W = s->cam.width;
#pragma omp parallel num_threads(nt)
    {
        double lst[4] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
        for (int yy = 0; yy < h; ++yy) {
            for (int xx = 0; xx < w; ++xx) {
                int pixel = (y0 + yy) * W + (x0 + xx);
                float acc[3] = {0, 0, 0};
                double accd[3] = {0, 0, 0};
                for (int it = first_iter; it < first_iter + n_iter; ++it) {
                    if (f64) {
                        V3<double> c;
                        render_path<double>(*s, *opt, it, pixel, c, lst);
                        accd[0] += c.x;
                        accd[1] += c.y;
                        accd[2] += c.z;
                    } else {
                        V3<float> c;
                        render_path<float>(*s, *opt, it, pixel, c, lst);
                        acc[0] += c.x;
                        acc[1] += c.y;
                        acc[2] += c.z;
                    }
                    lst[3] += 1;
                }
                float* o = image + (size_t(yy) * w + xx) * 3;
                for (int c = 0; c < 3; ++c) o[c] = f64 ? float(accd[c]) : acc[c];
            }
        }
#pragma omp critical
        for (int k = 0; k < 4; ++k) st[k] += lst[k];
    }
    if (stats)
        for (int k = 0; k < 4; ++k) stats[k] = st[k];
    return 0;
}

// sendImageToPBO (src/kernels/image_kernels.cu:6-46)
void orc_tonemap(const float* img, int n_pix, float iter, int color_mode, uint8_t* rgba) {
    float inv = 1.0f / iter;
    for (int i = 0; i < n_pix; ++i) {
        float p[3] = {img[i * 3] * inv, img[i * 3 + 1] * inv, img[i * 3 + 2] * inv};
        if (color_mode == 0) {
            for (int c = 0; c < 3; ++c) p[c] = p[c] / (p[c] + 1.0f);
        } else if (color_mode == 1) {
            agx(p);
        } else {
            acesfilm(p);
        }
        for (int c = 0; c < 3; ++c) p[c] = std::pow(p[c], 0.45f);
        for (int c = 0; c < 3; ++c) rgba[i * 4 + c] = uint8_t(gclamp(int(double(p[c]) * 255.0), 0, 255));
        rgba[i * 4 + 3] = 0;
    }
}

}  // extern "C"
