// device_math.cuh -- float vector math, RNG and shading pieces of the render path, for the
// device. Evaluation order follows glm 0.9.6 / sutil as the reference uses them, so a kernel
// compiled with --fmad=false computes every +,-,*,/,sqrt exactly as the reference's host
// build does; only the transcendental functions (sinf, cosf, atan2f, acosf, atanf, powf,
// log2f) come from CUDA's math library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lux {

#define LUX_DI __device__ __forceinline__
#define LUX_HDI __host__ __device__ __forceinline__

// include/utilities.h:13-16, include/shaders/cook_torrance.h:13, src/shaders/cook_torrance.cu:3-4
constexpr float kPI = 3.1415926535897932384626422832795028841971f;
constexpr float kTWO_PI = 6.2831853071795864769252867665590057683943f;
constexpr float kSQRT13 = 0.5773502691896257645091487805019574556476f;
constexpr float kEPS_UTIL = 0.00001f;
constexpr float kINV_PI = 0.3183098f;
constexpr float kEPS_CT = 1e-30f;
constexpr float kPDF_CLAMP = 1e-5f;
constexpr double kM_PI_SHADE = 3.14159;  // src/kernels/shade_path.cu:23
constexpr float kGLASS_EPS = 0.01f;      // src/kernels/shade_path.cu:24
constexpr float kSPEC_ROUGH = 0.05f;     // src/kernels/shade_path.cu:25
constexpr int kRR_MIN_DEPTH = 3;         // include/config.h:7
constexpr float kMT_EPS = 1.1920929E-7F; // src/intersections/mesh_isect.cu:34

struct f3 {
    float x, y, z;
};
LUX_HDI f3 mk(float x, float y, float z) { return f3{x, y, z}; }
LUX_HDI f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
LUX_HDI f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
LUX_HDI f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
LUX_HDI f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
LUX_HDI f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
LUX_HDI f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
LUX_HDI f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
// glm 0.9.6 min/max/clamp (func_common.inl:409-472)
LUX_HDI float gmin(float a, float b) { return a < b ? a : b; }
LUX_HDI float gmax(float a, float b) { return a > b ? a : b; }
LUX_HDI float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
LUX_HDI int gclampi(int x, int lo, int hi) { return (x > lo ? x : lo) < hi ? (x > lo ? x : lo) : hi; }
LUX_HDI float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LUX_HDI f3 cross(f3 a, f3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
LUX_DI f3 normalize(f3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
LUX_DI float length(f3 v) { return sqrtf(dot(v, v)); }
LUX_HDI f3 vmix(f3 x, f3 y, float a) { return x + a * (y - x); }
LUX_HDI f3 reflect(f3 I, f3 N) { return I - N * dot(N, I) * 2.0f; }
LUX_DI f3 refract(f3 I, f3 N, float eta) {
    float d = dot(N, I);
    float k = 1.0f - eta * eta * (1.0f - d * d);
    return (eta * I - (eta * d + sqrtf(k)) * N) * float(k >= 0.0f);
}
LUX_DI f3 vpow(f3 v, float e) { return {powf(v.x, e), powf(v.y, e), powf(v.z, e)}; }
LUX_DI f3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

// glm mat4 * vec4 with the matrix given as 4 columns of 3 floats (rows 0..2):
// (m0*v0 + m1*v1) + (m2*v2 + m3*w), every operation rounded on its own.
LUX_DI f3 xform(const float* m, f3 p, float w) {
    f3 r;
    r.x = __fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[3], p.y)),
                    __fadd_rn(__fmul_rn(m[6], p.z), __fmul_rn(m[9], w)));
    r.y = __fadd_rn(__fadd_rn(__fmul_rn(m[1], p.x), __fmul_rn(m[4], p.y)),
                    __fadd_rn(__fmul_rn(m[7], p.z), __fmul_rn(m[10], w)));
    r.z = __fadd_rn(__fadd_rn(__fmul_rn(m[2], p.x), __fmul_rn(m[5], p.y)),
                    __fadd_rn(__fmul_rn(m[8], p.z), __fmul_rn(m[11], w)));
    return r;
}

// ---- RNG: utilhash (include/intersections.h:13-22), makeSeededRandomEngine
// (include/common.h:38-47), thrust minstd_rand + uniform_real_distribution<float>(0,1).
LUX_HDI uint32_t utilhash(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}
// Path state is streamed: each kernel reads and writes a path's fields once, and a wave's
// state (about 1.4 GB at 1080p) does not fit in L2. Evict-first loads and stores
// (ld/st.global.cs) keep it from pushing the BVH nodes and triangle records, which every
// traversal reads again and again, out of L2.
LUX_DI float4 ld_stream(const float4* p) { return __ldcs(p); }
LUX_DI int ld_stream(const int* p) { return __ldcs(p); }
LUX_DI void st_stream(float4* p, float4 v) { __stcs(p, v); }
LUX_DI void st_stream(int* p, int v) { __stcs(p, v); }

struct Rng {
    uint32_t x;
    LUX_HDI static uint32_t mod_m(uint64_t v) {
        // v mod (2^31 - 1) for v < 2^62 without division
        uint64_t r = (v & 0x7fffffffull) + (v >> 31);
        r = (r & 0x7fffffffull) + (r >> 31);
        return uint32_t(r >= 0x7fffffffull ? r - 0x7fffffffull : r);
    }
    LUX_HDI static Rng seeded(int iter, int index, int depth) {
        uint32_t k = (1u << 31) | (uint32_t(depth) << 22) | uint32_t(iter);
        uint32_t s = utilhash(k) ^ utilhash(uint32_t(index));
        Rng r;
        uint32_t m = mod_m(s);
        r.x = m == 0u ? 1u : m;
        return r;
    }
    LUX_HDI uint32_t next() {
        x = mod_m(uint64_t(x) * 48271ull);
        return x;
    }
    // Three steps at once: x * 48271^3 mod (2^31 - 1), 48271^3 mod (2^31 - 1) = 1291394886.
    LUX_HDI void skip3() { x = mod_m(uint64_t(x) * 1291394886ull); }
    // (float(x - 1) / (1 + float(max - min))) * (1 - 0) + 0; the divisor rounds to 2^31
    LUX_DI float u01() {
        uint32_t v = next();
        return __fmul_rn(float(v - 1u), 4.656612873077392578125e-10f);
    }
};

// cudaUtils::select_from_cdf (src/common.cu:3-15)
LUX_DI int select_from_cdf(const float* __restrict__ cdf, int size, float xi) {
    int low = 0, high = size - 1;
    while (low < high) {
        int mid = low + (high - low) / 2;
        if (__ldg(cdf + mid) < xi) low = mid + 1;
        else high = mid;
    }
    return low;
}

// select_from_cdf over a bracket from a guide table. guide[j] = select_from_cdf(cdf, size, j/m)
// for j in 0..m (m a power of two, so j = floor(xi * m) and j/m are exact). The answer is
// monotone in xi, so for xi in [j/m, (j+1)/m] it lies in [guide[j], guide[j+1]], and the same
// first-index-not-below-xi search over that bracket returns the same index with far fewer
// dependent loads.
LUX_DI int select_from_cdf_guided(const float* __restrict__ cdf, const int* __restrict__ guide, int m, float xi) {
    int j = int(xi * float(m));
    j = j < 0 ? 0 : (j > m - 1 ? m - 1 : j);
    int low = __ldg(guide + j), high = __ldg(guide + j + 1);
    while (low < high) {
        int mid = low + (high - low) / 2;
        if (__ldg(cdf + mid) < xi) low = mid + 1;
        else high = mid;
    }
    return low;
}

// OptiX any-hit hash (src/optixshaders/optix_triangle.cu:41-49)
LUX_HDI uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

}  // namespace lux
