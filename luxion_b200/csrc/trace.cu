// trace.cu -- ray traversal of the two-level compressed 8-wide BVH on sm_100a.
//
// Replaces the reference's OptiX launch (src/pathtrace.cu:238-258, device programs in
// src/optixshaders/optix_triangle.cu:52-366) and its disabled software path
// (src/kernels/compute_intersections.cu:6-87, src/intersections/mesh_isect.cu:6-149).
//
// Design:
//  * persistent warps: lanes without a ray take the next ones from a global cursor with one
//    atomicAdd per warp (ballot/popc), and a warp leaves its inner loop to refill as soon as
//    fewer than kRefill lanes are still traversing (Aila & Laine's while-while with dynamic
//    fetch);
//  * the traversal stack keeps its top kShStack entries in shared memory (one column per
//    thread, conflict-free) and spills deeper entries to local memory;
//  * node groups / triangle groups as in Ylitie et al. 2017: a stack entry is a node's
//    remaining internal-child hits (ordered by ray octant) or a set of leaf records;
//  * two levels: the TLAS is traversed with the world ray; a TLAS leaf pushes a marker and
//    continues in the instance's BLAS with the object-space ray the reference uses
//    (inverseTransform * (o,1), (d,0), src/intersections/mesh_isect.cu:15-16);
//  * the triangle test is the reference's Moller-Trumbore (mesh_isect.cu:78-137) with every
//    operation rounded on its own, so t, u, v and the hit triangle match the CPU oracle bit
//    for bit on the same rays; equal t is resolved toward the lowest (instance, primitive);
//  * alpha mask / blend any-hit (optix_triangle.cu:317-366) is evaluated on candidate hits of
//    instances whose material is not opaque.
// Box tests are conservative: child boxes are quantised outward at build time and a child is
// entered while tnear <= tfar * (1 + 2^-17), so no triangle the exact test accepts is skipped.

#include "device_scene.h"
#include "device_math.cuh"
#include "bvh8.h"
#include "launch.h"

#include <array>
#include <map>
#include <mutex>

namespace lux {

namespace {

constexpr int kShStack = 16;
constexpr int kLocStack = 48;
static_assert(kShStack + kLocStack == kTraversalStack, "the scene build bounds the stack by kTraversalStack");
constexpr int kRefill = 20;
// environment occlusion rays (any hit, mode 2) refill below this many traversing lanes
constexpr int kRefillOcclusion = 24;
constexpr uint32_t kTagMask = 3u << 30;
constexpr uint32_t kTagNode = 0u;
constexpr uint32_t kTagTri = 1u << 30;
constexpr uint32_t kTagInst = 2u << 30;
constexpr uint32_t kTagMarker = 3u << 30;
constexpr uint32_t kRecMask = 0xffu;
// fewer lanes than this with triangles to test: push the triangle groups and keep
// traversing nodes (the postponement of Ylitie et al. 2017); 6 and a refill threshold of 20
// lanes were the fastest of the values tried on the 1M-triangle 1080p workload (3, 4 and 6;
// 16, 18, 20, 22, 24 and 28), and 24 for the occlusion rays (16, 20, 24, 28 and 32)
constexpr int kPostpone = 6;
// Slab acceptance tnear <= tfar * kWiden (tnear >= 0): a relative margin of 2^-17, far above
// the few-ulp rounding of the plane distances.
constexpr float kWiden = 1.0f + 1.0f / 131072.0f;
static_assert(kMaxLeafPrims == 1, "visit_node marks one triangle per leaf slot");

struct TRay {
    f3 o, d, idir;
    uint32_t oct;
};

// Reciprocal for the box tests only (the triangle test uses the direction itself): the
// hardware approximation, at most 1 ulp off, scales both slab distances of an axis by the same
// factor within 2^-23 of 1, far inside the 2^-17 acceptance margin.
// A component below 2^-66 in magnitude (zero and subnormals included) is raised to 2^-66 with
// its sign. An exact zero would give an infinite reciprocal, that axis's slab distances would
// then be NaN, and fminf / fmaxf drop NaN operands: the axis would stop culling, and in a
// world-space tree the ray would sweep a whole slab of the scene (a camera on an axis-aligned
// plane makes such rays, one pixel column of them). With 2^-66 the axis culls every box that
// does not hold the origin's coordinate to within 2^-66 * tmax, and keeps every box that holds
// it with a margin m for t up to m * 2^66: boxes are padded by far more than the 2^-66 * t a
// ray this close to the axis plane drifts within the scene.
LUX_DI float rcp_box(float x) {
    const float c = copysignf(fmaxf(fabsf(x), 1.35525271560688054e-20f), x);  // 2^-66
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(c));
    return r;
}

LUX_DI TRay make_ray(f3 o, f3 d) {
    TRay r;
    r.o = o;
    r.d = d;
    r.idir = mk(rcp_box(d.x), rcp_box(d.y), rcp_box(d.z));
    r.oct = (__float_as_uint(r.idir.x) >> 31) | ((__float_as_uint(r.idir.y) >> 31) << 1) |
            ((__float_as_uint(r.idir.z) >> 31) << 2);
    return r;
}

// Byte s of w as the float 2^23 + 256 * byte: one byte permute builds 0x4B00bb00. The 2^23
// bias is folded into the per-node plane constant (visit_node), so no add removes it.
LUX_DI float ubyte_biased(uint32_t w, int s) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7504u | (uint32_t(s) << 4))); }

// Three-operand max / min (sm_100 and later): one instruction where two fmaxf / fminf would
// be, with their NaN rule (a NaN operand is dropped).
LUX_DI float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
LUX_DI float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Intersect the 8 child boxes of node ni. Returns internal-child hits as a key mask
// (bit slot ^ oct), leaf hits as a slot mask, the node's leaf-slot mask, child_base and
// tri_base.
LUX_DI void visit_node(const uint4* __restrict__ nodes, uint32_t ni, const TRay& r, float tmax, uint32_t& keys,
                       uint32_t& imask, uint32_t& child_base, uint32_t& tri_base, uint32_t& trimask,
                       uint32_t& leafmask) {
    const uint4* n = nodes + size_t(ni) * 5;
    uint4 w0 = __ldg(n + 0), w1 = __ldg(n + 1), w2 = __ldg(n + 2), w3 = __ldg(n + 3), w4 = __ldg(n + 4);
    float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    float sx = __uint_as_float((w0.w & 0xffu) << 23);
    float sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
    imask = w0.w >> 24;
    child_base = w1.x;
    tri_base = w1.y;
    // plane q of an axis lies at t = q * a + b with a = scale * idir, b = (p - o) * idir.
    // It is evaluated as fma(2^23 + 256 q, a / 256, b - 2^15 a): a / 256 is exact, and the
    // rounding of the folded constant adds at most 2^-9 of a quantisation step (the host pads
    // every plane by at least 1 % of a step).
    float ax = sx * r.idir.x * 0.00390625f, ay = sy * r.idir.y * 0.00390625f, az = sz * r.idir.z * 0.00390625f;
    float bx = (px - r.o.x) * r.idir.x, by = (py - r.o.y) * r.idir.y, bz = (pz - r.o.z) * r.idir.z;
    bx = fmaf(-8388608.0f, ax, bx);
    by = fmaf(-8388608.0f, ay, by);
    bz = fmaf(-8388608.0f, az, bz);
    // near/far quantised planes per axis, by ray octant
    const bool fx = r.oct & 1, fy = r.oct & 2, fz = r.oct & 4;
    uint32_t nx0 = fx ? w3.z : w2.x, nx1 = fx ? w3.w : w2.y, fx0 = fx ? w2.x : w3.z, fx1 = fx ? w2.y : w3.w;
    uint32_t ny0 = fy ? w4.x : w2.z, ny1 = fy ? w4.y : w2.w, fy0 = fy ? w2.z : w4.x, fy1 = fy ? w2.w : w4.y;
    uint32_t nz0 = fz ? w4.z : w3.x, nz1 = fz ? w4.w : w3.y, fz0 = fz ? w3.x : w4.z, fz1 = fz ? w3.y : w4.w;
    uint32_t hits = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int b = s & 3;
        uint32_t wnx = s < 4 ? nx0 : nx1, wny = s < 4 ? ny0 : ny1, wnz = s < 4 ? nz0 : nz1;
        uint32_t wfx = s < 4 ? fx0 : fx1, wfy = s < 4 ? fy0 : fy1, wfz = s < 4 ? fz0 : fz1;
        float tnx = fmaf(ubyte_biased(wnx, b), ax, bx), tny = fmaf(ubyte_biased(wny, b), ay, by),
              tnz = fmaf(ubyte_biased(wnz, b), az, bz);
        float tfx = fmaf(ubyte_biased(wfx, b), ax, bx), tfy = fmaf(ubyte_biased(wfy, b), ay, by),
              tfz = fmaf(ubyte_biased(wfz, b), az, bz);
        float tn = max3f(tnx, tny, fmaxf(tnz, 0.0f));
        float tf = min3f(tfx, tfy, fminf(tfz, tmax));
        if (tn <= tf * kWiden) hits |= 1u << s;
    }
    leafmask = w1.z & 0xffu;
    hits &= imask | leafmask;
    trimask = hits & leafmask;
    uint32_t ih = hits & imask;  // to key order: bit s moves to bit s ^ oct
    if (r.oct & 1) ih = ((ih & 0x55u) << 1) | ((ih >> 1) & 0x55u);
    if (r.oct & 2) ih = ((ih & 0x33u) << 2) | ((ih >> 2) & 0x33u);
    if (r.oct & 4) ih = ((ih & 0x0Fu) << 4) | ((ih >> 4) & 0x0Fu);
    keys = ih;
}

struct Best {
    float t;
    int inst, prim;
    float u, v;
};

LUX_DI bool better(float t, int inst, int prim, const Best& b) {
    if (b.inst < 0) return true;
    if (t < b.t) return true;
    return t == b.t && (inst < b.inst || (inst == b.inst && prim < b.prim));
}

// Moller-Trumbore exactly as src/intersections/mesh_isect.cu:78-115, single-rounded ops, on a
// triangle record (v0 with the triangle index in w, e1, e2) and the ray (ro, d) of the
// triangle's object space.
LUX_DI bool mt_core(float4 a4, float4 e14, float4 e24, f3 ro, f3 d, float& t, float& u, float& v, int& prim) {
    prim = __float_as_int(a4.w);
    const f3 e1 = mk(e14.x, e14.y, e14.z), e2 = mk(e24.x, e24.y, e24.z);
    // cross(d, e2) = (d.y*e2.z - e2.y*d.z, d.z*e2.x - e2.z*d.x, d.x*e2.y - e2.x*d.y)
    f3 c = mk(__fsub_rn(__fmul_rn(d.y, e2.z), __fmul_rn(e2.y, d.z)), __fsub_rn(__fmul_rn(d.z, e2.x), __fmul_rn(e2.z, d.x)),
              __fsub_rn(__fmul_rn(d.x, e2.y), __fmul_rn(e2.x, d.y)));
    float det = __fadd_rn(__fadd_rn(__fmul_rn(e1.x, c.x), __fmul_rn(e1.y, c.y)), __fmul_rn(e1.z, c.z));
    if (det > -kMT_EPS && det < kMT_EPS) return false;
    float inv = __frcp_rn(det);
    f3 a = mk(__fsub_rn(ro.x, a4.x), __fsub_rn(ro.y, a4.y), __fsub_rn(ro.z, a4.z));
    u = __fmul_rn(inv, __fadd_rn(__fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y)), __fmul_rn(a.z, c.z)));
    if (u < -kMT_EPS || u > 1.0f + kMT_EPS) return false;
    // cross(a, e1)
    c = mk(__fsub_rn(__fmul_rn(a.y, e1.z), __fmul_rn(e1.y, a.z)), __fsub_rn(__fmul_rn(a.z, e1.x), __fmul_rn(e1.z, a.x)),
           __fsub_rn(__fmul_rn(a.x, e1.y), __fmul_rn(e1.x, a.y)));
    v = __fmul_rn(inv, __fadd_rn(__fadd_rn(__fmul_rn(d.x, c.x), __fmul_rn(d.y, c.y)), __fmul_rn(d.z, c.z)));
    float uv = __fadd_rn(u, v);
    if ((v < 0.0f && fabsf(v) > kMT_EPS) || (uv > 1.0f && fabsf(__fsub_rn(uv, 1.0f)) > kMT_EPS)) return false;
    t = __fmul_rn(inv, __fadd_rn(__fadd_rn(__fmul_rn(e2.x, c.x), __fmul_rn(e2.y, c.y)), __fmul_rn(e2.z, c.z)));
    return t > kMT_EPS;
}

LUX_DI bool mt_test(const float4* __restrict__ prims, uint32_t rec, const TRay& r, float& t, float& u, float& v,
                    int& prim) {
    const float4* q = prims + size_t(rec) * 3;
    return mt_core(__ldg(q), __ldg(q + 1), __ldg(q + 2), r.o, r.d, t, u, v, prim);
}

// Any-hit program (src/optixshaders/optix_triangle.cu:317-366): true = accept the hit.
LUX_DI bool alpha_accept(const DevScene& S, const DevInstance& I, int inst, int prim, float bu, float bv, f3 wdir,
                         int pixel, int iter) {
    const DevMaterial& m = S.mats[I.material];
    if (m.alpha_mode == 0) return true;
    float alpha = m.alpha;
    if (m.flags & kMatAlbedoTex) {
        float ux = 0.0f, uy = 0.0f;
        if (I.flags & kInstHasUVs) {
            const uint32_t* id = S.idx + (size_t(I.idx_base) + prim) * 3;
            uint32_t i0 = I.vert_base + id[0], i1 = I.vert_base + id[1], i2 = I.vert_base + id[2];
            float bA = 1.0f - bu - bv;
            ux = bA * S.uv[i0 * 2] + bu * S.uv[i1 * 2] + bv * S.uv[i2 * 2];
            uy = bA * S.uv[i0 * 2 + 1] + bu * S.uv[i1 * 2 + 1] + bv * S.uv[i2 * 2 + 1];
        }
        ux = ux * m.albedo_tt.scale[0];
        uy = uy * m.albedo_tt.scale[1];
        if (m.albedo_tt.rotation != 0.0f) {
            float c = cosf(m.albedo_tt.rotation), s = sinf(m.albedo_tt.rotation);
            float nx = c * ux - s * uy, ny = s * ux + c * uy;
            ux = nx;
            uy = ny;
        }
        ux = ux + m.albedo_tt.offset[0];
        uy = uy + m.albedo_tt.offset[1];
        float4 tx = tex2D<float4>(cudaTextureObject_t(m.albedo_tex), ux, uy);
        alpha *= tx.w;
    }
    if (m.alpha_mode == 1) return !(alpha < m.alpha_cutoff);
    uint32_t h = hash_u32(uint32_t(pixel) ^ hash_u32(uint32_t(iter)));
    h = hash_u32(h ^ __float_as_uint(wdir.x));
    h = hash_u32(h ^ __float_as_uint(wdir.y));
    h = hash_u32(h ^ __float_as_uint(wdir.z));
    h = hash_u32(h ^ uint32_t(I.key));  // the instance's index within its own scene
    h = hash_u32(h ^ uint32_t(prim));
    float rnd = float(h >> 8) * (1.0f / 16777216.0f);
    return !(rnd >= alpha);
}

// Traversal state of one lane. Two-level layout: wo, wd hold the world ray (its reciprocals are
// recomputed when the traversal leaves an instance) and cur the ray of the current level.
// Single-level layout: cur is the world ray throughout, and wo, wd hold the object-space ray of
// the instance `inst` whose triangles were tested last.
struct Lane {
    f3 wo, wd;          // world ray (two-level) / object ray of `inst` (single-level)
    TRay cur;           // ray of the current level (world in the TLAS, object space in a BLAS)
    float tmax;
    Best best;
    uint2 g;            // node group: x = first internal child, y = imask << 8 | remaining hit keys
    uint2 t;            // leaf group: x = first record, y = tag (kTagTri / kTagInst) | leaf-slot
                        // mask << 8 | remaining hit slots
    int sp;             // stack depth
    int inst;           // current instance (-1 in the TLAS)
    int inst_flags;
    uint32_t inst_prim_base;
    int key;            // path id (wave rays) or pixel (rays given directly): the alpha-blend
                        // hash key, resolved only when an alpha-blended instance is tested
    int work;           // BVH heatmap (mode 3): node visits + triangle tests
    bool done;
};

struct TraceArgs {
    DevScene S;
    DevWave W;
    Segs G;      // the (lane, bounce) segments of the launch
    int mode;    // 0 radiance, 1 DL shadow, 2 env shadow, 3 BVH heatmap of radiance rays
    int nee;     // radiance pass: 0 none, 1 DL, 2 env
    const float* ext_rays;  // lux_trace_rays: rays given directly (n * 8 floats)
    uint32_t* ext_hits;     // and hits written directly (n * 5 words)
    int ext_n;
    int ext_iter;
    int* ext_fetch;
};

template <int MODE, bool SINGLE>
struct Tracer {
    const DevScene& S;
    uint2 (*sh)[kTraceBlock];  // shared stack [kShStack][block]
    uint2 loc[kLocStack];
    int tid;
    int* err;
    const TraceArgs& A;  // the launch's arguments, in parameter space like S

    LUX_DI void push(Lane& L, uint2 e) {
        if (L.sp < kShStack) sh[L.sp][tid] = e;
        else if (L.sp < kShStack + kLocStack) loc[L.sp - kShStack] = e;
        else {
            atomicOr(err, 1);
            return;
        }
        ++L.sp;
    }
    LUX_DI uint2 pop(Lane& L) {
        --L.sp;
        return L.sp < kShStack ? sh[L.sp][tid] : loc[L.sp - kShStack];
    }

    LUX_DI void start(Lane& L, f3 o, f3 d, float tmax, uint32_t root) {
        L.wo = o;
        L.wd = d;
        L.cur = make_ray(o, d);
        L.tmax = tmax;
        L.best.t = -1.0f;
        L.best.inst = -1;
        L.best.prim = -1;
        L.best.u = L.best.v = 0.0f;
        L.sp = 0;
        L.inst = -1;
        L.inst_flags = 0;
        L.inst_prim_base = 0;
        L.done = false;
        L.work = 0;
        // root group: a single internal child (slot 0) = the TLAS root, at key oct
        L.g = make_uint2(root, (1u << 8) | (1u << L.cur.oct));
        L.t = make_uint2(0u, 0u);
    }

    LUX_DI float limit(const Lane& L) const { return (MODE != 2 && L.best.inst >= 0) ? L.best.t : L.tmax; }
    static LUX_DI f3 world_o(const Lane& L) { return SINGLE ? L.cur.o : L.wo; }
    static LUX_DI f3 world_d(const Lane& L) { return SINGLE ? L.cur.d : L.wd; }

    // Node phase: visit the nearest remaining child of the node group.
    LUX_DI void visit(Lane& L) {
        uint32_t keys = L.g.y & 0xffu;
        uint32_t key = __ffs(keys) - 1;
        keys &= keys - 1;
        uint32_t slot = key ^ L.cur.oct;
        uint32_t imask = L.g.y >> 8;
        uint32_t child = L.g.x + __popc(imask & ((1u << slot) - 1u));
        if (keys) push(L, make_uint2(L.g.x, (imask << 8) | keys));
        uint32_t nkeys, nimask, cbase, tbase, tmask, lmask;
        visit_node(S.nodes, child, L.cur, limit(L), nkeys, nimask, cbase, tbase, tmask, lmask);
        if (MODE == 3) ++L.work;
        L.g = make_uint2(cbase, (nimask << 8) | nkeys);
        if (tmask) {
            if (SINGLE) L.t = make_uint2(tbase, kTagTri | (lmask << 8) | tmask);
            else if (L.inst >= 0) L.t = make_uint2(L.inst_prim_base + tbase, kTagTri | (lmask << 8) | tmask);
            else L.t = make_uint2(tbase, kTagInst | (lmask << 8) | tmask);
        }
    }

    // Triangle phase: test the lowest triangle of the leaf group.
    LUX_DI void test_one(Lane& L) {
        uint32_t m = L.t.y & kRecMask;
        const uint32_t lm = (L.t.y >> 8) & 0xffu;
        int k = __ffs(m) - 1;
        m &= m - 1;
        L.t.y = m ? (kTagTri | (lm << 8) | m) : 0u;
        k = __popc(lm & ((1u << k) - 1u));  // the slot's record: its rank among the leaf slots
        float t, u, v;
        int prim;
        if (MODE == 3) ++L.work;
        if (SINGLE) {
            // the record names its instance; the object-space ray is rebuilt when it changes,
            // exactly as entering the instance from a TLAS leaf builds it
            const float4* q = S.prims + size_t(L.t.x + uint32_t(k)) * 3;
            const float4 a4 = __ldg(q), e14 = __ldg(q + 1), e24 = __ldg(q + 2);
            const int inst = __float_as_int(e14.w);
            if (inst != L.inst) {
                const DevInstance& I = S.insts[inst];
                const float4* mq = reinterpret_cast<const float4*>(I.Minv);
                const float4 m0 = __ldg(mq), m1 = __ldg(mq + 1), m2 = __ldg(mq + 2);
                const float Minv[12] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w, m2.x, m2.y, m2.z, m2.w};
                L.wo = xform(Minv, L.cur.o, 1.0f);
                L.wd = xform(Minv, L.cur.d, 0.0f);
                L.inst = inst;
                L.inst_flags = __ldg(&I.flags);
            }
            if (!mt_core(a4, e14, e24, L.wo, L.wd, t, u, v, prim)) return;
        } else {
            if (!mt_test(S.prims, L.t.x + uint32_t(k), L.cur, t, u, v, prim)) return;
        }
        if (!(t <= L.tmax)) return;
        if (MODE != 2 && !better(t, L.inst, prim, L.best)) return;
        if (L.inst_flags & kInstAnyHit) {
            int pixel = L.key, iter = A.ext_iter;
            if (A.ext_rays == nullptr) {  // key = path id: pixel in s2.w, iteration in s3.w
                pixel = __float_as_int(A.W.s2[L.key].w);
                iter = __float_as_int(A.W.s3[L.key].w);
            }
            if (!alpha_accept(S, S.insts[L.inst], L.inst, prim, u, v, world_d(L), pixel, iter)) return;
        }
        L.best.t = t;
        L.best.inst = L.inst;
        L.best.prim = prim;
        L.best.u = u;
        L.best.v = v;
        if (MODE == 2) L.done = true;
    }

    // Instance phase: enter the lowest instance of a TLAS leaf group. The world-level node
    // group and the rest of the leaf group wait on the stack under a marker.
    LUX_DI void enter(Lane& L) {
        uint32_t m = L.t.y & kRecMask;
        const uint32_t lm = (L.t.y >> 8) & 0xffu;
        int k = __ffs(m) - 1;
        m &= m - 1;
        const int slot_k = k;
        k = __popc(lm & ((1u << slot_k) - 1u));
        // the instance's leaf record: transform and BLAS root in one dependent 64-byte load
        const float4* q = S.tlas_leaf + size_t(L.t.x + uint32_t(k)) * 4;
        const float4 r0 = __ldg(q), r1 = __ldg(q + 1), r2 = __ldg(q + 2);
        const uint4 e = __ldg(reinterpret_cast<const uint4*>(q + 3));
        if (L.g.y & 0xffu) push(L, L.g);
        if (m) push(L, make_uint2(L.t.x, kTagInst | (lm << 8) | m));
        push(L, make_uint2(0u, kTagMarker));
        const float Minv[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
        L.cur = make_ray(xform(Minv, L.wo, 1.0f), xform(Minv, L.wd, 0.0f));
        L.inst = int(e.w);
        L.inst_flags = int(e.z);
        L.inst_prim_base = e.y;
        L.g = make_uint2(e.x, (1u << 8) | (1u << L.cur.oct));
        L.t = make_uint2(0u, 0u);
    }

    // Pop phase: take the next group from the stack; the ray is done when it is empty.
    LUX_DI void next(Lane& L) {
        while (true) {
            if (L.sp == 0) {
                L.done = true;
                return;
            }
            uint2 e = pop(L);
            uint32_t tag = e.y & kTagMask;
            if (tag == kTagMarker) {
                L.cur = make_ray(L.wo, L.wd);
                L.inst = -1;
                L.inst_flags = 0;
                continue;
            }
            if (tag == kTagNode) L.g = e;
            else L.t = e;
            return;
        }
    }
};


// World normal of a radiance hit as the closest-hit program computes it
// (src/optixshaders/optix_triangle.cu:170-192,224): interpolated vertex normals when the
// mesh has them, else the geometric normal, then the normal transform of the instance.
LUX_DI f3 hit_world_normal(const DevScene& S, int inst, int prim, float bu, float bv) {
    const DevInstance& I = S.insts[inst];
    const uint32_t* id = S.idx + (size_t(I.idx_base) + prim) * 3;
    uint32_t i0 = I.vert_base + __ldg(id), i1 = I.vert_base + __ldg(id + 1), i2 = I.vert_base + __ldg(id + 2);
    f3 n;
    if (I.flags & kInstHasNormals) {
        float bA = __fsub_rn(__fsub_rn(1.0f, bu), bv);
        f3 nA = ld3(S.nrm + i0 * 3), nB = ld3(S.nrm + i1 * 3), nC = ld3(S.nrm + i2 * 3);
        f3 s = mk(__fadd_rn(__fadd_rn(__fmul_rn(bA, nA.x), __fmul_rn(bu, nB.x)), __fmul_rn(bv, nC.x)),
                  __fadd_rn(__fadd_rn(__fmul_rn(bA, nA.y), __fmul_rn(bu, nB.y)), __fmul_rn(bv, nC.y)),
                  __fadd_rn(__fadd_rn(__fmul_rn(bA, nA.z), __fmul_rn(bu, nB.z)), __fmul_rn(bv, nC.z)));
        float l2 = __fadd_rn(__fadd_rn(__fmul_rn(s.x, s.x), __fmul_rn(s.y, s.y)), __fmul_rn(s.z, s.z));
        float il = __fdiv_rn(1.0f, __fsqrt_rn(l2));
        n = mk(__fmul_rn(s.x, il), __fmul_rn(s.y, il), __fmul_rn(s.z, il));
    } else {
        f3 A = ld3(S.pos + i0 * 3), B = ld3(S.pos + i1 * 3), C = ld3(S.pos + i2 * 3);
        f3 e1 = mk(__fsub_rn(B.x, A.x), __fsub_rn(B.y, A.y), __fsub_rn(B.z, A.z));
        f3 e2 = mk(__fsub_rn(C.x, A.x), __fsub_rn(C.y, A.y), __fsub_rn(C.z, A.z));
        f3 c = mk(__fsub_rn(__fmul_rn(e1.y, e2.z), __fmul_rn(e2.y, e1.z)), __fsub_rn(__fmul_rn(e1.z, e2.x), __fmul_rn(e2.z, e1.x)),
                  __fsub_rn(__fmul_rn(e1.x, e2.y), __fmul_rn(e2.x, e1.y)));
        float l2 = __fadd_rn(__fadd_rn(__fmul_rn(c.x, c.x), __fmul_rn(c.y, c.y)), __fmul_rn(c.z, c.z));
        float il = __fdiv_rn(1.0f, __fsqrt_rn(l2));
        n = mk(__fmul_rn(c.x, il), __fmul_rn(c.y, il), __fmul_rn(c.z, il));
    }
    f3 w = xform(I.MinvT, n, 0.0f);
    float l2 = __fadd_rn(__fadd_rn(__fmul_rn(w.x, w.x), __fmul_rn(w.y, w.y)), __fmul_rn(w.z, w.z));
    float il = __fdiv_rn(1.0f, __fsqrt_rn(l2));
    return mk(__fmul_rn(w.x, il), __fmul_rn(w.y, il), __fmul_rn(w.z, il));
}

template <int MODE, bool SINGLE>
// The arguments stay in parameter space (__grid_constant__): the tracer reads the scene
// through a reference to them, which would otherwise copy the struct to local memory.
// Seven 128-thread blocks per SM (at most 73 registers) measured faster than six (80) and
// eight (64, with spills).
__global__ void __launch_bounds__(kTraceBlock, 7) k_trace(const __grid_constant__ TraceArgs A) {
    __shared__ uint2 stack[kShStack][kTraceBlock];
    // work of segment k: items [seg_first[k], seg_first[k + 1]) of the launch's list
    __shared__ int seg_first[kMaxSegs + 1];
    const bool ext = A.ext_rays != nullptr;
    if (threadIdx.x == 0) {
        int t = 0;
        seg_first[0] = 0;
        for (int k = 0; k < kMaxSegs; ++k) {
            if (!ext && k < A.G.n) {
                const WaveCounters* c = A.W.ctr + A.G.lane[k];
                t += (MODE == 0 || MODE == 3) ? *(volatile const int*)&c->count[A.G.bounce[k]]
                                              : *(volatile const int*)&c->shadow[A.G.bounce[k]];
            }
            seg_first[k + 1] = t;
        }
    }
    __syncthreads();
    Tracer<MODE, SINGLE> T{A.S, stack, {}, int(threadIdx.x), &(A.W.ctr + A.G.lane[0])->error, A};
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int total;
    int* cursor;
    // the cursor of the first segment's (lane, bounce) serves the whole launch: no other
    // launch of this kind covers that lane at that bounce
    if (ext) {
        total = A.ext_n;
        cursor = A.ext_fetch;
    } else if (MODE == 0 || MODE == 3) {
        total = seg_first[kMaxSegs];
        cursor = &(A.W.ctr + A.G.lane[0])->fetch_r[A.G.bounce[0]];
    } else {
        total = seg_first[kMaxSegs];
        cursor = &(A.W.ctr + A.G.lane[0])->fetch_s[A.G.bounce[0]];
    }
    Lane L;
    bool active = false;
    bool exhausted = false;  // warp-uniform: the cursor has passed the end of the work list
    bool pending = false;    // the lane's ray is done and its result not yet written
    int item = 0;
    // Every lane of the warp runs every phase below (lanes without a ray or without work for
    // a phase are predicated off), so the ballots see the whole warp.
    while (true) {
        // Results of the rays that finished, written by all such lanes of the warp together
        // (at least 32 - kRefill of them, or the last ones): a lane that finishes keeps its
        // ray state untouched until the refill below replaces it.
        if (pending) {
            pending = false;
            if (ext) {
                uint32_t* h = A.ext_hits + size_t(item) * 5;
                if (MODE == 2) {
                    h[0] = __float_as_uint(L.best.inst >= 0 ? 1.0f : -1.0f);
                    h[1] = h[2] = 0xffffffffu;
                    h[3] = h[4] = 0u;
                } else if (MODE == 3) {
                    h[0] = __float_as_uint(L.best.inst >= 0 ? L.best.t : -1.0f);
                    h[1] = uint32_t(L.best.inst);
                    h[2] = uint32_t(L.best.prim);
                    h[3] = uint32_t(L.work);
                    h[4] = 0u;
                } else {
                    h[0] = __float_as_uint(L.best.inst >= 0 ? L.best.t : -1.0f);
                    h[1] = uint32_t(L.best.inst);
                    h[2] = uint32_t(L.best.prim);
                    h[3] = __float_as_uint(L.best.inst >= 0 ? L.best.u : 0.0f);
                    h[4] = __float_as_uint(L.best.inst >= 0 ? L.best.v : 0.0f);
                }
            } else if (MODE == 0) {
                bool hit = L.best.inst >= 0;
                st_stream(&A.W.hit[item], make_float4(hit ? L.best.t : -1.0f, L.best.u, L.best.v, __int_as_float(L.best.inst)));
                st_stream(&A.W.hit_prim[item], L.best.prim);
                if (hit && A.nee) {
                    // shadow ray of the raygen program (src/optixshaders/optix_triangle.cu:82-132)
                    f3 n = hit_world_normal(A.S, L.best.inst, L.best.prim, L.best.u, L.best.v);
                    const f3 wo = Tracer<MODE, SINGLE>::world_o(L), wd = Tracer<MODE, SINGLE>::world_d(L);
                    f3 hp = mk(__fadd_rn(wo.x, __fmul_rn(L.best.t, wd.x)), __fadd_rn(wo.y, __fmul_rn(L.best.t, wd.y)),
                               __fadd_rn(wo.z, __fmul_rn(L.best.t, wd.z)));
                    f3 so = mk(__fadd_rn(hp.x, __fmul_rn(n.x, 1e-4f)), __fadd_rn(hp.y, __fmul_rn(n.y, 1e-4f)),
                               __fadd_rn(hp.z, __fmul_rn(n.z, 1e-4f)));
                    // the segment of this slot: its lane, then the segment holding that lane
                    int k = 0;
                    if (A.G.n > 1) {
                        const int ln = item / A.W.lane_stride;
                        while (k + 1 < A.G.n && A.G.lane[k] != ln) ++k;
                    }
                    const int bk = A.G.bounce[k], lk = A.G.lane[k];
                    int pid = ld_stream(&A.W.queue[bk & 1][item]);
                    float4 ns = ld_stream(&A.W.s4[pid]);
                    f3 sd;
                    float tmax;
                    if (A.nee == 2) {
                        sd = mk(ns.x, ns.y, ns.z);
                        tmax = 1e16f;
                    } else {
                        f3 ld = mk(__fsub_rn(ns.x, so.x), __fsub_rn(ns.y, so.y), __fsub_rn(ns.z, so.z));
                        float dl = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ld.x, ld.x), __fmul_rn(ld.y, ld.y)), __fmul_rn(ld.z, ld.z)));
                        float il = __fdiv_rn(1.0f, dl);
                        sd = mk(__fmul_rn(ld.x, il), __fmul_rn(ld.y, il), __fmul_rn(ld.z, il));
                        tmax = __fadd_rn(__fmul_rn(dl, 1.0001f), 1e-4f);
                    }
                    // append to the lane's shadow queue, aggregated over the lanes of the
                    // warp that append to the same one; the ray is stored at its queue
                    // position, beside the slot it belongs to, so the occlusion launch reads
                    // rays contiguously and without first reading the slot
                    const unsigned am = __match_any_sync(__activemask(), lk);
                    int leader = __ffs(am) - 1;
                    int b2 = 0;
                    if (lane == leader) b2 = atomicAdd(&(A.W.ctr + lk)->shadow[bk], __popc(am));
                    b2 = __shfl_sync(am, b2, leader);
                    const size_t q = size_t(lk) * A.W.lane_stride + b2 + __popc(am & ((1u << lane) - 1u));
                    st_stream(&A.W.sh_o[q], make_float4(so.x, so.y, so.z, tmax));
                    st_stream(&A.W.sh_d[q], make_float4(sd.x, sd.y, sd.z, 0.0f));
                    st_stream(&A.W.sh_queue[q], item);
                }
            } else if (MODE == 1) {
                bool hit = L.best.inst >= 0;
                st_stream(&A.W.sh_hit[item], make_float4(hit ? L.best.t : -1.0f, L.best.u, L.best.v, __int_as_float(L.best.inst)));
                st_stream(&A.W.sh_prim[item], L.best.prim);
            } else if (MODE == 3) {
                // drawBVH (src/kernels/draw_bvh.cu:33): color += count * 0.001 on every channel
                int pid = A.W.queue[A.G.bounce[0] & 1][item];  // the heatmap traces one wave
                float4 c = A.W.s3[pid];
                const float h = float(L.work) * 0.001f;
                A.W.s3[pid] = make_float4(c.x + h, c.y + h, c.z + h, c.w);
            } else {
                st_stream(&A.W.sh_hit[item], make_float4(L.best.inst >= 0 ? 1.0f : -1.0f, 0.0f, 0.0f, __int_as_float(-1)));
            }
        }
        unsigned need = __ballot_sync(FULL, !active);
        if (need && !exhausted) {
            int base = 0;
            if (lane == 0) base = atomicAdd(cursor, __popc(need));
            base = __shfl_sync(FULL, base, 0);
            if (base + __popc(need) >= total) exhausted = true;
            if (!active) {
                int r = base + __popc(need & ((1u << lane) - 1u));
                if (r < total) {
                    item = r;
                    f3 o, d;
                    float tmax;
                    uint32_t root = A.S.tlas_root;
                    L.key = 0;
                    if (ext) {
                        const float* ry = A.ext_rays + size_t(r) * 8;
                        o = mk(ry[0], ry[1], ry[2]);
                        d = mk(ry[4], ry[5], ry[6]);
                        tmax = MODE == 1 ? ry[3] : 1e16f;
                        L.key = __float_as_int(ry[7]);
                    } else if (MODE == 0 || MODE == 3) {
                        int k = 0;
                        while (k + 1 < A.G.n && r >= seg_first[k + 1]) ++k;
                        item = A.G.lane[k] * A.W.lane_stride + (r - seg_first[k]);  // absolute slot
                        int pid = ld_stream(&A.W.queue[A.G.bounce[k] & 1][item]);
                        float4 a = ld_stream(&A.W.s0[pid]), b = ld_stream(&A.W.s1[pid]);
                        o = mk(a.x, a.y, a.z);
                        d = mk(b.x, b.y, b.z);
                        tmax = 1e16f;
                        L.key = pid;
                        if (A.W.path_job) root = A.W.jobs[A.W.path_job[pid]].tlas_root;
                    } else {
                        int k = 0;
                        while (k + 1 < A.G.n && r >= seg_first[k + 1]) ++k;
                        const size_t q = size_t(A.G.lane[k]) * A.W.lane_stride + (r - seg_first[k]);
                        int slot = ld_stream(&A.W.sh_queue[q]);
                        item = slot;
                        float4 a = ld_stream(&A.W.sh_o[q]), b = ld_stream(&A.W.sh_d[q]);
                        o = mk(a.x, a.y, a.z);
                        d = mk(b.x, b.y, b.z);
                        tmax = a.w;
                        int pid = ld_stream(&A.W.queue[A.G.bounce[k] & 1][slot]);
                        L.key = pid;
                        if (A.W.path_job) root = A.W.jobs[A.W.path_job[pid]].tlas_root;
                    }
                    T.start(L, o, d, tmax, root);
                    active = true;
                }
            }
        }
        if (!__any_sync(FULL, active)) break;
        while (true) {
            // node phase
            if (active && (L.g.y & 0xffu)) T.visit(L);
            // triangle phase, postponed while too few lanes have triangles and others nodes
            while (true) {
                const bool want = active && (L.t.y & kTagMask) == kTagTri;
                const unsigned wm = __ballot_sync(FULL, want);
                if (!wm) break;
                const bool nodes = active && (L.g.y & 0xffu);
                if (__popc(wm) < kPostpone && __any_sync(FULL, nodes)) {
                    // lanes with nodes left push their triangles; the others keep them
                    if (want && nodes) {
                        T.push(L, L.t);
                        L.t = make_uint2(0u, 0u);
                    }
                    break;
                }
                if (want) T.test_one(L);
                if (MODE == 2 && want && L.done) {
                    L.t = make_uint2(0u, 0u);
                    L.g = make_uint2(0u, 0u);
                }
            }
            // instance phase
            if (active && !L.done && (L.t.y & kTagMask) == kTagInst) T.enter(L);
            // pop phase
            if (active && !L.done && !(L.g.y & 0xffu) && !(L.t.y & kRecMask)) T.next(L);
            if (active && L.done) {
                active = false;
                pending = true;
            }
            const unsigned am = __ballot_sync(FULL, active);
            if (!am) break;
            if (__popc(am) < (MODE == 2 ? kRefillOcclusion : kRefill) && !exhausted) break;
        }
    }
}

}  // namespace

// Persistent grid of each traversal kind: SMs x resident blocks per SM. The answer depends on
// the device, so it is cached per device ordinal, under a lock (contexts on several devices and
// several host threads ask for it).
int trace_grid_blocks(int mode, bool single) {
    static std::mutex mu;
    static std::map<int, std::array<int, 8>> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    int& cached = cache[dev][mode * 2 + (single ? 1 : 0)];
    if (cached == 0) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (single) {
            if (mode == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<0, true>, kTraceBlock, 0);
            else if (mode == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<1, true>, kTraceBlock, 0);
            else if (mode == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<2, true>, kTraceBlock, 0);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<3, true>, kTraceBlock, 0);
        } else {
            if (mode == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<0, false>, kTraceBlock, 0);
            else if (mode == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<1, false>, kTraceBlock, 0);
            else if (mode == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<2, false>, kTraceBlock, 0);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trace<3, false>, kTraceBlock, 0);
        }
        cached = sms * (per > 0 ? per : 1);
    }
    return cached;
}

namespace {
template <bool SINGLE>
void launch_mode(int mode, int grid, cudaStream_t st, const TraceArgs& A) {
    if (mode == 0) k_trace<0, SINGLE><<<grid, kTraceBlock, 0, st>>>(A);
    else if (mode == 1) k_trace<1, SINGLE><<<grid, kTraceBlock, 0, st>>>(A);
    else if (mode == 2) k_trace<2, SINGLE><<<grid, kTraceBlock, 0, st>>>(A);
    else k_trace<3, SINGLE><<<grid, kTraceBlock, 0, st>>>(A);
}
}  // namespace

cudaError_t launch_trace(const DevScene& S, const DevWave& W, int bounce, int mode, int nee, cudaStream_t st,
                         int grid) {
    return launch_trace_segs(S, W, one_seg(bounce), mode, nee, st, grid);
}

cudaError_t launch_trace_segs(const DevScene& S, const DevWave& W, const Segs& G, int mode, int nee, cudaStream_t st,
                              int grid) {
    if (G.n < 1 || G.n > kMaxSegs) return cudaErrorInvalidValue;
    TraceArgs A{S, W, G, mode, nee, nullptr, nullptr, 0, 0, nullptr};
    const bool single = S.single_level != 0;
    if (grid <= 0) grid = trace_grid_blocks(mode, single);
    if (single) launch_mode<true>(mode, grid, st, A);
    else launch_mode<false>(mode, grid, st, A);
    return cudaGetLastError();
}

cudaError_t launch_trace_ext(const DevScene& S, const DevWave& W, const float* rays, uint32_t* hits, int n, int mode,
                             int iter, int* fetch, cudaStream_t st) {
    TraceArgs A{S, W, one_seg(0), mode, 0, rays, hits, n, iter, fetch};
    const bool single = S.single_level != 0;
    const int grid = trace_grid_blocks(mode, single);
    if (single) launch_mode<true>(mode, grid, st, A);
    else launch_mode<false>(mode, grid, st, A);
    return cudaGetLastError();
}

}  // namespace lux
