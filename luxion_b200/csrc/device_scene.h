// device_scene.h -- HBM layout of a resident scene and of one wavefront, shared by the host
// side (context.cpp) and the kernels.
//
// Scene (read-only during rendering):
//   nodes   BVH8 nodes (80 B, bvh8.h) of every mesh's BLAS, then the TLAS over instances
//   prims   3 x float4 per leaf primitive record in BVH order: (v0, prim id), e1, e2 with
//           e1 = v1 - v0 and e2 = v2 - v0 rounded once on the host, exactly the values the
//           Moller-Trumbore test of src/intersections/mesh_isect.cu:79-82 computes
//   insts   per instance: object<->world matrices, mesh bases, material, flags
//   pos/nrm/uv/idx  shading attributes in the input order (single index stream)
//   mats    uber-shader materials with bound texture objects
//   light tables: emissive-area CDF, per-emissive-instance triangle CDFs, HDRI CDFs
// Wavefront (per path id, SoA of float4 so each field is one 16-byte load):
//   s0 = origin, last_pdf    s1 = direction, flags    s2 = throughput, pixel
//   s3 = radiance, iteration s4 = NEE sample (DL point or env direction)
// plus two path-id queues, per-slot hit records and the shadow-ray queue.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lux {

enum InstFlags : int { kInstHasNormals = 1, kInstHasUVs = 2, kInstAnyHit = 4 };

// 16-byte aligned (192 bytes): traversal reads Minv as three float4.
struct alignas(16) DevInstance {
    float M[12];      // object -> world, columns 0..3 of the 4x4 (rows 0..2)
    float Minv[12];   // world -> object
    float MinvT[12];  // inverse transpose (normal transform)
    int mesh;
    int material;
    uint32_t blas_root;   // node index of the mesh's BLAS root
    uint32_t prim_base;   // first primitive record of the mesh
    uint32_t vert_base;   // first vertex of the mesh in pos/nrm/uv
    uint32_t idx_base;    // first index triplet of the mesh
    int flags;            // InstFlags
    int num_tris;
    int key;              // index of the instance within its own scene (alpha-blend hash key)
};

enum MatFlags : int { kMatAlbedoTex = 1, kMatEmissiveTex = 2, kMatNormalTex = 4, kMatMRTex = 8 };

struct DevTexTransform {
    float offset[2];
    float scale[2];
    float rotation;
};

struct DevMaterial {
    float color[3];
    float alpha;
    float emission[3];  // emission_color * emission_strength, rounded as the shader does
    float roughness;
    float metallic;
    float transmission;
    float ior;
    float alpha_cutoff;
    int alpha_mode;
    int flags;  // MatFlags
    int pad[2];
    unsigned long long albedo_tex, emissive_tex, normal_tex, mr_tex;
    DevTexTransform albedo_tt, emissive_tt, normal_tt, mr_tt;
};

struct DevScene {
    const uint4* nodes;
    const float4* prims;
    const DevInstance* insts;
    const uint32_t* tlas_prims;  // TLAS leaf records -> instance index
    // per TLAS leaf record, what entering its instance needs in one 64-byte load: the
    // world -> object matrix (12 floats, as DevInstance::Minv) in three float4, then
    // (blas_root, prim_base, flags, instance) as int bits
    const float4* tlas_leaf;
    uint32_t tlas_root;
    int num_insts;
    // 1: nodes under tlas_root are one world-space BVH over instanced triangles; its leaf
    // records carry their instance in e1.w and are tested in that instance's object space.
    // 0: two levels, a TLAS over instances (tlas_leaf records) above per-mesh BLASes.
    int single_level;
    const float* pos;
    const float* nrm;
    const float* uv;
    const uint32_t* idx;
    const DevMaterial* mats;
    // light sampling tables (src/scene/scene_precompute.cpp:22-124)
    const int* emissive_inst;
    const float* emissive_prefix;
    const float* tri_prefix;      // concatenated per emissive instance
    const int* tri_prefix_off;    // offset of each emissive instance's table
    int num_emissive;
    float total_area;
    const float* marginal;
    const float* conditional;
    const int* marginal_guide;     // guide_marg + 1 entries (select_from_cdf_guided)
    const int* conditional_guide;  // guide_cond + 1 entries per row
    int guide_marg, guide_cond;
    int env_w, env_h;
    unsigned long long env_tex;
    int has_env;
    float morton_bmin[3], morton_bmax[3];
};

struct DevCamera {
    float pos[3], view[3], right[3], up[3];
    float pixel_length[2];
    int width, height;
};

struct DevOptions {
    int dl;             // -dmis
    int env;            // -emis
    float env_intensity;
    int trace_depth;
    int color_mode;
    int precision;
    int material_debug;  // LUX_MATDEBUG_* (trace depth is 1 when set)
};

// Per-bounce device counters, zeroed once per wave (one memset):
//   count[b]     queue length entering bounce b (count[0] = paths of the wave)
//   shadow[b]    shadow rays queued at bounce b
//   fetch_r[b], fetch_s[b]  work-fetch cursors of the persistent trace kernels
//   error        sticky error word (bit 0: traversal stack overflow)
constexpr int kMaxDepth = 64;
struct WaveCounters {
    int count[kMaxDepth + 1];
    int shadow[kMaxDepth];
    int fetch_r[kMaxDepth];
    int fetch_s[kMaxDepth];
    int error;
    int pad[3];
};

// One render job of the shared wavefront (job engine): a scene, a camera and resolution, a
// sample count and a trace depth, and its own accumulation buffers (3 floats per pixel;
// comp only in the compensated form).
struct DevJob {
    int scene;
    int width, height, npix;
    int trace_depth;
    int first_iter;       // iteration of the job's sample 0 (1-based, as the reference's iter)
    uint32_t tlas_root;   // TLAS root of the job's scene in the concatenated node array
    int pad;
    float* image;
    float* comp;
    float pos[3], view[3], right[3], up[3];
    float pixel_length[2];
};

// A wave segment: samples [sample0, sample0 + nsamples) of one job. Its paths occupy
// [path0, path0 + nsamples * npix) sample-major; pix0 is the prefix of the wave's segment
// pixel counts (the accumulate kernel's index space).
struct DevSegment {
    int job;
    int sample0;
    int nsamples;
    int path0;
    int pix0;
};
constexpr int kMaxSegments = 256;

// Waves in flight together (wave pipelining). A wave lives in a lane: lane l owns paths and
// slots [l * lane_stride, (l + 1) * lane_stride) of every per-path and per-slot array (state,
// queues, hit and shadow records) and the counters ctr[l]. Path ids and slots are absolute, so
// a kernel finds a lane's data at its offset. One bounce-step launch covers up to kMaxSegs
// segments, each a lane at its own bounce; the single-wave paths use one segment, lane 0.
constexpr int kMaxSegs = 4;
struct Segs {
    int n;                  // segments, 1 .. kMaxSegs
    int lane[kMaxSegs];
    int bounce[kMaxSegs];   // the lane's bounce (depth after shading = bounce + 1)
    int compact[kMaxSegs];  // shade: append survivors to the lane's next queue
};
inline Segs one_seg(int bounce, int compact = 1) {
    Segs g{};
    g.n = 1;
    g.lane[0] = 0;
    g.bounce[0] = bounce;
    g.compact[0] = compact;
    return g;
}

struct DevWave {
    float4* s0;
    float4* s1;
    float4* s2;
    float4* s3;
    float4* s4;
    int* queue[2];
    float4* hit;      // per slot: t, u, v, instance (int bits)
    int* hit_prim;    // per slot
    float4* sh_o;     // per shadow-queue position: shadow origin, tmax
    float4* sh_d;     // per shadow-queue position: shadow direction
    int* sh_queue;    // per shadow-queue position: the slot the shadow ray belongs to
    float4* sh_hit;   // per slot: DL hit t, u, v, instance; env: occlusion in .x
    int* sh_prim;
    uint32_t* keys;   // Morton keys (ray sorting)
    uint32_t* keys_alt;
    int* queue_alt;
    WaveCounters* ctr;  // one per lane
    int* wave_iter;   // per wave of a render call: first iteration, samples
    // job engine only (null for a single-job context):
    const DevScene* scenes;    // per resident scene: geometry of the concatenated arrays + its lights
    const DevJob* jobs;
    const DevSegment* segs;    // the wave's segments, wave_hdr[0] of them
    int* wave_hdr;             // [0] segments, [1] paths, [2] pixels over the segments
    int* path_job;             // job of each path
    int npix;         // pixels of the job
    int width, height;
    int max_paths;    // paths of one lane
    int lane_stride;  // paths (and slots) per lane; lanes = allocated / lane_stride
};

}  // namespace lux
