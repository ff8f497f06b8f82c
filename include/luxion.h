/*
 * luxion.h -- C-ABI of the B200 wavefront path tracer.
 *
 * The entry points replace the render path of seabiscuit-iv/luxion:
 *   pathtraceInit(Scene*)         include/pathtrace/pathtrace_buffers.h:5,
 *                                 src/pathtrace/pathtrace_buffers.cu:21-140   -> lux_init
 *   pathtrace(uchar4*, int, int)  include/pathtrace.h:13, src/pathtrace.cu:97  -> lux_render_iter
 *   pathtraceFree()               include/pathtrace/pathtrace_buffers.h:6,
 *                                 src/pathtrace/pathtrace_buffers.cu:142-177  -> lux_free
 *   copyImageToHost()             include/pathtrace/pathtrace_buffers.h:7,
 *                                 src/pathtrace/pathtrace_buffers.cu:180-190  -> lux_copy_image
 *   PathTracerOptions             include/pathtrace/pathtracer_options.h:3-21 -> lux_options
 *   checkCUDAError (exit on error) include/common.h:16-36                    -> status codes +
 *                                                                              lux_last_error
 *
 * Conventions: plain C types only; every call returns LUX_OK (0) or a negative status and
 * never exits the process.  The caller owns every host buffer it passes; a context owns its
 * device memory.  A context is used by one host thread at a time; distinct contexts may run
 * concurrently on distinct streams.
 */
#ifndef LUXION_H
#define LUXION_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUX_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------------- */
enum {
    LUX_OK = 0,
    LUX_ERR_INVALID = -1,     /* bad argument or malformed scene                           */
    LUX_ERR_CUDA = -2,        /* a CUDA runtime call failed (text in lux_last_error)        */
    LUX_ERR_NO_DEVICE = -3,   /* no sm_100 device visible                                  */
    LUX_ERR_OOM = -4,         /* device allocation failed or the HBM budget is exceeded    */
    LUX_ERR_UNSUPPORTED = -5, /* option combination not implemented                        */
    LUX_ERR_TIMEOUT = -6,     /* a bounded device wait gave up (status read from device)   */
    LUX_ERR_STATE = -7        /* call out of order (e.g. render before init)               */
};

/* ---- scene description (POD views of caller-owned host memory) ------------------------- */

/* Texel storage formats. The reference stores every texture as float4 with hardware
 * bilinear filtering, wrap addressing and normalised coordinates (src/texture.cu:12-69). */
enum {
    LUX_TEX_RGBA8 = 0,    /* 4 x u8 unorm                    */
    LUX_TEX_RGBA16 = 1,   /* 4 x u16 unorm                   */
    LUX_TEX_RGBA32F = 2,  /* 4 x f32                         */
    LUX_TEX_RGBA16F = 3   /* 4 x f16 (IEEE binary16)         */
};

typedef struct lux_texture_desc {
    int32_t width, height;
    int32_t format;          /* LUX_TEX_*                                                   */
    int32_t _pad;
    const void* data;        /* width*height texels, row-major, 4 channels                  */
} lux_texture_desc;

/* KHR_texture_transform: uv*scale -> rotate -> +offset (src/material_queries.cu:3-17). */
typedef struct lux_tex_transform {
    float offset[2];
    float scale[2];
    float rotation;
} lux_tex_transform;

enum { LUX_ALPHA_OPAQUE = 0, LUX_ALPHA_MASK = 1, LUX_ALPHA_BLEND = 2 };

/* Mirrors the fields of the reference Material the uber-shader reads
 * (include/sceneStructs.h:94-131). Texture indices are -1 when absent. */
typedef struct lux_material_desc {
    float color[3];
    int32_t albedo_tex;
    float alpha;
    int32_t alpha_mode;      /* LUX_ALPHA_*                                                 */
    float alpha_cutoff;
    float emission_strength;
    float emission_color[3];
    int32_t emissive_tex;
    float roughness;
    float metallic;
    int32_t normal_tex;
    int32_t metallic_roughness_tex;
    float transmission;
    float ior;
    lux_tex_transform albedo_tt, emissive_tt, normal_tt, metallic_roughness_tt;
} lux_material_desc;

/* One triangle mesh in object space. A single index stream addresses positions, normals and
 * uvs, as the reference's glTF loader does (src/scene/scene_load_gltf.cpp:430). */
typedef struct lux_mesh_desc {
    int32_t num_verts;
    int32_t num_tris;
    const float* positions;  /* num_verts * 3                                               */
    const float* normals;    /* num_verts * 3, or NULL (geometric normals are used)          */
    const float* uvs;        /* num_verts * 2, or NULL (uv = 0, tangent = +x)                */
    const uint32_t* indices; /* num_tris * 3                                                */
} lux_mesh_desc;

/* One placed mesh (a reference Geom, include/sceneStructs.h:66-79). Matrices are 4x4
 * column-major, the glm layout. When has_inverse is 0 the library derives inverse and
 * inverse-transpose itself. */
typedef struct lux_instance_desc {
    int32_t mesh;
    int32_t material;
    int32_t has_inverse;
    int32_t _pad;
    float transform[16];
    float inverse[16];
    float inv_transpose[16];
} lux_instance_desc;

/* Pinhole camera, the reference Camera (include/sceneStructs.h:133-143). */
typedef struct lux_camera_desc {
    int32_t width, height;
    float position[3];
    float look_at[3];
    float view[3];
    float up[3];
    float right[3];
    float fov[2];
    float pixel_length[2];
} lux_camera_desc;

typedef struct lux_scene_desc {
    int32_t num_meshes, num_instances, num_materials, num_textures;
    const lux_mesh_desc* meshes;
    const lux_instance_desc* instances;
    const lux_material_desc* materials;
    const lux_texture_desc* textures;
    lux_camera_desc camera;
    int32_t trace_depth;     /* RenderState::traceDepth (include/sceneStructs.h:145-151)      */
    /* Environment map (an HDRI); env_data NULL means none. RGBA texels; the reference keeps
     * the alpha channel and feeds it to the CDF weight (src/scene/scene_precompute.cpp:88). */
    int32_t env_width, env_height;
    int32_t env_format;      /* LUX_TEX_RGBA32F or LUX_TEX_RGBA16F                          */
    const void* env_data;
} lux_scene_desc;

/* ---- options (PathTracerOptions + CLI flags -dmis -emis) -------------------------------- */
enum { LUX_TONEMAP_REINHARD = 0, LUX_TONEMAP_AGX = 1, LUX_TONEMAP_ACES = 2 };
enum { LUX_PRECISION_PLAIN = 0, LUX_PRECISION_COMPENSATED = 1 };
/* How scene textures are held in HBM. FLOAT converts 8/16-bit texels to float4 exactly as
 * the reference's upload does (src/texture.cu:17-27), so filtered values match it; UNORM8
 * keeps 8-bit texels as they are (4 B/texel, filtered by the hardware unorm path); HALF
 * stores IEEE binary16 (the precision form). */
enum { LUX_TEXSTORE_FLOAT = 0, LUX_TEXSTORE_UNORM8 = 1, LUX_TEXSTORE_HALF = 2 };
/* Material debug views (PathTracerOptions::material_debug_mode, include/pathtrace/
 * pathtracer_options.h:5; render_material_debug_mode, src/material_debug_render.cu:3-26):
 * trace depth 1, a camera hit shows one material channel, the display skips tone mapping. */
enum {
    LUX_MATDEBUG_OFF = 0,
    LUX_MATDEBUG_ALBEDO = 1,
    LUX_MATDEBUG_NORMAL = 2,     /* shading normal * 0.5 + 0.5                          */
    LUX_MATDEBUG_NORMAL_MAP = 3, /* raw normal-map texel, (0.5, 0.5, 1) without one      */
    LUX_MATDEBUG_ROUGHNESS = 4,
    LUX_MATDEBUG_METALLIC = 5,
    LUX_MATDEBUG_ALPHA = 6
};

typedef struct lux_options {
    int32_t direct_light_sampling;       /* -dmis                                            */
    int32_t env_importance_sampling;     /* -emis                                            */
    int32_t color_mode;                  /* LUX_TONEMAP_*, default ACES                       */
    float envmap_intensity;              /* default 1                                        */
    int32_t trace_depth;                 /* 0: take scene trace_depth                        */
    int32_t ray_sorting;                 /* 1: Morton-sort each bounce's queue (RAY_SORTING)  */
    int32_t precision;                   /* LUX_PRECISION_*                                  */
    int32_t spp_per_wave;                /* samples kept in flight together; 0 = automatic    */
    int32_t use_graph;                   /* 1: replay the bounce loop as a CUDA graph         */
    int32_t texture_storage;             /* LUX_TEXSTORE_*                                    */
    int32_t device;                      /* CUDA device ordinal                              */
    void* stream;                        /* cudaStream_t to launch on; NULL = a private one  */
    int32_t material_debug_mode;         /* LUX_MATDEBUG_*                                   */
    int32_t debug_bvh;                   /* 1: BVH heatmap of camera rays (PathTracerOptions::
                                          * debug_bvh, src/kernels/draw_bvh.cu:6-35): each
                                          * sample adds (BVH8 node visits + triangle tests)
                                          * * 0.001 to every channel of its pixel             */
    int32_t bvh_layout;                  /* LUX_BVH_*: how a scene build lays out its BVH     */
} lux_options;

/* BVH layout of a scene build. Both give the same hits bit for bit (every triangle is tested
 * in its instance's object space, as the reference does, src/intersections/mesh_isect.cu:15-16):
 * SINGLE_LEVEL builds one world-space BVH per scene over all instanced triangles, so traversal
 * never switches instances; TWO_LEVEL builds one BLAS per mesh and a TLAS over the instances
 * (the reference's GAS/IAS structure), which keeps one copy of a mesh that many instances
 * share. AUTO takes SINGLE_LEVEL unless the instanced triangles are both more than twice the
 * meshes' and more than 16M. */
enum { LUX_BVH_AUTO = 0, LUX_BVH_TWO_LEVEL = 1, LUX_BVH_SINGLE_LEVEL = 2 };

typedef struct lux_ctx lux_ctx;
typedef struct lux_scene lux_scene;

/* Fill *opt with the reference defaults (include/pathtrace/pathtracer_options.h:3-11). */
void lux_default_options(lux_options* opt);

/* pathtraceInit: upload the scene, build the acceleration structure and the light CDFs,
 * allocate every per-path buffer. The context owns the scene it built. */
int lux_init(const lux_scene_desc* scene, const lux_options* opt, lux_ctx** out);

/* A resident scene: geometry, BVH, materials, textures and light CDFs on one device, built
 * once. The reference does this work at load, before the first pathtraceInit: mesh uploads and
 * acceleration builds in main() (src/main.cpp:199-274) and the light precompute
 * (src/scene/scene_precompute.cpp:22-124). Of the options only device, texture_storage,
 * precision and bvh_layout shape the build; every context made on the scene must use the same
 * device, texture_storage and precision. */
int lux_scene_create(const lux_scene_desc* scene, const lux_options* opt, lux_scene** out);
/* pathtraceInit on a resident scene (src/pathtrace/pathtrace_buffers.cu:21-140): allocate only
 * the per-pixel and per-path state for `camera` (any resolution; NULL = the description's
 * camera) and take the trace depth from opt (0 = the description's). No scene work is done, so
 * the reference's pathtraceFree(); pathtraceInit() on every camera or option reset
 * (src/app/render_loop.cpp:122-126) costs allocations only. The context holds a reference to
 * the scene. */
int lux_init_on_scene(lux_scene* scene, const lux_camera_desc* camera, const lux_options* opt, lux_ctx** out);
/* Drop the caller's reference: the scene is freed once no context uses it. NULL is accepted. */
int lux_scene_free(lux_scene* scene);
/* Device bytes the scene holds (geometry, BVH, tables, textures). */
int64_t lux_scene_device_bytes(const lux_scene* scene);

/* Host wall time of the stages of a scene build (no counterpart in the reference). The
 * geometry (vertex upload, then every BLAS, then instances and TLAS) is built on one thread
 * while the textures upload on another and the light tables are built on a third. */
typedef struct lux_scene_stats {
    double ms_total;          /* the whole build, to the last upload                          */
    double ms_geometry;       /* upload + BLAS + TLAS                                          */
    double ms_upload;         /* vertex data to the device                                     */
    double ms_blas;           /* triangle boxes, every mesh's BVH8, triangle records (device)   */
    double ms_tlas;           /* instance records, instance boxes, TLAS (device)               */
    double ms_tables;         /* light CDFs and materials (host)                               */
    double ms_textures;       /* textures and environment map                                  */
    int64_t device_bytes;
    int64_t blas_nodes, tlas_nodes;
} lux_scene_stats;
int lux_scene_get_stats(const lux_scene* scene, lux_scene_stats* out);
/* The same for the scene a context renders (the one lux_init built, or the resident one). */
int lux_get_scene_stats(lux_ctx* ctx, lux_scene_stats* out);

/* pathtrace: render one sample per pixel. iter is 1-based and seeds the RNG exactly like
 * the reference (include/common.h:38-47). The sample is added to the FP32 accumulation
 * image. If rgba8_dev is not NULL it receives the tonemapped image of the running mean
 * (sendImageToPBO, src/kernels/image_kernels.cu:6-46); it is a device pointer, as the
 * reference's PBO is. */
int lux_render_iter(lux_ctx* ctx, int iter, uint8_t* rgba8_dev);

/* Render n_iter samples, iterations first_iter .. first_iter+n_iter-1, keeping up to
 * spp_per_wave of them in flight together; the image equals n_iter lux_render_iter calls. */
int lux_render(lux_ctx* ctx, int first_iter, int n_iter);

/* copyImageToHost: the accumulation SUM (not the mean), W*H*3 floats. */
int lux_copy_image(lux_ctx* ctx, float* rgb_host);
/* The same sum copied to device memory of the context's device (rgb_dev: W*H*3 floats), on
 * the context's stream and without waiting for it: for combining the images of several GPUs
 * with a device collective. */
int lux_copy_image_device(lux_ctx* ctx, float* rgb_dev);

/* Tonemapped RGBA8 of the running mean into a host buffer (W*H*4 bytes). */
int lux_copy_rgba8(lux_ctx* ctx, uint8_t* rgba_host);

/* Zero the accumulation image (the reference re-inits on camera change,
 * src/app/render_loop.cpp:122-126). */
int lux_reset(lux_ctx* ctx);

/* Replace the camera of a live context (same resolution) and zero the image. */
int lux_set_camera(lux_ctx* ctx, const lux_camera_desc* cam);

/* pathtraceFree: release everything; NULL is accepted (idempotent, like the reference). */
int lux_free(lux_ctx* ctx);

/* Thread-local text of the last failing call. */
const char* lux_last_error(void);

/* ---- statistics of the last lux_render / lux_render_iter call --------------------------- */
typedef struct lux_stats {
    double rays_radiance;     /* radiance rays traced                                        */
    double rays_shadow;       /* NEE shadow rays traced (DL + env)                           */
    double path_bounces;      /* queue entries shaded                                        */
    double samples;           /* pixel-samples rendered                                      */
    double ms_total;          /* device time of the call (CUDA events)                       */
    double ms_trace;          /* summed device time of the trace kernels                     */
    double ms_shade;          /* summed device time of the shade kernels                     */
    double ms_camera;         /* summed device time of camera generation                     */
    double ms_accum;          /* summed device time of accumulation                          */
    double ms_sort;           /* summed device time of Morton keys + sort                    */
    double launches_trace, launches_shade, launches_camera, launches_accum, launches_sort;
    double kernel_launches;   /* every kernel this library launched in the call              */
} lux_stats;

/* Per-kernel CUDA-event timing is recorded only while enabled (off by default). */
int lux_enable_timing(lux_ctx* ctx, int on);
int lux_get_stats(lux_ctx* ctx, lux_stats* out);

/* Queue lengths of the last wave rendered: paths[b] = paths entering bounce b (paths[0] = the
 * wave's camera paths; paths[b+1] = survivors of bounce b, the reference's num_paths after the
 * compaction of src/pathtrace.cu:316-322), shadow[b] = shadow rays traced at bounce b. Entries
 * up to max_bounces are written (the rest of each array is left alone). */
int lux_wave_counts(lux_ctx* ctx, int* paths, int* shadow, int max_bounces);

/* ---- kernel-level entry points used by the parity suite --------------------------------- */

/* Closest-hit / any-hit trace of caller rays through the device BVH.
 * rays: n * 8 floats (origin xyz, tmax, direction xyz, pixel-as-float-bits).
 * mode 0: closest hit (radiance; pixel and iter key the alpha-blend hash);
 * mode 1: closest hit with tmax (DL shadow); mode 2: any hit (env shadow);
 * mode 3: closest hit as mode 0, counting the traversal's work (the BVH heatmap's count, node
 * visits plus triangle tests), which replaces u: word 3 holds the count, word 4 is 0.
 * hits: n * 5 words (t as f32 bits, instance, prim, u bits, v bits); t=-1 on a miss; for
 * mode 2 only word 0 is meaningful (1.0 occluded, -1.0 free). Host buffers. */
int lux_trace_rays(lux_ctx* ctx, const float* rays, int n, int mode, int iter, uint32_t* hits);

/* lux_trace_rays_static: lux_trace_rays for callers that must not allocate device memory on
 * the call. No counterpart in the reference. Same arguments, results and errors as
 * lux_trace_rays, for n <= LUX_TRACE_STATIC_MAX_RAYS; a larger n is rejected with
 * LUX_ERR_INVALID before any device work.
 * Who needs it: a host that has given the device's free memory to its own pool or to other
 * tenants under a fixed budget, where a per-call cudaMalloc can fail in the middle of a
 * request; and a host that keeps other work running on other streams of the device, which
 * the per-call cudaFree of lux_trace_rays stalls (cudaFree waits for the whole device).
 * Rays and hits are staged through one fixed array of 256 + 52 * LUX_TRACE_STATIC_MAX_RAYS
 * bytes (about 3.25 MiB) compiled into the library, one copy per device. Its address is
 * looked up (cudaGetSymbolAddress) on every call; the first call on a device may load the
 * library's device code there, so make that first call before any stream capture begins on
 * that device.
 * Must start at zero: the traversal's work cursor in that array and the context's traversal
 * error word; the call clears both on the context's stream before its launch. Nothing else
 * carries over from one call to the next.
 * Calls that overlap on one device (two threads, or two contexts on the same device) share
 * the array and race: the library does not lock it, so serialise such calls. */
#define LUX_TRACE_STATIC_MAX_RAYS 65536
int lux_trace_rays_static(lux_ctx* ctx, const float* rays, int n, int mode, int iter, uint32_t* hits);

/* Device allocations the library has made since it was loaded, on all devices: cudaMalloc,
 * stream-ordered and pool allocations, CUDA arrays. A diagnostics hook with no counterpart in
 * the reference; the tests use it to show that lux_trace_rays_static allocates nothing. */
int64_t lux_device_alloc_count(void);

/* BVH8 build parity (no counterpart in the reference; its builder is fill_bvh,
 * src/mesh/bvh_build.cu:15-318): build the compressed 8-wide BVH over n = tree_begin[num_trees]
 * boxes (6 floats each: min xyz, max xyz) grouped into trees [tree_begin[t], tree_begin[t+1])
 * with the device builder (on_device = 1, the one every scene build uses) or the host builder
 * (0, needs no device). Trees are laid out one after another; child_base is absolute, tri_base
 * relative to the tree's first box. nodes: room for `capacity` 80-byte nodes; order: n leaf
 * records -> box index; roots, depth: per tree; *num_nodes: nodes written. Host buffers. */
int lux_bvh8_build(const float* boxes, const int* tree_begin, int num_trees, int on_device, void* nodes,
                   int capacity, uint32_t* order, uint32_t* roots, int* depth, int* num_nodes);

/* Morton keys of caller rays (src/morton_codes.cu:13-24, src/kernels/intersection_precompute.cu:6-33):
 * rays as in lux_trace_rays; keys: n u32. Host buffers. */
int lux_morton_keys(lux_ctx* ctx, const float* rays, int n, uint32_t* keys);

/* One bounce of the wavefront on caller state, for the shade parity test. The caller gives
 * n paths (path state, 24 floats each, layout LUX_PS_*) and the traced hits for them
 * (10 words each: radiance hit, then shadow hit / occlusion), the bounce depth after the
 * increment, and whether compaction is on. The kernel updates the states in place and
 * writes the survivor path indices; *n_out receives their number. Host buffers. */
enum {
    LUX_PS_ORIGIN = 0, LUX_PS_DIR = 3, LUX_PS_COLOR = 6, LUX_PS_THROUGHPUT = 9,
    LUX_PS_DL = 12, LUX_PS_ENV = 15, LUX_PS_PIXEL = 18, LUX_PS_KILL = 19,
    LUX_PS_SPECULAR = 20, LUX_PS_LAST_PDF = 21, LUX_PS_FLOATS = 24
};
int lux_shade_step(lux_ctx* ctx, int iter, int depth, int compact, float* paths, int n,
                   const uint32_t* hits, int* survivors, int* n_out);

/* Light samples (sampleDirectLight, src/kernels/sample_direct_light.cu:9-101) for n paths of
 * the given pixels at bounce depth: out n*6 floats (DL point xyz, env dir xyz). */
int lux_light_samples(lux_ctx* ctx, int iter, int depth, const int* pixels, int n, float* out);

/* Light-CDF tables as built on the device side (emissive prefix, per-mesh triangle prefix of
 * each emissive instance concatenated, HDRI marginal, HDRI conditional), for CDF parity. */
int lux_get_cdfs(lux_ctx* ctx, float* emissive_prefix, float* tri_prefix, float* marginal,
                 float* conditional, float* total_area);

/* Device-side minstd stream: n uniforms of the engine seeded by (iter, index, depth)
 * into a host buffer, for RNG parity. */
int lux_rng_stream(int iter, int index, int depth, int n, float* out);

/* Bilinear texture fetches of a scene texture (index -1: the environment map) at n (u, v)
 * pairs; out n*4 floats. */
int lux_sample_texture(lux_ctx* ctx, int tex, const float* uv, int n, float* out);

/* ---- job engine: many render jobs in one shared wavefront (no counterpart in the reference)
 *
 * The batching and serving forms. An engine keeps several scenes resident on one device
 * (their acceleration structures, materials, textures and light tables concatenated) and
 * renders any number of jobs -- each a scene, a camera with its own resolution, a sample count
 * and a trace depth -- in waves whose paths come from many jobs at once. Every wave is one
 * graph replay: camera rays for the wave's job segments, depth x (trace, shade, shadow trace),
 * and a per-job accumulation in sample order. A job's image is therefore the same bit for bit
 * whether it renders alone or among others, and the same as lux_render of that scene and
 * camera in a single-job context. Lighting options (-dmis, -emis, envmap intensity, precision,
 * texture storage) are the engine's; ray sorting is not used.
 * Jobs are admitted in submission order while the engine's device memory (scenes + wave
 * buffers + admitted jobs' images) stays within hbm_budget_bytes; the others wait queued.
 * An engine is driven by one host thread. */
typedef struct lux_engine lux_engine;

typedef struct lux_job_desc {
    int32_t scene;            /* index of a resident scene                                     */
    int32_t spp;              /* samples per pixel                                             */
    int32_t trace_depth;      /* 0: the scene's trace_depth                                    */
    int32_t first_iter;       /* iteration of the first sample (1-based, the reference's iter); 0 = 1 */
    lux_camera_desc camera;   /* resolution and pose                                           */
} lux_job_desc;

enum { LUX_SCHED_FIFO = 0, LUX_SCHED_SHORTEST_FIRST = 1 };

typedef struct lux_engine_config {
    int64_t hbm_budget_bytes; /* admission limit on the engine's device memory; 0 = unlimited   */
    int32_t max_paths;        /* paths per wave; 0 = autotune over a few sizes on the first waves */
    int32_t max_jobs;         /* job table capacity (live jobs); 0 = 4096                       */
    int32_t schedule;         /* LUX_SCHED_*: order in which admitted jobs fill a wave            */
    int32_t trace_blocks;     /* persistent trace grid in blocks; 0 = full occupancy (autotuned with max_paths) */
} lux_engine_config;

enum { LUX_JOB_QUEUED = 0, LUX_JOB_ACTIVE = 1, LUX_JOB_DONE = 2, LUX_JOB_RELEASED = 3 };

typedef struct lux_job_status {
    int32_t state;            /* LUX_JOB_*                                                     */
    int32_t spp_done;         /* samples accumulated so far, as an image read now holds them    */
    int32_t spp;
    int32_t waves;            /* waves the job took part in                                     */
    double t_submit_ms, t_admit_ms, t_done_ms;   /* engine clock (ms since creation)            */
} lux_job_status;

typedef struct lux_engine_stats {
    int64_t waves;
    double samples;           /* pixel samples rendered                                         */
    double rays;              /* radiance + shadow rays traced                                  */
    double ms_device;         /* summed device time of the steps (CUDA events)                  */
    int64_t device_bytes;     /* scenes + wave buffers + live job images                        */
    int64_t scene_bytes;
    int32_t max_paths;        /* wave size in use (autotuned when configured 0)                 */
    int32_t trace_blocks;     /* persistent trace grid in use                                   */
    int32_t jobs_queued, jobs_active, jobs_done;
} lux_engine_stats;

int lux_engine_create(const lux_scene_desc* const* scenes, int num_scenes, const lux_options* opt,
                      const lux_engine_config* cfg, lux_engine** out);
/* Queue a job; *job_id identifies it from then on. */
int lux_engine_submit(lux_engine* e, const lux_job_desc* job, int* job_id);
/* Admit what fits and advance the shared wavefront; return how many jobs completed (*done_jobs
 * may be NULL). The first waves (the autotuning ones) run one whole wave per call; after them
 * up to four waves are in flight: a call starts a new wave when a lane is free and there is
 * work, advances every wave in flight by three bounces, and accumulates the waves that are
 * through, in the order they started. Such a call returns while its step runs on the device,
 * after finishing the step before it: the jobs a step completes are reported (*done_jobs,
 * LUX_JOB_DONE) by the next call, and a job's spp_done counts the samples whose accumulation
 * has been enqueued, which an image read back now holds. *idle is set to 1 when there was
 * nothing to render and nothing left to report. */
int lux_engine_step(lux_engine* e, int* done_jobs, int* idle);
/* Step until every submitted job is done. */
int lux_engine_run(lux_engine* e);
int lux_engine_job_status(lux_engine* e, int job_id, lux_job_status* out);
/* The job's FP32 accumulation sum (width*height*3), at any point of its progress. */
int lux_engine_copy_image(lux_engine* e, int job_id, float* rgb_host);
/* Free a finished (or queued) job's device memory. */
int lux_engine_release(lux_engine* e, int job_id);
int lux_engine_get_stats(lux_engine* e, lux_engine_stats* out);
/* The engine clock (ms since creation), the time base of lux_job_status. */
double lux_engine_clock_ms(lux_engine* e);
int lux_engine_free(lux_engine* e);

/* Pure wave planner (host only, used by the engine; exposed for tests): given each live job's
 * pixels per sample and samples left, in the order they may fill the wave, choose how many
 * samples each contributes to a wave of `capacity` paths with at most `max_segments` segments.
 * A job contributes only whole samples and only if at least one fits. Returns the number of
 * segments; take[i] receives job i's samples. */
int lux_plan_wave(const int* npix, const int* remaining, int njobs, int capacity, int max_segments, int* take);

/* ---- procedural scenes (host only; no device needed) ------------------------------------ */
typedef struct lux_host_scene lux_host_scene;

/* Cornell box, 36 triangles, 256x256 (the 36-triangle config of the baseline). */
lux_host_scene* lux_scene_cornell36(int width, int height);

/* Random instanced scene: num_instances icospheres / displaced grids with total_tris
 * triangles, random materials, value-noise textures and an HDRI; seeded. */
typedef struct lux_random_scene_params {
    uint64_t seed;
    int32_t num_instances;
    int32_t total_tris;
    int32_t min_tris, max_tris;
    int32_t num_emissive;
    int32_t num_textures;
    int32_t texture_size;
    int32_t env_width, env_height;   /* 0 for no HDRI                                       */
    int32_t width, height;
    int32_t trace_depth;
    int32_t env_half;                /* 1: store the HDRI as RGBA16F                         */
    int32_t tex_half;                /* 1: store base-colour textures as RGBA16F             */
} lux_random_scene_params;
void lux_default_random_scene_params(lux_random_scene_params* p);
lux_host_scene* lux_scene_random(const lux_random_scene_params* p);

/* Furnace: a closed unit icosphere (vertex normals on) under a constant environment of 1,
 * made of smooth white metal (metallic 1, roughness 0.01, base colour 1, so Schlick F = 1). */
lux_host_scene* lux_scene_furnace(int width, int height, int subdiv);
/* The same furnace with the sphere made of *mat; vertex_normals 0 drops the vertex normals, so
 * the sphere shades with its geometric (facet) normals and stays exactly convex. */
lux_host_scene* lux_scene_furnace_material(int width, int height, int subdiv, const lux_material_desc* mat,
                                           int vertex_normals);
/* The material the procedural scenes start from: the reference glTF defaults for base colour
 * 1, roughness 1, metallic 0, ior 1.55 (src/scene/scene_load_gltf.cpp:85-89,177). */
void lux_default_material(lux_material_desc* m);

/* A pinhole camera at pos looking at look (world up +y) with vertical field of view fovy_deg
 * at width x height, set up as the reference's scene loader does from a camera's position,
 * look-at point and fov: pixelLength = 2 tan(fovy/2) (aspect, 1) / resolution. */
void lux_make_camera(int width, int height, const float pos[3], const float look[3], float fovy_deg,
                     lux_camera_desc* out);

const lux_scene_desc* lux_scene_get_desc(const lux_host_scene* s);
/* Total triangles over all instances. */
int64_t lux_scene_instanced_tris(const lux_host_scene* s);
void lux_scene_destroy(lux_host_scene* s);

#ifdef __cplusplus
}
#endif
#endif /* LUXION_H */
