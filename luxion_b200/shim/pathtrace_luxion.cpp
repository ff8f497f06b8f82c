// pathtrace_luxion.cpp -- the reference's render-path functions on top of libluxion.
//
// A maintainer adds this file to the reference (seabiscuit-iv/luxion) in place of
// src/pathtrace.cu and src/pathtrace/pathtrace_buffers.cu, and links it with
//   -I<this repository>/include -L<this repository>/luxion_b200/_lib -lluxion
// It defines, with the reference's signatures and meaning:
//   void pathtraceInit(Scene*)            include/pathtrace/pathtrace_buffers.h:5
//   void pathtrace(uchar4*, int, int)     include/pathtrace.h:13
//   void pathtraceFree()                  include/pathtrace/pathtrace_buffers.h:6
//   void copyImageToHost()                include/pathtrace/pathtrace_buffers.h:7
// The reference's scene loader, options singleton and application loop stay as they are.
//
// Lifecycle. The reference builds meshes, textures and acceleration structures once at load
// (src/main.cpp:199-274) and calls pathtraceFree(); pathtraceInit() on every camera or option
// reset (src/app/render_loop.cpp:122-126). Here the first pathtraceInit for a Scene builds the
// resident device scene (lux_scene_create: upload, BVH, light tables, textures) and keeps it;
// every pathtraceInit makes a render context on it (lux_init_on_scene: per-pixel state only),
// and pathtraceFree releases that context. luxionReleaseScene() frees the resident scene.
//
// Textures. TextureHandler keeps its float4 texels private but exposes each texture object
// (include/texture.h:17-33), and main() has uploaded them (TextureHandler::load_textures_on_device)
// before the first pathtraceInit. The texels are read back from the CUDA array behind each
// texture object, so the reference needs no change to its headers.
#include "luxion.h"

#include "pathtrace.h"  // the reference's declarations of the four functions defined below
#include "scene.h"
#include "texture.h"
#include "pathtrace/pathtracer_options.h"

#include <cuda_runtime.h>

#include <type_traits>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

lux_ctx* g_ctx = nullptr;
lux_scene* g_resident = nullptr;
const Scene* g_resident_of = nullptr;
Scene* g_scene = nullptr;

// The reference's error behaviour (checkCUDAError, include/common.h:16-36): print and exit.
void lux_check(int rc, const char* what) {
    if (rc != LUX_OK) {
        std::fprintf(stderr, "%s: %s\n", what, lux_last_error());
        std::exit(EXIT_FAILURE);
    }
}

lux_tex_transform tex_transform(const TextureTransform& s) {
    lux_tex_transform t;
    t.offset[0] = s.offset.x;
    t.offset[1] = s.offset.y;
    t.scale[0] = s.scale.x;
    t.scale[1] = s.scale.y;
    t.rotation = s.rotation;
    return t;
}

lux_camera_desc camera_of(const Camera& c) {
    lux_camera_desc d;
    d.width = c.resolution.x;
    d.height = c.resolution.y;
    const glm::vec3* v[5] = {&c.position, &c.lookAt, &c.view, &c.up, &c.right};
    float* o[5] = {d.position, d.look_at, d.view, d.up, d.right};
    for (int k = 0; k < 5; ++k) {
        o[k][0] = v[k]->x;
        o[k][1] = v[k]->y;
        o[k][2] = v[k]->z;
    }
    d.fov[0] = c.fov.x;
    d.fov[1] = c.fov.y;
    d.pixel_length[0] = c.pixelLength.x;
    d.pixel_length[1] = c.pixelLength.y;
    return d;
}

// Build the resident device scene from the reference Scene (the mesh geoms, their materials,
// the uploaded textures and the environment map).
void build_resident(const Scene* scene) {
    std::vector<lux_mesh_desc> meshes;
    std::vector<lux_instance_desc> insts;
    std::vector<std::vector<uint32_t>> idx;
    std::map<std::string, int> by_label;  // geoms that share a mesh share its BLAS (src/main.cpp:199-216)
    for (const Geom& g : scene->geoms) {
        if (g.type != GeomType::MESH || !g.mesh.h_valid) continue;
        const Mesh& m = g.mesh;
        auto it = by_label.find(m.label);
        int mi;
        if (it != by_label.end()) {
            mi = it->second;
        } else {
            // the glTF loader writes one index stream (v_indices == n_indices == uv_indices,
            // src/scene/scene_load_gltf.cpp:430), the single-index form lux_mesh_desc takes
            idx.emplace_back();
            for (const Triangle& t : m.h_triangles)
                idx.back().insert(idx.back().end(), {t.v_indices[0], t.v_indices[1], t.v_indices[2]});
            lux_mesh_desc md;
            md.num_verts = m.num_verts;
            md.num_tris = m.num_triangles;
            md.positions = &m.h_verts[0].x;
            md.normals = m.has_normal_buffers ? &m.h_normals[0].x : nullptr;
            md.uvs = m.has_uvs ? &m.h_uvs[0].x : nullptr;
            md.indices = nullptr;  // set once idx stops growing
            mi = int(meshes.size());
            meshes.push_back(md);
            by_label[m.label] = mi;
        }
        lux_instance_desc in;
        std::memset(&in, 0, sizeof(in));
        in.mesh = mi;
        in.material = g.materialid;
        in.has_inverse = 1;
        std::memcpy(in.transform, &g.transform[0][0], 64);  // glm matrices are column-major
        std::memcpy(in.inverse, &g.inverseTransform[0][0], 64);
        std::memcpy(in.inv_transpose, &g.invTranspose[0][0], 64);
        insts.push_back(in);
    }
    for (size_t k = 0; k < meshes.size(); ++k) meshes[k].indices = idx[k].data();

    // materials, field for field (include/sceneStructs.h:94-131)
    std::vector<lux_material_desc> mats;
    for (const Material& m : scene->materials) {
        lux_material_desc d;
        std::memset(&d, 0, sizeof(d));
        d.color[0] = m.color.x;
        d.color[1] = m.color.y;
        d.color[2] = m.color.z;
        d.albedo_tex = m.albedo_tex;
        d.alpha = m.alpha;
        d.alpha_mode = int32_t(m.alpha_mode);
        d.alpha_cutoff = m.alpha_cutoff;
        d.emission_strength = m.emission.emission_strength;
        d.emission_color[0] = m.emission.emission_color.x;
        d.emission_color[1] = m.emission.emission_color.y;
        d.emission_color[2] = m.emission.emission_color.z;
        d.emissive_tex = m.emission.emissive_tex;
        d.roughness = m.roughness;
        d.metallic = m.metallic;
        d.normal_tex = m.normal_tex;
        d.metallic_roughness_tex = m.metallic_roughness_tex;
        d.transmission = m.transmission;
        d.ior = m.indexOfRefraction;
        d.albedo_tt = tex_transform(m.albedo_tex_transform);
        d.emissive_tt = tex_transform(m.emission.emissive_tex_transform);
        d.normal_tt = tex_transform(m.normal_tex_transform);
        d.metallic_roughness_tt = tex_transform(m.metallic_roughness_tex_transform);
        mats.push_back(d);
    }

    // textures: read the float4 texels back from the CUDA array behind each texture object
    const TextureHandler& th = TextureHandler::get();
    std::vector<std::vector<float4>> texels(th.host_textures.size());
    std::vector<lux_texture_desc> texs;
    for (size_t i = 0; i < th.host_textures.size(); ++i) {
        const TextureData& t = th.host_textures[i];
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        if (cudaGetTextureObjectResourceDesc(&rd, t.tex) != cudaSuccess || rd.resType != cudaResourceTypeArray) {
            std::fprintf(stderr, "pathtraceInit: texture %zu is not an uploaded CUDA array\n", i);
            std::exit(EXIT_FAILURE);
        }
        texels[i].resize(size_t(t.width) * t.height);
        const size_t row = size_t(t.width) * sizeof(float4);
        if (cudaMemcpy2DFromArray(texels[i].data(), row, rd.res.array.array, 0, 0, row, size_t(t.height),
                                  cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fprintf(stderr, "pathtraceInit: reading texture %zu back failed\n", i);
            std::exit(EXIT_FAILURE);
        }
        lux_texture_desc d;
        d.width = t.width;
        d.height = t.height;
        d.format = LUX_TEX_RGBA32F;
        d._pad = 0;
        d.data = texels[i].data();
        texs.push_back(d);
    }

    lux_scene_desc sd;
    std::memset(&sd, 0, sizeof(sd));
    sd.num_meshes = int32_t(meshes.size());
    sd.num_instances = int32_t(insts.size());
    sd.num_materials = int32_t(mats.size());
    sd.num_textures = int32_t(texs.size());
    sd.meshes = meshes.data();
    sd.instances = insts.data();
    sd.materials = mats.data();
    sd.textures = texs.empty() ? nullptr : texs.data();
    sd.camera = camera_of(scene->state.camera);
    sd.trace_depth = scene->state.traceDepth;
    if (!scene->exr_data.empty()) {
        sd.env_width = scene->exr_width;
        sd.env_height = scene->exr_height;
        sd.env_format = LUX_TEX_RGBA32F;
        sd.env_data = &scene->exr_data[0].x;
    }
    lux_options opt;
    lux_default_options(&opt);  // float texels, plain FP32: what the reference renders with
    lux_check(lux_scene_create(&sd, &opt, &g_resident), "pathtraceInit");
    g_resident_of = scene;
}

}  // namespace

// Frees the resident scene the shim keeps (call at exit, where main() frees its meshes).
void luxionReleaseScene() {
    if (g_ctx) {
        lux_free(g_ctx);
        g_ctx = nullptr;
    }
    lux_scene_free(g_resident);
    g_resident = nullptr;
    g_resident_of = nullptr;
}

void pathtraceInit(Scene* scene) {
    g_scene = scene;
    if (!g_resident || g_resident_of != scene) {
        luxionReleaseScene();
        build_resident(scene);
    }
    // options: PathTracerOptions -> lux_options (set before init, as the reference requires)
    const PathTracerOptions* o = PathTracerOptions::Get();
    lux_options opt;
    lux_default_options(&opt);
    opt.direct_light_sampling = o->direct_light_sampling;                   // -dmis
    opt.env_importance_sampling = o->environment_map_importance_sampling;   // -emis
    opt.color_mode = o->color_mode;
    opt.envmap_intensity = o->envmap_intensity;
    opt.trace_depth = scene->state.traceDepth;
    opt.material_debug_mode = o->material_debug_mode;                       // ImGui debug views
    opt.debug_bvh = o->debug_bvh ? 1 : 0;
    const lux_camera_desc cam = camera_of(scene->state.camera);
    lux_check(lux_init_on_scene(g_resident, &cam, &opt, &g_ctx), "pathtraceInit");
}

void pathtrace(uchar4* pbo, int /*frame*/, int iter) {  // iter is 1-based (src/app/render_loop.cpp:131-136)
    lux_check(lux_render_iter(g_ctx, iter, reinterpret_cast<uint8_t*>(pbo)), "pathtrace");
}

void pathtraceFree() {  // idempotent, and called before the first init, as in the reference
    if (g_ctx) {
        lux_free(g_ctx);
        g_ctx = nullptr;
    }
}

void copyImageToHost() {  // the FP32 accumulation sum, not the mean
    lux_check(lux_copy_image(g_ctx, &g_scene->state.image[0].x), "copyImageToHost");
}

// The definitions above must be the reference's functions, not overloads of them.
static_assert(std::is_same<decltype(&pathtraceInit), void (*)(Scene*)>::value, "pathtraceInit signature");
static_assert(std::is_same<decltype(&pathtrace), void (*)(uchar4*, int, int)>::value, "pathtrace signature");
static_assert(std::is_same<decltype(&pathtraceFree), void (*)()>::value, "pathtraceFree signature");
static_assert(std::is_same<decltype(&copyImageToHost), void (*)()>::value, "copyImageToHost signature");
