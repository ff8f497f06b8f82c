// ref_loader.cpp -- host harness around the reference's own glTF/EXR loader, for loader parity.
//
// Test infrastructure only (built into oracle/_ref/libluxref.so with the reference's sources,
// compiled unmodified). ref_load_gltf constructs the reference Scene from a .glb file
// (Scene::Scene, src/scene/scene.cpp:22-49 -> Scene::loadFromGLTF,
// src/scene/scene_load_gltf.cpp:61-529, which also reads the EXR environment map with tinyexr)
// and exposes what it loaded as a lux_scene_desc: one mesh and one instance per mesh Geom, in
// the loader's order, the materials, the float4 texels the loader handed to TextureHandler, the
// camera, the trace depth and the environment texels.
#define private public  // TextureHandler keeps the loaded texels in a private member
#include "texture.h"
#undef private
#include "scene.h"

#include "../../include/luxion.h"

#include <cstring>
#include <vector>

namespace {

struct Loaded {
    Scene* scene = nullptr;
    std::vector<lux_mesh_desc> meshes;
    std::vector<std::vector<uint32_t>> idx;
    std::vector<lux_instance_desc> insts;
    std::vector<lux_material_desc> mats;
    std::vector<std::vector<float>> texels;
    std::vector<lux_texture_desc> texs;
    lux_scene_desc desc;
};

lux_tex_transform tt(const TextureTransform& s) {
    lux_tex_transform t;
    t.offset[0] = s.offset.x;
    t.offset[1] = s.offset.y;
    t.scale[0] = s.scale.x;
    t.scale[1] = s.scale.y;
    t.rotation = s.rotation;
    return t;
}

}  // namespace

extern "C" void* ref_load_gltf(const char* path, const char* exr) {
    TextureHandler& th = TextureHandler::get();
    th.host_textures.clear();
    th.host_texture_data.clear();
    Loaded* L = new Loaded();
    L->scene = new Scene(path, exr && exr[0] ? exr : nullptr);
    const Scene& S = *L->scene;
    for (const Geom& g : S.geoms) {
        if (g.type != GeomType::MESH || !g.mesh.h_valid) continue;
        const Mesh& m = g.mesh;
        L->idx.emplace_back();
        for (const Triangle& t : m.h_triangles)
            L->idx.back().insert(L->idx.back().end(), {t.v_indices[0], t.v_indices[1], t.v_indices[2]});
        lux_mesh_desc md;
        md.num_verts = m.num_verts;
        md.num_tris = m.num_triangles;
        md.positions = &m.h_verts[0].x;
        md.normals = m.has_normal_buffers ? &m.h_normals[0].x : nullptr;
        md.uvs = m.has_uvs ? &m.h_uvs[0].x : nullptr;
        md.indices = nullptr;
        L->meshes.push_back(md);
        lux_instance_desc in;
        std::memset(&in, 0, sizeof(in));
        in.mesh = int(L->meshes.size()) - 1;
        in.material = g.materialid;
        in.has_inverse = 1;
        std::memcpy(in.transform, &g.transform[0][0], 64);
        std::memcpy(in.inverse, &g.inverseTransform[0][0], 64);
        std::memcpy(in.inv_transpose, &g.invTranspose[0][0], 64);
        L->insts.push_back(in);
    }
    for (size_t k = 0; k < L->meshes.size(); ++k) L->meshes[k].indices = L->idx[k].data();
    for (const Material& m : S.materials) {
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
        d.albedo_tt = tt(m.albedo_tex_transform);
        d.emissive_tt = tt(m.emission.emissive_tex_transform);
        d.normal_tt = tt(m.normal_tex_transform);
        d.metallic_roughness_tt = tt(m.metallic_roughness_tex_transform);
        L->mats.push_back(d);
    }
    for (size_t i = 0; i < th.host_textures.size(); ++i) {
        const std::vector<glm::vec4>& src = th.host_texture_data[i];
        L->texels.emplace_back(src.size() * 4);
        std::memcpy(L->texels.back().data(), src.data(), src.size() * sizeof(glm::vec4));
        lux_texture_desc d;
        d.width = th.host_textures[i].width;
        d.height = th.host_textures[i].height;
        d.format = LUX_TEX_RGBA32F;
        d._pad = 0;
        d.data = nullptr;
        L->texs.push_back(d);
    }
    for (size_t i = 0; i < L->texs.size(); ++i) L->texs[i].data = L->texels[i].data();
    lux_scene_desc& sd = L->desc;
    std::memset(&sd, 0, sizeof(sd));
    sd.num_meshes = int32_t(L->meshes.size());
    sd.num_instances = int32_t(L->insts.size());
    sd.num_materials = int32_t(L->mats.size());
    sd.num_textures = int32_t(L->texs.size());
    sd.meshes = L->meshes.data();
    sd.instances = L->insts.data();
    sd.materials = L->mats.data();
    sd.textures = L->texs.empty() ? nullptr : L->texs.data();
    const Camera& c = S.state.camera;
    sd.camera.width = c.resolution.x;
    sd.camera.height = c.resolution.y;
    const glm::vec3* v[5] = {&c.position, &c.lookAt, &c.view, &c.up, &c.right};
    float* o[5] = {sd.camera.position, sd.camera.look_at, sd.camera.view, sd.camera.up, sd.camera.right};
    for (int k = 0; k < 5; ++k) {
        o[k][0] = v[k]->x;
        o[k][1] = v[k]->y;
        o[k][2] = v[k]->z;
    }
    sd.camera.fov[0] = c.fov.x;
    sd.camera.fov[1] = c.fov.y;
    sd.camera.pixel_length[0] = c.pixelLength.x;
    sd.camera.pixel_length[1] = c.pixelLength.y;
    sd.trace_depth = S.state.traceDepth;
    if (!S.exr_data.empty()) {
        sd.env_width = S.exr_width;
        sd.env_height = S.exr_height;
        sd.env_format = LUX_TEX_RGBA32F;
        sd.env_data = &S.exr_data[0].x;
    }
    return L;
}

extern "C" const lux_scene_desc* ref_loaded_desc(void* h) { return h ? &static_cast<Loaded*>(h)->desc : nullptr; }

extern "C" void ref_loaded_free(void* h) {
    Loaded* L = static_cast<Loaded*>(h);
    if (!L) return;
    delete L->scene;
    delete L;
}
