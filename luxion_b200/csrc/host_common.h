// host_common.h -- host-side pieces shared by the single-job context (context.cpp) and the
// job engine (engine.cpp): error reporting, device allocation, textures and the host-side
// scene build with its upload.
#pragma once

#include "../../include/luxion.h"
#include "bvh8.h"
#include "device_scene.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <functional>
#include <string>
#include <vector>

namespace lux {

extern thread_local std::string g_err;
// record msg for lux_last_error() and return code
int fail(int code, const std::string& msg);

inline double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

#define LUX_CUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            return ::lux::fail(e_ == cudaErrorMemoryAllocation ? LUX_ERR_OOM : LUX_ERR_CUDA, \
                               std::string(#call) + ": " + cudaGetErrorString(e_));         \
        }                                                                                   \
    } while (0)

// Counts every device allocation the library makes (lux_device_alloc_count).
void note_device_alloc();

// Small page-locked host blocks (wave counters, iteration words, build counters) from a
// process-wide free list: cudaMallocHost and cudaFreeHost cost tens to hundreds of
// microseconds each and synchronise, and every context and scene build needs a few such
// blocks. A block is kept by size class (a power of two of at least 256 bytes) when put back
// and never returned to the system. Put a block back only when no copy into or out of it is
// still queued on any stream.
void* pinned_get(size_t bytes);
void pinned_put(void* p, size_t bytes);

template <class T>
int dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return LUX_OK;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
    if (e != cudaSuccess) return fail(LUX_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    note_device_alloc();
    return LUX_OK;
}
template <class T>
int upload(T** p, const T* src, size_t n) {
    int rc = dalloc(p, n);
    if (rc) return rc;
    if (n) LUX_CUDA(cudaMemcpy(*p, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return LUX_OK;
}

struct DevTex {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t obj = 0;
    size_t bytes = 0;
};
// CUDA arrays of destroyed textures are kept, per device, channel format and size, for the
// next texture of that shape (up to kTexArrayKeep bytes per device; beyond that they are
// freed): cudaMallocArray and cudaFreeArray synchronise the device and cost far more than the
// copy into an array, and a renderer that reloads or replaces scenes meets the same texture
// shapes again. tex_array_get takes a kept array or allocates one; tex_array_put keeps or
// frees it. Put an array back only when no copy or kernel can still use it.
constexpr size_t kTexArrayKeep = size_t(2) << 30;
cudaError_t tex_array_get(cudaArray_t* arr, const cudaChannelFormatDesc& fd, size_t width, size_t height);
void tex_array_put(cudaArray_t arr);

inline void destroy_texture(DevTex& t) {
    if (t.obj) cudaDestroyTextureObject(t.obj);
    if (t.arr) tex_array_put(t.arr);
    t = DevTex{};
}

// Allocator whose value-less construct leaves trivially constructible elements uninitialised:
// the large host arrays of a scene are sized once and first written (and paged in) by the
// threads that fill them, not zero-filled by one thread beforehand.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

// The host-built part of a resident scene: materials (textures are created on the device here
// because materials hold their texture objects) and the light tables. The geometry (vertex
// data, BVHs, triangle and instance records) is built on the device by build_geometry.
struct HostScene {
    std::vector<DevMaterial> mats;
    std::vector<int> emissive;        // emissive instances (scene-local)
    std::vector<float> emissive_prefix, tri_prefix, marginal, conditional;
    std::vector<int> marginal_guide, conditional_guide;  // guide tables of the HDRI CDFs
    int guide_marg = 0, guide_cond = 0;
    std::vector<int> tri_off;
    float total_area = 0.0f;
    int env_w = 0, env_h = 0;
    unsigned long long env_tex = 0;
    bool has_env = false;
    float morton_bmin[3] = {0, 0, 0}, morton_bmax[3] = {0, 0, 0};
    double ms_tables = 0, ms_textures = 0;  // light tables + materials; texture thread
};

// Device allocation that the owner records (and frees with everything else it owns).
using DevAlloc = std::function<int(void** p, size_t bytes)>;

// What build_geometry reports besides the DevScene geometry fields.
struct GeometryBuild {
    std::vector<uint32_t> tlas_root;      // per scene
    std::vector<int64_t> instanced_tris;  // per scene
    std::vector<int> inst_base;           // per scene (+ total): first instance in the concatenation
    std::vector<int> max_blas_depth;      // per scene
    uint32_t blas_nodes = 0, tlas_nodes = 0;
    double ms_upload = 0, ms_blas = 0, ms_tlas = 0, ms_total = 0;  // host wall time per stage
    bool single_level = false;
    size_t bytes = 0;                     // device bytes allocated through alloc
};

// Device geometry of ns scenes concatenated (geometry.cpp): vertex data and, by layout
// (LUX_BVH_*), either every mesh's BLAS and every scene's TLAS or one world-space BVH per scene
// over its instanced triangles, built on the device, triangle records, instance records (materials
// offset by material_base[s]) and TLAS leaf records. Fills S.nodes, prims, insts, tlas_prims,
// tlas_leaf, tlas_root (scene 0), num_insts, pos, nrm, uv, idx. Runs on stream st and returns
// once the build has finished.
int build_geometry(const lux_scene_desc* const* scenes, int ns, const std::vector<int>& material_base, int layout,
                   const DevAlloc& alloc, cudaStream_t st, DevScene& S, GeometryBuild& G);

// Check a scene description (sizes, index ranges, references, environment format).
int validate_scene_desc(const lux_scene_desc& d);

// Host-side build of one validated scene description with the given options (texture
// storage, precision, which light tables -dmis / -emis require): textures, materials, light
// tables and the Morton box. Textures are appended to texs and created on a second thread;
// the environment map goes to env. device_work, when given, runs on that thread after the
// textures and its status is returned like a texture failure. The thread is joined before the
// function returns.
int build_host_scene(const lux_scene_desc& d, const lux_options& opt, std::vector<DevTex>& texs, DevTex& env,
                     HostScene& H, const std::function<int()>& device_work = nullptr);

// Upload the light tables of a host scene and set its environment and Morton box fields.
// Owner provides up(T** dst, const T* src, size_t n), which records the allocation.
template <class Owner>
int upload_scene_lights(Owner* C, const HostScene& H, DevScene& S) {
    int rc;
    float* f = nullptr;
    int* ei = nullptr;
    if ((rc = C->up(&ei, H.emissive.data(), H.emissive.size()))) return rc;
    S.emissive_inst = ei;
    if ((rc = C->up(&f, H.emissive_prefix.data(), H.emissive_prefix.size()))) return rc;
    S.emissive_prefix = f;
    if ((rc = C->up(&f, H.tri_prefix.data(), H.tri_prefix.size()))) return rc;
    S.tri_prefix = f;
    if ((rc = C->up(&ei, H.tri_off.data(), H.tri_off.size()))) return rc;
    S.tri_prefix_off = ei;
    S.num_emissive = int(H.emissive.size());
    S.total_area = H.total_area;
    if (H.has_env) {
        if ((rc = C->up(&f, H.marginal.data(), H.marginal.size()))) return rc;
        S.marginal = f;
        if ((rc = C->up(&f, H.conditional.data(), H.conditional.size()))) return rc;
        S.conditional = f;
        int* g = nullptr;
        if ((rc = C->up(&g, H.marginal_guide.data(), H.marginal_guide.size()))) return rc;
        S.marginal_guide = g;
        if ((rc = C->up(&g, H.conditional_guide.data(), H.conditional_guide.size()))) return rc;
        S.conditional_guide = g;
        S.guide_marg = H.guide_marg;
        S.guide_cond = H.guide_cond;
        S.env_w = H.env_w;
        S.env_h = H.env_h;
        S.env_tex = H.env_tex;
        S.has_env = 1;
    }
    for (int a = 0; a < 3; ++a) {
        S.morton_bmin[a] = H.morton_bmin[a];
        S.morton_bmax[a] = H.morton_bmax[a];
    }
    return LUX_OK;
}

// Upload the materials of a host scene.
template <class Owner>
int upload_scene_materials(Owner* C, const HostScene& H, DevScene& S) {
    DevMaterial* dm = nullptr;
    if (int rc = C->up(&dm, H.mats.data(), H.mats.size())) return rc;
    S.mats = dm;
    return LUX_OK;
}

}  // namespace lux
