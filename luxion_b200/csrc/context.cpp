// context.cpp -- host side of the C-ABI (include/luxion.h): scene upload, acceleration
// structure build, light tables, wavefront buffers and the device-side bounce loop.
//
// Reference mapping:
//   lux_init         pathtraceInit (src/pathtrace/pathtrace_buffers.cu:21-140) together with
//                    the per-mesh uploads and acceleration builds main() does before it
//                    (src/main.cpp:199-274) and the scene precompute
//                    (src/scene/scene_precompute.cpp:22-124)
//   lux_render_iter  pathtrace (src/pathtrace.cu:97-367): one sample per pixel
//   lux_render       the same loop, several samples in flight per wave
//   lux_free         pathtraceFree (src/pathtrace/pathtrace_buffers.cu:142-177)
//   lux_copy_image   copyImageToHost (src/pathtrace/pathtrace_buffers.cu:180-190)
// Unlike the reference, no step of a bounce returns to the host: queue lengths live in
// device counters that the kernels read, so a whole wave is one stream of launches that can
// be captured once as a CUDA graph and replayed.

#include "../../include/luxion.h"
#include "bvh8.h"
#include "bvh_gpu.h"
#include "device_scene.h"
#include "launch.h"
#include "host_common.h"

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

using namespace lux;

namespace lux {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

}  // namespace lux


// A resident scene: geometry, acceleration structure, materials, textures and light tables on
// one device. The reference builds these once at load (mesh uploads and acceleration builds in
// src/main.cpp:199-274, the light precompute in src/scene/scene_precompute.cpp:22-124); render
// contexts made on it allocate only their per-pixel state. Reference counted: the creator's
// handle and every context on the scene hold one reference each.
struct lux_scene {
    int device = 0;
    DevScene S{};
    std::vector<void*> allocs;
    std::vector<DevTex> texs;
    DevTex env;
    // what the build depended on: a context must render with the same choices
    int precision = LUX_PRECISION_PLAIN;
    int texture_storage = LUX_TEXSTORE_FLOAT;
    int trace_depth = 0;          // the description's RenderState::traceDepth
    lux_camera_desc camera{};     // the description's camera
    bool has_emissive = false;    // -dmis is possible
    // host copies for CDF queries
    std::vector<float> h_emissive_prefix, h_tri_prefix, h_marginal, h_conditional;
    float h_total_area = 0.0f;
    int64_t instanced_tris = 0;
    size_t scene_bytes = 0;
    lux_scene_stats stats{};     // stage times of the build
    std::atomic<int> refs{1};

    // Device memory of the scene: stream-ordered from the library's pool on the scene's own
    // stream (the geometry is built on it), so building and freeing a scene never waits for
    // the whole device; host tables are copied on the same stream.
    cudaStream_t stream = nullptr;
    template <class T>
    int alloc(T** p, size_t n) {
        *p = nullptr;
        if (n == 0) return LUX_OK;
        cudaError_t e = scratch_alloc(reinterpret_cast<void**>(p), n * sizeof(T), stream);
        if (e != cudaSuccess) return fail(LUX_ERR_OOM, std::string("device allocation: ") + cudaGetErrorString(e));
        allocs.push_back(*p);
        scene_bytes += n * sizeof(T);
        return LUX_OK;
    }
    template <class T>
    int up(T** p, const T* src, size_t n) {
        if (int rc = alloc(p, n)) return rc;
        if (n) LUX_CUDA(cudaMemcpyAsync(*p, src, n * sizeof(T), cudaMemcpyHostToDevice, stream));
        return LUX_OK;
    }
};

// Waves of one render call whose first iteration and size the device table holds; a longer
// call runs in chunks of this many waves.
constexpr int kWaveTab = 4096;
// Lanes (waves in flight) of a pipelined render call.
constexpr int kMaxLanes = lux::kMaxSegs;

struct lux_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    lux_scene* scene = nullptr;   // holds one reference
    lux_options opt{};
    DevOptions dopt{};
    DevCamera cam{};
    DevScene S{};
    DevWave W{};
    int width = 0, height = 0, npix = 0;
    int spp_per_wave = 1;
    int accumulated = 0;
    // owned device memory (per-pixel and per-path state only)
    std::vector<void*> allocs;
    float* image = nullptr;
    float* comp = nullptr;
    uint8_t* rgba = nullptr;
    void* sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    int* h_wave_iter = nullptr;          // pinned, two ints per wave of the current call
    WaveCounters* h_ctr = nullptr;       // pinned, one per wave of the current call
    int h_cap = 0;
    // lanes of the wave arrays (waves in flight at once) and the lane of the last wave rendered
    int lanes = 1;
    int last_lane = 0;
    void* wave_block = nullptr;  // the wave arrays' allocation (wave_block_get)
    size_t wave_block_bytes = 0;
    // graphs: per wave size (one wave at a time), and per (waves, last wave size) of a
    // pipelined call; both hold device and page-locked host pointers of this context
    std::map<int, cudaGraphExec_t> graphs;
    std::map<std::pair<int, int>, cudaGraphExec_t> pgraphs;  // (waves, last wave size)
    std::map<std::pair<int, int>, int> pseen;                // call shapes launched eagerly
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        graphs.clear();
        for (auto& g : pgraphs) cudaGraphExecDestroy(g.second);
        pgraphs.clear();
        pseen.clear();
    }
    // stats of the last call
    lux_stats stats{};
    bool timing = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> kev;

    // per-pixel and per-path state: stream-ordered from the library's device memory pool, so
    // a context is made and freed without device-wide synchronisation, and the next context
    // reuses the memory (the reference's pathtraceFree / pathtraceInit on every reset)
    template <class T>
    int alloc(T** p, size_t n) {
        *p = nullptr;
        if (n == 0) return LUX_OK;
        cudaError_t e = scratch_alloc(reinterpret_cast<void**>(p), n * sizeof(T), stream);
        if (e != cudaSuccess) return fail(LUX_ERR_OOM, std::string("device allocation: ") + cudaGetErrorString(e));
        allocs.push_back(*p);
        return LUX_OK;
    }
};

namespace {

float half_bits_to_float(uint16_t h) {
    __half_raw r;
    r.x = h;
    return __half2float(__half(r));
}

// Upload one texture. storage LUX_TEXSTORE_FLOAT converts 8/16-bit unorm texels to float4 as
// TextureHandler::load_textures_on_device does (c/255, c/65535; src/texture.cu:12-69; on the
// device, texconv.cu),
// LUX_TEXSTORE_HALF converts them to binary16, LUX_TEXSTORE_UNORM8 keeps 8-bit texels (16-bit
// ones become float4). Binary16 texels stay binary16 under every storage.
// The texture uploads of one scene build run asynchronously on one stream: host texels are
// copied to device staging (pool memory, freed once the stream has drained), converted there,
// and copied into their CUDA arrays; one synchronisation ends the batch.
struct TexStage {
    cudaStream_t st = nullptr;
    std::vector<void*> staging;
    TexStage() = default;
    TexStage(const TexStage&) = delete;
    TexStage& operator=(const TexStage&) = delete;
    int begin() {
        LUX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        return LUX_OK;
    }
    int finish() {
        if (!st) return LUX_OK;
        cudaError_t e = cudaStreamSynchronize(st);
        release();
        if (e != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("texture upload: ") + cudaGetErrorString(e));
        return LUX_OK;
    }
    void release() {
        for (void* p : staging) scratch_free(p, st);
        staging.clear();
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        st = nullptr;
    }
    ~TexStage() { release(); }
    int get(void** p, size_t bytes) {
        cudaError_t e = scratch_alloc(p, bytes, st);
        if (e != cudaSuccess) return fail(LUX_ERR_OOM, std::string("texture staging: ") + cudaGetErrorString(e));
        staging.push_back(*p);
        return LUX_OK;
    }
};

int make_texture(const lux_texture_desc& t, DevTex& out, int storage, TexStage& stage) {
    if (t.width <= 0 || t.height <= 0 || !t.data) return fail(LUX_ERR_INVALID, "empty texture");
    const size_t n = size_t(t.width) * t.height * 4;
    const void* src = t.data;
    int fmt = t.format;
    // conversions run on the device: the texels are uploaded as they are and converted there
    const bool to_half = storage == LUX_TEXSTORE_HALF && t.format != LUX_TEX_RGBA16F;
    const bool to_float = (storage == LUX_TEXSTORE_FLOAT && t.format == LUX_TEX_RGBA8) ||
                          (storage != LUX_TEXSTORE_HALF && t.format == LUX_TEX_RGBA16);
    const void* dev_src = nullptr;
    if (to_half || to_float) {
        const size_t in_bytes = t.format == LUX_TEX_RGBA8 ? 1 : (t.format == LUX_TEX_RGBA32F ? 4 : 2);
        void *s_in = nullptr, *s_out = nullptr;
        if (int rc = stage.get(&s_in, n * in_bytes)) return rc;
        if (int rc = stage.get(&s_out, n * (to_half ? 2 : 4))) return rc;
        LUX_CUDA(cudaMemcpyAsync(s_in, t.data, n * in_bytes, cudaMemcpyHostToDevice, stage.st));
        LUX_CUDA(launch_convert_texels(s_in, t.format, to_half ? 1 : 0, s_out, n, stage.st));
        dev_src = s_out;
        fmt = to_half ? LUX_TEX_RGBA16F : LUX_TEX_RGBA32F;
    }
    cudaChannelFormatDesc fd;
    size_t texel;
    cudaTextureReadMode rm = cudaReadModeElementType;
    switch (fmt) {
        case LUX_TEX_RGBA8:
            fd = cudaCreateChannelDesc<uchar4>();
            texel = 4;
            rm = cudaReadModeNormalizedFloat;
            break;
        case LUX_TEX_RGBA16:
            fd = cudaCreateChannelDesc<ushort4>();
            texel = 8;
            rm = cudaReadModeNormalizedFloat;
            break;
        case LUX_TEX_RGBA16F:
            fd = cudaCreateChannelDescHalf4();
            texel = 8;
            break;
        case LUX_TEX_RGBA32F:
            fd = cudaCreateChannelDesc<float4>();
            texel = 16;
            break;
        default:
            return fail(LUX_ERR_INVALID, "unknown texture format");
    }
    LUX_CUDA(tex_array_get(&out.arr, fd, size_t(t.width), size_t(t.height)));
    if (dev_src)
        LUX_CUDA(cudaMemcpy2DToArrayAsync(out.arr, 0, 0, dev_src, size_t(t.width) * texel, size_t(t.width) * texel,
                                          t.height, cudaMemcpyDeviceToDevice, stage.st));
    else
        LUX_CUDA(cudaMemcpy2DToArrayAsync(out.arr, 0, 0, src, size_t(t.width) * texel, size_t(t.width) * texel,
                                          t.height, cudaMemcpyHostToDevice, stage.st));
    out.bytes = size_t(t.width) * t.height * texel;
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = out.arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = rm;
    td.normalizedCoords = 1;
    LUX_CUDA(cudaCreateTextureObject(&out.obj, &rd, &td, nullptr));
    return LUX_OK;
}

// Run fn(lo, hi) over [0, n) split into contiguous chunks, one per host thread. It runs while
// the geometry and texture threads of a scene build launch device work, so it leaves them
// three cores: a launching thread that waits for a core stalls the device behind it.
template <class F>
void parallel_chunks(int n, F fn, int min_chunk = 64) {
    const unsigned hw = std::thread::hardware_concurrency();
    unsigned nt = std::max(1u, std::min(hw > 4 ? hw - 3 : 1u, 64u));
    nt = std::max(1u, std::min(nt, unsigned((n + min_chunk - 1) / min_chunk)));
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(fn, int(int64_t(n) * t / nt), int(int64_t(n) * (t + 1) / nt));
    fn(0, int(int64_t(n) / nt));
    for (auto& t : th) t.join();
}

// The environment texels the HDRI CDF is built from: the values the env texture holds on the
// device, so that with binary16 storage the importance-sampling tables follow the stored map.
// Returns the scene's own array when it already holds those values, else fills `tmp`.
const float* env_texels(const lux_scene_desc& d, int storage, std::vector<float>& tmp) {
    const size_t n = size_t(d.env_width) * d.env_height * 4;
    if (d.env_format != LUX_TEX_RGBA16F && storage != LUX_TEXSTORE_HALF) return static_cast<const float*>(d.env_data);
    tmp.resize(n);
    const int rows = d.env_height;
    const size_t row = size_t(d.env_width) * 4;
    parallel_chunks(rows, [&](int y0, int y1) {
        for (size_t i = size_t(y0) * row; i < size_t(y1) * row; ++i) {
            if (d.env_format == LUX_TEX_RGBA16F)
                tmp[i] = half_bits_to_float(static_cast<const uint16_t*>(d.env_data)[i]);
            else
                tmp[i] = __half2float(__float2half_rn(static_cast<const float*>(d.env_data)[i]));
        }
    });
    return tmp.data();
}

// Emissive-area and HDRI CDFs as Scene::precompute_emissive_mesh_area and
// precompute_hdri_emission build them (src/scene/scene_precompute.cpp:22-124): sequential
// prefix sums in T, then normalised. T = float reproduces the reference bit for bit; the
// precision form uses T = double and rounds the final tables to float.
template <class T>
bool light_tables(const lux_scene_desc& d, const float* env, std::vector<int>& emissive,
                  std::vector<float>& eprefix, std::vector<std::vector<float>>& tri_prefix, float& total_area,
                  std::vector<float>& marginal, std::vector<float>& conditional) {
    const float kEPS = 0.00001f;
    T area = T(0);
    std::vector<T> ep;
    emissive.clear();
    tri_prefix.assign(d.num_instances, {});
    for (int i = 0; i < d.num_instances; ++i) {
        const lux_material_desc& mat = d.materials[d.instances[i].material];
        float ec = std::sqrt(mat.emission_color[0] * mat.emission_color[0] + mat.emission_color[1] * mat.emission_color[1] +
                             mat.emission_color[2] * mat.emission_color[2]);
        if (ec * mat.emission_strength > kEPS) emissive.push_back(i);  // only these tables are read
    }
    // each emissive instance's triangle CDF on its own thread; the instance totals then chain
    // in instance order, as the sequential loop adds them
    std::vector<T> inst_area(emissive.size());
    parallel_chunks(int(emissive.size()), [&](int e0, int e1) {
        for (int e = e0; e < e1; ++e) {
            const int i = emissive[e];
            const lux_instance_desc& in = d.instances[i];
            const lux_mesh_desc& m = d.meshes[in.mesh];
            T cum = T(0);
            std::vector<T> tp(m.num_tris);
            for (int k = 0; k < m.num_tris; ++k) {
                T P[3][3];
                for (int c = 0; c < 3; ++c) {
                    const float* v = m.positions + size_t(m.indices[k * 3 + c]) * 3;
                    for (int r = 0; r < 3; ++r) {
                        T a0 = T(in.transform[0 * 4 + r]) * T(v[0]), a1 = T(in.transform[1 * 4 + r]) * T(v[1]);
                        T a2 = T(in.transform[2 * 4 + r]) * T(v[2]), a3 = T(in.transform[3 * 4 + r]) * T(1);
                        P[c][r] = (a0 + a1) + (a2 + a3);
                    }
                }
                T u[3], v[3];
                for (int r = 0; r < 3; ++r) {
                    u[r] = P[1][r] - P[0][r];
                    v[r] = P[2][r] - P[0][r];
                }
                T cx = u[1] * v[2] - v[1] * u[2], cy = u[2] * v[0] - v[2] * u[0], cz = u[0] * v[1] - v[0] * u[1];
                cum += T(0.5) * std::sqrt(cx * cx + cy * cy + cz * cz);
                tp[k] = cum;
            }
            tri_prefix[i].resize(m.num_tris);
            for (int k = 0; k < m.num_tris; ++k) tri_prefix[i][k] = float(tp[k] / cum);
            inst_area[e] = cum;
        }
    }, 1);
    for (size_t e = 0; e < emissive.size(); ++e) {
        area += inst_area[e];
        ep.push_back(area);
    }
    eprefix.resize(ep.size());
    for (size_t k = 0; k < ep.size(); ++k) eprefix[k] = float(ep[k] / area);
    total_area = float(area);
    marginal.clear();
    conditional.clear();
    if (!d.env_data) return true;
    const int W = d.env_width, H = d.env_height;
    const float kPI = 3.1415926535897932384626422832795028841971f;
    // rows are independent; only the row totals chain, in row order
    std::vector<T> cond(size_t(W) * H), marg(H), rows(H);
    parallel_chunks(H, [&](int y0, int y1) {
        for (int y = y0; y < y1; ++y) {
            T rt = T(0);
            T theta = T(kPI) * (T(y) + T(0.5f)) / T(H);
            T st = std::sin(theta);
            T* cy = &cond[size_t(y) * W];
            for (int x = 0; x < W; ++x) {
                const float* p = &env[(size_t(y) * W + x) * 4];
                T a = T(p[0]) * T(p[0]), b = T(p[1]) * T(p[1]), c = T(p[2]) * T(p[2]), dd = T(p[3]) * T(p[3]);
                T e = std::sqrt((a + b) + (c + dd));
                rt += e * st;
                cy[x] = rt;
            }
            if (rt > T(0)) {
                for (int x = 0; x < W; ++x) cy[x] /= rt;
            } else {
                for (int x = 0; x < W; ++x) cy[x] = T(x + 1) / T(W);
            }
            cy[W - 1] = T(1);
            rows[y] = rt;
        }
    });
    T total = T(0);
    for (int y = 0; y < H; ++y) {
        total += rows[y];
        marg[y] = total;
    }
    if (total == T(0)) return false;  // the reference exits: "HDRI has emission of 0.0f"
    for (int y = 0; y < H; ++y) marg[y] /= total;
    marg[H - 1] = T(1);
    marginal.resize(H);
    conditional.resize(size_t(W) * H);
    for (int y = 0; y < H; ++y) marginal[y] = float(marg[y]);
    parallel_chunks(H, [&](int y0, int y1) {
        for (size_t k = size_t(y0) * W; k < size_t(y1) * W; ++k) conditional[k] = float(cond[k]);
    });
    return true;
}

// Guide table of one CDF (select_from_cdf_guided): g[j] = first i with cdf[i] >= j/m, or n-1.
void cdf_guide(const float* cdf, int n, int m, int* g) {
    int i = 0;
    for (int j = 0; j <= m; ++j) {
        const float t = float(j) / float(m);  // exact: m is a power of two
        while (i < n - 1 && cdf[i] < t) ++i;
        g[j] = i;
    }
}

int pow2_at_least(int v) {
    int m = 1;
    while (m < v && m < (1 << 16)) m <<= 1;
    return m;
}

}  // namespace

int lux::build_host_scene(const lux_scene_desc& d, const lux_options& opt, std::vector<DevTex>& texs,
                          DevTex& env, HostScene& H, const std::function<int()>& device_work) {
    // ---- textures and the environment map, on their own thread during the light tables ----
    const size_t tex0 = texs.size();
    texs.resize(tex0 + d.num_textures);
    int dev = 0;
    cudaGetDevice(&dev);
    int tex_rc = LUX_OK;
    std::string tex_err;
    const auto t0 = std::chrono::steady_clock::now();
    std::thread texer([&]() {
        if (cudaSetDevice(dev) != cudaSuccess) {
            tex_rc = fail(LUX_ERR_CUDA, "cudaSetDevice failed on the texture thread");
            tex_err = g_err;
            return;
        }
        {
            TexStage stage;
            tex_rc = stage.begin();
            for (int t = 0; t < d.num_textures && tex_rc == LUX_OK; ++t)
                tex_rc = make_texture(d.textures[t], texs[tex0 + t], opt.texture_storage, stage);
            if (tex_rc == LUX_OK && d.env_data) {
                lux_texture_desc et{d.env_width, d.env_height, d.env_format, 0, d.env_data};
                tex_rc = make_texture(et, env, opt.texture_storage == LUX_TEXSTORE_HALF ? LUX_TEXSTORE_HALF : LUX_TEXSTORE_FLOAT,
                                      stage);
            }
            const int frc = stage.finish();
            if (tex_rc == LUX_OK) tex_rc = frc;
        }
        H.ms_textures = ms_since(t0);
        if (tex_rc == LUX_OK && device_work) tex_rc = device_work();
        if (tex_rc) tex_err = g_err;
    });
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) t.join();
        }
    } joiner{texer};

    // ---- light tables ----
    std::vector<float> envt_tmp;
    const float* envt = d.env_data ? env_texels(d, opt.texture_storage, envt_tmp) : nullptr;
    std::vector<std::vector<float>> tri_prefix;
    bool env_ok;
    if (opt.precision == LUX_PRECISION_COMPENSATED)
        env_ok = light_tables<double>(d, envt, H.emissive, H.emissive_prefix, tri_prefix, H.total_area, H.marginal,
                                      H.conditional);
    else
        env_ok = light_tables<float>(d, envt, H.emissive, H.emissive_prefix, tri_prefix, H.total_area, H.marginal,
                                     H.conditional);
    if (!env_ok) return fail(LUX_ERR_INVALID, "environment map has no emission");
    if (d.env_data) {
        // about one marginal entry and four conditional entries per guide cell
        const int W = d.env_width, Hh = d.env_height;
        H.guide_marg = pow2_at_least(Hh);
        H.guide_cond = pow2_at_least(std::max(1, W / 4));
        H.marginal_guide.resize(size_t(H.guide_marg) + 1);
        cdf_guide(H.marginal.data(), Hh, H.guide_marg, H.marginal_guide.data());
        H.conditional_guide.resize(size_t(H.guide_cond + 1) * Hh);
        parallel_chunks(Hh, [&](int y0, int y1) {
            for (int y = y0; y < y1; ++y)
                cdf_guide(H.conditional.data() + size_t(y) * W, W, H.guide_cond,
                          H.conditional_guide.data() + size_t(y) * (H.guide_cond + 1));
        });
    }
    H.tri_off.clear();
    H.tri_prefix.clear();
    for (int e : H.emissive) {
        H.tri_off.push_back(int(H.tri_prefix.size()));
        H.tri_prefix.insert(H.tri_prefix.end(), tri_prefix[e].begin(), tri_prefix[e].end());
    }
    if (opt.direct_light_sampling && (H.emissive.empty() || H.total_area < 0.00001f))
        return fail(LUX_ERR_INVALID, "-dmis requires the scene to contain emissive geometry");
    if (opt.env_importance_sampling && !d.env_data)
        return fail(LUX_ERR_INVALID, "-emis requires an environment map");
    H.ms_tables = ms_since(t0);
    // ---- materials + textures ----
    texer.join();
    if (tex_rc) return fail(tex_rc, tex_err);
    std::vector<DevMaterial>& mats = H.mats;
    mats.assign(d.num_materials, DevMaterial{});
    for (int k = 0; k < d.num_materials; ++k) {
        const lux_material_desc& s = d.materials[k];
        DevMaterial& m = mats[k];
        std::memset(&m, 0, sizeof(m));
        for (int c = 0; c < 3; ++c) {
            m.color[c] = s.color[c];
            m.emission[c] = s.emission_color[c] * s.emission_strength;
        }
        m.alpha = s.alpha;
        m.roughness = s.roughness;
        m.metallic = s.metallic;
        m.transmission = s.transmission;
        m.ior = s.ior;
        m.alpha_cutoff = s.alpha_cutoff;
        m.alpha_mode = s.alpha_mode;
        auto tex_of = [&](int t, int flag, unsigned long long& obj) -> int {
            if (t < 0) return LUX_OK;
            if (t >= d.num_textures) return fail(LUX_ERR_INVALID, "material texture index out of range");
            obj = texs[tex0 + t].obj;
            m.flags |= flag;
            return LUX_OK;
        };
        int rc = tex_of(s.albedo_tex, kMatAlbedoTex, m.albedo_tex);
        rc = rc ? rc : tex_of(s.emissive_tex, kMatEmissiveTex, m.emissive_tex);
        rc = rc ? rc : tex_of(s.normal_tex, kMatNormalTex, m.normal_tex);
        rc = rc ? rc : tex_of(s.metallic_roughness_tex, kMatMRTex, m.mr_tex);
        if (rc) return rc;
        auto tt = [](const lux_tex_transform& a, DevTexTransform& b) {
            b.offset[0] = a.offset[0];
            b.offset[1] = a.offset[1];
            b.scale[0] = a.scale[0];
            b.scale[1] = a.scale[1];
            b.rotation = a.rotation;
        };
        tt(s.albedo_tt, m.albedo_tt);
        tt(s.emissive_tt, m.emissive_tt);
        tt(s.normal_tt, m.normal_tt);
        tt(s.metallic_roughness_tt, m.mr_tt);
    }
    if (d.env_data) {
        H.env_w = d.env_width;
        H.env_h = d.env_height;
        H.env_tex = env.obj;
        H.has_env = true;
    }
    // Morton box: the first instance's mesh bounds padded by 1e-5 (EPSILON of
    // include/utilities.h:16), in that instance's object space
    if (d.num_instances > 0) {
        const lux_mesh_desc& m0 = d.meshes[d.instances[0].mesh];
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int v = 0; v < m0.num_verts; ++v)
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], m0.positions[size_t(v) * 3 + a]);
                hi[a] = std::max(hi[a], m0.positions[size_t(v) * 3 + a]);
            }
        for (int a = 0; a < 3; ++a) {
            H.morton_bmin[a] = lo[a] - 0.00001f;
            H.morton_bmax[a] = hi[a] + 0.00001f;
        }
    }
    return LUX_OK;
}

namespace {

// Host build and upload of the scene; device_work runs on the build's device thread.
int build_scene(lux_scene* R, const lux_scene_desc& d, const lux_options& opt, const std::function<int()>& device_work) {
    const auto t_start = std::chrono::steady_clock::now();
    // The device geometry (vertex uploads, every BVH) is built on its own thread and stream,
    // while this thread builds the light tables and the texture thread uploads the textures.
    const int dev = R->device;
    GeometryBuild G;
    DevScene geo{};
    int geo_rc = LUX_OK;
    std::string geo_err;
    std::thread geom([&]() {
        if (cudaSetDevice(dev) != cudaSuccess) {
            geo_rc = fail(LUX_ERR_CUDA, "geometry thread set-up failed");
            geo_err = g_err;
            return;
        }
        const lux_scene_desc* one = &d;
        geo_rc = build_geometry(&one, 1, std::vector<int>{0}, opt.bvh_layout,
                                [&](void** p, size_t bytes) { return R->alloc(reinterpret_cast<char**>(p), bytes); },
                                R->stream, geo, G);
        if (geo_rc) geo_err = g_err;
    });
    HostScene H;
    int rc = build_host_scene(d, opt, R->texs, R->env, H, device_work);
    geom.join();
    if (rc) return rc;
    if (geo_rc) return fail(geo_rc, geo_err);
    R->instanced_tris = G.instanced_tris[0];
    lux_scene_stats& st = R->stats;
    st.ms_geometry = G.ms_total;
    st.ms_upload = G.ms_upload;
    st.ms_blas = G.ms_blas;
    st.ms_tlas = G.ms_tlas;
    st.ms_tables = H.ms_tables;
    st.ms_textures = H.ms_textures;
    st.blas_nodes = int64_t(G.blas_nodes);
    st.tlas_nodes = int64_t(G.tlas_nodes);
    R->h_emissive_prefix = H.emissive_prefix;
    R->h_tri_prefix = H.tri_prefix;
    R->h_marginal = H.marginal;
    R->h_conditional = H.conditional;
    R->h_total_area = H.total_area;
    R->has_emissive = !H.emissive.empty() && H.total_area >= 0.00001f;
    for (const DevTex& t : R->texs) R->scene_bytes += t.bytes;
    R->scene_bytes += R->env.bytes;
    R->S = geo;
    if ((rc = upload_scene_materials(R, H, R->S))) return rc;
    if ((rc = upload_scene_lights(R, H, R->S))) return rc;
    LUX_CUDA(cudaStreamSynchronize(R->stream));
    st.ms_total = ms_since(t_start);
    st.device_bytes = int64_t(R->scene_bytes);
    return LUX_OK;
}

void scene_release(lux_scene* R) {
    if (!R || --R->refs > 0) return;
    cudaSetDevice(R->device);
    // no copy into the textures is left in flight when their arrays go back for reuse
    if (R->stream) cudaStreamSynchronize(R->stream);
    for (auto& t : R->texs) destroy_texture(t);
    destroy_texture(R->env);
    for (void* p : R->allocs) scratch_free(p, R->stream);
    if (R->stream) {
        cudaStreamSynchronize(R->stream);
        cudaStreamDestroy(R->stream);
    }
    delete R;
}

// Checks shared by lux_scene_create and lux_init: options, and the device (made current).
int check_options_and_device(const lux_options& o) {
    if (o.texture_storage < LUX_TEXSTORE_FLOAT || o.texture_storage > LUX_TEXSTORE_HALF)
        return fail(LUX_ERR_INVALID, "unknown texture storage");
    if (o.precision != LUX_PRECISION_PLAIN && o.precision != LUX_PRECISION_COMPENSATED)
        return fail(LUX_ERR_INVALID, "unknown precision");
    if (o.bvh_layout < LUX_BVH_AUTO || o.bvh_layout > LUX_BVH_SINGLE_LEVEL)
        return fail(LUX_ERR_INVALID, "unknown BVH layout");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LUX_ERR_NO_DEVICE, "no CUDA device");
    if (o.device < 0 || o.device >= ndev) return fail(LUX_ERR_INVALID, "device ordinal out of range");
    // one attribute, not cudaGetDeviceProperties, which fills every field of the struct
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, o.device);
    if (major < 10) return fail(LUX_ERR_NO_DEVICE, "an sm_100 device is required");
    LUX_CUDA(cudaSetDevice(o.device));
    return LUX_OK;
}

// Build a resident scene; device_work (may be empty) runs on the build's device thread after
// the textures, overlapping the acceleration-structure build.
int scene_create(const lux_scene_desc& d, const lux_options& o, const std::function<int()>& device_work,
                 lux_scene** out) {
    *out = nullptr;
    lux_scene* R = new lux_scene();
    R->device = o.device;
    if (cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete R;
        return fail(LUX_ERR_CUDA, "cudaStreamCreate failed");
    }
    R->precision = o.precision;
    R->texture_storage = o.texture_storage;
    R->trace_depth = d.trace_depth;
    R->camera = d.camera;
    int rc = build_scene(R, d, o, device_work);
    if (rc) {
        std::string keep = g_err;
        scene_release(R);
        g_err = keep;
        return rc;
    }
    *out = R;
    return LUX_OK;
}

// Freed wave blocks kept per device and size class (up to kBlockKeep bytes per device) for the
// next context of about the same wave size: the reference re-creates its render state on every
// camera reset, and a block of a few GB from the memory pool can cost tens of ms once the pool
// has been churned by other sizes. Sizes are rounded up to kBlockGrain, and wave sizes cluster
// near 8M paths whatever the resolution, so most contexts share a class or two (a 1080p wave of
// 4 spp is 8.29M paths, one of 512x512 at 32 spp 8.39M: classes 41 and 42). A request takes the
// smallest kept block of its class or up to a quarter larger, so neighbouring classes share
// blocks. On a miss the device's kept blocks go back to the pool first, where the new block can
// reuse their memory. Blocks come back only after the context's stream has drained.
constexpr size_t kBlockKeep = size_t(16) << 30;
constexpr size_t kBlockGrain = size_t(128) << 20;
std::mutex g_block_mu;
std::multimap<std::pair<int, size_t>, void*> g_blocks;
std::map<int, size_t> g_block_bytes;

size_t block_class(size_t bytes) { return (bytes + kBlockGrain - 1) / kBlockGrain * kBlockGrain; }

// *cap receives the capacity of the block returned (its class), which wave_block_put takes back.
void* wave_block_get(int dev, size_t bytes, cudaStream_t st, size_t* cap) {
    const size_t cls = block_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_block_mu);
        auto it = g_blocks.lower_bound({dev, cls});
        if (it != g_blocks.end() && it->first.first == dev && it->first.second <= cls + cls / 4) {
            void* p = it->second;
            *cap = it->first.second;
            g_block_bytes[dev] -= it->first.second;
            g_blocks.erase(it);
            return p;
        }
        for (auto jt = g_blocks.begin(); jt != g_blocks.end();) {
            if (jt->first.first == dev) {
                scratch_free(jt->second, st);
                g_block_bytes[dev] -= jt->first.second;
                jt = g_blocks.erase(jt);
            } else {
                ++jt;
            }
        }
    }
    void* p = nullptr;
    if (scratch_alloc(&p, cls, st) != cudaSuccess) return nullptr;
    *cap = cls;
    return p;
}

void wave_block_put(int dev, void* p, size_t bytes, cudaStream_t st) {
    if (!p) return;
    const size_t cls = block_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_block_mu);
        if (g_block_bytes[dev] + cls <= kBlockKeep) {
            g_blocks.insert({{dev, cls}, p});
            g_block_bytes[dev] += cls;
            return;
        }
    }
    scratch_free(p, st);
}

// The wave's arrays are carved from one allocation (each 256-byte aligned), so that a
// context costs one allocation and one free for its whole path state.
// Wave arrays for `lanes` waves of max_paths paths each (lane l: paths and slots
// [l * max_paths, (l + 1) * max_paths)), counters per lane, and the table of the waves of a
// render call. Replaces an earlier allocation (the graphs captured on it are dropped).
int alloc_wave(lux_ctx* C, int max_paths, int lanes) {
    DevWave& W = C->W;
    if (C->wave_block) {
        if (C->stream) cudaStreamSynchronize(C->stream);
        C->drop_graphs();
        wave_block_put(C->device, C->wave_block, C->wave_block_bytes, C->stream);
        C->wave_block = nullptr;
        C->wave_block_bytes = 0;
    }
    std::memset(&W, 0, sizeof(W));
    const size_t n1 = size_t(max_paths), n = n1 * size_t(lanes);
    size_t off = 0;
    std::vector<std::pair<void**, size_t>> parts;
    auto take = [&](auto*& p, size_t count) {
        off = (off + 255) & ~size_t(255);
        parts.emplace_back(reinterpret_cast<void**>(&p), off);
        off += count * sizeof(*p);
    };
    take(W.s0, n);
    take(W.s1, n);
    take(W.s2, n);
    take(W.s3, n);
    take(W.s4, n);
    take(W.queue[0], n);
    take(W.queue[1], n);
    take(W.hit, n);
    take(W.hit_prim, n);
    take(W.sh_o, n);
    take(W.sh_d, n);
    take(W.sh_queue, n);
    take(W.sh_hit, n);
    take(W.sh_prim, n);
    take(W.ctr, size_t(lanes));
    take(W.wave_iter, 2 * size_t(kWaveTab));
    char* sort_temp = nullptr;
    if (C->opt.ray_sorting) {  // ray sorting runs one wave at a time, in lane 0
        take(W.keys, n1);
        take(W.keys_alt, n1);
        take(W.queue_alt, n1);
        C->sort_temp_bytes = morton_sort_temp_bytes(max_paths);
        take(sort_temp, C->sort_temp_bytes);
    }
    size_t cap = 0;
    char* base = static_cast<char*>(wave_block_get(C->device, off, C->stream, &cap));
    if (!base) return fail(LUX_ERR_OOM, "device allocation of the path state failed");
    C->wave_block = base;
    C->wave_block_bytes = cap;
    for (auto& pt : parts) *pt.first = base + pt.second;
    if (C->opt.ray_sorting) C->sort_temp = sort_temp;
    W.npix = C->npix;
    W.width = C->width;
    W.height = C->height;
    W.max_paths = max_paths;
    W.lane_stride = max_paths;
    C->lanes = lanes;
    C->last_lane = 0;
    return LUX_OK;
}

// Enqueue one wave of ns samples starting at iteration W.wave_iter[0].
int enqueue_wave(lux_ctx* C, int ns, const cudaEvent_t* ev) {
    cudaStream_t st = C->stream;
    DevWave& W = C->W;
    const int n = ns * C->npix;
    const int depth = C->dopt.trace_depth;
    const int nee = C->dopt.env ? 2 : (C->dopt.dl ? 1 : 0);
    int k = 0;
    auto rec = [&]() {
        if (ev) cudaEventRecord(ev[k], st);
        ++k;
    };
    LUX_CUDA(cudaMemsetAsync(W.ctr, 0, sizeof(WaveCounters), st));
    rec();
    LUX_CUDA(launch_camera(C->S, W, C->dopt, C->cam, n, 0, W.wave_iter, st));
    rec();
    for (int b = 0; b < depth; ++b) {
        if (C->opt.ray_sorting) LUX_CUDA(launch_morton_sort(C->S, W, b, C->sort_temp, C->sort_temp_bytes, st));
        rec();
        if (C->opt.debug_bvh) {
            // BVH heatmap: the counting traversal writes the camera ray's colour; no shading
            LUX_CUDA(launch_trace(C->S, W, b, 3, 0, st));
            rec();
            rec();
            continue;
        }
        LUX_CUDA(launch_trace(C->S, W, b, 0, nee, st));
        if (nee) LUX_CUDA(launch_trace(C->S, W, b, nee == 2 ? 2 : 1, 0, st));
        rec();
        LUX_CUDA(launch_shade(C->S, W, C->dopt, b, (b + 1) < depth ? 1 : 0, st));
        rec();
    }
    LUX_CUDA(launch_accumulate(W, 0, C->image, C->comp, ns, C->opt.precision == LUX_PRECISION_COMPENSATED, st));
    rec();
    return LUX_OK;
}

int events_needed(const lux_ctx* C) { return 3 + 3 * C->dopt.trace_depth; }

// ---- pipelined waves ------------------------------------------------------------------------
// After the first bounces almost every path of a wave has ended (Russian roulette), but each
// of its remaining bounces still costs a full launch of traversal, occlusion and shading whose
// time is the latency of a few rays. Several waves are therefore kept in flight, one per lane:
// wave w starts at step w * P and runs bounce t - w * P at step t, and every step is one set of
// launches over all waves in flight (launch_trace_segs / launch_shade_segs). With L lanes and
// P = ceil(depth / L), lane w % L is free again when wave w starts. Every path is computed as in
// the one-wave schedule, waves end in order and each is accumulated as it ends, in sample
// order, so the image is the same bit for bit.
int lanes_wanted(const lux_ctx* C) {
    const int depth = C->dopt.trace_depth;
    if (C->opt.ray_sorting || C->opt.debug_bvh || depth < 2) return 1;
    return std::min(kMaxLanes, depth);
}

// Events of a timed call: (event, what the interval that it ends measured).
enum { kSpanNone = 0, kSpanCamera, kSpanTrace, kSpanShade, kSpanAccum };
struct Spans {
    lux_ctx* C;
    std::vector<std::pair<int, int>> marks;
    int mark(int what) {
        if (!C->timing) return LUX_OK;
        const size_t i = marks.size();
        if (i >= C->kev.size()) {
            C->kev.emplace_back();
            LUX_CUDA(cudaEventCreate(&C->kev.back()));
        }
        LUX_CUDA(cudaEventRecord(C->kev[i], C->stream));
        marks.emplace_back(int(i), what);
        return LUX_OK;
    }
};

// Waves [0, nw) of the call (table entries of W.wave_iter), the last one of ns_last samples;
// counters of wave w are copied to h_ctr[h0 + w] when it ends.
int enqueue_pipelined(lux_ctx* C, int nw, int ns_last, int h0, Spans* sp) {
    cudaStream_t st = C->stream;
    DevWave& W = C->W;
    const int D = C->dopt.trace_depth, L = C->lanes, P = (D + L - 1) / L;
    const int nee = C->dopt.env ? 2 : (C->dopt.dl ? 1 : 0);
    const int steps = (nw - 1) * P + D;
    auto ns_of = [&](int w) { return w == nw - 1 ? ns_last : C->spp_per_wave; };
    if (sp) if (int rc_ = sp->mark(kSpanNone)) return rc_;
    for (int t = 0; t < steps; ++t) {
        if (t % P == 0 && t / P < nw) {
            const int w = t / P, lane = w % L;
            LUX_CUDA(cudaMemsetAsync(W.ctr + lane, 0, sizeof(WaveCounters), st));
            LUX_CUDA(launch_camera(C->S, W, C->dopt, C->cam, ns_of(w) * C->npix, lane, W.wave_iter + 2 * w, st));
            if (sp) if (int rc_ = sp->mark(kSpanCamera)) return rc_;
        }
        Segs G{};
        const int w_lo = std::max(0, (t - D) / P), w_hi = std::min(nw - 1, t / P);
        for (int w = w_lo; w <= w_hi; ++w) {
            const int b = t - w * P;
            if (b < 0 || b >= D) continue;
            if (G.n == kMaxSegs) return fail(LUX_ERR_STATE, "wave schedule: too many waves in flight");
            G.lane[G.n] = w % L;
            G.bounce[G.n] = b;
            G.compact[G.n] = (b + 1) < D ? 1 : 0;
            ++G.n;
        }
        LUX_CUDA(launch_trace_segs(C->S, W, G, 0, nee, st));
        if (nee) LUX_CUDA(launch_trace_segs(C->S, W, G, nee == 2 ? 2 : 1, 0, st));
        if (sp) if (int rc_ = sp->mark(kSpanTrace)) return rc_;
        LUX_CUDA(launch_shade_segs(C->S, W, C->dopt, G, st));
        if (sp) if (int rc_ = sp->mark(kSpanShade)) return rc_;
        // the wave that ran its last bounce: counters out, then its samples into the image
        const int we = t - (D - 1);
        if (we >= 0 && we % P == 0 && we / P < nw) {
            const int w = we / P, lane = w % L;
            LUX_CUDA(cudaMemcpyAsync(&C->h_ctr[h0 + w], W.ctr + lane, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
            LUX_CUDA(launch_accumulate(W, lane, C->image, C->comp, ns_of(w),
                                       C->opt.precision == LUX_PRECISION_COMPENSATED, st));
            if (sp) if (int rc_ = sp->mark(kSpanAccum)) return rc_;
            C->last_lane = lane;
        }
    }
    return LUX_OK;
}

// Stats of a finished call from the waves' counters and, when timed, the marked spans.
int finish_stats(lux_ctx* C, int nwaves, int n_iter, const Spans* sp, int steps) {
    const int depth = C->dopt.trace_depth;
    const bool nee = C->dopt.dl || C->dopt.env;
    const int spw = C->spp_per_wave;
    for (int w = 0; w < nwaves; ++w) {
        const WaveCounters& c = C->h_ctr[w];
        if (c.error) return fail(LUX_ERR_UNSUPPORTED, "traversal stack overflow");
        for (int b = 0; b < depth; ++b) {
            C->stats.rays_radiance += c.count[b];
            C->stats.path_bounces += c.count[b];
            C->stats.rays_shadow += c.shadow[b];
        }
        const int ns = std::min(spw, n_iter - w * spw);
        C->stats.samples += double(ns) * C->npix;
    }
    C->stats.launches_camera += nwaves;
    C->stats.launches_accum += nwaves;
    C->stats.launches_trace += steps * (nee ? 2 : 1);
    C->stats.launches_shade += steps;
    if (sp) {
        for (size_t i = 1; i < sp->marks.size(); ++i) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, C->kev[sp->marks[i - 1].first], C->kev[sp->marks[i].first]);
            switch (sp->marks[i].second) {
                case kSpanCamera: C->stats.ms_camera += t; break;
                case kSpanTrace: C->stats.ms_trace += t; break;
                case kSpanShade: C->stats.ms_shade += t; break;
                case kSpanAccum: C->stats.ms_accum += t; break;
                default: break;
            }
        }
    }
    C->stats.kernel_launches = C->stats.launches_camera + C->stats.launches_accum + C->stats.launches_trace +
                               C->stats.launches_shade + C->stats.launches_sort;
    return LUX_OK;
}

// A render call of several waves with `lanes` of them in flight (enqueue_pipelined).
int run_pipelined(lux_ctx* C, int first_iter, int n_iter, int nwaves, int lanes) {
    cudaStream_t st = C->stream;
    const int spw = C->spp_per_wave;
    if (C->lanes < lanes)
        if (int rc = alloc_wave(C, spw * C->npix, lanes)) return rc;
    const int D = C->dopt.trace_depth, P = (D + C->lanes - 1) / C->lanes;
    std::memset(&C->stats, 0, sizeof(C->stats));
    Spans spans{C, {}};
    LUX_CUDA(cudaEventRecord(C->ev[0], st));
    int steps = 0;
    for (int c0 = 0; c0 < nwaves; c0 += kWaveTab) {
        const int nw = std::min(kWaveTab, nwaves - c0);
        int ns_last = 0;
        for (int w = 0; w < nw; ++w) {
            const int it0 = first_iter + (c0 + w) * spw;
            ns_last = std::min(spw, first_iter + n_iter - it0);
            C->h_wave_iter[2 * (c0 + w)] = it0;
            C->h_wave_iter[2 * (c0 + w) + 1] = ns_last;
        }
        LUX_CUDA(cudaMemcpyAsync(C->W.wave_iter, &C->h_wave_iter[2 * c0], 2 * sizeof(int) * size_t(nw),
                                 cudaMemcpyHostToDevice, st));
        // the graph bakes in the chunk's counter copies (h_ctr + c0) and its wave count. A call
        // shape is captured when it comes again: a context that renders once (a cold start,
        // a one-off job) would spend more on capturing and instantiating than replay saves.
        const std::pair<int, int> key{(c0 / kWaveTab) * (kWaveTab + 1) + nw, ns_last};
        const bool replay = C->opt.use_graph && !C->timing && (C->pgraphs.count(key) || C->pseen[key]++ > 0);
        if (replay) {
            auto it = C->pgraphs.find(key);
            if (it == C->pgraphs.end()) {
                cudaGraph_t g;
                LUX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                int rc = enqueue_pipelined(C, nw, ns_last, c0, nullptr);
                cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (rc) return rc;
                if (ce != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
                cudaGraphExec_t ge;
                cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
                it = C->pgraphs.emplace(key, ge).first;
            }
            LUX_CUDA(cudaGraphLaunch(it->second, st));
        } else {
            if (int rc = enqueue_pipelined(C, nw, ns_last, c0, C->timing ? &spans : nullptr)) return rc;
        }
        steps += (nw - 1) * P + D;
        C->last_lane = (nw - 1) % C->lanes;
    }
    LUX_CUDA(cudaEventRecord(C->ev[1], st));
    LUX_CUDA(cudaEventSynchronize(C->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, C->ev[0], C->ev[1]);
    C->stats.ms_total = ms;
    if (int rc = finish_stats(C, nwaves, n_iter, C->timing ? &spans : nullptr, steps)) return rc;
    C->accumulated += n_iter;
    return LUX_OK;
}

int run_waves(lux_ctx* C, int first_iter, int n_iter) {
    if (n_iter <= 0) return LUX_OK;
    cudaStream_t st = C->stream;
    const int spw = C->spp_per_wave;
    const int nwaves = (n_iter + spw - 1) / spw;
    if (C->h_cap < nwaves) {
        // the previous call ended with a synchronize, so no copy uses the old blocks; graphs
        // of pipelined calls copy counters into them, so they go too
        C->drop_graphs();
        pinned_put(C->h_ctr, sizeof(WaveCounters) * size_t(C->h_cap));
        pinned_put(C->h_wave_iter, sizeof(int) * 2 * size_t(C->h_cap));
        C->h_ctr = nullptr;
        C->h_wave_iter = nullptr;
        C->h_cap = 0;
        C->h_ctr = static_cast<WaveCounters*>(pinned_get(sizeof(WaveCounters) * size_t(nwaves)));
        C->h_wave_iter = static_cast<int*>(pinned_get(sizeof(int) * 2 * size_t(nwaves)));
        if (!C->h_ctr || !C->h_wave_iter) return fail(LUX_ERR_OOM, "page-locked host allocation failed");
        C->h_cap = nwaves;
    }
    const int want = lanes_wanted(C);
    if (want > 1 && nwaves > 1) return run_pipelined(C, first_iter, n_iter, nwaves, want);
    C->last_lane = 0;
    const int epw = events_needed(C);
    if (C->timing && int(C->kev.size()) < epw * nwaves) {
        size_t have = C->kev.size();
        C->kev.resize(size_t(epw) * nwaves);
        for (size_t i = have; i < C->kev.size(); ++i) LUX_CUDA(cudaEventCreate(&C->kev[i]));
    }
    std::memset(&C->stats, 0, sizeof(C->stats));
    LUX_CUDA(cudaEventRecord(C->ev[0], st));
    for (int w = 0; w < nwaves; ++w) {
        int it0 = first_iter + w * spw;
        int ns = std::min(spw, first_iter + n_iter - it0);
        // the wave's first iteration reaches the camera kernel through a device word, so a
        // captured graph stays valid for every wave of the same size
        C->h_wave_iter[2 * w] = it0;
        C->h_wave_iter[2 * w + 1] = ns;
        LUX_CUDA(cudaMemcpyAsync(C->W.wave_iter, &C->h_wave_iter[2 * w], 2 * sizeof(int), cudaMemcpyHostToDevice, st));
        if (C->opt.use_graph && !C->timing) {
            auto it = C->graphs.find(ns);
            if (it == C->graphs.end()) {
                cudaGraph_t g;
                LUX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                int rc = enqueue_wave(C, ns, nullptr);
                cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (rc) return rc;
                if (ce != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
                cudaGraphExec_t ge;
                cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
                it = C->graphs.emplace(ns, ge).first;
            }
            LUX_CUDA(cudaGraphLaunch(it->second, st));
        } else {
            int rc = enqueue_wave(C, ns, C->timing ? &C->kev[size_t(w) * epw] : nullptr);
            if (rc) return rc;
        }
        LUX_CUDA(cudaMemcpyAsync(&C->h_ctr[w], C->W.ctr, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
    }
    LUX_CUDA(cudaEventRecord(C->ev[1], st));
    LUX_CUDA(cudaEventSynchronize(C->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, C->ev[0], C->ev[1]);
    C->stats.ms_total = ms;
    const int depth = C->dopt.trace_depth;
    const bool nee = C->dopt.dl || C->dopt.env;
    const int sort_launches = 1 + 4 * 3;
    for (int w = 0; w < nwaves; ++w) {
        const WaveCounters& c = C->h_ctr[w];
        if (c.error) return fail(LUX_ERR_UNSUPPORTED, "traversal stack overflow");
        for (int b = 0; b < depth; ++b) {
            C->stats.rays_radiance += c.count[b];
            C->stats.path_bounces += c.count[b];
            C->stats.rays_shadow += c.shadow[b];
        }
        int ns = std::min(spw, n_iter - w * spw);
        C->stats.samples += double(ns) * C->npix;
        C->stats.launches_camera += 1;
        C->stats.launches_accum += 1;
        C->stats.launches_trace += depth * (nee ? 2 : 1);
        C->stats.launches_shade += depth;
        C->stats.launches_sort += C->opt.ray_sorting ? depth * sort_launches : 0;
        if (C->timing) {
            const cudaEvent_t* e = &C->kev[size_t(w) * epw];
            float t;
            cudaEventElapsedTime(&t, e[0], e[1]);
            C->stats.ms_camera += t;
            for (int b = 0; b < depth; ++b) {
                cudaEventElapsedTime(&t, e[1 + 3 * b], e[2 + 3 * b]);
                C->stats.ms_sort += t;
                cudaEventElapsedTime(&t, e[2 + 3 * b], e[3 + 3 * b]);
                C->stats.ms_trace += t;
                cudaEventElapsedTime(&t, e[3 + 3 * b], e[4 + 3 * b]);
                C->stats.ms_shade += t;
            }
            cudaEventElapsedTime(&t, e[1 + 3 * depth], e[2 + 3 * depth]);
            C->stats.ms_accum += t;
        }
    }
    C->stats.kernel_launches = C->stats.launches_camera + C->stats.launches_accum + C->stats.launches_trace +
                               C->stats.launches_shade + C->stats.launches_sort;
    C->accumulated += n_iter;
    return LUX_OK;
}

struct Tmp {
    std::vector<void*> p;
    ~Tmp() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    T* get(size_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        note_device_alloc();
        p.push_back(q);
        return static_cast<T*>(q);
    }
};

}  // namespace

int lux::validate_scene_desc(const lux_scene_desc& d) {
    if (d.num_instances <= 0 || d.num_meshes <= 0 || !d.meshes || !d.instances)
        return fail(LUX_ERR_INVALID, "scene has no geometry");
    if (d.num_materials <= 0 || !d.materials) return fail(LUX_ERR_INVALID, "scene has no materials");
    if (d.camera.width <= 0 || d.camera.height <= 0) return fail(LUX_ERR_INVALID, "camera resolution must be positive");
    if (d.num_textures < 0 || (d.num_textures > 0 && !d.textures)) return fail(LUX_ERR_INVALID, "bad texture list");
    for (int i = 0; i < d.num_meshes; ++i) {
        const lux_mesh_desc& m = d.meshes[i];
        if (m.num_tris <= 0 || m.num_verts <= 0 || !m.positions || !m.indices)
            return fail(LUX_ERR_INVALID, "mesh " + std::to_string(i) + " is empty");
        for (int k = 0; k < m.num_tris * 3; ++k)
            if (m.indices[k] >= uint32_t(m.num_verts))
                return fail(LUX_ERR_INVALID, "mesh " + std::to_string(i) + " index out of range");
    }
    for (int i = 0; i < d.num_instances; ++i) {
        if (d.instances[i].mesh < 0 || d.instances[i].mesh >= d.num_meshes || d.instances[i].material < 0 ||
            d.instances[i].material >= d.num_materials)
            return fail(LUX_ERR_INVALID, "instance " + std::to_string(i) + " references a missing mesh or material");
    }
    if (d.env_data && (d.env_width <= 0 || d.env_height <= 0 ||
                       (d.env_format != LUX_TEX_RGBA32F && d.env_format != LUX_TEX_RGBA16F)))
        return fail(LUX_ERR_INVALID, "environment map must be RGBA32F or RGBA16F with a positive size");
    return LUX_OK;
}

namespace {
std::atomic<int64_t> g_device_allocs{0};
}

void lux::note_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }

namespace {
std::mutex g_pinned_mu;
std::map<size_t, std::vector<void*>> g_pinned_free;
size_t pinned_class(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
}
}  // namespace

void* lux::pinned_get(size_t bytes) {
    const size_t c = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        auto it = g_pinned_free.find(c);
        if (it != g_pinned_free.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, c) != cudaSuccess) return nullptr;
    return p;
}

namespace {
struct TexShape {
    int device, x, y, z, w, kind;
    size_t width, height;
    bool operator<(const TexShape& o) const {
        return std::tie(device, x, y, z, w, kind, width, height) <
               std::tie(o.device, o.x, o.y, o.z, o.w, o.kind, o.width, o.height);
    }
};
std::mutex g_arr_mu;
std::map<TexShape, std::vector<cudaArray_t>> g_arr_free;
std::map<int, size_t> g_arr_bytes;  // kept bytes per device
TexShape tex_shape(int dev, const cudaChannelFormatDesc& fd, size_t w, size_t h) {
    return TexShape{dev, fd.x, fd.y, fd.z, fd.w, int(fd.f), w, h};
}
size_t tex_bytes(const cudaChannelFormatDesc& fd, size_t w, size_t h) {
    return size_t(fd.x + fd.y + fd.z + fd.w) / 8 * w * h;
}
}  // namespace

cudaError_t lux::tex_array_get(cudaArray_t* arr, const cudaChannelFormatDesc& fd, size_t width, size_t height) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_arr_mu);
        auto it = g_arr_free.find(tex_shape(dev, fd, width, height));
        if (it != g_arr_free.end() && !it->second.empty()) {
            *arr = it->second.back();
            it->second.pop_back();
            g_arr_bytes[dev] -= tex_bytes(fd, width, height);
            return cudaSuccess;
        }
    }
    e = cudaMallocArray(arr, &fd, width, height);
    if (e == cudaSuccess) note_device_alloc();
    return e;
}

void lux::tex_array_put(cudaArray_t arr) {
    if (!arr) return;
    int dev = 0;
    cudaChannelFormatDesc fd;
    cudaExtent ext;
    unsigned flags = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaArrayGetInfo(&fd, &ext, &flags, arr) != cudaSuccess || flags != 0 ||
        ext.depth != 0) {
        cudaFreeArray(arr);
        return;
    }
    const size_t bytes = tex_bytes(fd, ext.width, ext.height);
    {
        std::lock_guard<std::mutex> lk(g_arr_mu);
        if (g_arr_bytes[dev] + bytes <= kTexArrayKeep) {
            g_arr_free[tex_shape(dev, fd, ext.width, ext.height)].push_back(arr);
            g_arr_bytes[dev] += bytes;
            return;
        }
    }
    cudaFreeArray(arr);
}

void lux::pinned_put(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free[pinned_class(bytes)].push_back(p);
}

extern "C" {

int64_t lux_device_alloc_count(void) { return g_device_allocs.load(std::memory_order_relaxed); }

void lux_default_options(lux_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->color_mode = LUX_TONEMAP_ACES;
    o->envmap_intensity = 1.0f;
    o->use_graph = 1;
    o->texture_storage = LUX_TEXSTORE_FLOAT;
}

const char* lux_last_error(void) { return lux::g_err.c_str(); }

}  // extern "C"

namespace {

// The context fields that follow from the options and the camera, and its stream; no device
// memory yet. scene_depth is the scene description's trace depth.
// Context options that need no device: trace depth and the debug views.
int check_ctx_options(const lux_options& o, const lux_camera_desc& cd, int scene_depth) {
    if (cd.width <= 0 || cd.height <= 0) return fail(LUX_ERR_INVALID, "camera resolution must be positive");
    int tdepth = o.trace_depth > 0 ? o.trace_depth : scene_depth;
    if (tdepth <= 0 || tdepth > kMaxDepth) return fail(LUX_ERR_INVALID, "trace depth must be in 1..64");
    if (o.material_debug_mode < LUX_MATDEBUG_OFF || o.material_debug_mode > LUX_MATDEBUG_ALPHA)
        return fail(LUX_ERR_INVALID, "material_debug_mode must be in 0..6");
    if (o.debug_bvh != 0 && o.debug_bvh != 1) return fail(LUX_ERR_INVALID, "debug_bvh must be 0 or 1");
    if (o.debug_bvh && o.material_debug_mode)
        return fail(LUX_ERR_UNSUPPORTED, "the BVH heatmap and a material debug view are exclusive");
    return LUX_OK;
}

int ctx_prepare(const lux_options& o, const lux_camera_desc& cd, int scene_depth, lux_ctx** out) {
    *out = nullptr;
    if (int rc = check_ctx_options(o, cd, scene_depth)) return rc;
    int tdepth = o.trace_depth > 0 ? o.trace_depth : scene_depth;
    // debug views trace camera rays only (src/pathtrace.cu:107 forces trace depth 1 for the
    // material views); their camera rays are seeded with that depth as well
    if (o.material_debug_mode || o.debug_bvh) tdepth = 1;
    lux_ctx* C = new lux_ctx();
    C->device = o.device;
    C->opt = o;
    C->dopt.dl = o.direct_light_sampling ? 1 : 0;
    C->dopt.env = o.env_importance_sampling ? 1 : 0;
    C->dopt.env_intensity = o.envmap_intensity;
    C->dopt.trace_depth = tdepth;
    C->dopt.color_mode = o.color_mode;
    C->dopt.precision = o.precision;
    C->dopt.material_debug = o.material_debug_mode;
    C->width = cd.width;
    C->height = cd.height;
    C->npix = C->width * C->height;
    for (int a = 0; a < 3; ++a) {
        C->cam.pos[a] = cd.position[a];
        C->cam.view[a] = cd.view[a];
        C->cam.right[a] = cd.right[a];
        C->cam.up[a] = cd.up[a];
    }
    C->cam.pixel_length[0] = cd.pixel_length[0];
    C->cam.pixel_length[1] = cd.pixel_length[1];
    C->cam.width = cd.width;
    C->cam.height = cd.height;
    if (o.stream) {
        C->stream = static_cast<cudaStream_t>(o.stream);
    } else {
        if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete C;
            return fail(LUX_ERR_CUDA, "cudaStreamCreate failed");
        }
        C->own_stream = true;
    }
    // samples kept in flight together: about 8M paths, at least one sample
    int spw = o.spp_per_wave > 0 ? o.spp_per_wave : std::max(1, (8 << 20) / C->npix);
    spw = std::max(1, std::min(spw, 1 << 16));
    C->spp_per_wave = spw;
    *out = C;
    return LUX_OK;
}

// Per-pixel and per-path device memory of a context (the part pathtraceInit allocates,
// src/pathtrace/pathtrace_buffers.cu:21-140).
int ctx_alloc(lux_ctx* C) {
    // The lanes of waves in flight come with the context, in one block. A wave holds about 8M
    // paths whatever the resolution, so most contexts ask for one size class, and a freed
    // context's block serves the next. (Giving a small image one lane here and its other lanes
    // at its first render of several waves made two classes alternate in a stream of mixed
    // sizes: each miss sent the kept blocks back to the pool, and a sequence of 64 plain renders
    // of mixed sizes took 3.7 s instead of 1.4.)
    const int lanes = lanes_wanted(C);
    int r = alloc_wave(C, C->spp_per_wave * C->npix, lanes);
    if (!r) r = C->alloc(&C->image, size_t(C->npix) * 3);
    if (!r && C->opt.precision == LUX_PRECISION_COMPENSATED) r = C->alloc(&C->comp, size_t(C->npix) * 3);
    if (!r) r = C->alloc(&C->rgba, size_t(C->npix) * 4);
    if (!r && cudaMemsetAsync(C->image, 0, size_t(C->npix) * 3 * sizeof(float), C->stream) != cudaSuccess)
        r = fail(LUX_ERR_CUDA, "memset");
    if (!r && C->comp && cudaMemsetAsync(C->comp, 0, size_t(C->npix) * 3 * sizeof(float), C->stream) != cudaSuccess)
        r = fail(LUX_ERR_CUDA, "memset");
    return r;
}

// The scene-dependent option checks of a context on R.
int check_ctx_on_scene(const lux_scene* R, const lux_options& o) {
    if (o.device != R->device) return fail(LUX_ERR_INVALID, "the context's device differs from the scene's");
    if (o.precision != R->precision) return fail(LUX_ERR_INVALID, "precision differs from the scene's build");
    if (o.texture_storage != R->texture_storage)
        return fail(LUX_ERR_INVALID, "texture storage differs from the scene's build");
    if (o.direct_light_sampling && !R->has_emissive)
        return fail(LUX_ERR_INVALID, "-dmis requires the scene to contain emissive geometry");
    if (o.env_importance_sampling && !R->S.has_env) return fail(LUX_ERR_INVALID, "-emis requires an environment map");
    return LUX_OK;
}

int ctx_finish(lux_ctx* C) {
    if (cudaEventCreate(&C->ev[0]) != cudaSuccess || cudaEventCreate(&C->ev[1]) != cudaSuccess)
        return fail(LUX_ERR_CUDA, "cudaEventCreate failed");
    // occupancy queries happen here, never inside a stream capture
    for (int m = 0; m < 4; ++m) trace_grid_blocks(m, C->S.single_level != 0);
    shade_grid_blocks();
    if (cudaStreamSynchronize(C->stream) != cudaSuccess) return fail(LUX_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    if (cudaGetLastError() != cudaSuccess) return fail(LUX_ERR_CUDA, "context set-up failed");
    return LUX_OK;
}

}  // namespace

extern "C" {

int lux_scene_create(const lux_scene_desc* scene, const lux_options* opt, lux_scene** out) {
    if (!out) return fail(LUX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scene) return fail(LUX_ERR_INVALID, "scene is NULL");
    if (int rc = validate_scene_desc(*scene)) return rc;
    lux_options o;
    if (opt) o = *opt;
    else lux_default_options(&o);
    if (int rc = check_options_and_device(o)) return rc;
    // -dmis / -emis are checked per context (lux_init_on_scene), not against the scene build
    o.direct_light_sampling = 0;
    o.env_importance_sampling = 0;
    int rc = scene_create(*scene, o, nullptr, out);
    if (rc) return rc;
    if (cudaDeviceSynchronize() != cudaSuccess) {
        lux_scene_free(*out);
        *out = nullptr;
        return fail(LUX_ERR_CUDA, "scene build failed");
    }
    return LUX_OK;
}

int lux_scene_free(lux_scene* scene) {
    scene_release(scene);
    return LUX_OK;
}

int64_t lux_scene_device_bytes(const lux_scene* scene) { return scene ? int64_t(scene->scene_bytes) : 0; }

int lux_scene_get_stats(const lux_scene* scene, lux_scene_stats* out) {
    if (!scene || !out) return fail(LUX_ERR_INVALID, "NULL argument");
    *out = scene->stats;
    return LUX_OK;
}

int lux_get_scene_stats(lux_ctx* C, lux_scene_stats* out) {
    if (!C || !out) return fail(LUX_ERR_INVALID, "NULL argument");
    *out = C->scene->stats;
    return LUX_OK;
}

int lux_init_on_scene(lux_scene* R, const lux_camera_desc* camera, const lux_options* opt, lux_ctx** out) {
    if (!out) return fail(LUX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!R) return fail(LUX_ERR_INVALID, "scene is NULL");
    lux_options o;
    if (opt) o = *opt;
    else lux_default_options(&o);
    if (int rc = check_ctx_options(o, camera ? *camera : R->camera, R->trace_depth)) return rc;
    if (int rc = check_options_and_device(o)) return rc;
    if (int rc = check_ctx_on_scene(R, o)) return rc;
    lux_ctx* C = nullptr;
    if (int rc = ctx_prepare(o, camera ? *camera : R->camera, R->trace_depth, &C)) return rc;
    ++R->refs;
    C->scene = R;
    C->S = R->S;
    int rc = ctx_alloc(C);
    if (!rc) rc = ctx_finish(C);
    if (rc) {
        std::string keep = g_err;
        lux_free(C);
        g_err = keep;
        return rc;
    }
    *out = C;
    return LUX_OK;
}

int lux_init(const lux_scene_desc* scene, const lux_options* opt, lux_ctx** out) {
    if (!out) return fail(LUX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scene) return fail(LUX_ERR_INVALID, "scene is NULL");
    const lux_scene_desc& d = *scene;
    if (int rc = validate_scene_desc(d)) return rc;
    lux_options o;
    if (opt) o = *opt;
    else lux_default_options(&o);
    if (int rc = check_ctx_options(o, d.camera, d.trace_depth)) return rc;
    if (int rc = check_options_and_device(o)) return rc;
    lux_ctx* C = nullptr;
    if (int rc = ctx_prepare(o, d.camera, d.trace_depth, &C)) return rc;
    auto bail = [&](int rc) {
        std::string keep = g_err;
        lux_free(C);
        g_err = keep;
        return rc;
    };
    // The wave buffers and the image do not depend on the scene: the scene build's device
    // thread allocates them after the textures, while this thread builds the BVHs.
    lux_scene* R = nullptr;
    int rc = scene_create(d, o, [&]() { return ctx_alloc(C); }, &R);
    if (rc) return bail(rc);
    C->scene = R;  // the creation's reference passes to the context
    C->S = R->S;
    if ((rc = check_ctx_on_scene(R, o))) return bail(rc);
    if ((rc = ctx_finish(C))) return bail(rc);
    *out = C;
    return LUX_OK;
}

int lux_render(lux_ctx* C, int first_iter, int n_iter) {
    if (!C) return fail(LUX_ERR_STATE, "context is NULL");
    if (first_iter < 1 || n_iter < 0) return fail(LUX_ERR_INVALID, "iterations are 1-based and n_iter >= 0");
    cudaSetDevice(C->device);
    return run_waves(C, first_iter, n_iter);
}

int lux_render_iter(lux_ctx* C, int iter, uint8_t* rgba8_dev) {
    if (!C) return fail(LUX_ERR_STATE, "context is NULL");
    if (iter < 1) return fail(LUX_ERR_INVALID, "iter is 1-based");
    cudaSetDevice(C->device);
    int save = C->spp_per_wave;
    C->spp_per_wave = 1;
    int rc = run_waves(C, iter, 1);
    C->spp_per_wave = save;
    if (rc) return rc;
    if (rgba8_dev) {
        LUX_CUDA(launch_tonemap(C->image, rgba8_dev, C->npix, float(iter), C->opt.material_debug_mode ? -1 : C->opt.color_mode, C->stream));
        LUX_CUDA(cudaStreamSynchronize(C->stream));
    }
    return LUX_OK;
}

int lux_copy_image(lux_ctx* C, float* rgb_host) {
    if (!C || !rgb_host) return fail(LUX_ERR_INVALID, "NULL argument");
    cudaSetDevice(C->device);
    LUX_CUDA(cudaMemcpyAsync(rgb_host, C->image, size_t(C->npix) * 3 * sizeof(float), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    return LUX_OK;
}

int lux_copy_image_device(lux_ctx* C, float* rgb_dev) {
    if (!C || !rgb_dev) return fail(LUX_ERR_INVALID, "NULL argument");
    LUX_CUDA(cudaSetDevice(C->device));
    LUX_CUDA(cudaMemcpyAsync(rgb_dev, C->image, size_t(C->npix) * 3 * sizeof(float), cudaMemcpyDeviceToDevice,
                             C->stream));
    return LUX_OK;
}

int lux_copy_rgba8(lux_ctx* C, uint8_t* rgba_host) {
    if (!C || !rgba_host) return fail(LUX_ERR_INVALID, "NULL argument");
    cudaSetDevice(C->device);
    float it = float(std::max(1, C->accumulated));
    LUX_CUDA(launch_tonemap(C->image, C->rgba, C->npix, it, C->opt.material_debug_mode ? -1 : C->opt.color_mode, C->stream));
    LUX_CUDA(cudaMemcpyAsync(rgba_host, C->rgba, size_t(C->npix) * 4, cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    return LUX_OK;
}

int lux_reset(lux_ctx* C) {
    if (!C) return fail(LUX_ERR_STATE, "context is NULL");
    cudaSetDevice(C->device);
    LUX_CUDA(cudaMemsetAsync(C->image, 0, size_t(C->npix) * 3 * sizeof(float), C->stream));
    if (C->comp) LUX_CUDA(cudaMemsetAsync(C->comp, 0, size_t(C->npix) * 3 * sizeof(float), C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    C->accumulated = 0;
    return LUX_OK;
}

int lux_set_camera(lux_ctx* C, const lux_camera_desc* cd) {
    if (!C || !cd) return fail(LUX_ERR_INVALID, "NULL argument");
    if (cd->width != C->width || cd->height != C->height) return fail(LUX_ERR_INVALID, "resolution cannot change");
    for (int a = 0; a < 3; ++a) {
        C->cam.pos[a] = cd->position[a];
        C->cam.view[a] = cd->view[a];
        C->cam.right[a] = cd->right[a];
        C->cam.up[a] = cd->up[a];
    }
    C->cam.pixel_length[0] = cd->pixel_length[0];
    C->cam.pixel_length[1] = cd->pixel_length[1];
    // camera parameters are baked into captured graphs
    C->drop_graphs();
    return lux_reset(C);
}

int lux_free(lux_ctx* C) {
    if (!C) return LUX_OK;
    cudaSetDevice(C->device);
    if (C->stream) cudaStreamSynchronize(C->stream);
    C->drop_graphs();
    for (void* p : C->allocs) scratch_free(p, C->stream);
    wave_block_put(C->device, C->wave_block, C->wave_block_bytes, C->stream);
    pinned_put(C->h_wave_iter, sizeof(int) * 2 * size_t(C->h_cap));
    pinned_put(C->h_ctr, sizeof(WaveCounters) * size_t(C->h_cap));
    for (auto e : C->kev) cudaEventDestroy(e);
    if (C->ev[0]) cudaEventDestroy(C->ev[0]);
    if (C->ev[1]) cudaEventDestroy(C->ev[1]);
    if (C->own_stream && C->stream) cudaStreamDestroy(C->stream);
    lux_scene* R = C->scene;
    delete C;
    scene_release(R);
    return LUX_OK;
}

int lux_enable_timing(lux_ctx* C, int on) {
    if (!C) return fail(LUX_ERR_STATE, "context is NULL");
    C->timing = on != 0;
    return LUX_OK;
}

int lux_get_stats(lux_ctx* C, lux_stats* out) {
    if (!C || !out) return fail(LUX_ERR_INVALID, "NULL argument");
    *out = C->stats;
    return LUX_OK;
}

int lux_wave_counts(lux_ctx* C, int* paths, int* shadow, int max_bounces) {
    if (!C || !paths || !shadow || max_bounces < 0) return fail(LUX_ERR_INVALID, "bad arguments");
    LUX_CUDA(cudaSetDevice(C->device));
    WaveCounters hc;
    LUX_CUDA(cudaMemcpyAsync(&hc, C->W.ctr + C->last_lane, sizeof(hc), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    const int n = std::min(max_bounces, kMaxDepth);
    for (int b = 0; b < n; ++b) {
        paths[b] = hc.count[b];
        shadow[b] = hc.shadow[b];
    }
    return LUX_OK;
}

// ---- kernel-level entry points -------------------------------------------------------
int lux_trace_rays(lux_ctx* C, const float* rays, int n, int mode, int iter, uint32_t* hits) {
    if (!C || (!rays && n > 0) || (!hits && n > 0) || n < 0 || mode < 0 || mode > 3)
        return fail(LUX_ERR_INVALID, "bad arguments");
    if (n == 0) return LUX_OK;
    cudaSetDevice(C->device);
    Tmp t;
    float* dr = t.get<float>(size_t(n) * 8);
    uint32_t* dh = t.get<uint32_t>(size_t(n) * 5);
    int* fetch = t.get<int>(1);
    if (!dr || !dh || !fetch) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(cudaMemcpyAsync(dr, rays, size_t(n) * 8 * sizeof(float), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(cudaMemsetAsync(fetch, 0, sizeof(int), C->stream));
    LUX_CUDA(cudaMemsetAsync(C->W.ctr, 0, sizeof(WaveCounters), C->stream));
    LUX_CUDA(launch_trace_ext(C->S, C->W, dr, dh, n, mode, iter, fetch, C->stream));
    LUX_CUDA(cudaMemcpyAsync(hits, dh, size_t(n) * 5 * sizeof(uint32_t), cudaMemcpyDeviceToHost, C->stream));
    WaveCounters hc;
    LUX_CUDA(cudaMemcpyAsync(&hc, C->W.ctr, sizeof(hc), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    if (hc.error) return fail(LUX_ERR_UNSUPPORTED, "traversal stack overflow");
    return LUX_OK;
}

int lux_trace_rays_static(lux_ctx* C, const float* rays, int n, int mode, int iter, uint32_t* hits) {
    if (!C || (!rays && n > 0) || (!hits && n > 0) || n < 0 || mode < 0 || mode > 3)
        return fail(LUX_ERR_INVALID, "bad arguments");
    if (n > LUX_TRACE_STATIC_MAX_RAYS)
        return fail(LUX_ERR_INVALID, "lux_trace_rays_static: n = " + std::to_string(n) +
                                         " exceeds LUX_TRACE_STATIC_MAX_RAYS (" +
                                         std::to_string(LUX_TRACE_STATIC_MAX_RAYS) +
                                         "); split the batch or call lux_trace_rays");
    if (n == 0) return LUX_OK;
    LUX_CUDA(cudaSetDevice(C->device));
    TraceScratch sc;
    LUX_CUDA(trace_static_scratch(C->device, sc));
    LUX_CUDA(cudaMemcpyAsync(sc.rays, rays, size_t(n) * 8 * sizeof(float), cudaMemcpyHostToDevice, C->stream));
    // the work cursor and the traversal error word must start at zero
    LUX_CUDA(cudaMemsetAsync(sc.cursor, 0, sizeof(int), C->stream));
    LUX_CUDA(cudaMemsetAsync(C->W.ctr, 0, sizeof(WaveCounters), C->stream));
    LUX_CUDA(launch_trace_ext(C->S, C->W, sc.rays, sc.hits, n, mode, iter, sc.cursor, C->stream));
    LUX_CUDA(cudaMemcpyAsync(hits, sc.hits, size_t(n) * 5 * sizeof(uint32_t), cudaMemcpyDeviceToHost, C->stream));
    WaveCounters hc;
    LUX_CUDA(cudaMemcpyAsync(&hc, C->W.ctr, sizeof(hc), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    if (hc.error) return fail(LUX_ERR_UNSUPPORTED, "traversal stack overflow");
    return LUX_OK;
}

int lux_morton_keys(lux_ctx* C, const float* rays, int n, uint32_t* keys) {
    if (!C || n < 0 || (n > 0 && (!rays || !keys))) return fail(LUX_ERR_INVALID, "bad arguments");
    if (n == 0) return LUX_OK;
    cudaSetDevice(C->device);
    Tmp t;
    float* dr = t.get<float>(size_t(n) * 8);
    uint32_t* dk = t.get<uint32_t>(size_t(n));
    if (!dr || !dk) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(cudaMemcpyAsync(dr, rays, size_t(n) * 8 * sizeof(float), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(launch_morton_ext(C->S, dr, dk, n, C->stream));
    LUX_CUDA(cudaMemcpyAsync(keys, dk, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    return LUX_OK;
}

int lux_shade_step(lux_ctx* C, int iter, int depth, int compact, float* paths, int n, const uint32_t* hits,
                   int* survivors, int* n_out) {
    if (!C || n < 0 || !n_out || (n > 0 && (!paths || !hits || !survivors))) return fail(LUX_ERR_INVALID, "bad arguments");
    *n_out = 0;
    if (n == 0) return LUX_OK;
    cudaSetDevice(C->device);
    Tmp t;
    float* dp = t.get<float>(size_t(n) * LUX_PS_FLOATS);
    uint32_t* dh = t.get<uint32_t>(size_t(n) * 10);
    int* ds = t.get<int>(size_t(n));
    int* dn = t.get<int>(1);
    if (!dp || !dh || !ds || !dn) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(cudaMemcpyAsync(dp, paths, size_t(n) * LUX_PS_FLOATS * sizeof(float), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(cudaMemcpyAsync(dh, hits, size_t(n) * 10 * sizeof(uint32_t), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(cudaMemsetAsync(dn, 0, sizeof(int), C->stream));
    LUX_CUDA(launch_shade_ext(C->S, C->dopt, dp, dh, n, iter, depth, compact, ds, dn, C->stream));
    LUX_CUDA(cudaMemcpyAsync(paths, dp, size_t(n) * LUX_PS_FLOATS * sizeof(float), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaMemcpyAsync(n_out, dn, sizeof(int), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    LUX_CUDA(cudaMemcpy(survivors, ds, size_t(*n_out) * sizeof(int), cudaMemcpyDeviceToHost));
    return LUX_OK;
}

int lux_light_samples(lux_ctx* C, int iter, int depth, const int* pixels, int n, float* out) {
    if (!C || n < 0 || (n > 0 && (!pixels || !out))) return fail(LUX_ERR_INVALID, "bad arguments");
    if (n == 0) return LUX_OK;
    cudaSetDevice(C->device);
    Tmp t;
    int* dp = t.get<int>(size_t(n));
    float* dout = t.get<float>(size_t(n) * 6);
    if (!dp || !dout) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(cudaMemcpyAsync(dp, pixels, size_t(n) * sizeof(int), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(launch_light_ext(C->S, C->dopt, iter, depth, dp, n, dout, C->stream));
    LUX_CUDA(cudaMemcpyAsync(out, dout, size_t(n) * 6 * sizeof(float), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    return LUX_OK;
}

int lux_get_cdfs(lux_ctx* C, float* ep, float* tp, float* mg, float* cd, float* ta) {
    if (!C) return fail(LUX_ERR_STATE, "context is NULL");
    cudaSetDevice(C->device);
    DevScene& S = C->S;
    if (ep && S.num_emissive) LUX_CUDA(cudaMemcpy(ep, S.emissive_prefix, C->scene->h_emissive_prefix.size() * 4, cudaMemcpyDeviceToHost));
    if (tp && !C->scene->h_tri_prefix.empty()) LUX_CUDA(cudaMemcpy(tp, S.tri_prefix, C->scene->h_tri_prefix.size() * 4, cudaMemcpyDeviceToHost));
    if (mg && S.has_env) LUX_CUDA(cudaMemcpy(mg, S.marginal, C->scene->h_marginal.size() * 4, cudaMemcpyDeviceToHost));
    if (cd && S.has_env) LUX_CUDA(cudaMemcpy(cd, S.conditional, C->scene->h_conditional.size() * 4, cudaMemcpyDeviceToHost));
    if (ta) *ta = S.total_area;
    return LUX_OK;
}

int lux_rng_stream(int iter, int index, int depth, int n, float* out) {
    if (n < 0 || (n > 0 && !out)) return fail(LUX_ERR_INVALID, "bad arguments");
    if (n == 0) return LUX_OK;
    Tmp t;
    float* d = t.get<float>(size_t(n));
    if (!d) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(launch_rng_ext(iter, index, depth, n, d, 0));
    LUX_CUDA(cudaMemcpy(out, d, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost));
    return LUX_OK;
}

int lux_sample_texture(lux_ctx* C, int tex, const float* uv, int n, float* out) {
    if (!C || n < 0 || (n > 0 && (!uv || !out))) return fail(LUX_ERR_INVALID, "bad arguments");
    if (tex < -1 || tex >= int(C->scene->texs.size())) return fail(LUX_ERR_INVALID, "texture index out of range");
    if (tex == -1 && !C->S.has_env) return fail(LUX_ERR_INVALID, "no environment map");
    if (n == 0) return LUX_OK;
    cudaSetDevice(C->device);
    Tmp t;
    float* du = t.get<float>(size_t(n) * 2);
    float* dout = t.get<float>(size_t(n) * 4);
    if (!du || !dout) return fail(LUX_ERR_OOM, "temporary allocation failed");
    LUX_CUDA(cudaMemcpyAsync(du, uv, size_t(n) * 2 * sizeof(float), cudaMemcpyHostToDevice, C->stream));
    LUX_CUDA(launch_tex_ext(tex < 0 ? C->scene->env.obj : C->scene->texs[tex].obj, du, n, dout, C->stream));
    LUX_CUDA(cudaMemcpyAsync(out, dout, size_t(n) * 4 * sizeof(float), cudaMemcpyDeviceToHost, C->stream));
    LUX_CUDA(cudaStreamSynchronize(C->stream));
    return LUX_OK;
}

}  // extern "C"
