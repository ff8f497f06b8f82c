// engine.cpp -- the job engine: many render jobs over resident scenes in one shared wavefront
// (the batching and serving forms; C-ABI in include/luxion.h, lux_engine_*).
//
// Scenes are built with the same host code as a single-job context (build_host_scene) and
// concatenated: node, primitive, instance, TLAS-leaf, vertex, index and material arrays are
// appended with their cross-references offset. Each scene keeps its own light tables and
// environment map, reachable through a per-scene DevScene in device memory whose geometry
// pointers are the concatenated arrays. A wave is a list of segments (job, sample range);
// the kernels find a path's job from W.path_job and take its camera, depth, scene lights and
// TLAS root from there. The wave's launches are captured once per (trace depth, wave size,
// trace grid) and replayed.
//
// Because every path is seeded by its job-local iteration and pixel, and a job's samples are
// accumulated in order, the image of a job does not depend on the other jobs of its waves
// nor on how its samples were split across waves.

#include "host_common.h"
#include "launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <string>
#include <tuple>
#include <vector>

using namespace lux;

namespace {

struct EngineJob {
    lux_job_desc desc{};
    int state = LUX_JOB_QUEUED;
    int slot = -1;  // row of the device job table while admitted
    int spp_sched = 0, spp_done = 0, waves = 0;
    int spp_final = 0;  // samples whose accumulation has completed on the device
    int depth = 0;
    int npix = 0;
    size_t bytes = 0;
    float* image = nullptr;
    float* comp = nullptr;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

// A wave in flight (after autotuning, up to kEngineLanes at once): its lane, the depth it runs
// to, the next bounce, its paths and the (job id, samples) it renders.
struct Flight {
    int lane = 0;
    int depth = 0;
    int bounce = 0;
    int paths = 0;
    std::vector<std::pair<int, int>> part;
};
constexpr int kEngineLanes = kMaxSegs;
// bounces every wave in flight advances per lux_engine_step (six, with half the host round
// trips, served 4 to 7 % more requests per second but rendered the batched mix 5 % slower:
// a lane frees up half as often, so fewer waves overlap)
constexpr int kStepBounces = 3;

double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct lux_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    lux_options opt{};
    DevOptions dopt{};
    lux_engine_config cfg{};
    std::chrono::steady_clock::time_point t0;
    // resident scenes
    std::vector<DevTex> texs;
    std::vector<DevTex> envs;
    std::vector<int> scene_depth;
    std::vector<uint32_t> scene_root;
    DevScene S{};                 // concatenated geometry (kernel argument of trace and shade)
    DevScene* scenes_d = nullptr; // per-scene views
    // wave
    DevWave W{};
    int paths_alloc = 0;          // wave buffers are sized for this many paths
    int max_paths = 0;            // wave size in use
    int trace_blocks = 0;         // persistent trace grid in use
    DevJob* jobs_d = nullptr;
    DevJob* jobs_h = nullptr;     // pinned mirror, one row per slot
    DevSegment* segs_d = nullptr; // per lane, kMaxSegments each
    // pinned, per lane and twice (by step parity): a wave planned while the step before is
    // still on the device must not overwrite a table whose copy that step has not yet made
    DevSegment* segs_h = nullptr; // kMaxSegments per lane
    int* hdr_h = nullptr;         // 4 ints per lane
    WaveCounters* ctr_h = nullptr;  // pinned, per lane, twice (by step parity)
    int lanes = kEngineLanes;
    std::deque<Flight> flight;    // waves in flight, in start order
    int max_jobs = 0;
    std::vector<int> free_slots;
    std::vector<EngineJob> jobs;  // by job id
    std::deque<int> queued;
    std::vector<int> active;
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> graphs;  // (depth, wave size, trace grid)
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // Pipelined steps: a call enqueues its step and then finishes the step before it, so the
    // device runs one step while the host finishes the last and serves finished jobs.
    cudaEvent_t step_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // (start, end) by parity
    int step_par = 0;
    bool pend_valid = false;  // a step is enqueued whose accumulated waves await bookkeeping
    int pend_par = 0;
    std::vector<Flight> pend_fin;
    cudaStream_t copy_stream = nullptr;  // read-back of finished jobs' images
    // autotuning of (wave size, trace grid) on the first waves
    std::vector<std::pair<int, int>> tune_cands;
    std::vector<double> tune_cost;  // device ms per path of each candidate's wave
    size_t tune_next = 0;
    // memory accounting and stats
    std::vector<void*> allocs;
    int64_t scene_bytes = 0, wave_bytes = 0, job_bytes = 0;
    lux_engine_stats stats{};

    template <class T>
    int alloc(T** p, size_t n) {
        int rc = dalloc(p, n);
        if (rc == LUX_OK && *p) allocs.push_back(*p);
        wave_bytes += int64_t(n * sizeof(T));
        return rc;
    }
    template <class T>
    int up(T** p, const T* src, size_t n) {
        int rc = upload(p, src, n);
        if (rc == LUX_OK && *p) allocs.push_back(*p);
        scene_bytes += int64_t(n * sizeof(T));
        return rc;
    }
    // device allocation counted as scene memory (the device-built geometry)
    int up_alloc(char** p, size_t n) {
        int rc = dalloc(p, n);
        if (rc == LUX_OK && *p) allocs.push_back(*p);
        scene_bytes += int64_t(n);
        return rc;
    }
    int64_t device_bytes() const { return scene_bytes + wave_bytes + job_bytes; }
};

namespace {

// Admitted jobs with samples still to schedule, in the order they fill a wave.
int order_jobs(const lux_engine* E, std::vector<int>& order) {
    order.clear();
    for (int id : E->active) {
        const EngineJob& j = E->jobs[id];
        if (j.spp_sched < j.desc.spp) order.push_back(id);
    }
    if (E->cfg.schedule == LUX_SCHED_SHORTEST_FIRST) {
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            const EngineJob& x = E->jobs[a];
            const EngineJob& y = E->jobs[b];
            return double(x.npix) * (x.desc.spp - x.spp_sched) < double(y.npix) * (y.desc.spp - y.spp_sched);
        });
    }
    return int(order.size());
}

int enqueue_wave(lux_engine* E, int depth, int wave_paths, int trace_grid) {
    cudaStream_t st = E->stream;
    const int nee = E->dopt.env ? 2 : (E->dopt.dl ? 1 : 0);
    LUX_CUDA(cudaMemsetAsync(E->W.ctr, 0, sizeof(WaveCounters), st));
    LUX_CUDA(launch_camera_jobs(E->W, E->dopt, wave_paths, 0, st));
    for (int b = 0; b < depth; ++b) {
        LUX_CUDA(launch_trace(E->S, E->W, b, 0, nee, st, trace_grid));
        if (nee) LUX_CUDA(launch_trace(E->S, E->W, b, nee == 2 ? 2 : 1, 0, st, trace_grid));
        LUX_CUDA(launch_shade(E->S, E->W, E->dopt, b, 1, st));
    }
    LUX_CUDA(launch_accumulate_jobs(E->W, E->opt.precision == LUX_PRECISION_COMPENSATED, 0, st));
    return LUX_OK;
}

// Admit queued jobs in submission order while a job-table row is free and the device memory
// stays within the budget: allocate and clear the job's image (stream-ordered) and write its
// row of the job table.
int admit(lux_engine* E) {
    while (!E->queued.empty()) {
        const int id = E->queued.front();
        EngineJob& j = E->jobs[id];
        if (E->free_slots.empty()) break;
        if (E->cfg.hbm_budget_bytes > 0 && E->device_bytes() + int64_t(j.bytes) > E->cfg.hbm_budget_bytes) break;
        const size_t n = size_t(j.npix) * 3;
        LUX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&j.image), n * sizeof(float), E->stream));
        note_device_alloc();
        LUX_CUDA(cudaMemsetAsync(j.image, 0, n * sizeof(float), E->stream));
        if (E->opt.precision == LUX_PRECISION_COMPENSATED) {
            LUX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&j.comp), n * sizeof(float), E->stream));
            note_device_alloc();
            LUX_CUDA(cudaMemsetAsync(j.comp, 0, n * sizeof(float), E->stream));
        }
        j.slot = E->free_slots.back();
        E->free_slots.pop_back();
        DevJob& dj = E->jobs_h[j.slot];
        std::memset(&dj, 0, sizeof(dj));
        const lux_camera_desc& c = j.desc.camera;
        dj.scene = j.desc.scene;
        dj.width = c.width;
        dj.height = c.height;
        dj.npix = j.npix;
        dj.trace_depth = j.depth;
        dj.first_iter = j.desc.first_iter > 0 ? j.desc.first_iter : 1;
        dj.tlas_root = E->scene_root[j.desc.scene];
        dj.image = j.image;
        dj.comp = j.comp;
        for (int a = 0; a < 3; ++a) {
            dj.pos[a] = c.position[a];
            dj.view[a] = c.view[a];
            dj.right[a] = c.right[a];
            dj.up[a] = c.up[a];
        }
        dj.pixel_length[0] = c.pixel_length[0];
        dj.pixel_length[1] = c.pixel_length[1];
        LUX_CUDA(cudaMemcpyAsync(E->jobs_d + j.slot, &dj, sizeof(DevJob), cudaMemcpyHostToDevice, E->stream));
        j.state = LUX_JOB_ACTIVE;
        j.t_admit = now_ms(E->t0);
        E->job_bytes += int64_t(j.bytes);
        E->active.push_back(id);
        E->queued.pop_front();
    }
    return LUX_OK;
}

void free_job_memory(lux_engine* E, EngineJob& j) {
    if (j.image) cudaFreeAsync(j.image, E->stream);
    if (j.comp) cudaFreeAsync(j.comp, E->stream);
    j.image = j.comp = nullptr;
    if (j.slot >= 0) {
        E->free_slots.push_back(j.slot);
        j.slot = -1;
        E->job_bytes -= int64_t(j.bytes);
    }
}

}  // namespace

extern "C" {

int lux_plan_wave(const int* npix, const int* remaining, int njobs, int capacity, int max_segments, int* take) {
    if (njobs < 0 || capacity < 0 || max_segments < 0 || (njobs > 0 && (!npix || !remaining || !take)))
        return fail(LUX_ERR_INVALID, "bad arguments");
    int used = 0, segs = 0;
    for (int i = 0; i < njobs; ++i) {
        take[i] = 0;
        if (segs >= max_segments || remaining[i] <= 0 || npix[i] <= 0) continue;
        const int fit = (capacity - used) / npix[i];
        if (fit <= 0) continue;
        take[i] = std::min(remaining[i], fit);
        used += take[i] * npix[i];
        ++segs;
    }
    return segs;
}

int lux_engine_create(const lux_scene_desc* const* scenes, int num_scenes, const lux_options* opt,
                      const lux_engine_config* cfg, lux_engine** out) {
    if (!out) return fail(LUX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scenes || num_scenes <= 0) return fail(LUX_ERR_INVALID, "no scenes");
    for (int i = 0; i < num_scenes; ++i) {
        if (!scenes[i]) return fail(LUX_ERR_INVALID, "scene " + std::to_string(i) + " is NULL");
        if (int rc = validate_scene_desc(*scenes[i])) return rc;
        if (scenes[i]->trace_depth < 0 || scenes[i]->trace_depth > kMaxDepth)
            return fail(LUX_ERR_INVALID, "trace depth must be in 1..64");
    }
    lux_options o;
    if (opt) o = *opt;
    else lux_default_options(&o);
    if (o.texture_storage < LUX_TEXSTORE_FLOAT || o.texture_storage > LUX_TEXSTORE_HALF)
        return fail(LUX_ERR_INVALID, "unknown texture storage");
    if (o.bvh_layout < LUX_BVH_AUTO || o.bvh_layout > LUX_BVH_SINGLE_LEVEL)
        return fail(LUX_ERR_INVALID, "unknown BVH layout");
    if (o.material_debug_mode || o.debug_bvh)
        return fail(LUX_ERR_UNSUPPORTED, "debug views are rendered by lux_init contexts, not by the engine");
    lux_engine_config c{};
    if (cfg) c = *cfg;
    if (c.max_paths < 0 || c.max_jobs < 0 || c.trace_blocks < 0 || c.hbm_budget_bytes < 0)
        return fail(LUX_ERR_INVALID, "negative engine configuration value");
    if (c.schedule != LUX_SCHED_FIFO && c.schedule != LUX_SCHED_SHORTEST_FIRST)
        return fail(LUX_ERR_INVALID, "unknown schedule");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LUX_ERR_NO_DEVICE, "no CUDA device");
    if (o.device < 0 || o.device >= ndev) return fail(LUX_ERR_INVALID, "device ordinal out of range");
    // one attribute, not cudaGetDeviceProperties, which fills every field of the struct
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, o.device);
    if (major < 10) return fail(LUX_ERR_NO_DEVICE, "an sm_100 device is required");
    LUX_CUDA(cudaSetDevice(o.device));

    lux_engine* E = new lux_engine();
    E->t0 = std::chrono::steady_clock::now();
    E->device = o.device;
    E->opt = o;
    E->cfg = c;
    E->dopt.dl = o.direct_light_sampling ? 1 : 0;
    E->dopt.env = o.env_importance_sampling ? 1 : 0;
    E->dopt.env_intensity = o.envmap_intensity;
    E->dopt.trace_depth = 0;  // per job
    E->dopt.color_mode = o.color_mode;
    E->dopt.precision = o.precision;
    auto bail = [&](int rc) {
        std::string keep = g_err;
        lux_engine_free(E);
        g_err = keep;
        return rc;
    };
    if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(LUX_ERR_CUDA, "cudaStreamCreate failed"));

    // ---- scenes: geometry of all scenes built on the device at once, then each scene's
    // textures, materials and light tables ----
    std::vector<HostScene> hs(num_scenes);
    std::vector<int> mat_base(num_scenes, 0);
    for (int i = 1; i < num_scenes; ++i) mat_base[i] = mat_base[i - 1] + scenes[i - 1]->num_materials;
    GeometryBuild G;
    if (int rc = build_geometry(scenes, num_scenes, mat_base, o.bvh_layout,
                                [&](void** p, size_t bytes) { return E->up_alloc(reinterpret_cast<char**>(p), bytes); },
                                E->stream, E->S, G))
        return bail(rc);
    E->envs.resize(num_scenes);
    std::vector<DevMaterial> mats;
    for (int i = 0; i < num_scenes; ++i) {
        if (int rc = build_host_scene(*scenes[i], o, E->texs, E->envs[i], hs[i])) return bail(rc);
        E->scene_depth.push_back(scenes[i]->trace_depth);
        E->scene_root.push_back(G.tlas_root[i]);
        for (int& e : hs[i].emissive) e += G.inst_base[i];  // emissive instances in the concatenation
        mats.insert(mats.end(), hs[i].mats.begin(), hs[i].mats.end());
    }
    {
        DevMaterial* dm = nullptr;
        if (int rc = E->up(&dm, mats.data(), mats.size())) return bail(rc);
        E->S.mats = dm;
    }
    std::vector<DevScene> views(num_scenes);
    for (int i = 0; i < num_scenes; ++i) {
        DevScene& v = views[i];
        v = E->S;
        v.tlas_root = E->scene_root[i];
        if (int rc = upload_scene_lights(E, hs[i], v)) return bail(rc);
    }
    if (int rc = E->up(&E->scenes_d, views.data(), views.size())) return bail(rc);
    for (const DevTex& t : E->texs) E->scene_bytes += int64_t(t.bytes);
    for (const DevTex& t : E->envs) E->scene_bytes += int64_t(t.bytes);

    // ---- wave buffers ----
    static const int kTuneSizes[] = {2 << 20, 4 << 20, 8 << 20};
    E->paths_alloc = c.max_paths > 0 ? c.max_paths : kTuneSizes[2];
    DevWave& W = E->W;
    const int L = E->lanes;
    const size_t n = size_t(E->paths_alloc) * size_t(L);  // lane l: paths [l * paths_alloc, ...)
    int rc;
    if ((rc = E->alloc(&W.s0, n)) || (rc = E->alloc(&W.s1, n)) || (rc = E->alloc(&W.s2, n)) ||
        (rc = E->alloc(&W.s3, n)) || (rc = E->alloc(&W.s4, n)) || (rc = E->alloc(&W.queue[0], n)) ||
        (rc = E->alloc(&W.queue[1], n)) || (rc = E->alloc(&W.hit, n)) || (rc = E->alloc(&W.hit_prim, n)) ||
        (rc = E->alloc(&W.sh_o, n)) || (rc = E->alloc(&W.sh_d, n)) || (rc = E->alloc(&W.sh_queue, n)) ||
        (rc = E->alloc(&W.sh_hit, n)) || (rc = E->alloc(&W.sh_prim, n)) || (rc = E->alloc(&W.ctr, size_t(L))) ||
        (rc = E->alloc(&W.wave_iter, 4)) || (rc = E->alloc(&W.path_job, n)) ||
        (rc = E->alloc(&E->segs_d, size_t(kMaxSegments) * L)) || (rc = E->alloc(&W.wave_hdr, size_t(4) * L)))
        return bail(rc);
    E->max_jobs = c.max_jobs > 0 ? c.max_jobs : 4096;
    if ((rc = E->alloc(&E->jobs_d, size_t(E->max_jobs)))) return bail(rc);
    W.scenes = E->scenes_d;
    W.jobs = E->jobs_d;
    W.segs = E->segs_d;
    W.max_paths = E->paths_alloc;
    W.lane_stride = E->paths_alloc;
    if (cudaMallocHost(&E->jobs_h, sizeof(DevJob) * E->max_jobs) != cudaSuccess ||
        cudaMallocHost(&E->segs_h, sizeof(DevSegment) * kMaxSegments * 2 * L) != cudaSuccess ||
        cudaMallocHost(&E->hdr_h, sizeof(int) * 4 * 2 * L) != cudaSuccess ||
        cudaMallocHost(&E->ctr_h, sizeof(WaveCounters) * 2 * L) != cudaSuccess)
        return bail(fail(LUX_ERR_OOM, "pinned host allocation failed"));
    for (int s = E->max_jobs - 1; s >= 0; --s) E->free_slots.push_back(s);
    cudaEventCreate(&E->ev[0]);
    cudaEventCreate(&E->ev[1]);
    for (auto& pe : E->step_ev)
        for (cudaEvent_t& e : pe)
            if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(LUX_ERR_CUDA, "event creation failed"));
    if (cudaStreamCreateWithFlags(&E->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(LUX_ERR_CUDA, "stream creation failed"));
    // occupancy queries happen here, never inside a stream capture
    for (int m = 0; m < 3; ++m) trace_grid_blocks(m, E->S.single_level != 0);
    shade_grid_blocks();
    const int full = trace_grid_blocks(0, E->S.single_level != 0);
    if (c.max_paths > 0 || c.trace_blocks > 0) {
        E->max_paths = E->paths_alloc;
        E->trace_blocks = c.trace_blocks > 0 ? c.trace_blocks : full;
    } else {
        // candidates: wave sizes, at the full traversal grid (one trial wave each: a grid of 4
        // blocks per SM won trials on the job mix of its trial wave and then ran the mix 16 %
        // slower; every measurement of the kernel itself favours the full grid)
        for (int sz : kTuneSizes) E->tune_cands.push_back({sz, full});
        E->max_paths = E->tune_cands[0].first;
        E->trace_blocks = E->tune_cands[0].second;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(LUX_ERR_CUDA, cudaGetErrorString(cudaGetLastError())));
    *out = E;
    return LUX_OK;
}

int lux_engine_submit(lux_engine* E, const lux_job_desc* job, int* job_id) {
    if (!E || !job || !job_id) return fail(LUX_ERR_INVALID, "NULL argument");
    *job_id = -1;
    if (job->scene < 0 || job->scene >= int(E->scene_root.size())) return fail(LUX_ERR_INVALID, "scene index out of range");
    if (job->spp <= 0) return fail(LUX_ERR_INVALID, "spp must be positive");
    if (job->camera.width <= 0 || job->camera.height <= 0) return fail(LUX_ERR_INVALID, "camera resolution must be positive");
    if (job->first_iter < 0) return fail(LUX_ERR_INVALID, "first_iter must be >= 0");
    const int depth = job->trace_depth > 0 ? job->trace_depth : E->scene_depth[job->scene];
    if (depth <= 0 || depth > kMaxDepth) return fail(LUX_ERR_INVALID, "trace depth must be in 1..64");
    const int64_t npix = int64_t(job->camera.width) * job->camera.height;
    if (npix > E->paths_alloc) return fail(LUX_ERR_INVALID, "one sample of the job exceeds the wave size");
    EngineJob j;
    j.desc = *job;
    j.depth = depth;
    j.npix = int(npix);
    j.bytes = size_t(npix) * 3 * sizeof(float) * (E->opt.precision == LUX_PRECISION_COMPENSATED ? 2 : 1);
    if (E->cfg.hbm_budget_bytes > 0 && E->scene_bytes + E->wave_bytes + int64_t(j.bytes) > E->cfg.hbm_budget_bytes)
        return fail(LUX_ERR_OOM, "the job does not fit in the HBM budget even alone");
    j.t_submit = now_ms(E->t0);
    E->jobs.push_back(j);
    *job_id = int(E->jobs.size()) - 1;
    E->queued.push_back(*job_id);
    return LUX_OK;
}

}  // extern "C"

namespace {

// The wave's view of the engine's arrays in lane `lane`: its own segment table and header.
DevWave lane_view(const lux_engine* E, int lane) {
    DevWave W = E->W;
    W.segs = E->segs_d + size_t(lane) * kMaxSegments;
    W.wave_hdr = E->W.wave_hdr + size_t(lane) * 4;
    return W;
}

// Plan the next wave into lane `lane`'s host tables and copy them to the device: returns its
// segments (0: nothing to render) with its size, depth, paths and (job id, samples) parts.
int plan_next(lux_engine* E, int lane, int& wave_paths, int& depth, int& path0,
              std::vector<std::pair<int, int>>& part) {
    std::vector<int> order;
    const int nj = order_jobs(E, order);
    // The wave is filled from the scene of the job first in line, then from the other jobs in
    // their order: paths of one scene share that scene's BVH in L2, where a wave over many
    // resident scenes makes traversal fetch several at once.
    if (nj > 1) {
        const int head_scene = E->jobs[order[0]].desc.scene;
        std::stable_partition(order.begin(), order.end(),
                              [&](int id) { return E->jobs[id].desc.scene == head_scene; });
    }
    std::vector<int> np(nj), rem(nj), take(nj);
    for (int i = 0; i < nj; ++i) {
        const EngineJob& j = E->jobs[order[i]];
        np[i] = j.npix;
        rem[i] = j.desc.spp - j.spp_sched;
    }
    wave_paths = E->max_paths;
    int nsegs = lux_plan_wave(np.data(), rem.data(), nj, wave_paths, kMaxSegments, take.data());
    if (nsegs <= 0 && nj > 0) {
        // one sample of every waiting job exceeds the wave size in use (a small autotuning
        // candidate): this wave takes the full allocated size
        wave_paths = E->paths_alloc;
        nsegs = lux_plan_wave(np.data(), rem.data(), nj, wave_paths, kMaxSegments, take.data());
    }
    if (nsegs <= 0) return 0;
    const size_t buf = size_t(E->step_par) * E->lanes + lane;
    DevSegment* segs_h = E->segs_h + buf * kMaxSegments;
    int* hdr_h = E->hdr_h + buf * 4;
    path0 = 0;
    depth = 0;
    part.clear();
    int pix0 = 0, k = 0;
    for (int i = 0; i < nj; ++i) {
        if (!take[i]) continue;
        EngineJob& j = E->jobs[order[i]];
        segs_h[k] = DevSegment{j.slot, j.spp_sched, take[i], path0, pix0};
        path0 += take[i] * j.npix;
        pix0 += j.npix;
        depth = std::max(depth, j.depth);
        j.spp_sched += take[i];
        part.push_back({order[i], take[i]});
        ++k;
    }
    hdr_h[0] = k;
    hdr_h[1] = path0;
    hdr_h[2] = pix0;
    cudaStream_t st = E->stream;
    LUX_CUDA(cudaMemcpyAsync(E->segs_d + size_t(lane) * kMaxSegments, segs_h, sizeof(DevSegment) * k,
                             cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaMemcpyAsync(E->W.wave_hdr + size_t(lane) * 4, hdr_h, sizeof(int) * 4, cudaMemcpyHostToDevice, st));
    return k;
}

// Samples a wave adds to its jobs, counted when its accumulation is enqueued: an image read
// back in stream order (which waits for everything enqueued) then holds spp_done samples.
void count_wave(lux_engine* E, const std::vector<std::pair<int, int>>& part) {
    for (auto& pr : part) {
        EngineJob& j = E->jobs[pr.first];
        j.spp_done += pr.second;
        j.waves += 1;
    }
}

// Bookkeeping of a wave whose accumulation has completed on the device (its counters copied to
// c): rays, samples, and the jobs it completed (every sample's accumulation completed).
int finish_wave(lux_engine* E, const WaveCounters& c, int depth, int paths, const std::vector<std::pair<int, int>>& part) {
    if (c.error) return fail(LUX_ERR_UNSUPPORTED, "traversal stack overflow");
    const double t = now_ms(E->t0);
    double rays = 0;
    for (int b = 0; b < depth; ++b) rays += double(c.count[b]) + double(c.shadow[b]);
    E->stats.waves += 1;
    E->stats.samples += double(paths);
    E->stats.rays += rays;
    int done = 0;
    for (auto& pr : part) {
        EngineJob& j = E->jobs[pr.first];
        j.spp_final += pr.second;
        if (j.state == LUX_JOB_ACTIVE && j.spp_final == j.desc.spp) {
            j.state = LUX_JOB_DONE;
            j.t_done = t;
            ++done;
        }
    }
    if (done) {
        std::vector<int> keep;
        for (int id : E->active)
            if (E->jobs[id].state == LUX_JOB_ACTIVE) keep.push_back(id);
        E->active.swap(keep);
    }
    return done;
}

// One wave start to end, as a CUDA graph (the autotuning waves).
int step_one_wave(lux_engine* E, bool tuning, int* done_jobs, int* idle) {
    int wave_paths = 0, depth = 0, path0 = 0;
    std::vector<std::pair<int, int>> part;
    const int k = plan_next(E, 0, wave_paths, depth, path0, part);
    if (k < 0) return k;
    if (k == 0) {
        if (idle) *idle = 1;
        return LUX_OK;
    }
    cudaStream_t st = E->stream;
    auto key = std::make_tuple(depth, wave_paths, E->trace_blocks);
    auto it = E->graphs.find(key);
    if (it == E->graphs.end()) {
        cudaGraph_t g;
        LUX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_wave(E, depth, wave_paths, E->trace_blocks);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (rc) return rc;
        if (ce != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        cudaGraphExec_t ge;
        cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return fail(LUX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        it = E->graphs.emplace(key, ge).first;
    }
    LUX_CUDA(cudaEventRecord(E->ev[0], st));
    LUX_CUDA(cudaGraphLaunch(it->second, st));
    LUX_CUDA(cudaEventRecord(E->ev[1], st));
    LUX_CUDA(cudaMemcpyAsync(E->ctr_h, E->W.ctr, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, E->ev[0], E->ev[1]);
    E->stats.ms_device += ms;
    if (tuning) {
        // cost per traced ray (radiance and shadow): the tuning waves hold different jobs, whose
        // depths and survival differ, so a cost per path compares the jobs more than the settings
        double rays = 0;
        for (int b = 0; b < depth; ++b) rays += double(E->ctr_h->count[b]) + double(E->ctr_h->shadow[b]);
        E->tune_cost.push_back(double(ms) / std::max(1.0, rays));
        if (++E->tune_next == E->tune_cands.size()) {
            size_t best = size_t(std::min_element(E->tune_cost.begin(), E->tune_cost.end()) - E->tune_cost.begin());
            E->max_paths = E->tune_cands[best].first;
            E->trace_blocks = E->tune_cands[best].second;
        }
    }
    count_wave(E, part);
    const int done = finish_wave(E, *E->ctr_h, depth, path0, part);
    if (done < 0) return done;
    if (done_jobs) *done_jobs = done;
    return LUX_OK;
}

// Bookkeeping of the pipelined step enqueued last: waits for its end event, then counts its
// device time and finishes the waves it accumulated (their counters in its parity's buffers).
int finish_pending(lux_engine* E, int* done) {
    *done = 0;
    if (!E->pend_valid) return LUX_OK;
    E->pend_valid = false;
    const int p = E->pend_par;
    LUX_CUDA(cudaEventSynchronize(E->step_ev[p][1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, E->step_ev[p][0], E->step_ev[p][1]);
    E->stats.ms_device += ms;
    std::vector<Flight> fin = std::move(E->pend_fin);
    E->pend_fin.clear();
    for (const Flight& f : fin) {
        const int d = finish_wave(E, E->ctr_h[size_t(p) * E->lanes + f.lane], f.depth, f.paths, f.part);
        if (d < 0) return d;
        *done += d;
    }
    return LUX_OK;
}

// Waves in flight (after autotuning): start a wave in a free lane when there is work, advance
// every wave in flight by kStepBounces bounces in launches that cover all of them, then
// accumulate the waves that are through, in start order, so each job's samples add up in
// sample order as in step_one_wave. A wave that ends before an older one keeps its lane until
// the older one is done.
int step_pipelined(lux_engine* E, int* done_jobs, int* idle) {
    cudaStream_t st = E->stream;
    const int nee = E->dopt.env ? 2 : (E->dopt.dl ? 1 : 0);
    if (int(E->flight.size()) < E->lanes) {
        int lane = 0;
        for (; lane < E->lanes; ++lane) {
            bool used = false;
            for (const Flight& f : E->flight) used = used || f.lane == lane;
            if (!used) break;
        }
        Flight f;
        int wave_paths = 0;
        const int k = plan_next(E, lane, wave_paths, f.depth, f.paths, f.part);
        if (k < 0) return k;
        if (k > 0) {
            f.lane = lane;
            LUX_CUDA(cudaMemsetAsync(E->W.ctr + lane, 0, sizeof(WaveCounters), st));
            LUX_CUDA(launch_camera_jobs(lane_view(E, lane), E->dopt, wave_paths, lane, st));
            E->flight.push_back(std::move(f));
        }
    }
    if (E->flight.empty()) {
        // nothing in flight: the step enqueued last, if any, is the last to finish
        int done = 0;
        if (int rc = finish_pending(E, &done)) return rc;
        if (done_jobs) *done_jobs = done;
        if (idle && done == 0) *idle = 1;
        return LUX_OK;
    }
    const int par = E->step_par;
    E->step_par ^= 1;
    LUX_CUDA(cudaEventRecord(E->step_ev[par][0], st));
    for (int s = 0; s < kStepBounces; ++s) {
        Segs G{};
        for (const Flight& f : E->flight) {
            if (f.bounce >= f.depth) continue;
            G.lane[G.n] = f.lane;
            G.bounce[G.n] = f.bounce;
            G.compact[G.n] = 1;  // each path stops at its own job's depth
            ++G.n;
        }
        if (G.n == 0) break;
        LUX_CUDA(launch_trace_segs(E->S, E->W, G, 0, nee, st, E->trace_blocks));
        if (nee) LUX_CUDA(launch_trace_segs(E->S, E->W, G, nee == 2 ? 2 : 1, 0, st, E->trace_blocks));
        LUX_CUDA(launch_shade_segs(E->S, E->W, E->dopt, G, st));
        for (Flight& f : E->flight)
            if (f.bounce < f.depth) ++f.bounce;
    }
    std::vector<Flight> fin;
    while (!E->flight.empty() && E->flight.front().bounce >= E->flight.front().depth) {
        Flight f = std::move(E->flight.front());
        E->flight.pop_front();
        LUX_CUDA(launch_accumulate_jobs(lane_view(E, f.lane), E->opt.precision == LUX_PRECISION_COMPENSATED, f.lane, st));
        LUX_CUDA(cudaMemcpyAsync(E->ctr_h + size_t(par) * E->lanes + f.lane, E->W.ctr + f.lane, sizeof(WaveCounters),
                                 cudaMemcpyDeviceToHost, st));
        count_wave(E, f.part);
        fin.push_back(std::move(f));
    }
    LUX_CUDA(cudaEventRecord(E->step_ev[par][1], st));
    // this step runs on the device while the one before it is finished here
    int done = 0;
    if (int rc = finish_pending(E, &done)) return rc;
    E->pend_valid = true;
    E->pend_par = par;
    E->pend_fin = std::move(fin);
    if (done_jobs) *done_jobs = done;
    return LUX_OK;
}

}  // namespace

extern "C" {

int lux_engine_step(lux_engine* E, int* done_jobs, int* idle) {
    if (!E) return fail(LUX_ERR_INVALID, "engine is NULL");
    if (done_jobs) *done_jobs = 0;
    if (idle) *idle = 0;
    LUX_CUDA(cudaSetDevice(E->device));
    if (int rc = admit(E)) return rc;
    // autotuning: the first waves try each candidate once, one wave at a time; then the
    // cheapest per path stays and waves run in flight together
    const bool tuning = E->tune_next < E->tune_cands.size();
    if (tuning) {
        E->max_paths = E->tune_cands[E->tune_next].first;
        E->trace_blocks = E->tune_cands[E->tune_next].second;
        return step_one_wave(E, true, done_jobs, idle);
    }
    return step_pipelined(E, done_jobs, idle);
}

int lux_engine_run(lux_engine* E) {
    if (!E) return fail(LUX_ERR_INVALID, "engine is NULL");
    while (!E->queued.empty() || !E->active.empty()) {
        int idle = 0;
        if (int rc = lux_engine_step(E, nullptr, &idle)) return rc;
        if (idle && E->active.empty() && !E->queued.empty())
            return fail(LUX_ERR_OOM, "queued jobs cannot be admitted within the HBM budget");
        if (idle && !E->active.empty()) return fail(LUX_ERR_STATE, "active jobs but nothing to render");
    }
    return LUX_OK;
}

int lux_engine_job_status(lux_engine* E, int id, lux_job_status* out) {
    if (!E || !out) return fail(LUX_ERR_INVALID, "NULL argument");
    if (id < 0 || id >= int(E->jobs.size())) return fail(LUX_ERR_INVALID, "unknown job");
    const EngineJob& j = E->jobs[id];
    out->state = j.state;
    out->spp_done = j.spp_done;
    out->spp = j.desc.spp;
    out->waves = j.waves;
    out->t_submit_ms = j.t_submit;
    out->t_admit_ms = j.t_admit;
    out->t_done_ms = j.t_done;
    return LUX_OK;
}

int lux_engine_copy_image(lux_engine* E, int id, float* rgb) {
    if (!E || !rgb) return fail(LUX_ERR_INVALID, "NULL argument");
    if (id < 0 || id >= int(E->jobs.size())) return fail(LUX_ERR_INVALID, "unknown job");
    const EngineJob& j = E->jobs[id];
    if (j.state == LUX_JOB_RELEASED) return fail(LUX_ERR_STATE, "job released");
    const size_t bytes = size_t(j.npix) * 3 * sizeof(float);
    if (j.state == LUX_JOB_QUEUED) {
        std::memset(rgb, 0, bytes);
        return LUX_OK;
    }
    LUX_CUDA(cudaSetDevice(E->device));
    if (j.state == LUX_JOB_DONE && E->copy_stream) {
        // its last accumulation is complete (the step's end event was waited for): read it back
        // on the side stream, without waiting for the step now running
        LUX_CUDA(cudaMemcpyAsync(rgb, j.image, bytes, cudaMemcpyDeviceToHost, E->copy_stream));
        LUX_CUDA(cudaStreamSynchronize(E->copy_stream));
        return LUX_OK;
    }
    LUX_CUDA(cudaMemcpyAsync(rgb, j.image, bytes, cudaMemcpyDeviceToHost, E->stream));
    LUX_CUDA(cudaStreamSynchronize(E->stream));
    return LUX_OK;
}

int lux_engine_release(lux_engine* E, int id) {
    if (!E) return fail(LUX_ERR_INVALID, "engine is NULL");
    if (id < 0 || id >= int(E->jobs.size())) return fail(LUX_ERR_INVALID, "unknown job");
    EngineJob& j = E->jobs[id];
    if (j.state == LUX_JOB_ACTIVE) return fail(LUX_ERR_STATE, "job still rendering");
    if (j.state == LUX_JOB_RELEASED) return LUX_OK;
    if (j.state == LUX_JOB_QUEUED) E->queued.erase(std::find(E->queued.begin(), E->queued.end(), id));
    LUX_CUDA(cudaSetDevice(E->device));
    free_job_memory(E, j);
    j.state = LUX_JOB_RELEASED;
    return LUX_OK;
}

int lux_engine_get_stats(lux_engine* E, lux_engine_stats* out) {
    if (!E || !out) return fail(LUX_ERR_INVALID, "NULL argument");
    *out = E->stats;
    out->device_bytes = E->device_bytes();
    out->scene_bytes = E->scene_bytes;
    out->max_paths = E->max_paths;
    out->trace_blocks = E->trace_blocks;
    out->jobs_queued = int(E->queued.size());
    out->jobs_active = int(E->active.size());
    int done = 0;
    for (const EngineJob& j : E->jobs) done += j.state == LUX_JOB_DONE;
    out->jobs_done = done;
    return LUX_OK;
}

double lux_engine_clock_ms(lux_engine* E) { return E ? now_ms(E->t0) : 0.0; }

int lux_engine_free(lux_engine* E) {
    if (!E) return LUX_OK;
    cudaSetDevice(E->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    for (EngineJob& j : E->jobs) free_job_memory(E, j);
    if (E->stream) cudaStreamSynchronize(E->stream);
    for (auto& g : E->graphs) cudaGraphExecDestroy(g.second);
    for (DevTex& t : E->texs) destroy_texture(t);
    for (DevTex& t : E->envs) destroy_texture(t);
    for (void* p : E->allocs) cudaFree(p);
    if (E->jobs_h) cudaFreeHost(E->jobs_h);
    if (E->segs_h) cudaFreeHost(E->segs_h);
    if (E->hdr_h) cudaFreeHost(E->hdr_h);
    if (E->ctr_h) cudaFreeHost(E->ctr_h);
    for (cudaEvent_t e : E->ev)
        if (e) cudaEventDestroy(e);
    for (auto& pe : E->step_ev)
        for (cudaEvent_t e : pe)
            if (e) cudaEventDestroy(e);
    if (E->copy_stream) {
        cudaStreamSynchronize(E->copy_stream);
        cudaStreamDestroy(E->copy_stream);
    }
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
    return LUX_OK;
}

}  // extern "C"
