// launch.h -- host-callable launchers of the kernels (defined in trace.cu, shade.cu, sort.cu).
#pragma once

#include <cuda_runtime.h>
#include "device_scene.h"

namespace lux {

constexpr int kTraceBlock = 128;
constexpr int kShadeBlock = 128;

// persistent traversal grid of `mode` for the two-level or the single-level layout
int trace_grid_blocks(int mode, bool single = false);
int shade_grid_blocks();

// persistent trace of bounce `bounce`: mode 0 radiance (queues shadow rays when nee != 0:
// 1 DL, 2 env), 1 DL shadow rays, 2 env occlusion rays
// grid > 0 overrides the persistent grid (blocks), for the job engine's autotuner
cudaError_t launch_trace(const DevScene& S, const DevWave& W, int bounce, int mode, int nee, cudaStream_t st,
                         int grid = 0);
// the same over several (lane, bounce) segments of waves in flight, in one launch
cudaError_t launch_trace_segs(const DevScene& S, const DevWave& W, const Segs& G, int mode, int nee, cudaStream_t st,
                              int grid = 0);
// trace caller rays (device buffers), n * 8 floats -> n * 5 words; fetch is a zeroed int
cudaError_t launch_trace_ext(const DevScene& S, const DevWave& W, const float* rays, uint32_t* hits, int n, int mode,
                             int iter, int* fetch, cudaStream_t st);

// the fixed scratch of lux_trace_rays_static on `device` (trace_static.cu), which must be the
// current device on the first call for it: cursor, then LUX_TRACE_STATIC_MAX_RAYS rays and hits
struct TraceScratch {
    int* cursor;
    float* rays;
    uint32_t* hits;
};
cudaError_t trace_static_scratch(int device, TraceScratch& out);
size_t trace_static_scratch_bytes();

// camera rays for paths [0, n) of a wave in lane `lane` (+ NEE sample of bounce 0), queue 0 =
// identity; wave_iter: the wave's first iteration and sample count (device)
cudaError_t launch_camera(const DevScene& S, const DevWave& W, const DevOptions& O, const DevCamera& cam, int n,
                          int lane, const int* wave_iter, cudaStream_t st);
// shade bounce `bounce` (depth = bounce + 1 after the increment of src/pathtrace.cu:264)
cudaError_t launch_shade(const DevScene& S, const DevWave& W, const DevOptions& O, int bounce, int compact,
                         cudaStream_t st);
// the same over several (lane, bounce) segments of waves in flight, in one launch
cudaError_t launch_shade_segs(const DevScene& S, const DevWave& W, const DevOptions& O, const Segs& G,
                              cudaStream_t st);
// job engine: camera rays of the wave's segments (W.segs, counts read from W.wave_hdr) into lane
// `lane`, and the per-job accumulation of that lane's segments in sample order
cudaError_t launch_camera_jobs(const DevWave& W, const DevOptions& O, int max_paths, int lane, cudaStream_t st);
cudaError_t launch_accumulate_jobs(const DevWave& W, int compensated, int lane, cudaStream_t st);
// image[p] (+comp) += radiance of every sample of the wave in lane `lane`, in sample order
cudaError_t launch_accumulate(const DevWave& W, int lane, float* image, float* comp, int nsamples, int compensated,
                              cudaStream_t st);
cudaError_t launch_tonemap(const float* image, uint8_t* rgba, int npix, float iter, int color_mode, cudaStream_t st);

// n texel channels at src (device) of format fmt (LUX_TEX_RGBA8/16/32F) to float (c / 255,
// c / 65535) or, with to_half, to binary16 at dst (device); texconv.cu
cudaError_t launch_convert_texels(const void* src, int fmt, int to_half, void* dst, size_t n, cudaStream_t st);

// Morton keys of the bounce's queue and a stable LSD radix sort of the queue by key
cudaError_t launch_morton_sort(const DevScene& S, DevWave& W, int bounce, void* temp, size_t temp_bytes,
                               cudaStream_t st);
size_t morton_sort_temp_bytes(int max_paths);
cudaError_t launch_morton_ext(const DevScene& S, const float* rays, uint32_t* keys, int n, cudaStream_t st);

// kernel-level parity entry points (device buffers)
cudaError_t launch_shade_ext(const DevScene& S, const DevOptions& O, float* paths, const uint32_t* hits, int n,
                             int iter, int depth, int compact, int* survivors, int* n_out, cudaStream_t st);
cudaError_t launch_light_ext(const DevScene& S, const DevOptions& O, int iter, int depth, const int* pixels, int n,
                             float* out, cudaStream_t st);
cudaError_t launch_rng_ext(int iter, int index, int depth, int n, float* out, cudaStream_t st);
cudaError_t launch_tex_ext(unsigned long long tex, const float* uv, int n, float* out, cudaStream_t st);

}  // namespace lux
