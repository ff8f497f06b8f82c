/*
 * lux_oracle.h -- C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a scalar CPU restatement of the seabiscuit-iv/luxion render path. Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load it, always as
 * the checker of the CUDA path, never as a substitute for it. It is pinned against the
 * reference's own hot-path sources compiled for the host (oracle/ref/, built into
 * oracle/_ref/) through golden vectors under tests/golden/.
 *
 * Layouts (rays, hits, path states) are the ones documented in include/luxion.h.
 */
#ifndef LUX_ORACLE_H
#define LUX_ORACLE_H

#include <stdint.h>
#include "../include/luxion.h"

#ifdef __cplusplus
extern "C" {
#endif

uint32_t orc_utilhash(uint32_t a);
void orc_rng_stream(int iter, int index, int depth, int n, float* out);
int orc_select_from_cdf(const float* cdf, int size, float xi);

/* Batch evaluation of the uber-shader pieces for known-answer tests.
 * in: n records of 16 floats: wo(3) n(3) wi(3) albedo(3) roughness metallic ior transmission
 * out: n records of 16 floats: BRDF(3) BTDF(3) shade(3) PDF D G F_dielectric(cos=n.wo)
 *      F_schlick_r FresnelMix_r pad */
void orc_eval_bsdf(const float* in, int n, float* out);
/* Lobe sampling: in n records of 16 floats as above (wi ignored) plus seeds (iter, index,
 * depth) in seeds[3n]; out n*4 floats: sample_dir xyz, uniforms consumed. */
void orc_sample_bsdf(const float* in, const int* seeds, int n, float* out);
/* cosine hemisphere: normals n*3, seeds 3n -> out n*3 */
void orc_hemisphere(const float* normals, const int* seeds, int n, float* out);

typedef struct orc_scene orc_scene;
/* cdf_f64: 1 builds the light CDFs in FP64 (precision form), 0 in FP32 like the reference.
 * tex_storage: LUX_TEXSTORE_* of the CUDA path being checked. */
orc_scene* orc_scene_create(const lux_scene_desc* desc, int cdf_f64, int tex_storage);
void orc_scene_destroy(orc_scene* s);
int orc_get_cdfs(orc_scene* s, float* emissive_prefix, float* tri_prefix, float* marginal,
                 float* conditional, float* total_area);
/* sizes: [num_emissive, tri_prefix_len, env_h, env_w] */
void orc_cdf_sizes(orc_scene* s, int* sizes);

/* mode 0 radiance, 1 DL shadow (tmax), 2 env occlusion; brute: 1 tests every triangle */
void orc_trace(orc_scene* s, const float* rays, int n, int mode, int iter, uint32_t* hits,
               int brute);
void orc_morton(orc_scene* s, const float* rays, int n, uint32_t* keys);
void orc_light_samples(orc_scene* s, const lux_options* opt, int iter, int depth,
                       const int* pixels, int n, float* out);
void orc_camera_rays(orc_scene* s, int iter, const int* pixels, int n, float* paths);
void orc_shade_step(orc_scene* s, const lux_options* opt, int iter, int depth, int compact,
                    float* paths, int n, const uint32_t* hits, int* survivors, int* n_out);
/* Texture fetch emulating CUDA bilinear filtering (tex -1 = environment map). */
void orc_sample_texture(orc_scene* s, int tex, const float* uv, int n, float* out);

/* Full render of iterations first_iter..first_iter+n_iter-1 over the pixel crop
 * [x0,x0+w) x [y0,y0+h) of the full-resolution camera. image: w*h*3 floats receiving the
 * accumulation SUM in iteration order. f64: 1 runs the FP64 integrator. threads: OpenMP
 * threads (0 = all). stats[4]: radiance rays, shadow rays, path-bounces, samples. */
int orc_render(orc_scene* s, const lux_options* opt, int first_iter, int n_iter, int x0,
               int y0, int w, int h, int f64, int threads, float* image, double* stats);
void orc_tonemap(const float* image_sum, int n_pix, float iter, int color_mode, uint8_t* rgba);

#ifdef __cplusplus
}
#endif
#endif
