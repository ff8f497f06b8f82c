"""ctypes mirror of include/luxion.h (the C-ABI of the render path).

The structures below must match the C declarations field for field; the CPU tests check
their sizes and offsets against a C compiler's view of the header.
"""
from __future__ import annotations

import ctypes as C

c_float_p = C.POINTER(C.c_float)
c_u32_p = C.POINTER(C.c_uint32)
c_int_p = C.POINTER(C.c_int)

LUX_OK = 0
STATUS_NAMES = {
    0: "LUX_OK",
    -1: "LUX_ERR_INVALID",
    -2: "LUX_ERR_CUDA",
    -3: "LUX_ERR_NO_DEVICE",
    -4: "LUX_ERR_OOM",
    -5: "LUX_ERR_UNSUPPORTED",
    -6: "LUX_ERR_TIMEOUT",
    -7: "LUX_ERR_STATE",
}

TEX_RGBA8, TEX_RGBA16, TEX_RGBA32F, TEX_RGBA16F = 0, 1, 2, 3
ALPHA_OPAQUE, ALPHA_MASK, ALPHA_BLEND = 0, 1, 2
TONEMAP_REINHARD, TONEMAP_AGX, TONEMAP_ACES = 0, 1, 2
PRECISION_PLAIN, PRECISION_COMPENSATED = 0, 1
TEXSTORE_FLOAT, TEXSTORE_UNORM8, TEXSTORE_HALF = 0, 1, 2
(MATDEBUG_OFF, MATDEBUG_ALBEDO, MATDEBUG_NORMAL, MATDEBUG_NORMAL_MAP, MATDEBUG_ROUGHNESS, MATDEBUG_METALLIC,
 MATDEBUG_ALPHA) = range(7)
TRACE_STATIC_MAX_RAYS = 65536  # LUX_TRACE_STATIC_MAX_RAYS

# path-state layout (LUX_PS_*)
PS_ORIGIN, PS_DIR, PS_COLOR, PS_THROUGHPUT = 0, 3, 6, 9
PS_DL, PS_ENV, PS_PIXEL, PS_KILL, PS_SPECULAR, PS_LAST_PDF, PS_FLOATS = 12, 15, 18, 19, 20, 21, 24


class TextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("format", C.c_int32),
                ("_pad", C.c_int32), ("data", C.c_void_p)]


class TexTransform(C.Structure):
    _fields_ = [("offset", C.c_float * 2), ("scale", C.c_float * 2), ("rotation", C.c_float)]


class MaterialDesc(C.Structure):
    _fields_ = [("color", C.c_float * 3), ("albedo_tex", C.c_int32), ("alpha", C.c_float),
                ("alpha_mode", C.c_int32), ("alpha_cutoff", C.c_float),
                ("emission_strength", C.c_float), ("emission_color", C.c_float * 3),
                ("emissive_tex", C.c_int32), ("roughness", C.c_float), ("metallic", C.c_float),
                ("normal_tex", C.c_int32), ("metallic_roughness_tex", C.c_int32),
                ("transmission", C.c_float), ("ior", C.c_float),
                ("albedo_tt", TexTransform), ("emissive_tt", TexTransform),
                ("normal_tt", TexTransform), ("metallic_roughness_tt", TexTransform)]


class MeshDesc(C.Structure):
    _fields_ = [("num_verts", C.c_int32), ("num_tris", C.c_int32), ("positions", c_float_p),
                ("normals", c_float_p), ("uvs", c_float_p), ("indices", c_u32_p)]


class InstanceDesc(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("material", C.c_int32), ("has_inverse", C.c_int32),
                ("_pad", C.c_int32), ("transform", C.c_float * 16), ("inverse", C.c_float * 16),
                ("inv_transpose", C.c_float * 16)]


class CameraDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("position", C.c_float * 3),
                ("look_at", C.c_float * 3), ("view", C.c_float * 3), ("up", C.c_float * 3),
                ("right", C.c_float * 3), ("fov", C.c_float * 2), ("pixel_length", C.c_float * 2)]


class SceneDesc(C.Structure):
    _fields_ = [("num_meshes", C.c_int32), ("num_instances", C.c_int32),
                ("num_materials", C.c_int32), ("num_textures", C.c_int32),
                ("meshes", C.POINTER(MeshDesc)), ("instances", C.POINTER(InstanceDesc)),
                ("materials", C.POINTER(MaterialDesc)), ("textures", C.POINTER(TextureDesc)),
                ("camera", CameraDesc), ("trace_depth", C.c_int32),
                ("env_width", C.c_int32), ("env_height", C.c_int32), ("env_format", C.c_int32),
                ("env_data", C.c_void_p)]


BVH_AUTO, BVH_TWO_LEVEL, BVH_SINGLE_LEVEL = 0, 1, 2


class Options(C.Structure):
    _fields_ = [("direct_light_sampling", C.c_int32), ("env_importance_sampling", C.c_int32),
                ("color_mode", C.c_int32), ("envmap_intensity", C.c_float),
                ("trace_depth", C.c_int32), ("ray_sorting", C.c_int32),
                ("precision", C.c_int32), ("spp_per_wave", C.c_int32),
                ("use_graph", C.c_int32), ("texture_storage", C.c_int32), ("device", C.c_int32),
                ("stream", C.c_void_p), ("material_debug_mode", C.c_int32), ("debug_bvh", C.c_int32),
                ("bvh_layout", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rays_radiance", "rays_shadow", "path_bounces", "samples", "ms_total", "ms_trace",
        "ms_shade", "ms_camera", "ms_accum", "ms_sort", "launches_trace", "launches_shade",
        "launches_camera", "launches_accum", "launches_sort", "kernel_launches")]


class SceneStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("ms_total", "ms_geometry", "ms_upload", "ms_blas", "ms_tlas", "ms_tables",
                                          "ms_textures")] + \
        [("device_bytes", C.c_int64), ("blas_nodes", C.c_int64), ("tlas_nodes", C.c_int64)]


class RandomSceneParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("num_instances", C.c_int32), ("total_tris", C.c_int32),
                ("min_tris", C.c_int32), ("max_tris", C.c_int32), ("num_emissive", C.c_int32),
                ("num_textures", C.c_int32), ("texture_size", C.c_int32),
                ("env_width", C.c_int32), ("env_height", C.c_int32), ("width", C.c_int32),
                ("height", C.c_int32), ("trace_depth", C.c_int32), ("env_half", C.c_int32),
                ("tex_half", C.c_int32)]


class JobDesc(C.Structure):
    _fields_ = [("scene", C.c_int32), ("spp", C.c_int32), ("trace_depth", C.c_int32),
                ("first_iter", C.c_int32), ("camera", CameraDesc)]


SCHED_FIFO, SCHED_SHORTEST_FIRST = 0, 1
JOB_QUEUED, JOB_ACTIVE, JOB_DONE, JOB_RELEASED = 0, 1, 2, 3


class EngineConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_paths", C.c_int32), ("max_jobs", C.c_int32),
                ("schedule", C.c_int32), ("trace_blocks", C.c_int32)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("spp_done", C.c_int32), ("spp", C.c_int32), ("waves", C.c_int32),
                ("t_submit_ms", C.c_double), ("t_admit_ms", C.c_double), ("t_done_ms", C.c_double)]


class EngineStats(C.Structure):
    _fields_ = [("waves", C.c_int64), ("samples", C.c_double), ("rays", C.c_double), ("ms_device", C.c_double),
                ("device_bytes", C.c_int64), ("scene_bytes", C.c_int64), ("max_paths", C.c_int32),
                ("trace_blocks", C.c_int32), ("jobs_queued", C.c_int32), ("jobs_active", C.c_int32),
                ("jobs_done", C.c_int32)]


def default_options(**kw) -> Options:
    """PathTracerOptions defaults (include/pathtrace/pathtracer_options.h:3-11)."""
    o = Options()
    o.direct_light_sampling = 0
    o.env_importance_sampling = 0
    o.color_mode = TONEMAP_ACES
    o.envmap_intensity = 1.0
    o.trace_depth = 0
    o.ray_sorting = 0
    o.precision = PRECISION_PLAIN
    o.spp_per_wave = 0
    o.use_graph = 1
    o.texture_storage = TEXSTORE_FLOAT
    o.bvh_layout = BVH_AUTO
    o.device = 0
    o.stream = None
    o.material_debug_mode = MATDEBUG_OFF
    o.debug_bvh = 0
    for k, v in kw.items():
        setattr(o, k, v)
    return o
