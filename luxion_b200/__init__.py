"""luxion_b200 -- B200-native wavefront path tracer behind the luxion render-path interface.

The product is the C-ABI library ``_lib/libluxion.so`` (include/luxion.h). This module is a
thin ctypes mirror of the reference's host interface for the render path:

    pathtraceInit(scene)      include/pathtrace/pathtrace_buffers.h:5
    pathtrace(pbo, frame, it) include/pathtrace.h:13
    pathtraceFree()           include/pathtrace/pathtrace_buffers.h:6
    copyImageToHost()         include/pathtrace/pathtrace_buffers.h:7
    PathTracerOptions         include/pathtrace/pathtracer_options.h:3-21

plus an object API (``Renderer``) for callers that want several contexts. Every call goes
through the CUDA library; there is no CPU fallback: when the library is missing or no
sm_100 device is visible the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _ffi
from ._ffi import (CameraDesc, EngineConfig, EngineStats, JobDesc, JobStatus, Options, RandomSceneParams,
                   SceneDesc, Stats, c_float_p, c_int_p, c_u32_p, default_options)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libluxion.so")
_lib: Optional[C.CDLL] = None

# every symbol include/luxion.h declares, with its ctypes signature
_P = C.c_void_p
SIGNATURES = {
    "lux_default_options": (None, [C.POINTER(Options)]),
    "lux_init": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(Options), C.POINTER(_P)]),
    "lux_scene_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(Options), C.POINTER(_P)]),
    "lux_init_on_scene": (C.c_int, [_P, C.POINTER(CameraDesc), C.POINTER(Options), C.POINTER(_P)]),
    "lux_scene_free": (C.c_int, [_P]),
    "lux_scene_device_bytes": (C.c_int64, [_P]),
    "lux_scene_get_stats": (C.c_int, [_P, C.POINTER(_ffi.SceneStats)]),
    "lux_get_scene_stats": (C.c_int, [_P, C.POINTER(_ffi.SceneStats)]),
    "lux_render_iter": (C.c_int, [_P, C.c_int, _P]),
    "lux_render": (C.c_int, [_P, C.c_int, C.c_int]),
    "lux_copy_image": (C.c_int, [_P, c_float_p]),
    "lux_copy_rgba8": (C.c_int, [_P, C.POINTER(C.c_uint8)]),
    "lux_reset": (C.c_int, [_P]),
    "lux_set_camera": (C.c_int, [_P, C.POINTER(CameraDesc)]),
    "lux_free": (C.c_int, [_P]),
    "lux_last_error": (C.c_char_p, []),
    "lux_enable_timing": (C.c_int, [_P, C.c_int]),
    "lux_get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "lux_wave_counts": (C.c_int, [_P, c_int_p, c_int_p, C.c_int]),
    "lux_copy_image_device": (C.c_int, [_P, C.c_void_p]),
    "lux_trace_rays": (C.c_int, [_P, c_float_p, C.c_int, C.c_int, C.c_int, c_u32_p]),
    "lux_trace_rays_static": (C.c_int, [_P, c_float_p, C.c_int, C.c_int, C.c_int, c_u32_p]),
    "lux_device_alloc_count": (C.c_int64, []),
    "lux_morton_keys": (C.c_int, [_P, c_float_p, C.c_int, c_u32_p]),
    "lux_bvh8_build": (C.c_int, [c_float_p, c_int_p, C.c_int, C.c_int, C.c_void_p, C.c_int, c_u32_p, c_u32_p, c_int_p,
                                 c_int_p]),
    "lux_shade_step": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, c_float_p, C.c_int, c_u32_p, c_int_p, c_int_p]),
    "lux_light_samples": (C.c_int, [_P, C.c_int, C.c_int, c_int_p, C.c_int, c_float_p]),
    "lux_get_cdfs": (C.c_int, [_P, c_float_p, c_float_p, c_float_p, c_float_p, c_float_p]),
    "lux_rng_stream": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, c_float_p]),
    "lux_sample_texture": (C.c_int, [_P, C.c_int, c_float_p, C.c_int, c_float_p]),
    "lux_engine_create": (C.c_int, [C.POINTER(C.POINTER(SceneDesc)), C.c_int, C.POINTER(Options),
                                    C.POINTER(EngineConfig), C.POINTER(_P)]),
    "lux_engine_submit": (C.c_int, [_P, C.POINTER(JobDesc), c_int_p]),
    "lux_engine_step": (C.c_int, [_P, c_int_p, c_int_p]),
    "lux_engine_run": (C.c_int, [_P]),
    "lux_engine_job_status": (C.c_int, [_P, C.c_int, C.POINTER(JobStatus)]),
    "lux_engine_copy_image": (C.c_int, [_P, C.c_int, c_float_p]),
    "lux_engine_release": (C.c_int, [_P, C.c_int]),
    "lux_engine_get_stats": (C.c_int, [_P, C.POINTER(EngineStats)]),
    "lux_engine_clock_ms": (C.c_double, [_P]),
    "lux_engine_free": (C.c_int, [_P]),
    "lux_plan_wave": (C.c_int, [c_int_p, c_int_p, C.c_int, C.c_int, C.c_int, c_int_p]),
    "lux_make_camera": (None, [C.c_int, C.c_int, c_float_p, c_float_p, C.c_float, C.POINTER(CameraDesc)]),
    "lux_scene_cornell36": (_P, [C.c_int, C.c_int]),
    "lux_default_random_scene_params": (None, [C.POINTER(RandomSceneParams)]),
    "lux_scene_random": (_P, [C.POINTER(RandomSceneParams)]),
    "lux_scene_furnace": (_P, [C.c_int, C.c_int, C.c_int]),
    "lux_scene_furnace_material": (_P, [C.c_int, C.c_int, C.c_int, C.POINTER(_ffi.MaterialDesc), C.c_int]),
    "lux_default_material": (None, [C.POINTER(_ffi.MaterialDesc)]),
    "lux_scene_get_desc": (C.POINTER(SceneDesc), [_P]),
    "lux_scene_instanced_tris": (C.c_int64, [_P]),
    "lux_scene_destroy": (None, [_P]),
}


class LuxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ffi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load the CUDA library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"luxion CUDA library missing: {LIB_PATH}")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise LuxError(rc, lib().lux_last_error().decode(errors="replace"))


def ptr(a: np.ndarray, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


# ---- procedural scenes (host only) ---------------------------------------------------------
class HostScene:
    """Host-side scene description produced by the library's procedural generators."""

    def __init__(self, handle):
        if not handle:
            raise LuxError(-1, "scene generation failed")
        self._h = handle

    @property
    def desc(self) -> SceneDesc:
        return lib().lux_scene_get_desc(self._h).contents

    @property
    def desc_ptr(self):
        return lib().lux_scene_get_desc(self._h)

    @property
    def instanced_tris(self) -> int:
        return int(lib().lux_scene_instanced_tris(self._h))

    @property
    def width(self) -> int:
        return self.desc.camera.width

    @property
    def height(self) -> int:
        return self.desc.camera.height

    def close(self):
        if self._h:
            lib().lux_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cornell36(width: int = 256, height: int = 256) -> HostScene:
    return HostScene(lib().lux_scene_cornell36(width, height))


def random_scene(**kw) -> HostScene:
    p = RandomSceneParams()
    lib().lux_default_random_scene_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return HostScene(lib().lux_scene_random(C.byref(p)))


def furnace(width: int = 64, height: int = 64, subdiv: int = 16, vertex_normals: bool = True,
            **material) -> HostScene:
    """White furnace: a unit icosphere under a constant environment of 1. Without material
    keywords the sphere is smooth white metal (lux_scene_furnace); keywords (color, roughness,
    metallic, ior, transmission, ...) override the reference glTF default material."""
    if not material and vertex_normals:
        return HostScene(lib().lux_scene_furnace(width, height, subdiv))
    m = _ffi.MaterialDesc()
    lib().lux_default_material(C.byref(m))
    for k, v in material.items():
        if k == "color":
            m.color[:] = [float(x) for x in v]
        else:
            setattr(m, k, v)
    return HostScene(lib().lux_scene_furnace_material(width, height, subdiv, C.byref(m), 1 if vertex_normals else 0))


def bvh8_build(boxes: np.ndarray, tree_begin, on_device: bool):
    """Build the 8-wide BVH over boxes (n x 6: min, max) grouped into trees (lux_bvh8_build).
    Returns (nodes as an n_nodes x 80 uint8 array, leaf order, roots, depths)."""
    boxes = np.ascontiguousarray(boxes, np.float32)
    tb = np.ascontiguousarray(tree_begin, np.int32)
    n, g = int(tb[-1]), len(tb) - 1
    cap = max(2 * n, 16)
    nodes = np.zeros((cap, 80), np.uint8)
    order = np.zeros(n, np.uint32)
    roots = np.zeros(g, np.uint32)
    depth = np.zeros(g, np.int32)
    nn = C.c_int(0)
    _check(lib().lux_bvh8_build(ptr(boxes), ptr(tb, C.c_int), g, 1 if on_device else 0, nodes.ctypes.data, cap,
                                ptr(order, C.c_uint32), ptr(roots, C.c_uint32), ptr(depth, C.c_int), C.byref(nn)))
    return nodes[: nn.value], order, roots, depth


# ---- renderer -------------------------------------------------------------------------------
class ResidentScene:
    """A scene built once on the device (lux_scene_create): geometry, BVH, materials, textures
    and light tables. Renderers made on it (Renderer(resident, ...)) allocate only per-pixel
    state, as the reference's pathtraceInit does after main() has built the scene."""

    def __init__(self, scene, options: Optional[Options] = None, **kw):
        self.scene = scene
        self.options = options if options is not None else default_options(**kw)
        h = C.c_void_p()
        _check(lib().lux_scene_create(scene.desc_ptr, C.byref(self.options), C.byref(h)))
        self._h = h

    @property
    def width(self) -> int:
        return self.scene.width

    @property
    def height(self) -> int:
        return self.scene.height

    @property
    def device_bytes(self) -> int:
        return int(lib().lux_scene_device_bytes(self._h))

    def build_stats(self) -> dict:
        """Stage times of the scene build (lux_scene_get_stats)."""
        st = _ffi.SceneStats()
        _check(lib().lux_scene_get_stats(self._h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in _ffi.SceneStats._fields_}

    def compatible(self, opt: Options) -> bool:
        """Whether a context with these options can render on this build (the options that
        shape a build are the same)."""
        keys = ("device", "precision", "texture_storage", "bvh_layout")
        return all(getattr(opt, k) == getattr(self.options, k) for k in keys)

    def close(self):
        if getattr(self, "_h", None):
            lib().lux_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Renderer:
    """One render context (lux_ctx): a scene plus its accumulation image. `scene` is a host
    scene (built and owned by the context, lux_init) or a ResidentScene (shared, lux_init_on_scene,
    optionally with another camera of any resolution)."""

    def __init__(self, scene, options: Optional[Options] = None, camera: Optional[CameraDesc] = None, **kw):
        self.scene = scene
        self.options = options if options is not None else default_options(**kw)
        h = C.c_void_p()
        if isinstance(scene, ResidentScene):
            _check(lib().lux_init_on_scene(scene._h, C.byref(camera) if camera is not None else None,
                                           C.byref(self.options), C.byref(h)))
        else:
            if camera is not None:
                raise LuxError(-1, "a camera override needs a ResidentScene")
            _check(lib().lux_init(scene.desc_ptr, C.byref(self.options), C.byref(h)))
        self._h = h
        self.width = camera.width if camera is not None else scene.width
        self.height = camera.height if camera is not None else scene.height

    def render_iter(self, it: int, rgba8_dev: int = 0):
        _check(lib().lux_render_iter(self._h, it, C.c_void_p(rgba8_dev) if rgba8_dev else None))

    def render(self, first_iter: int, n_iter: int):
        _check(lib().lux_render(self._h, first_iter, n_iter))

    def image_sum(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 3), np.float32)
        _check(lib().lux_copy_image(self._h, ptr(out)))
        return out

    def image_sum_into(self, out: np.ndarray) -> np.ndarray:
        """The accumulation sum into a caller's float32 (height, width, 3) array."""
        if out.dtype != np.float32 or out.shape != (self.height, self.width, 3) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (height, width, 3)")
        _check(lib().lux_copy_image(self._h, ptr(out)))
        return out

    def rgba8(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.uint8)
        _check(lib().lux_copy_rgba8(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def reset(self):
        _check(lib().lux_reset(self._h))

    def set_camera(self, cam: CameraDesc):
        _check(lib().lux_set_camera(self._h, C.byref(cam)))

    def enable_timing(self, on: bool = True):
        _check(lib().lux_enable_timing(self._h, 1 if on else 0))

    def stats(self) -> dict:
        s = Stats()
        _check(lib().lux_get_stats(self._h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in Stats._fields_}

    def scene_stats(self) -> dict:
        """Stage times of the build of the scene this context renders (lux_get_scene_stats)."""
        st = _ffi.SceneStats()
        _check(lib().lux_get_scene_stats(self._h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in _ffi.SceneStats._fields_}

    def copy_image_device(self, dev_ptr: int):
        """Copy the accumulation sum (W*H*3 floats) to device memory at dev_ptr, on the
        context's stream, without waiting."""
        _check(lib().lux_copy_image_device(self._h, C.c_void_p(dev_ptr)))

    def wave_counts(self, max_bounces: int = 64):
        """(paths entering each bounce, shadow rays per bounce) of the last wave rendered."""
        p = np.zeros(max_bounces, np.int32)
        sh = np.zeros(max_bounces, np.int32)
        _check(lib().lux_wave_counts(self._h, ptr(p, C.c_int), ptr(sh, C.c_int), max_bounces))
        return p, sh

    # kernel-level entry points (parity suite)
    def trace_rays(self, rays: np.ndarray, mode: int = 0, it: int = 1) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        hits = np.zeros((n, 5), np.uint32)
        _check(lib().lux_trace_rays(self._h, ptr(rays), n, mode, it, ptr(hits, C.c_uint32)))
        return hits

    def trace_rays_static(self, rays: np.ndarray, mode: int = 0, it: int = 1) -> np.ndarray:
        """trace_rays through the library's fixed device scratch (no device allocation on the
        call), for at most TRACE_STATIC_MAX_RAYS rays; overlapping calls on one device race."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        hits = np.zeros((n, 5), np.uint32)
        _check(lib().lux_trace_rays_static(self._h, ptr(rays), n, mode, it, ptr(hits, C.c_uint32)))
        return hits

    def morton_keys(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        keys = np.zeros(rays.shape[0], np.uint32)
        _check(lib().lux_morton_keys(self._h, ptr(rays), rays.shape[0], ptr(keys, C.c_uint32)))
        return keys

    def shade_step(self, paths: np.ndarray, hits: np.ndarray, it: int, depth: int, compact: int = 1):
        paths = np.ascontiguousarray(paths, np.float32).copy()
        hits = np.ascontiguousarray(hits, np.uint32)
        n = paths.shape[0]
        surv = np.zeros(max(n, 1), np.int32)
        nout = C.c_int(0)
        _check(lib().lux_shade_step(self._h, it, depth, compact, ptr(paths), n, ptr(hits, C.c_uint32),
                                    ptr(surv, C.c_int), C.byref(nout)))
        return paths, surv[: nout.value].copy()

    def light_samples(self, pixels: np.ndarray, it: int, depth: int) -> np.ndarray:
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((pixels.shape[0], 6), np.float32)
        _check(lib().lux_light_samples(self._h, it, depth, ptr(pixels, C.c_int), pixels.shape[0], ptr(out)))
        return out

    def cdfs(self, sizes) -> dict:
        ne, ntp, eh, ew = sizes
        ep = np.zeros(max(ne, 1), np.float32)
        tp = np.zeros(max(ntp, 1), np.float32)
        mg = np.zeros(max(eh, 1), np.float32)
        cd = np.zeros(max(eh * ew, 1), np.float32)
        ta = C.c_float(0)
        _check(lib().lux_get_cdfs(self._h, ptr(ep), ptr(tp), ptr(mg), ptr(cd), C.byref(ta)))
        return {"emissive_prefix": ep[:ne], "tri_prefix": tp[:ntp], "marginal": mg[:eh],
                "conditional": cd[: eh * ew], "total_area": ta.value}

    def sample_texture(self, tex: int, uv: np.ndarray) -> np.ndarray:
        uv = np.ascontiguousarray(uv, np.float32)
        out = np.zeros((uv.shape[0], 4), np.float32)
        _check(lib().lux_sample_texture(self._h, tex, ptr(uv), uv.shape[0], ptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().lux_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """The job engine (lux_engine_*): resident scenes, many jobs in one shared wavefront.

    Each scene is a HostScene or SceneBuilder (anything with desc_ptr). A job is a scene index,
    a camera (defaulting to the scene's own), samples per pixel and a trace depth; its image
    equals the single-job render of the same scene, camera and samples bit for bit."""

    def __init__(self, scenes, options: Optional[Options] = None, hbm_budget_bytes: int = 0, max_paths: int = 0,
                 max_jobs: int = 0, schedule: int = _ffi.SCHED_FIFO, trace_blocks: int = 0):
        self._scenes = list(scenes)
        ptrs = (C.POINTER(SceneDesc) * len(self._scenes))(*[sc.desc_ptr for sc in self._scenes])
        self.options = options if options is not None else default_options()
        cfg = EngineConfig()
        cfg.hbm_budget_bytes, cfg.max_paths, cfg.max_jobs = hbm_budget_bytes, max_paths, max_jobs
        cfg.schedule, cfg.trace_blocks = schedule, trace_blocks
        h = _P()
        _check(lib().lux_engine_create(ptrs, len(self._scenes), C.byref(self.options), C.byref(cfg), C.byref(h)))
        self._h = h
        self._sizes = {}

    def submit(self, scene: int, spp: int, trace_depth: int = 0, first_iter: int = 1,
               camera: Optional[CameraDesc] = None) -> int:
        j = JobDesc()
        j.scene, j.spp, j.trace_depth, j.first_iter = scene, spp, trace_depth, first_iter
        j.camera = camera if camera is not None else self._scenes[scene].desc.camera
        jid = C.c_int()
        _check(lib().lux_engine_submit(self._h, C.byref(j), C.byref(jid)))
        self._sizes[jid.value] = (j.camera.height, j.camera.width)
        return jid.value

    def step(self):
        """Render one wave; returns (jobs completed in it, idle)."""
        done, idle = C.c_int(), C.c_int()
        _check(lib().lux_engine_step(self._h, C.byref(done), C.byref(idle)))
        return done.value, bool(idle.value)

    def run(self):
        _check(lib().lux_engine_run(self._h))

    def status(self, job: int) -> dict:
        st = JobStatus()
        _check(lib().lux_engine_job_status(self._h, job, C.byref(st)))
        return {n: getattr(st, n) for n, _ in JobStatus._fields_}

    def image(self, job: int) -> np.ndarray:
        h, w = self._sizes[job]
        out = np.empty((h, w, 3), np.float32)
        _check(lib().lux_engine_copy_image(self._h, job, ptr(out)))
        return out

    def release(self, job: int):
        _check(lib().lux_engine_release(self._h, job))

    def stats(self) -> dict:
        st = EngineStats()
        _check(lib().lux_engine_get_stats(self._h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in EngineStats._fields_}

    def clock_ms(self) -> float:
        return float(lib().lux_engine_clock_ms(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().lux_engine_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_camera(width: int, height: int, pos, look, fovy_deg: float = 45.0) -> CameraDesc:
    """A pinhole camera (lux_make_camera) at pos looking at look, world up +y."""
    p = (C.c_float * 3)(*[float(x) for x in pos])
    q = (C.c_float * 3)(*[float(x) for x in look])
    cam = CameraDesc()
    lib().lux_make_camera(width, height, p, q, float(fovy_deg), C.byref(cam))
    return cam


def plan_wave(npix, remaining, capacity: int, max_segments: int = 256) -> np.ndarray:
    """The engine's wave planner (lux_plan_wave): samples each job contributes to one wave."""
    npix = np.ascontiguousarray(npix, np.int32)
    remaining = np.ascontiguousarray(remaining, np.int32)
    take = np.zeros(len(npix), np.int32)
    rc = lib().lux_plan_wave(ptr(npix, C.c_int), ptr(remaining, C.c_int), len(npix), capacity, max_segments,
                             ptr(take, C.c_int))
    if rc < 0:
        _check(rc)
    return take


def rng_stream(it: int, index: int, depth: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    _check(lib().lux_rng_stream(it, index, depth, n, ptr(out)))
    return out


# ---- reference-shaped module interface --------------------------------------------------------
class PathTracerOptions:
    """Singleton options, as include/pathtrace/pathtracer_options.h:3-21."""

    _instance: Optional["PathTracerOptions"] = None

    def __init__(self):
        self.debug_bvh = False
        self.material_debug_mode = 0
        self.color_mode = _ffi.TONEMAP_ACES
        self.envmap_intensity = 1.0
        self.direct_light_sampling = False
        self.environment_map_importance_sampling = False
        self.selected_material = 0

    @classmethod
    def Get(cls) -> "PathTracerOptions":
        if cls._instance is None:
            cls._instance = PathTracerOptions()
        return cls._instance

    def to_options(self, **kw) -> Options:
        return default_options(direct_light_sampling=int(self.direct_light_sampling),
                               env_importance_sampling=int(self.environment_map_importance_sampling),
                               color_mode=int(self.color_mode), envmap_intensity=float(self.envmap_intensity),
                               material_debug_mode=int(self.material_debug_mode), debug_bvh=int(bool(self.debug_bvh)),
                               **kw)


_state: Optional[Renderer] = None
_resident: Optional[ResidentScene] = None


def pathtraceInit(scene, **kw) -> None:
    """Allocate the per-pixel state for `scene` (src/pathtrace/pathtrace_buffers.cu:21-140).

    The scene's device build (upload, BVH, light tables, textures) is made on the first call
    for a scene object and kept, as the reference builds meshes and acceleration structures
    once at load (src/main.cpp:199-274): a pathtraceFree(); pathtraceInit() pair on a camera
    or option reset (src/app/render_loop.cpp:122-126) only reallocates per-pixel state.
    sceneRelease() drops the kept build."""
    global _state, _resident
    pathtraceFree()
    opt = PathTracerOptions.Get().to_options(**kw)
    if _resident is None or _resident.scene is not scene or not _resident.compatible(opt):
        sceneRelease()
        _resident = ResidentScene(scene, opt)
    _state = Renderer(_resident, opt)


def sceneRelease() -> None:
    """Free the device build pathtraceInit keeps (the reference frees meshes at exit)."""
    global _resident
    if _resident is not None:
        _resident.close()
        _resident = None


def pathtrace(pbo: int, frame: int, iteration: int) -> None:
    """One sample per pixel (src/pathtrace.cu:97-367). `pbo` is a device pointer or 0."""
    del frame  # unused by the reference as well
    if _state is None:
        raise LuxError(-7, "pathtrace called before pathtraceInit")
    _state.render_iter(iteration, pbo)


def pathtraceFree() -> None:
    global _state
    if _state is not None:
        _state.close()
        _state = None


def copyImageToHost() -> np.ndarray:
    """The FP32 accumulation sum (src/pathtrace/pathtrace_buffers.cu:180-190)."""
    if _state is None:
        raise LuxError(-7, "copyImageToHost called before pathtraceInit")
    return _state.image_sum()
