"""ctypes bindings of the CPU oracle (oracle/liblux_oracle.so) and of the reference's own
host-compiled render path (oracle/_ref/libluxref.so). Test infrastructure only: these
libraries check the CUDA path; they are never a substitute for it."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from luxion_b200._ffi import Options, SceneDesc, c_float_p, c_int_p, c_u32_p

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liblux_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libluxref.so")

_orc: Optional[C.CDLL] = None
_ref: Optional[C.CDLL] = None


def build_oracle() -> None:
    """Build the oracle (and, where the reference tree exists, the reference library)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j8", "all"], check=True,
                   capture_output=True)


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        P = C.c_void_p
        L.orc_utilhash.restype = C.c_uint32
        L.orc_utilhash.argtypes = [C.c_uint32]
        L.orc_rng_stream.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, c_float_p]
        L.orc_select_from_cdf.restype = C.c_int
        L.orc_select_from_cdf.argtypes = [c_float_p, C.c_int, C.c_float]
        L.orc_eval_bsdf.argtypes = [c_float_p, C.c_int, c_float_p]
        L.orc_sample_bsdf.argtypes = [c_float_p, c_int_p, C.c_int, c_float_p]
        L.orc_hemisphere.argtypes = [c_float_p, c_int_p, C.c_int, c_float_p]
        L.orc_scene_create.restype = P
        L.orc_scene_create.argtypes = [C.POINTER(SceneDesc), C.c_int, C.c_int]
        L.orc_scene_destroy.argtypes = [P]
        L.orc_get_cdfs.argtypes = [P, c_float_p, c_float_p, c_float_p, c_float_p, c_float_p]
        L.orc_cdf_sizes.argtypes = [P, c_int_p]
        L.orc_trace.argtypes = [P, c_float_p, C.c_int, C.c_int, C.c_int, c_u32_p, C.c_int]
        L.orc_morton.argtypes = [P, c_float_p, C.c_int, c_u32_p]
        L.orc_light_samples.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, c_int_p, C.c_int, c_float_p]
        L.orc_camera_rays.argtypes = [P, C.c_int, c_int_p, C.c_int, c_float_p]
        L.orc_shade_step.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, C.c_int, c_float_p, C.c_int,
                                     c_u32_p, c_int_p, c_int_p]
        L.orc_sample_texture.argtypes = [P, C.c_int, c_float_p, C.c_int, c_float_p]
        L.orc_render.restype = C.c_int
        L.orc_render.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.c_int, c_float_p, C.POINTER(C.c_double)]
        L.orc_tonemap.argtypes = [c_float_p, C.c_int, C.c_float, C.c_int, C.POINTER(C.c_uint8)]
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        P = C.c_void_p
        L.ref_utilhash.restype = C.c_uint32
        L.ref_utilhash.argtypes = [C.c_uint32]
        L.ref_rng_stream.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, c_float_p]
        L.ref_select_from_cdf.restype = C.c_int
        L.ref_select_from_cdf.argtypes = [c_float_p, C.c_int, C.c_float]
        L.ref_eval_bsdf.argtypes = [c_float_p, C.c_int, c_float_p]
        L.ref_sample_bsdf.argtypes = [c_float_p, c_int_p, C.c_int, c_float_p]
        L.ref_hemisphere.argtypes = [c_float_p, c_int_p, C.c_int, c_float_p]
        L.ref_scene_create.restype = P
        L.ref_scene_create.argtypes = [C.POINTER(SceneDesc)]
        L.ref_scene_destroy.argtypes = [P]
        L.ref_get_cdfs.argtypes = [P, c_float_p, c_float_p, c_float_p, c_float_p, c_float_p]
        L.ref_cdf_sizes.argtypes = [P, c_int_p]
        L.ref_trace.argtypes = [P, c_float_p, C.c_int, C.c_int, C.c_int, c_u32_p]
        L.ref_mesh_isect_t.argtypes = [P, c_float_p, C.c_int, c_float_p]
        L.ref_morton.argtypes = [P, c_float_p, C.c_int, c_float_p, c_float_p, c_u32_p]
        L.ref_light_samples.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, c_int_p, C.c_int, c_float_p]
        L.ref_camera_rays.argtypes = [P, C.c_int, c_int_p, C.c_int, c_float_p]
        L.ref_shade_step.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, C.c_int, c_float_p, C.c_int,
                                     c_u32_p, c_int_p, c_int_p]
        L.ref_render.restype = C.c_int
        L.ref_render.argtypes = [P, C.POINTER(Options), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, c_float_p, C.POINTER(C.c_double)]
        _ref = L
    return _ref


def f32p(a):
    return a.ctypes.data_as(c_float_p)


def u32p(a):
    return a.ctypes.data_as(c_u32_p)


def i32p(a):
    return a.ctypes.data_as(c_int_p)


class OracleScene:
    def __init__(self, host_scene, cdf_f64: int = 0, tex_storage: int = 0):
        self.host = host_scene
        self.h = orc().orc_scene_create(host_scene.desc_ptr, cdf_f64, tex_storage)

    def close(self):
        if self.h:
            orc().orc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cdf_sizes(self):
        s = np.zeros(4, np.int32)
        orc().orc_cdf_sizes(self.h, i32p(s))
        return [int(x) for x in s]

    def cdfs(self):
        ne, ntp, eh, ew = self.cdf_sizes()
        ep = np.zeros(max(ne, 1), np.float32)
        tp = np.zeros(max(ntp, 1), np.float32)
        mg = np.zeros(max(eh, 1), np.float32)
        cd = np.zeros(max(eh * ew, 1), np.float32)
        ta = np.zeros(1, np.float32)
        orc().orc_get_cdfs(self.h, f32p(ep), f32p(tp), f32p(mg), f32p(cd), f32p(ta))
        return {"emissive_prefix": ep[:ne], "tri_prefix": tp[:ntp], "marginal": mg[:eh],
                "conditional": cd[: eh * ew], "total_area": float(ta[0])}

    def trace(self, rays, mode=0, it=1, brute=False):
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 5), np.uint32)
        orc().orc_trace(self.h, f32p(rays), rays.shape[0], mode, it, u32p(hits), 1 if brute else 0)
        return hits

    def morton(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        keys = np.zeros(rays.shape[0], np.uint32)
        orc().orc_morton(self.h, f32p(rays), rays.shape[0], u32p(keys))
        return keys

    def light_samples(self, opt, pixels, it, depth):
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((pixels.shape[0], 6), np.float32)
        orc().orc_light_samples(self.h, C.byref(opt), it, depth, i32p(pixels), pixels.shape[0], f32p(out))
        return out

    def camera_rays(self, pixels, it):
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((pixels.shape[0], 24), np.float32)
        orc().orc_camera_rays(self.h, it, i32p(pixels), pixels.shape[0], f32p(out))
        return out

    def shade_step(self, opt, paths, hits, it, depth, compact=1):
        paths = np.ascontiguousarray(paths, np.float32).copy()
        hits = np.ascontiguousarray(hits, np.uint32)
        n = paths.shape[0]
        surv = np.zeros(max(n, 1), np.int32)
        nout = np.zeros(1, np.int32)
        orc().orc_shade_step(self.h, C.byref(opt), it, depth, compact, f32p(paths), n, u32p(hits), i32p(surv),
                             i32p(nout))
        return paths, surv[: nout[0]].copy()

    def sample_texture(self, tex, uv):
        uv = np.ascontiguousarray(uv, np.float32)
        out = np.zeros((uv.shape[0], 4), np.float32)
        orc().orc_sample_texture(self.h, tex, f32p(uv), uv.shape[0], f32p(out))
        return out

    def render(self, opt, first_iter, n_iter, crop=None, f64=False, threads=0):
        W, H = self.host.width, self.host.height
        x0, y0, w, h = crop if crop else (0, 0, W, H)
        img = np.zeros((h, w, 3), np.float32)
        st = np.zeros(4, np.float64)
        orc().orc_render(self.h, C.byref(opt), first_iter, n_iter, x0, y0, w, h, 1 if f64 else 0, threads,
                         f32p(img), st.ctypes.data_as(C.POINTER(C.c_double)))
        return img, st


class RefScene:
    def __init__(self, host_scene):
        self.host = host_scene
        self.h = ref().ref_scene_create(host_scene.desc_ptr)

    def close(self):
        if self.h:
            ref().ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cdfs(self):
        s = np.zeros(4, np.int32)
        ref().ref_cdf_sizes(self.h, i32p(s))
        ne, ntp, eh, ew = [int(x) for x in s]
        ep = np.zeros(max(ne, 1), np.float32)
        tp = np.zeros(max(ntp, 1), np.float32)
        mg = np.zeros(max(eh, 1), np.float32)
        cd = np.zeros(max(eh * ew, 1), np.float32)
        ta = np.zeros(1, np.float32)
        ref().ref_get_cdfs(self.h, f32p(ep), f32p(tp), f32p(mg), f32p(cd), f32p(ta))
        return {"emissive_prefix": ep[:ne], "tri_prefix": tp[:ntp], "marginal": mg[:eh],
                "conditional": cd[: eh * ew], "total_area": float(ta[0])}

    def trace(self, rays, mode=0, it=1):
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 5), np.uint32)
        ref().ref_trace(self.h, f32p(rays), rays.shape[0], mode, it, u32p(hits))
        return hits

    def mesh_isect_t(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        t = np.zeros(rays.shape[0], np.float32)
        ref().ref_mesh_isect_t(self.h, f32p(rays), rays.shape[0], f32p(t))
        return t

    def morton(self, rays, bmin, bmax):
        rays = np.ascontiguousarray(rays, np.float32)
        keys = np.zeros(rays.shape[0], np.uint32)
        ref().ref_morton(self.h, f32p(rays), rays.shape[0], f32p(np.asarray(bmin, np.float32)),
                         f32p(np.asarray(bmax, np.float32)), u32p(keys))
        return keys

    def light_samples(self, opt, pixels, it, depth):
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((pixels.shape[0], 6), np.float32)
        ref().ref_light_samples(self.h, C.byref(opt), it, depth, i32p(pixels), pixels.shape[0], f32p(out))
        return out

    def camera_rays(self, pixels, it):
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((pixels.shape[0], 24), np.float32)
        ref().ref_camera_rays(self.h, it, i32p(pixels), pixels.shape[0], f32p(out))
        return out

    def shade_step(self, opt, paths, hits, it, depth, compact=1):
        paths = np.ascontiguousarray(paths, np.float32).copy()
        hits = np.ascontiguousarray(hits, np.uint32)
        n = paths.shape[0]
        surv = np.zeros(max(n, 1), np.int32)
        nout = np.zeros(1, np.int32)
        ref().ref_shade_step(self.h, C.byref(opt), it, depth, compact, f32p(paths), n, u32p(hits), i32p(surv),
                             i32p(nout))
        return paths, surv[: nout[0]].copy()

    def render(self, opt, first_iter, n_iter, crop=None, threads=0):
        W, H = self.host.width, self.host.height
        x0, y0, w, h = crop if crop else (0, 0, W, H)
        img = np.zeros((h, w, 3), np.float32)
        st = np.zeros(4, np.float64)
        ref().ref_render(self.h, C.byref(opt), first_iter, n_iter, x0, y0, w, h, threads, f32p(img),
                         st.ctypes.data_as(C.POINTER(C.c_double)))
        return img, st


def camera_paths_to_rays(paths: np.ndarray) -> np.ndarray:
    """Path states (24 floats) -> ray records (origin, tmax, direction, pixel bits)."""
    n = paths.shape[0]
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = paths[:, 0:3]
    rays[:, 3] = 1e16
    rays[:, 4:7] = paths[:, 3:6]
    rays[:, 7] = paths[:, 18]
    return rays


def random_rays(n: int, lo, hi, seed: int = 0, pixel_base: int = 0) -> np.ndarray:
    """Rays with origins uniform in the box [lo, hi] and uniform directions."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e16
    rays[:, 4:7] = d.astype(np.float32)
    rays[:, 7] = (np.arange(n, dtype=np.int32) + pixel_base).view(np.float32)
    return rays
