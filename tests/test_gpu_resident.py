"""Resident scenes (lux_scene_create / lux_init_on_scene / lux_scene_free) through the C-ABI.

The reference builds its meshes and acceleration structures once at load and reallocates only
per-pixel buffers on every pathtraceFree(); pathtraceInit() (src/main.cpp:199-274,
src/app/render_loop.cpp:122-126). A context made on a resident scene must render exactly what
a context that built the scene itself renders, for any camera and resolution.
"""
import ctypes
import time

import numpy as np
import pytest

import luxion_b200 as lx
from luxion_b200 import _ffi
from luxion_b200._ffi import CameraDesc, default_options

pytestmark = pytest.mark.gpu


def small_random_scene(**kw):
    p = dict(seed=7, num_instances=8, total_tris=16000, min_tris=1000, max_tris=4000, num_emissive=2,
             num_textures=4, texture_size=64, env_width=128, env_height=64, width=40, height=32, trace_depth=6)
    p.update(kw)
    return lx.random_scene(**p)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def camera(w, h, pos, look, fov=45.0):
    c = CameraDesc()
    lx.lib().lux_make_camera(w, h, (ctypes.c_float * 3)(*pos), (ctypes.c_float * 3)(*look), fov, ctypes.byref(c))
    return c


def test_context_on_resident_scene_equals_own_build():
    s = small_random_scene()
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
    own = lx.Renderer(s, opt)
    own.render(1, 6)
    a = own.image_sum()
    own.close()
    R = lx.ResidentScene(s, opt)
    assert R.device_bytes > 0
    r = lx.Renderer(R, opt)
    r.render(1, 6)
    b = r.image_sum()
    r.close()
    R.close()
    assert np.array_equal(bits(a), bits(b))


def test_other_cameras_and_resolutions_on_one_scene():
    """Contexts of several resolutions on one resident scene render what a scene description
    carrying that camera renders in its own context."""
    s = small_random_scene()
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
    R = lx.ResidentScene(s, opt)
    d = s.desc
    saved = CameraDesc.from_buffer_copy(d.camera)
    try:
        for (w, h), pos in (((64, 48), (3.0, 6.0, 20.0)), ((17, 31), (-8.0, 4.0, 12.0))):
            cam = camera(w, h, pos, (0.0, 1.0, 0.0))
            r = lx.Renderer(R, opt, camera=cam)
            r.render(2, 3)
            a = r.image_sum()
            r.close()
            assert a.shape == (h, w, 3)
            d.camera = cam
            own = lx.Renderer(s, opt)
            own.render(2, 3)
            b = own.image_sum()
            own.close()
            d.camera = saved
            assert np.array_equal(bits(a), bits(b))
    finally:
        d.camera = saved
        R.close()


def test_scene_outlives_its_handle_while_contexts_use_it():
    s = small_random_scene()
    opt = default_options(direct_light_sampling=1)
    R = lx.ResidentScene(s, opt)
    r1 = lx.Renderer(R, opt)
    R.close()                      # the contexts keep the scene alive
    r1.render(1, 2)
    assert np.isfinite(r1.image_sum()).all()
    r1.close()


def test_contexts_must_match_the_build():
    s = small_random_scene()
    R = lx.ResidentScene(s, default_options())
    with pytest.raises(lx.LuxError, match="precision"):
        lx.Renderer(R, default_options(precision=_ffi.PRECISION_COMPENSATED))
    with pytest.raises(lx.LuxError, match="texture storage"):
        lx.Renderer(R, default_options(texture_storage=_ffi.TEXSTORE_HALF))
    no_env = lx.ResidentScene(small_random_scene(env_width=0, env_height=0), default_options())
    with pytest.raises(lx.LuxError, match="environment"):
        lx.Renderer(no_env, default_options(env_importance_sampling=1))
    no_env.close()
    R.close()


def test_reference_shaped_reinit_keeps_the_scene():
    """pathtraceFree(); pathtraceInit() on the same scene reuses its device build, and renders
    what a fresh build renders."""
    s = lx.cornell36(32, 32)
    lx.PathTracerOptions.Get().direct_light_sampling = True
    try:
        lx.pathtraceInit(s)
        built = lx._resident
        for it in range(1, 4):
            lx.pathtrace(0, 0, it)
        first = lx.copyImageToHost().copy()
        lx.pathtraceFree()
        lx.pathtraceInit(s)
        assert lx._resident is built
        for it in range(1, 4):
            lx.pathtrace(0, 0, it)
        again = lx.copyImageToHost()
    finally:
        lx.pathtraceFree()
        lx.sceneRelease()
        lx.PathTracerOptions.Get().direct_light_sampling = False
    assert np.array_equal(bits(first), bits(again))


def test_reinit_on_a_resident_1m_triangle_scene_is_cheap():
    """Building the 1M-triangle scene is the expensive part; a new 1080p context on it only
    allocates per-pixel and per-path state (measured here, bounded loosely)."""
    s = lx.random_scene(seed=0)
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
    R = lx.ResidentScene(s, opt)
    r = lx.Renderer(R, opt)     # first context: loads kernels, warms the allocator
    r.close()
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        r = lx.Renderer(R, opt)
        times.append((time.perf_counter() - t0) * 1e3)
        r.close()
    R.close()
    assert min(times) < 50.0, times
