"""The CPU oracle reproduces the golden vectors produced by the reference's own host-compiled
sources (tests/golden/make_golden.py), bit for bit."""
import ctypes as C
import os

import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200._ffi import default_options

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLD)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def small_random_scene():
    return lx.random_scene(seed=7, num_instances=8, total_tris=16000, min_tris=1000, max_tris=4000, num_emissive=2,
                           num_textures=4, texture_size=64, env_width=128, env_height=64, width=40, height=32,
                           trace_depth=6)


SCENES = {
    "cornell": (lambda: lx.cornell36(48, 48), lambda: default_options(direct_light_sampling=1)),
    "rand": (small_random_scene, lambda: default_options(direct_light_sampling=1, env_importance_sampling=1)),
}


def test_rng_streams(g):
    O = ol.orc()
    for (a, b, c), ref in zip(g["rng_seeds"], g["rng_streams"]):
        out = np.zeros(32, np.float32)
        O.orc_rng_stream(int(a), int(b), int(c), 32, ol.f32p(out))
        assert np.array_equal(bits(out), bits(ref))


def test_utilhash(g):
    O = ol.orc()
    assert [O.orc_utilhash(int(x)) for x in g["hash_in"]] == list(g["hash_out"])


def test_select_from_cdf(g):
    O = ol.orc()
    cdf = np.ascontiguousarray(g["cdf"])
    got = [O.orc_select_from_cdf(ol.f32p(cdf), len(cdf), C.c_float(float(x))) for x in g["cdf_xi"]]
    assert got == list(g["cdf_idx"])


def test_bsdf_eval(g):
    rec = np.ascontiguousarray(g["bsdf_in"])
    out = np.zeros_like(g["bsdf_out"])
    ol.orc().orc_eval_bsdf(ol.f32p(rec), len(rec), ol.f32p(out))
    ref = g["bsdf_out"]
    same = (bits(out) == bits(ref)) | (np.isnan(out) & np.isnan(ref))
    assert same.all()


def test_bsdf_sample_and_hemisphere(g):
    rec = np.ascontiguousarray(g["bsdf_in"])
    seeds = np.ascontiguousarray(g["sample_seeds"])
    out = np.zeros_like(g["sample_out"])
    ol.orc().orc_sample_bsdf(ol.f32p(rec), ol.i32p(seeds), len(seeds), ol.f32p(out))
    assert np.array_equal(bits(out), bits(g["sample_out"]))
    n = np.ascontiguousarray(g["hemi_n"])
    h = np.zeros_like(g["hemi_out"])
    ol.orc().orc_hemisphere(ol.f32p(n), ol.i32p(seeds[: len(n)]), len(n), ol.f32p(h))
    assert np.array_equal(bits(h), bits(g["hemi_out"]))


@pytest.fixture(scope="module", params=list(SCENES))
def scene(request):
    make, opt = SCENES[request.param]
    s = make()
    return request.param, s, ol.OracleScene(s), opt()


def test_cdfs(g, scene):
    tag, s, o, _ = scene
    cd = o.cdfs()
    for k in ("emissive_prefix", "tri_prefix", "marginal", "conditional"):
        assert np.array_equal(bits(np.asarray(cd[k], np.float32)), bits(g[f"{tag}_cdf_{k}"])), k
    assert np.float32(cd["total_area"]) == np.float32(g[f"{tag}_cdf_total_area"])


def test_camera_and_light_samples(g, scene):
    tag, s, o, opt = scene
    pix = np.arange(s.width * s.height, dtype=np.int32)
    assert np.array_equal(bits(o.camera_rays(pix, 3)[:, :19]), bits(g[f"{tag}_camera_it3"][:, :19]))
    for depth in (0, 1, 4):
        assert np.array_equal(bits(o.light_samples(opt, pix, 3, depth)), bits(g[f"{tag}_light_d{depth}"]))


def test_trace_hits(g, scene):
    tag, s, o, _ = scene
    rays = ol.camera_paths_to_rays(g[f"{tag}_camera_it3"])
    assert np.array_equal(o.trace(rays, 0, 3), g[f"{tag}_trace_cam"])
    rr = g[f"{tag}_rand_rays"]
    assert np.array_equal(o.trace(rr, 0, 3), g[f"{tag}_trace_rand_m0"])
    # any-hit: only the occlusion word is defined
    assert np.array_equal(o.trace(rr, 2, 3)[:, 0], g[f"{tag}_trace_rand_m2"][:, 0])
    assert np.array_equal(o.trace(g[f"{tag}_rand_rays_tmax"], 1, 3), g[f"{tag}_trace_rand_m1"])
    # the oracle's BVH and the brute-force loop agree
    assert np.array_equal(o.trace(rr, 0, 3, brute=True), g[f"{tag}_trace_rand_m0"])


def test_shade_step(g, scene):
    tag, s, o, opt = scene
    out, surv = o.shade_step(opt, g[f"{tag}_shade_in_paths"], g[f"{tag}_shade_in_hits"], 3, 1, 1)
    assert np.array_equal(np.sort(surv), g[f"{tag}_shade_survivors"])
    ref = g[f"{tag}_shade_out_paths"]
    assert np.array_equal(bits(out[:, :22]), bits(ref[:, :22]))


def test_render(g, scene):
    tag, s, o, opt = scene
    img, st = o.render(opt, 1, 2)
    assert np.array_equal(bits(img), bits(g[f"{tag}_render_2spp"]))
    assert np.array_equal(st, g[f"{tag}_render_stats"])


def test_morton(g, scene):
    tag, s, o, _ = scene
    assert np.array_equal(o.morton(g[f"{tag}_rand_rays"]), g[f"{tag}_morton"])
