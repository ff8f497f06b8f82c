"""The seeded workloads of the batching and serving forms (host only): sizes, ranges,
determinism, and the camera helper against the scene generator's own camera."""
import math

import numpy as np

import luxion_b200 as lx
from luxion_b200 import workloads


def test_make_camera_matches_the_generator():
    s = lx.random_scene(seed=0, total_tris=20000, num_instances=8, min_tris=1000, max_tris=5000, num_textures=1,
                        texture_size=16, env_width=16, env_height=8)
    c = s.desc.camera
    m = lx.make_camera(c.width, c.height, workloads.CAMERA_POS, workloads.CAMERA_LOOK, 45.0)
    for f in ("position", "view", "right", "up", "pixel_length", "fov"):
        assert np.array_equal(np.array(getattr(c, f)[:], np.float32), np.array(getattr(m, f)[:], np.float32)), f


def test_scene_params_respect_the_triangle_range():
    for t in (10_000, 50_000, 300_000, 2_000_000, 4_000_000):
        p = workloads.scene_params(t, 1)
        assert 4 <= p["num_instances"] <= 200 and p["min_tris"] < p["max_tris"]
        assert p["min_tris"] * p["num_instances"] <= t <= p["max_tris"] * p["num_instances"]


def test_batch_jobs_are_seeded_and_in_range():
    a, b = workloads.batch_jobs(8, 64, seed=3), workloads.batch_jobs(8, 64, seed=3)
    assert [(j["scene"], j["spp"], j["depth"], j["camera"].width) for j in a] == \
           [(j["scene"], j["spp"], j["depth"], j["camera"].width) for j in b]
    assert len(a) == 64
    for j in a:
        assert 0 <= j["scene"] < 8 and j["spp"] in workloads.BATCH_SPP and 4 <= j["depth"] <= 16
        assert (j["camera"].width, j["camera"].height) in workloads.BATCH_RESOLUTIONS


def test_request_stream_is_poisson_like_and_in_range():
    r = workloads.request_stream(16, 400, 50.0, seed=1)
    t = np.array([x["arrival_ms"] for x in r])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 20.0) < 4.0            # 50 requests per second
    for x in r:
        px = x["camera"].width * x["camera"].height
        assert 256 * 144 <= px <= 1920 * 1080 and 4 <= x["spp"] <= 256 and 0 <= x["scene"] < 16
        p = np.array(x["camera"].position[:])
        assert abs(math.hypot(p[0], p[2]) - math.hypot(0, 25)) < 1e-3 and abs(p[1] - 7) < 1e-6
