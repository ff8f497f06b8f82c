"""Seeded synthetic workloads of the batching and serving forms.

batch_*:   render jobs over 8 resident scenes of 10k to 2M triangles (the 1M-triangle scene
           generator with its materials, textures and HDRI, scaled), each job a resolution from
           {128^2, 256^2, 512^2, 1024^2, 1920x1080}, 1/4/16/64 spp and a trace depth of 4 to 16.
serving_*: 16 resident scenes of 50k to 4M triangles with a binary16 2048x1024 HDRI each, and a
           Poisson stream of requests with a random camera pose, a log-normal resolution between
           256^2 and 1920x1080 pixels and 4 to 256 spp.
Scenes are generated in parallel threads (the generator releases the interpreter while it runs).
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import os
from typing import List

import numpy as np

from . import make_camera, random_scene

BATCH_RESOLUTIONS = [(128, 128), (256, 256), (512, 512), (1024, 1024), (1920, 1080)]
BATCH_SPP = [1, 4, 16, 64]
CAMERA_POS = (0.0, 7.0, 25.0)   # the generator's camera: (0, 7, 25) looking at (0, 1, 0), fov 45
CAMERA_LOOK = (0.0, 1.0, 0.0)


def scene_params(total_tris: int, seed: int, env_half: bool = False) -> dict:
    """Generator parameters for a scene of about total_tris triangles with the 1M-triangle
    scene's layout: instances of a few thousand to tens of thousands of triangles."""
    ni = int(min(200, max(4, round(total_tris / 10000))))
    lo = max(200, total_tris // (ni * 4))
    hi = max(lo * 2, total_tris // ni * 4)
    return dict(seed=seed, total_tris=int(total_tris), num_instances=ni, min_tris=int(lo), max_tris=int(hi),
                num_emissive=min(12, ni // 2), env_half=int(env_half))


def make_scenes(params: List[dict], threads: int = 0):
    threads = threads or min(len(params), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda p: random_scene(**p), params))


def log_uniform_tris(rng, n, lo, hi):
    return [int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(n)]


def batch_scenes(seed: int = 0, n: int = 8, lo: int = 10_000, hi: int = 2_000_000):
    rng = np.random.default_rng(seed)
    tris = log_uniform_tris(rng, n, lo, hi)
    return make_scenes([scene_params(t, 1000 + seed * 100 + i) for i, t in enumerate(tris)]), tris


def batch_jobs(num_scenes: int, n: int = 64, seed: int = 0) -> List[dict]:
    rng = np.random.default_rng(seed + 1)
    jobs = []
    for _ in range(n):
        w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        jobs.append(dict(scene=int(rng.integers(num_scenes)), camera=make_camera(w, h, CAMERA_POS, CAMERA_LOOK, 45.0),
                         spp=int(BATCH_SPP[int(rng.integers(len(BATCH_SPP)))]), depth=int(rng.integers(4, 17))))
    return jobs


def serving_scenes(seed: int = 0, n: int = 16, lo: int = 50_000, hi: int = 4_000_000):
    rng = np.random.default_rng(seed + 7)
    tris = log_uniform_tris(rng, n, lo, hi)
    return make_scenes([scene_params(t, 5000 + seed * 100 + i, env_half=True) for i, t in enumerate(tris)]), tris


def request_stream(num_scenes: int, n: int, rate_per_s: float, seed: int = 0, depth: int = 12) -> List[dict]:
    """n requests with Poisson arrivals: arrival_ms, scene, camera (random azimuth around the
    scene at the generator's distance and height), spp in 4..256, and a trace depth."""
    rng = np.random.default_rng(seed + 11)
    t = 0.0
    lo, hi = math.log(256 * 256), math.log(1920 * 1080)
    out = []
    r = math.hypot(CAMERA_POS[0], CAMERA_POS[2])
    for _ in range(n):
        t += rng.exponential(1000.0 / rate_per_s)
        px = math.exp(min(hi, max(lo, rng.normal(0.5 * (lo + hi), (hi - lo) / 4))))
        w = int(min(1920, max(256, round(math.sqrt(px * 16 / 9)))))
        h = int(min(1080, max(144, round(w * 9 / 16))))
        a = rng.uniform(0, 2 * math.pi)
        pos = (r * math.sin(a), CAMERA_POS[1], r * math.cos(a))
        out.append(dict(arrival_ms=t, scene=int(rng.integers(num_scenes)),
                        camera=make_camera(w, h, pos, CAMERA_LOOK, 45.0), spp=int(rng.integers(4, 257)), depth=depth))
    return out
