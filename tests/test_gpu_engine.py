"""The job engine (batching and serving forms) against the single-job path, on the GPU.

A job's image must be the single-job render of the same scene, camera, samples and trace depth
bit for bit: alone, mixed with other jobs in one wave, split over many small waves, throttled
by the HBM budget, and at every point of its progress (progressive results)."""
import numpy as np
import pytest

import luxion_b200 as lx
from luxion_b200 import _ffi
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu

OPT = dict(direct_light_sampling=1, env_importance_sampling=1)


def scene(seed, w, h, tris=20000, depth=8):
    return lx.random_scene(seed=seed, num_instances=12, total_tris=tris, min_tris=500, max_tris=tris // 4,
                           num_emissive=3, num_textures=3, texture_size=32, env_width=64, env_height=32,
                           width=w, height=h, trace_depth=depth)


@pytest.fixture(scope="module")
def scenes():
    # scene "a" in two resolutions (the geometry depends on the seed only), and two others
    return {"a": scene(5, 48, 32), "a_small": scene(5, 24, 20), "b": scene(6, 32, 32, tris=8000, depth=6),
            "c": scene(7, 40, 24, tris=30000)}


def plain(sc, spp, first_iter=1, depth=0, **kw):
    r = lx.Renderer(sc, default_options(trace_depth=depth, **OPT, **kw))
    r.render(first_iter, spp)
    img = r.image_sum()
    r.close()
    return img


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def jobs_of(scenes):
    # (engine scene index, scene with the job's camera, spp, depth override, first_iter)
    return [(0, scenes["a"], 3, 0, 1), (1, scenes["b"], 5, 4, 1), (0, scenes["a_small"], 2, 0, 9),
            (2, scenes["c"], 4, 3, 1), (1, scenes["b"], 1, 0, 3)]


@pytest.mark.parametrize("max_paths,schedule", [(0, _ffi.SCHED_FIFO), (2000, _ffi.SCHED_FIFO),
                                                (5000, _ffi.SCHED_SHORTEST_FIRST)])
def test_mixed_jobs_equal_single_job_renders(scenes, max_paths, schedule):
    E = lx.Engine([scenes["a"], scenes["b"], scenes["c"]], default_options(**OPT), max_paths=max_paths,
                  schedule=schedule)
    ids = [E.submit(si, spp, trace_depth=depth, first_iter=it, camera=sc.desc.camera)
           for si, sc, spp, depth, it in jobs_of(scenes)]
    E.run()
    st = E.stats()
    for jid, (si, sc, spp, depth, it) in zip(ids, jobs_of(scenes)):
        s = E.status(jid)
        assert s["state"] == _ffi.JOB_DONE and s["spp_done"] == spp
        assert same(E.image(jid), plain(sc, spp, it, depth)), (jid, max_paths)
    if max_paths:
        assert st["waves"] > 1 and st["max_paths"] == max_paths
    E.close()


def test_job_alone_equals_job_in_the_mix(scenes):
    E1 = lx.Engine([scenes["a"], scenes["b"]], default_options(**OPT), max_paths=3000)
    j1 = E1.submit(1, 4, camera=scenes["b"].desc.camera)
    E1.run()
    alone = E1.image(j1)
    E1.close()
    E2 = lx.Engine([scenes["a"], scenes["b"]], default_options(**OPT), max_paths=3000)
    E2.submit(0, 3, camera=scenes["a"].desc.camera)
    j2 = E2.submit(1, 4, camera=scenes["b"].desc.camera)
    E2.submit(0, 2, camera=scenes["a_small"].desc.camera)
    E2.run()
    assert same(alone, E2.image(j2))
    E2.close()


def test_budget_queues_jobs_and_progressive_results(scenes):
    probe = lx.Engine([scenes["a"]], default_options(**OPT), max_paths=2000)
    base = probe.stats()["device_bytes"]
    probe.close()
    one_image = 48 * 32 * 3 * 4
    # room for one job image at a time, and 2000 paths per wave: one 48x32 sample per wave
    E = lx.Engine([scenes["a"]], default_options(**OPT), max_paths=2000, hbm_budget_bytes=base + one_image + 16)
    cam = scenes["a"].desc.camera
    j1, j2 = E.submit(0, 3, camera=cam), E.submit(0, 2, camera=cam, first_iter=4)
    # a step advances the waves in flight by a few bounces; step until the first one is in
    steps = 0
    while E.status(j1)["spp_done"] == 0:
        E.step()
        steps += 1
        assert steps < 64
    s1, s2 = E.status(j1), E.status(j2)
    assert s1["state"] == _ffi.JOB_ACTIVE and s1["spp_done"] == 1 and s2["state"] == _ffi.JOB_QUEUED
    assert same(E.image(j1), plain(scenes["a"], 1))          # progressive: 1 of 3 samples
    while E.status(j1)["state"] != _ffi.JOB_DONE:
        E.step()
    assert same(E.image(j1), plain(scenes["a"], 3))
    assert E.status(j2)["state"] == _ffi.JOB_QUEUED
    E.release(j1)
    E.run()
    assert same(E.image(j2), plain(scenes["a"], 2, first_iter=4))
    s2 = E.status(j2)
    assert s2["t_submit_ms"] <= s2["t_admit_ms"] <= s2["t_done_ms"]
    E.close()


def test_precision_form_in_the_engine(scenes):
    opt = default_options(precision=_ffi.PRECISION_COMPENSATED, texture_storage=_ffi.TEXSTORE_HALF, **OPT)
    E = lx.Engine([scenes["b"], scenes["c"]], opt, max_paths=2500)
    j = E.submit(1, 3, camera=scenes["c"].desc.camera)
    E.submit(0, 2, camera=scenes["b"].desc.camera)
    E.run()
    r = lx.Renderer(scenes["c"], default_options(precision=_ffi.PRECISION_COMPENSATED,
                                                 texture_storage=_ffi.TEXSTORE_HALF, **OPT))
    r.render(1, 3)
    assert same(E.image(j), r.image_sum())
    r.close()
    E.close()


def test_engine_argument_errors(scenes):
    E = lx.Engine([scenes["a"]], default_options(**OPT), max_paths=2000)
    cam = scenes["a"].desc.camera
    with pytest.raises(lx.LuxError):
        E.submit(1, 1, camera=cam)           # no such scene
    with pytest.raises(lx.LuxError):
        E.submit(0, 0)                       # no samples
    big = _ffi.CameraDesc.from_buffer_copy(cam)
    big.width = big.height = 64
    with pytest.raises(lx.LuxError):
        E.submit(0, 1, camera=big)           # one sample larger than the wave
    j = E.submit(0, 1)
    with pytest.raises(lx.LuxError):
        E.release(j + 5)
    E.step()
    E.close()


def test_serving_loop_latencies_and_images(scenes):
    from luxion_b200 import serving, workloads
    sc = [scenes["a"], scenes["b"]]
    reqs = workloads.request_stream(2, 8, 200.0, seed=4, depth=5)
    for r in reqs:       # small frames for a quick test
        r["camera"] = lx.make_camera(40, 24, r["camera"].position[:], workloads.CAMERA_LOOK, 45.0)
        r["spp"] = 1 + r["spp"] % 5
    E = lx.Engine(sc, default_options(**OPT), max_paths=4000, schedule=_ffi.SCHED_SHORTEST_FIRST)
    eng = serving.serve_engine(E, reqs, keep_images=True)
    E.close()
    plain = serving.serve_plain(sc, reqs, default_options(**OPT), keep_images=True)
    assert eng["requests"] == 8 and eng["p50_ms"] <= eng["p99_ms"] and eng["p50_ms"] > 0
    for i in range(8):
        assert same(eng["images"][i], plain["images"][i]), i
