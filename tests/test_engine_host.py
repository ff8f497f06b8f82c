"""Host logic of the job engine, on the CPU: the wave planner (lux_plan_wave) against a
restatement of its rule, and the engine's argument checks that need no device."""
import ctypes as C

import numpy as np
import pytest

import luxion_b200 as lx


def plan_py(npix, remaining, capacity, max_segments):
    take, used, segs = [0] * len(npix), 0, 0
    for i, (n, r) in enumerate(zip(npix, remaining)):
        if segs >= max_segments or r <= 0 or n <= 0:
            continue
        fit = (capacity - used) // n
        if fit <= 0:
            continue
        take[i] = min(r, fit)
        used += take[i] * n
        segs += 1
    return take


def test_plan_wave_matches_rule_on_random_mixes():
    rng = np.random.default_rng(0)
    sizes = np.array([128 * 128, 256 * 256, 512 * 512, 1024 * 1024, 1920 * 1080])
    for _ in range(300):
        n = int(rng.integers(1, 80))
        npix = rng.choice(sizes, n).astype(np.int32)
        rem = rng.choice([1, 4, 16, 64], n).astype(np.int32) * rng.integers(0, 2, n).astype(np.int32)
        cap = int(rng.choice([1 << 20, 4 << 20, 8 << 20, 16 << 20]))
        segs = int(rng.integers(1, 300))
        got = lx.plan_wave(npix, rem, cap, segs)
        assert list(got) == plan_py(list(npix), list(rem), cap, segs)
        assert int((got.astype(np.int64) * npix).sum()) <= cap
        assert np.count_nonzero(got) <= segs
        assert np.all(got <= np.maximum(rem, 0))


def test_plan_wave_skips_jobs_that_do_not_fit_and_fills_with_later_ones():
    # a 1080p sample does not fit next to two 1024^2 samples in 3M paths; the small job does
    got = lx.plan_wave([1024 * 1024, 1920 * 1080, 128 * 128], [2, 5, 64], 3 << 20)
    assert list(got) == [2, 0, 64]


def test_plan_wave_rejects_bad_arguments():
    L = lx.lib()
    take = (C.c_int * 1)()
    one = (C.c_int * 1)(1)
    assert L.lux_plan_wave(one, one, -1, 10, 4, take) == -1
    assert L.lux_plan_wave(None, None, 1, 10, 4, take) == -1
    assert L.lux_plan_wave(None, None, 0, 10, 4, None) == 0


def test_engine_needs_a_device_and_scenes():
    s = lx.random_scene(seed=1, num_instances=4, total_tris=4000, min_tris=500, max_tris=1500, num_emissive=1,
                        num_textures=1, texture_size=16, env_width=16, env_height=8, width=16, height=16)
    with pytest.raises(lx.LuxError) as e:
        lx.Engine([s])
    assert e.value.code == -3
    with pytest.raises(lx.LuxError) as e:
        lx.Engine([])
    assert e.value.code == -1
