"""lux_trace_rays_static, the trace entry point that stages rays and hits through the library's
fixed device scratch instead of per-call allocations, against lux_trace_rays on the same rays.

Named to be collected last, so that it also runs after every other test has used the device.
Two calls in a row, the second one smaller than the first, show that the work cursor is
cleared between calls and that no result of the first call shows through in the second."""
import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200 import _ffi
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu

LO, HI = [-12, 0, -12], [12, 5, 12]


@pytest.fixture(scope="module")
def renderer():
    s = lx.random_scene(seed=31, num_instances=30, total_tris=150000, min_tris=2000, max_tris=20000,
                        num_emissive=3, num_textures=4, texture_size=64, env_width=64, env_height=32,
                        width=64, height=48, trace_depth=8)
    r = lx.Renderer(s, default_options())
    yield r
    r.close()


def _rays(n, seed, mode):
    rays = ol.random_rays(n, LO, HI, seed=seed)
    if mode == 1:
        rays[:, 3] = np.random.default_rng(seed + 1).uniform(0.5, 20.0, n).astype(np.float32)
    return rays


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_two_calls_in_a_row_match_lux_trace_rays(renderer, mode):
    a, b = _rays(50000, 100 + mode, mode), _rays(20000, 200 + mode, mode)
    sa = renderer.trace_rays_static(a, mode, 3)
    sb = renderer.trace_rays_static(b, mode, 4)
    ra = renderer.trace_rays(a, mode, 3)
    rb = renderer.trace_rays(b, mode, 4)
    assert np.array_equal(sa, ra)
    assert np.array_equal(sb, rb)
    assert (ra[:, 0].view(np.float32) > 0).sum() > 1000   # the rays do hit the scene


def test_largest_batch_and_limits(renderer):
    n = _ffi.TRACE_STATIC_MAX_RAYS
    rays = _rays(n, 7, 0)
    assert np.array_equal(renderer.trace_rays_static(rays, 0, 5), renderer.trace_rays(rays, 0, 5))
    assert renderer.trace_rays_static(rays[:0], 0, 5).shape == (0, 5)
    with pytest.raises(lx.LuxError) as e:
        renderer.trace_rays_static(_rays(n + 1, 8, 0), 0, 5)
    assert e.value.code == -1 and "LUX_TRACE_STATIC_MAX_RAYS" in str(e.value)
    # the rejected call did no device work: the next call still matches
    small = _rays(1000, 9, 2)
    assert np.array_equal(renderer.trace_rays_static(small, 2, 6), renderer.trace_rays(small, 2, 6))


def test_static_call_allocates_no_device_memory(renderer):
    """The entry point's defining property: lux_trace_rays_static makes no device allocation
    (lux_device_alloc_count is unchanged across it), while lux_trace_rays makes its per-call
    temporaries."""
    rays = _rays(30000, 11, 0)
    renderer.trace_rays_static(rays, 0, 3)   # the device code and scratch are loaded
    count = lx.lib().lux_device_alloc_count
    before = count()
    for mode in (0, 1, 2):
        renderer.trace_rays_static(_rays(30000, 12 + mode, mode), mode, 3)
    assert count() == before
    renderer.trace_rays(rays, 0, 3)
    assert count() > before
